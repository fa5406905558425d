"""Synthetic generators and Grappolo's binary format (host side)."""
import numpy as np

from grappolo_b200 import graphs


def _check_csr(g):
    assert g.ptr[0] == 0 and np.all(np.diff(g.ptr) >= 0) and g.ptr[-1] == g.nnz
    heads = g.heads()
    # symmetric with equal weights both ways
    a = np.lexsort((g.tail, heads))
    b = np.lexsort((heads, g.tail))
    assert np.array_equal(heads[a], g.tail[b]) and np.array_equal(g.tail[a], heads[b])
    assert np.array_equal(g.weight[a], g.weight[b])
    # rows sorted by tail, no duplicates
    for v in range(min(g.num_vertices, 2000)):
        row = g.tail[g.ptr[v]:g.ptr[v + 1]]
        assert np.all(np.diff(row) > 0)


def test_planted_partition_shape():
    g = graphs.planted_partition(num_blocks=50, block_size=100, seed=3)
    assert g.num_vertices == 5000
    _check_csr(g)
    assert not np.any(g.heads() == g.tail)
    assert 12 <= g.nnz / g.num_vertices <= 17  # intra 12 + inter ~4 minus duplicates
    assert np.all(g.weight == 1.0)


def test_rmat_shape_and_weights():
    g = graphs.rmat(12, seed=5)
    assert g.num_vertices == 4096
    _check_csr(g)
    assert np.all((g.weight > 0) & (g.weight <= 1))
    assert np.diff(g.ptr).max() > 20 * np.diff(g.ptr).mean()  # skewed degrees


def test_generators_are_seeded():
    assert np.array_equal(graphs.rmat(10, seed=1).tail, graphs.rmat(10, seed=1).tail)
    assert not np.array_equal(graphs.rmat(10, seed=1).tail, graphs.rmat(10, seed=2).tail)


def test_binary_round_trip(tmp_path):
    g = graphs.rmat(10, seed=2)
    p = tmp_path / 'g.bin'
    graphs.write_binary(g, str(p))
    h = graphs.read_binary(str(p))
    assert np.array_equal(g.ptr, h.ptr) and np.array_equal(g.tail, h.tail)
    assert np.array_equal(g.weight, h.weight)


def test_from_edges_keeps_self_loops_once():
    g = graphs.from_edges(3, [(0, 1), (1, 1), (1, 2)], weights=[1, 5, 2])
    assert g.nnz == 5
    row1 = g.tail[g.ptr[1]:g.ptr[2]]
    assert list(row1) == [0, 1, 2]
    assert g.num_edges == 3
