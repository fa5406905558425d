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


def test_union_lays_graphs_end_to_end():
    from grappolo_b200 import louvain
    a = graphs.planted_partition_mixed(50, 10, 0.2, 6, seed=1)
    b = graphs.planted_partition_mixed(70, 7, 0.3, 5, seed=2)
    voff, u = louvain.union([a, b])
    assert list(voff) == [0, 50, 120]
    assert u.num_vertices == 120 and u.nnz == a.nnz + b.nnz
    assert np.array_equal(u.ptr[:51], a.ptr)
    assert np.array_equal(u.tail[:a.nnz], a.tail)
    assert np.array_equal(u.tail[a.nnz:], b.tail + 50)
    assert np.array_equal(u.ptr[50:] - a.nnz, b.ptr)
    heads = u.heads()
    assert np.all((heads < 50) == (u.tail < 50))


def test_batch_specs_ranges():
    sp = graphs.batch_specs(512, seed=3)
    assert sp.shape == (512, 4)
    assert sp[:, 0].min() >= 500 and sp[:, 0].max() < 200000
    assert np.all(sp[:, 1] >= 20) and np.all(sp[:, 1] <= sp[:, 0])
    assert np.all((sp[:, 2] >= 0.1) & (sp[:, 2] <= 0.6))
    assert np.all((sp[:, 3] >= 6) & (sp[:, 3] <= 32))


def test_planted_batch_generator_on_cpu():
    """The device generator (run here with torch on the CPU): tails stay in
    their graph, rows sorted, no duplicates or self-loops, symmetric."""
    sp = graphs.batch_specs(6, seed=1, nv_range=(500, 3000))
    voff, ptr, tail, w = graphs.planted_batch_device(sp, device='cpu', group_pairs=20000)
    p = ptr.numpy()
    t = tail.numpy().astype(np.int64)
    assert p[0] == 0 and p[-1] == t.size and voff[-1] == p.size - 1
    heads = np.repeat(np.arange(p.size - 1), np.diff(p))
    g_of = np.searchsorted(voff, heads, side='right') - 1
    assert np.all((t >= voff[g_of]) & (t < voff[g_of + 1]))
    n = voff[-1]
    key = heads * n + t
    assert np.all(np.diff(key) > 0) and np.all(heads != t)
    assert np.array_equal(np.sort(t * n + heads), key)
    assert np.all(w.numpy() == 1.0)


def test_rmat_lean_generator_on_cpu():
    """The bounded-scratch R-MAT builder (torch on the CPU here): rows sorted
    by tail, no duplicates or self-loops, symmetric with equal weights, U(0,1]."""
    ptr, tail, w = graphs.rmat_device_lean(11, device='cpu', chunk=3000)
    p = ptr.numpy()
    t = tail.numpy().astype(np.int64)
    ww = w.numpy()
    nv = p.size - 1
    heads = np.repeat(np.arange(nv), np.diff(p))
    key = heads * nv + t
    assert np.all(np.diff(key) > 0) and np.all(heads != t)
    rev = t * nv + heads
    o = np.argsort(rev)
    assert np.array_equal(rev[o], key)
    assert np.array_equal(ww[o], ww)
    assert ww.min() > 0 and ww.max() <= 1
