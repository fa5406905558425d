"""Edge lists to CSR and binary graph files on the GPU, against the
reference's own outputs (tests/golden/csr_build.npz, karate.bin) and the
oracle.  Everything here is integer or index work, or moves weights without
arithmetic: results must be identical, entry for entry."""
import os

import numpy as np
import pytest

from grappolo_b200 import _lib, graphs, louvain
from _golden import csr_cases, load

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden')


def _cols(e):
    return e['head'], e['tail'], e['weight']


@pytest.mark.parametrize('case', csr_cases(), ids=lambda c: c[0])
def test_remove_edges(case):
    _, e = case
    out, nge = louvain.removeEdges(e['nv'], louvain._edges(e['head'], e['tail'], e['weight']))
    assert nge == e['nge']
    assert np.array_equal(out['head'], e['rm_head']) and np.array_equal(out['tail'], e['rm_tail'])
    assert np.array_equal(out['weight'], e['rm_weight'])


@pytest.mark.parametrize('case', csr_cases(), ids=lambda c: c[0])
def test_sort_edges_undirected_and_rows(case):
    _, e = case
    nv, n = e['nv'], e['nge']
    kept = louvain._edges(e['rm_head'][:n], e['rm_tail'][:n], e['rm_weight'][:n])
    ptrs, rows = louvain.SortEdgesUndirected(nv, kept)
    assert np.array_equal(ptrs, e['ptrs'])
    assert np.array_equal(rows['tail'], e['rows_tail'])
    assert np.array_equal(rows['weight'], e['rows_weight'])
    srt = louvain.SortNodeEdgesByIndex(nv, rows, ptrs)
    assert np.array_equal(srt['tail'], e['sorted_tail'])
    assert np.array_equal(srt['weight'], e['sorted_weight'])
    rp, raw = louvain.SortEdgesUndirected(nv, louvain._edges(*_cols(e)))
    assert np.array_equal(rp, e['raw_ptrs'])
    assert np.array_equal(raw['tail'], e['raw_tail']) and np.array_equal(raw['weight'],
                                                                          e['raw_weight'])


@pytest.mark.parametrize('case', csr_cases(), ids=lambda c: c[0])
@pytest.mark.parametrize('remove,sort', [(True, True), (True, False), (False, False)])
def test_build_csr_host_and_device(case, remove, sort):
    import torch
    _, e = case
    nv = e['nv']
    if remove:
        ptr_e = e['ptrs'][:nv + 1]
        tail_e, w_e = (e['sorted_tail'], e['sorted_weight']) if sort else \
            (e['rows_tail'], e['rows_weight'])
    else:
        ptr_e, tail_e, w_e = e['raw_ptrs'][:nv + 1], e['raw_tail'], e['raw_weight']
    g, ne = louvain.build_csr(nv, *_cols(e), remove_edges=remove, sort_rows=sort)
    assert ne == (e['nge'] if remove else len(e['head']))
    assert np.array_equal(g.ptr, ptr_e) and np.array_equal(g.tail, tail_e)
    assert np.array_equal(g.weight, w_e)
    dh = torch.tensor(e['head'], device='cuda')
    dt = torch.tensor(e['tail'], device='cuda')
    dw = torch.tensor(e['weight'], device='cuda')
    p, t, w = louvain.build_csr_device(nv, dh, dt, dw, remove_edges=remove, sort_rows=sort)
    assert np.array_equal(p.cpu().numpy(), ptr_e)
    assert np.array_equal(t.cpu().numpy(), tail_e) and np.array_equal(w.cpu().numpy(), w_e)


def test_build_csr_large_vs_oracle(oracle):
    """Three million edges with repeats and both orientations: the device
    build, and the host build from pageable arrays (72 MB in, 130 MB out: the
    staged copies), equal the oracle's removeEdges + fill + row sort."""
    import torch
    rng = np.random.default_rng(5)
    nv, ne = 200_000, 3_000_000
    h, t = rng.integers(0, nv, ne), rng.integers(0, nv, ne)
    k = ne // 4
    src, dst = rng.integers(0, ne, k), rng.integers(0, ne, k)
    h[dst], t[dst] = h[src], t[src]
    flip = rng.random(ne) < 0.5
    h, t = np.where(flip, t, h), np.where(flip, h, t)
    w = rng.uniform(0.1, 3.0, ne)
    rh, rt, rw, nge = oracle.remove_edges(nv, h, t, w)
    ptrs, sh, st, sw = oracle.sort_edges_undirected(nv, rh[:nge], rt[:nge], rw[:nge])
    _, ot, ow = oracle.sort_node_edges(nv, ptrs, sh, st, sw)
    p, dt, dw = louvain.build_csr_device(nv, torch.tensor(h, device='cuda'),
                                         torch.tensor(t, device='cuda'),
                                         torch.tensor(w, device='cuda'), True, True)
    assert np.array_equal(p.cpu().numpy(), ptrs[:nv + 1])
    assert np.array_equal(dt.cpu().numpy(), ot) and np.array_equal(dw.cpu().numpy(), ow)
    p2, dt2, _ = louvain.build_csr_device(nv, torch.tensor(h, device='cuda'),
                                          torch.tensor(t, device='cuda'), None, True, False)
    assert np.array_equal(p2.cpu().numpy(), ptrs[:nv + 1])
    assert np.array_equal(dt2.cpu().numpy(), st)
    g, nk = louvain.build_csr(nv, h, t, w, remove_edges=True, sort_rows=True)
    assert nk == nge and np.array_equal(g.ptr, ptrs[:nv + 1])
    assert np.array_equal(g.tail, ot) and np.array_equal(g.weight, ow)
    srt = louvain.SortNodeEdgesByIndex(nv, louvain._edges(sh, st, sw), ptrs)
    assert np.array_equal(srt['tail'], ot) and np.array_equal(srt['weight'], ow)


def test_build_csr_rejects_bad_ids():
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.build_csr(4, [0, 1, 5], [1, 2, 3])
    assert e.value.code == 1  # GLV_ERR_ARG
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.build_csr(4, [0, -1], [1, 2], remove_edges=False)
    assert e.value.code == 1


def test_empty_edge_list():
    g, ne = louvain.build_csr(5, [], [])
    assert ne == 0 and np.array_equal(g.ptr, np.zeros(6, dtype=np.int64))


def test_load_binary_device_golden():
    import torch
    p, t, w = louvain.load_binary_device(os.path.join(GOLDEN, 'karate.bin'))
    _, z = load('karate')
    assert np.array_equal(p.cpu().numpy(), z['ptr'])
    assert np.array_equal(t.cpu().numpy(), z['tail']) and np.array_equal(w.cpu().numpy(),
                                                                          z['weight'])
    assert t.dtype == torch.int32


def test_load_binary_device_then_cluster(tmp_path):
    """A 100k-vertex graph written to a binary file, streamed into the device
    and clustered there: the same communities as the host path on the same
    graph (verify mode)."""
    import torch
    g = graphs.planted_partition()
    path = str(tmp_path / 'pp.bin')
    graphs.write_binary(g, path)
    p, t, w = louvain.load_binary_device(path)
    assert np.array_equal(t.cpu().numpy(), g.tail.astype(np.int32))
    C = torch.empty(g.num_vertices, dtype=torch.int32, device='cuda')
    st = louvain.run_multiphase_device(g.num_vertices, p.data_ptr(), t.data_ptr(), w.data_ptr(),
                                       C.data_ptr(), mode=_lib.GLV_MODE_VERIFY)
    C1, s1 = louvain.run_multiphase_csr(g, mode=_lib.GLV_MODE_VERIFY)
    assert np.array_equal(C.cpu().numpy(), C1)
    assert st['final_modularity'] == s1['final_modularity']


def test_load_binary_device_many_chunks(tmp_path):
    """R-MAT scale 18 (7.6M entries): the file streams through the pinned
    buffers in two chunks."""
    g = graphs.rmat(18, seed=3)
    path = str(tmp_path / 'r18.bin')
    graphs.write_binary(g, path)
    p, t, w = louvain.load_binary_device(path)
    assert g.nnz > (1 << 22)  # more than one 4M-entry chunk
    assert np.array_equal(p.cpu().numpy(), g.ptr)
    assert np.array_equal(t.cpu().numpy(), g.tail.astype(np.int32))
    assert np.array_equal(w.cpu().numpy(), g.weight)


def test_load_binary_device_rejects_bad_files(tmp_path):
    bad = tmp_path / 'bad.bin'
    g = graphs.from_edges(3, [(0, 1), (1, 2)])
    graphs.write_binary(g, str(bad))
    raw = bytearray(bad.read_bytes())
    raw[24 + 4 * 8 + 8:24 + 4 * 8 + 16] = (7).to_bytes(8, 'little')  # a tail outside [0, 3)
    bad.write_bytes(bytes(raw))
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.load_binary_device(str(bad))
    assert e.value.code == 9  # GLV_ERR_IO
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.load_binary_device(str(tmp_path / 'missing.bin'))
    assert e.value.code == 9
