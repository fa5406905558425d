"""The allocation-free modularity entry point, against the allocating one.

glv_dev_modularity_static serves callers that cannot call cudaMalloc during a
run (their device memory belongs to a host framework's caching allocator, or
to a budget fixed at start-up).  It keeps its scratch in a static device array
and computes the modularity from the caller's device buffers.  This file is
collected last so that a failure here cannot stop the other GPU tests from
running first; it passes on its own in a fresh process and after them.
"""
import ctypes as ct

import numpy as np
import pytest

from grappolo_b200 import _lib, graphs, louvain

pytestmark = pytest.mark.gpu

MOD_REL_TOL = 1e-9  # the modularity tolerance the parity tests use


def _device_inputs(g, C):
    import torch
    dev = torch.device('cuda:0')
    vdeg = np.bincount(g.heads(), weights=g.weight, minlength=g.num_vertices)
    cdeg = np.zeros(g.num_vertices)
    ok = C >= 0
    np.add.at(cdeg, C[ok], vdeg[ok])
    t = {
        'ptr': torch.from_numpy(g.ptr.astype(np.int64)).to(dev),
        'tail': torch.from_numpy(g.tail.astype(np.int32)).to(dev),
        'w': torch.from_numpy(g.weight.astype(np.float64)).to(dev),
        'C': torch.from_numpy(C.astype(np.int32)).to(dev),
        'cdeg': torch.from_numpy(cdeg).to(dev),
        'out': torch.zeros(3, dtype=torch.float64, device=dev),
    }
    return t, 1.0 / vdeg.sum()


def _call(g, t, constant):
    import torch
    L = _lib.lib()
    rc = L.glv_dev_modularity_static(g.num_vertices, t['ptr'].data_ptr(), t['tail'].data_ptr(),
                                     t['w'].data_ptr(), t['C'].data_ptr(), t['cdeg'].data_ptr(),
                                     constant, t['out'].data_ptr(),
                                     ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc)
    torch.cuda.synchronize()
    return float(t['out'][0].item())


@pytest.mark.parametrize('weighted', [False, True])
def test_static_modularity_matches_allocating_entry(weighted):
    g = graphs.planted_partition(num_blocks=200, block_size=100, seed=4)
    if weighted:
        g = graphs.random_weights(g, seed=8)
    C = louvain.runMultiPhaseColoring(g, numThreads=1)
    expected = louvain.modularity(g, C)
    t, constant = _device_inputs(g, C)
    for _ in range(2):  # two calls in a row share the static scratch
        assert _call(g, t, constant) == pytest.approx(expected, rel=MOD_REL_TOL)


def _numpy_modularity(g, C, constant, cdeg):
    heads = g.heads()
    same = (C[heads] == C[g.tail]) & (C[heads] >= 0)
    exx = float(np.sum(g.weight[same]))
    a2 = float(np.sum(cdeg * cdeg))
    return exx * constant - a2 * constant * constant


def test_static_modularity_unlabelled_vertices_and_no_allocation():
    """Vertices labelled -1 belong to no community, so their entries add
    nothing to e_xx; and after its first call on a device the entry leaves the
    device's free memory unchanged."""
    import torch
    g = graphs.planted_partition(num_blocks=50, block_size=40, seed=6)
    C = louvain.runMultiPhaseColoring(g, numThreads=1).copy()
    rng = np.random.default_rng(3)
    C[rng.random(g.num_vertices) < 0.2] = -1  # edges between unlabelled vertices remain
    t, constant = _device_inputs(g, C)
    expected = _numpy_modularity(g, C, constant, t['cdeg'].cpu().numpy())
    assert _call(g, t, constant) == pytest.approx(expected, rel=MOD_REL_TOL)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    assert _call(g, t, constant) == pytest.approx(expected, rel=MOD_REL_TOL)
    assert torch.cuda.mem_get_info()[0] == free_before


def test_static_modularity_rejects_oversize():
    L = _lib.lib()
    too_many = 16_777_216 + 1
    rc = L.glv_dev_modularity_static(too_many, 1, 1, 1, 1, 1, 1.0, 1, None)
    assert rc == 8  # GLV_ERR_LIMIT, refused before any device work
    assert b'16,777,216' in L.glv_last_error()
