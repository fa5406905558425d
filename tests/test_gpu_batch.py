"""Batches of independent graphs in one run (glv_run_batch_csr) against the
same graphs run one at a time, and against the oracle.

Verify mode with integral weights must give every graph exactly the result of
its own one-thread run: community array, final modularity, iteration and
phase counts.  Fast mode must land where a fast run of the graph alone lands.
"""
import ctypes as ct

import numpy as np
import pytest

from grappolo_b200 import _lib, graphs, louvain

pytestmark = pytest.mark.gpu

FAST_Q_TOL = 1e-3  # |Q_fast - Q_reference| on graphs with clear communities


def _mixed_batch(seed=3, sizes=(600, 900, 1500, 2500, 4000, 7000, 12000, 800, 3000, 20000)):
    rng = np.random.default_rng(seed)
    out = []
    for k, nv in enumerate(sizes):
        block = int(rng.integers(20, 200))
        mu = float(rng.uniform(0.1, 0.6))
        deg = float(rng.uniform(6, 32))
        out.append(graphs.planted_partition_mixed(nv, block, mu, deg, seed=seed * 100 + k))
    return out


@pytest.mark.parametrize('coloring', [True, False])
def test_batch_verify_equals_single_runs(coloring):
    gs = _mixed_batch()
    Cs, st = louvain.run_batch(gs, coloring=coloring, mode=_lib.GLV_MODE_VERIFY)
    for k, g in enumerate(gs):
        C1, s1 = louvain.run_multiphase_csr(g, coloring=coloring, mode=_lib.GLV_MODE_VERIFY)
        assert np.array_equal(Cs[k], C1), k
        assert st['final_modularity'][k] == s1['final_modularity'], k
        assert st['iterations'][k] == s1['total_iterations'], k
        assert st['phases'][k] == s1['phases'], k
        assert st['clusters'][k] == s1['final_clusters'], k


def test_batch_verify_vs_oracle(oracle):
    gs = _mixed_batch(seed=5, sizes=(700, 3000, 9000))
    Cs, st = louvain.run_batch(gs, coloring=True, mode=_lib.GLV_MODE_VERIFY)
    for k, g in enumerate(gs):
        Co, so, _ = oracle.run_multiphase_coloring(g)
        assert np.array_equal(Cs[k], Co), k
        assert st['final_modularity'][k] == pytest.approx(so['final_mod'], rel=1e-12)


def test_batch_fast_mode_matches_single_runs(monkeypatch):
    """Fast mode's speculative colouring races, which spreads the final Q of
    weakly structured graphs by a few 1e-3 from run to run (the reference's
    own multi-thread runs spread the same way).  With the deterministic
    id-order colouring and integral weights every other fast-mode sum is exact,
    so a batched graph must get exactly the result of its own fast run."""
    monkeypatch.setenv('GRAPPOLO_B200_COLORING', 'id')
    gs = _mixed_batch(seed=7, sizes=(3000, 30000, 60000, 1200))
    Cs, st = louvain.run_batch(gs, coloring=True, mode=_lib.GLV_MODE_FAST)
    for k, g in enumerate(gs):
        C1, s1 = louvain.run_multiphase_csr(g, mode=_lib.GLV_MODE_FAST)
        assert np.array_equal(Cs[k], C1), k
        assert st['final_modularity'][k] == s1['final_modularity'], k
    assert np.all(st['done_seconds'] > 0)


def test_batch_rejects_cross_edges():
    gs = _mixed_batch(sizes=(600, 700))
    voff, u = louvain.union(gs)
    tail = u.tail.copy()
    tail[0] = voff[1] + 3  # row 0 of graph 0 points into graph 1
    C = np.zeros(u.num_vertices, dtype=np.int64)
    lp = lambda a: a.ctypes.data_as(ct.POINTER(ct.c_long))  # noqa: E731
    rc = _lib.lib().glv_run_batch_csr(2, lp(voff), lp(u.ptr), lp(tail),
                                      u.weight.ctypes.data_as(ct.POINTER(ct.c_double)), lp(C),
                                      1, 1000, 1e-6, 1e-4, _lib.GLV_MODE_FAST, None)
    assert rc == 1  # GLV_ERR_ARG
