"""Fast-mode coarsening without sorts (coarsen_hash.cuh) against the
sort-based coarsening (GRAPPOLO_B200_COARSEN=sort), which the verify-mode
tests pin to the reference's buildNextLevelGraphOpt bit for bit: the
per-community hash tables (GRAPPOLO_B200_COARSEN=hash, every level) and the
default, where a level of at most 16384 communities is folded into a dense
matrix and larger ones keep the sorts.

These paths leave the order of each sum's additions open (the hash tables
also the entry order inside a coarse row).  With integral weights every sum
is exact, and with the deterministic id-order colouring nothing else in fast
mode depends on either order, so whole multiphase runs must give the same
community array, modularity, and phase, iteration, cluster and level sizes
on every path.  On non-integral weights the sums may differ in the last bits:
the final modularity must agree to well inside the fast-mode tolerance.
"""
import numpy as np
import pytest

from grappolo_b200 import _lib, graphs, louvain
from _golden import load

pytestmark = pytest.mark.gpu


def _int_rmat(scale, seed):
    g = graphs.rmat(scale, seed=seed)
    return graphs.CSRGraph(g.ptr, g.tail, np.floor(g.weight * 4.0) + 1.0)


def _cases():
    yield 'hubs', load('hubs')[0]
    yield 'karate', load('karate')[0]
    yield 'mixed20k', graphs.planted_partition_mixed(20000, 50, 0.3, 12.0, seed=4)
    yield 'rmat14_int', _int_rmat(14, 9)
    yield 'rmat16_int', _int_rmat(16, 3)


def _run(monkeypatch, g, path):
    monkeypatch.setenv('GRAPPOLO_B200_COLORING', 'id')
    monkeypatch.setenv('GRAPPOLO_B200_AUTOTUNE', '0')
    if path:
        monkeypatch.setenv('GRAPPOLO_B200_COARSEN', path)
    else:
        monkeypatch.delenv('GRAPPOLO_B200_COARSEN', raising=False)
    return louvain.run_multiphase_csr(g, mode=_lib.GLV_MODE_FAST)


@pytest.mark.parametrize('path', ['hash', None])
@pytest.mark.parametrize('name,g', list(_cases()), ids=[c[0] for c in _cases()])
def test_coarsening_paths_equal_sorted_integral(name, g, path, monkeypatch):
    assert np.all(g.weight == np.floor(g.weight))
    C1, s1 = _run(monkeypatch, g, 'sort')
    C2, s2 = _run(monkeypatch, g, path)
    assert np.array_equal(C1, C2)
    for k in ('phases', 'total_iterations', 'final_clusters', 'final_modularity'):
        assert s1[k] == s2[k], k
    assert [(p['num_vertices'], p['nnz']) for p in s1['phase']] == \
        [(p['num_vertices'], p['nnz']) for p in s2['phase']]


@pytest.mark.parametrize('path', ['hash', None])
@pytest.mark.parametrize('scale', [14, 18])
def test_coarsening_paths_non_integral(scale, path, monkeypatch):
    g = graphs.rmat(scale, seed=2)
    _, s1 = _run(monkeypatch, g, 'sort')
    _, s2 = _run(monkeypatch, g, path)
    assert abs(s1['final_modularity'] - s2['final_modularity']) < 1e-4
