"""Balanced recolouring (coloring = 2, vBaseRedistribution) on the GPU against
the reference's own function (tests/golden/vbase.npz, from a copy with its
missing return added) and against the oracle restatement on larger graphs.
Colourings and, in verify mode, whole multiphase runs must be equal exactly.
Type 0 and the multiphase runs are pinned to the reference only on graphs
where its first-fit scan finds a colour for every vertex it moves
(tests/test_vbase_oracle.py); elsewhere the oracle is the checker."""
import numpy as np
import pytest

from grappolo_b200 import _lib, graphs, louvain
from _golden import vbase_cases

pytestmark = pytest.mark.gpu

FAST_Q_TOL = 1e-3


def _graphs():
    yield 'pp1000', graphs.planted_partition(num_blocks=20, block_size=50, intra_degree=10,
                                             inter_degree=3, seed=2)
    yield 'rmat12', graphs.rmat(12, seed=4)
    yield 'pp100k', graphs.planted_partition()
    yield 'rmat16', graphs.rmat(16, seed=6)
    yield 'star', graphs.from_edges(60, [(0, i) for i in range(1, 60)] + [(1, 2), (3, 4)])


@pytest.mark.parametrize('name,g', list(_graphs()))
@pytest.mark.parametrize('vtype', [0, 1])
def test_vbase_vs_oracle(oracle, name, g, vtype):
    col, mc = oracle.color_greedy(g)
    exp, moves, _ = oracle.vbase(g, col, mc + 1, vtype)
    out, n = louvain.vBaseRedistribution(g, col, mc + 1, vtype)
    assert n == moves
    assert np.array_equal(out, exp)


VBASE = vbase_cases()


@pytest.mark.parametrize('case', VBASE, ids=[c[0] for c in VBASE])
def test_vbase_golden(case):
    name, g, col, nc, exp, _ = case
    for vtype, want in exp.items():
        out, n = louvain.vBaseRedistribution(g, col, nc, vtype)
        assert np.array_equal(out, want), (name, vtype)
        assert n == int((want != col).sum())


@pytest.mark.parametrize('case', [c for c in VBASE if c[5] is not None],
                         ids=[c[0] for c in VBASE if c[5] is not None])
def test_multiphase_coloring2_golden(case):
    name, g, _, _, _, mp = case
    C, st = louvain.runMultiPhaseColoring(g, coloring=2, numThreads=1, stats=True)
    assert np.array_equal(C, mp['C'])
    assert (st['phases'], st['total_iterations'], st['final_clusters']) == \
        (mp['phases'], mp['total_iterations'], mp['final_clusters'])
    assert abs(st['final_modularity'] - mp['final_mod']) <= 5e-7  # printed with %lf


@pytest.mark.parametrize('name', ['pp1000', 'rmat12', 'pp100k'])
def test_multiphase_coloring2_verify(oracle, name):
    g = dict(_graphs())[name]
    C, st = louvain.runMultiPhaseColoring(g, coloring=2, numThreads=1, stats=True)
    Co, so, recs = oracle.run_multiphase_coloring(g, coloring=2)
    assert np.array_equal(C, Co)
    assert (st['phases'], st['total_iterations'], st['final_clusters']) == \
        (so['phases'], so['total_iterations'], so['final_clusters'])
    assert st['final_modularity'] == pytest.approx(so['final_mod'], rel=1e-12)


def test_multiphase_coloring2_fast(oracle):
    g = graphs.planted_partition(seed=4)
    _, st = louvain.runMultiPhaseColoring(g, coloring=2, numThreads=8, stats=True)
    _, so, _ = oracle.run_multiphase_coloring(g, coloring=2)
    assert abs(st['final_modularity'] - so['final_mod']) <= FAST_Q_TOL


def test_vbase_rejects_bad_colours():
    g = graphs.from_edges(3, [(0, 1), (1, 2)])
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.vBaseRedistribution(g, [0, 1, 5], 2)
    assert e.value.code == 1
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.vBaseRedistribution(g, [0, 1, 0], 2, type=3)
    assert e.value.code == 1
