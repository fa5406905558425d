"""The incomplete multi-hash max/min colouring (coloring = 3) on the GPU
against the reference's own output (tests/golden/mhash.npz) and the oracle.

Both sides draw their random values from the C library's rand(), so each
call is preceded by the same srand().  Verify mode (nThreads=1) must match
the reference's one-thread run bit for bit: the colouring, C_orig and the
summary.  Fast mode must land within FAST_Q_TOL of the reference's final
modularity on graphs with clear communities.
"""
import numpy as np
import pytest

from grappolo_b200 import _lib, graphs, louvain
from _golden import mhash_cases, srand

pytestmark = pytest.mark.gpu

FAST_Q_TOL = 1e-3  # |Q_fast - Q_reference| (absolute)


@pytest.mark.parametrize('case', mhash_cases(), ids=lambda c: c[0])
def test_multihash_coloring_verify(case):
    _, g, nc, exp = case
    srand(exp['seed'])
    col, mc, _ = louvain.algoColoringMultiHashMaxMin(g, nHash=2, nItrs=max(1, nc // 4))
    assert mc == int(exp['max_color'])
    assert np.array_equal(col, exp['color'])


@pytest.mark.parametrize('case', mhash_cases(), ids=lambda c: c[0])
def test_multiphase_multihash_verify(case):
    _, g, nc, exp = case
    srand(exp['seed'])
    C, st = louvain.runMultiPhaseColoring(g, coloring=3, numColors=nc, numThreads=1, stats=True)
    assert np.array_equal(C, exp['C'])
    assert (st['phases'], st['total_iterations'], st['final_clusters']) == \
        (int(exp['phases']), int(exp['itr']), int(exp['clusters']))
    assert abs(st['final_modularity'] - float(exp['mod'])) <= 5e-7  # reference prints %lf


@pytest.mark.parametrize('nc', [4, 16, 64])
def test_multihash_verify_vs_oracle_100k(oracle, nc):
    """A 100k-vertex planted partition: colouring and multiphase run, against
    the oracle restatement with the same rand() stream."""
    g = graphs.planted_partition()
    srand(21)
    col, mc, _ = louvain.algoColoringMultiHashMaxMin(g, nHash=2, nItrs=max(1, nc // 4))
    srand(21)
    col_o, mc_o = oracle.color_mhash(g, nc)
    assert mc == mc_o and np.array_equal(col, col_o)
    srand(22)
    C, st = louvain.runMultiPhaseColoring(g, coloring=3, numColors=nc, numThreads=1, stats=True)
    srand(22)
    Co, so, _ = oracle.run_multiphase_coloring(g, coloring=3, num_colors=nc)
    assert np.array_equal(C, Co)
    assert st['phases'] == so['phases'] and st['total_iterations'] == so['total_iterations']
    assert st['final_modularity'] == pytest.approx(so['final_mod'], rel=1e-12)


@pytest.mark.parametrize('nc', [4, 16])
def test_multihash_fast_mode(oracle, nc):
    g = graphs.planted_partition(seed=3)
    srand(31)
    _, st = louvain.runMultiPhaseColoring(g, coloring=3, numColors=nc, numThreads=8, stats=True)
    srand(31)
    _, so, _ = oracle.run_multiphase_coloring(g, coloring=3, num_colors=nc)
    assert abs(st['final_modularity'] - so['final_mod']) <= FAST_Q_TOL


def test_multihash_rejects_bad_arguments():
    g = graphs.from_edges(3, [(0, 1), (1, 2)])
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.algoColoringMultiHashMaxMin(g, nHash=0, nItrs=2)
    assert e.value.code == 1  # GLV_ERR_ARG
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.algoColoringMultiHashMaxMin(g, nHash=2, nItrs=1024)
    assert e.value.code == 4  # GLV_ERR_COLORS
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.runMultiPhaseColoring(g, coloring=4)
    assert e.value.code == 1  # GLV_ERR_ARG
