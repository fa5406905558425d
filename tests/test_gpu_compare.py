"""Community-comparison metrics on the GPU (glv_compare_communities,
glv_gini_coefficient) against the reference's own output
(tests/golden/compare.npz) and the oracle.  Pair counts are integers and must
be exact; precision, recall, F-score and Gini are computed from them with the
reference's expressions, so they equal the oracle's bit for bit and the
reference's printed values to their six decimals."""
import numpy as np
import pytest

from grappolo_b200 import _lib, graphs, louvain
from _golden import COMPARE_FLOATS, COMPARE_INTS, compare_cases, gini_cases

pytestmark = pytest.mark.gpu

PRINTED_TOL = 5e-7  # the reference prints these with %lf


@pytest.mark.parametrize('case', compare_cases(), ids=lambda c: c[0])
def test_comparison_golden(case, oracle):
    _, C1, C2, exp = case
    st, a, b = louvain.computeCommunityComparisons(C1, C2)
    for k in COMPARE_INTS:
        assert st[k] == int(exp[k]), k
    for k in COMPARE_FLOATS:
        assert abs(st[k] - float(exp[k])) <= PRINTED_TOL, k
    assert np.array_equal(a, exp['C1_after']) and np.array_equal(b, exp['C2_after'])
    o, _, _ = oracle.compare(C1, C2)
    for k in COMPARE_INTS + COMPARE_FLOATS:
        assert st[k] == o[k], k


@pytest.mark.parametrize('k', range(4))
def test_gini_golden(k):
    sizes, value, srt = gini_cases()[k]
    g, s = louvain.computeGiniCoefficient(sizes)
    assert g == value and np.array_equal(s, srt)


def test_comparison_large_vs_oracle(oracle):
    """One million vertices: planted blocks against a noisy copy, with -1
    entries on both sides; host and device entry points."""
    import torch
    rng = np.random.default_rng(7)
    n = 1_000_000
    C1 = np.arange(n) // 1000
    C2 = C1.copy()
    flip = rng.random(n) < 0.2
    C2[flip] = rng.integers(0, 2000, int(flip.sum()))
    C1[rng.integers(0, n, 500)] = -1
    C2[rng.integers(0, n, 700)] = -1
    st, a, b = louvain.computeCommunityComparisons(C1, C2)
    o, oa, ob = oracle.compare(C1, C2)
    for k in COMPARE_INTS + COMPARE_FLOATS:
        assert st[k] == o[k], k
    assert np.array_equal(a, oa) and np.array_equal(b, ob)
    d1 = torch.tensor(C1, device='cuda')
    d2 = torch.tensor(C2, device='cuda')
    sd = louvain.compare_communities_device(d1, d2)
    for k in COMPARE_INTS + COMPARE_FLOATS:
        assert sd[k] == o[k], k
    assert np.array_equal(d1.cpu().numpy(), oa)


def test_comparison_of_a_louvain_run(oracle):
    """The planted partition's blocks against the engine's own clustering."""
    g = graphs.planted_partition()
    C = louvain.runMultiPhaseColoring(g, numThreads=1)
    truth = np.arange(g.num_vertices) // 100
    st, _, _ = louvain.computeCommunityComparisons(truth, C)
    o, _, _ = oracle.compare(truth, C)
    for k in COMPARE_INTS + COMPARE_FLOATS:
        assert st[k] == o[k], k
    # Louvain merges planted blocks of 100 (the resolution limit), so pairs of
    # one block stay together (recall) while precision drops
    assert 0 < st['f_score'] <= 1 and st['recall'] >= st['precision']


def test_comparison_rejects_bad_labels():
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.computeCommunityComparisons([0, 1, -2], [0, 1, 1])
    assert e.value.code == 1
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.computeCommunityComparisons([0, 1, 1], [0, 1])
    assert e.value.code == 1
    with pytest.raises(_lib.GrappoloError) as e:
        louvain.computeGiniCoefficient([3, -1, 2])
    assert e.value.code == 1
