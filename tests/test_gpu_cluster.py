"""Hub rows on thread-block clusters (GRAPPOLO_B200_CLUSTER = blocks per
cluster; the autotuner's third candidate).  A cluster's blocks hold one hash
table in their shared memory, reached through distributed shared memory; a
row whose table needs more than one cluster's slots is split by community
into partitions (GRAPPOLO_B200_CLUSTER_PARTS at most), each a task that reads
the whole row, and the last partition to finish decides the row.

With integral weights every sum is exact in any order, so verify mode must
give the reference's one-thread results bit for bit on every cluster size,
including rows decided across partitions; fast mode must stay in the
reference's modularity range; batches must equal their graphs' own runs.
GRAPPOLO_B200_BLOCK_MAX=128 sends every row above 128 entries to the hub path.
"""
import json
import os

import numpy as np
import pytest

from grappolo_b200 import _lib, graphs, louvain
from _golden import load

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _cluster(monkeypatch, cl, parts, block_max='128'):
    monkeypatch.setenv('GRAPPOLO_B200_CLUSTER', cl)
    monkeypatch.setenv('GRAPPOLO_B200_CLUSTER_PARTS', parts)
    monkeypatch.setenv('GRAPPOLO_B200_AUTOTUNE', '0')
    if block_max:
        monkeypatch.setenv('GRAPPOLO_B200_BLOCK_MAX', block_max)


@pytest.mark.parametrize('cl,parts', [('1', '4'), ('2', '2'), ('4', '1'), ('8', '1'), ('16', '1')])
def test_cluster_rows_verify_golden(cl, parts, monkeypatch):
    _cluster(monkeypatch, cl, parts)
    for name in ('hubs', 'karate', 'pp1000'):  # the golden cases with integral weights
        g, z = load(name)
        C, st = louvain.runMultiPhaseColoring(g, numThreads=1, stats=True)
        assert st['hub_cluster'] == int(cl)
        assert np.array_equal(C, z['mpc_C']), name
        assert (st['phases'], st['total_iterations'], st['final_clusters']) == \
            (z['mpc_phases'], z['mpc_itr'], z['mpc_clusters']), name
        C, st = louvain.runMultiPhaseBasic(g, numThreads=1, stats=True)
        assert np.array_equal(C, z['mpb_C']), name


def _integral(g):
    # R-MAT's weights mapped to 1..4 (still symmetric): verify mode then runs
    # the persistent sweep, whose sums are exact in any order
    return graphs.CSRGraph(g.ptr, g.tail, np.floor(g.weight * 4.0) + 1.0)


@pytest.mark.parametrize('cl,parts', [('1', '8'), ('2', '1'), ('4', '2')])
def test_cluster_rows_verify_vs_oracle(cl, parts, monkeypatch, oracle):
    _cluster(monkeypatch, cl, parts)
    g = _integral(graphs.rmat(14, seed=9))
    C, st = louvain.runMultiPhaseColoring(g, numThreads=1, stats=True)
    assert st['hub_cluster'] == int(cl)
    Co, so, _ = oracle.run_multiphase_coloring(g)
    assert np.array_equal(C, Co)
    assert st['total_iterations'] == so['total_iterations']


@pytest.mark.parametrize('cl', ['2', '8'])
def test_cluster_rows_fast_rmat18(cl, monkeypatch):
    _cluster(monkeypatch, cl, '2', block_max=None)
    with open(os.path.join(HERE, 'golden', 'fast_pins.json')) as f:
        lo, hi = json.load(f)['rmat18']['printed_range']
    sys_path = os.path.join(HERE, 'golden')
    import sys
    sys.path.insert(0, sys_path)
    from make_fast_pins import make_graph
    g = make_graph('rmat18')
    C, st = louvain.run_multiphase_csr(g, mode=_lib.GLV_MODE_FAST)
    assert st['hub_cluster'] == int(cl)
    assert lo - 1e-3 <= st['final_modularity'] <= hi + 1e-3
    deg = np.diff(g.ptr)
    assert np.all(C[deg == 0] == -1)


def test_cluster_rows_batch_equals_single_runs(monkeypatch):
    _cluster(monkeypatch, '2', '2')
    rng = np.random.default_rng(11)
    gs = [graphs.planted_partition_mixed(int(nv), 40, 0.3, 24.0, seed=int(s))
          for nv, s in zip(rng.integers(800, 6000, 6), rng.integers(0, 1000, 6))]
    gs.append(load('hubs')[0])
    Cs, st = louvain.run_batch(gs, coloring=True, mode=_lib.GLV_MODE_VERIFY)
    for k, g in enumerate(gs):
        C1, s1 = louvain.run_multiphase_csr(g, coloring=True, mode=_lib.GLV_MODE_VERIFY)
        assert np.array_equal(Cs[k], C1), k
        assert st['iterations'][k] == s1['total_iterations'], k
