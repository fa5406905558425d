"""The sweep's autotuner: per graph it picks the hub threshold and the hub chunk
size by timing one sweep iteration of the level per candidate (state restored
after each trial) and caches the choice by the graph's signature.

* the choice does not change results: with tuning forced on a small verify-mode
  graph the community array still equals the reference's one-thread run
  (the pinned digest of tests/golden/pins.json);
* a second run on the same graph takes the cached choice;
* tuned runs are not slower than the default knobs (device sweep time per
  sweep, under the deterministic id-order colouring: with the speculative
  colouring's races the iteration count of R-MAT 20 varies about threefold
  from run to run), and fast-mode modularity stays within the reference's
  range.
"""
import hashlib
import json
import os
import sys

import pytest

from grappolo_b200 import _lib, graphs, louvain
from _golden import pins

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, 'golden'))
from make_fast_pins import make_graph  # noqa: E402


def test_tuning_leaves_verify_results_unchanged(monkeypatch):
    monkeypatch.setenv('GRAPPOLO_B200_AUTOTUNE_MIN', '0')  # tune even this small level
    g = graphs.planted_partition()
    C, st = louvain.runMultiPhaseColoring(g, numThreads=1, stats=True)
    pin = pins()['planted_100k']
    assert st['tuned_block_max'] > 0 and st['tuned_hub_chunk'] > 0
    assert hashlib.sha256(C.astype('<i8').tobytes()).hexdigest() == pin['c_orig_sha256']
    assert st['total_iterations'] == pin['total_iterations']


@pytest.mark.parametrize('name', ['rmat20', 'powerlaw1m'])
def test_tuned_not_slower_and_cached(monkeypatch, name):
    with open(os.path.join(HERE, 'golden', 'fast_pins.json')) as f:
        lo, hi = json.load(f)[name]['printed_range']
    g = make_graph(name)
    monkeypatch.setenv('GRAPPOLO_B200_COLORING', 'id')
    _lib.lib().glv_set_profiling(1)  # device time of the sweep launches
    try:
        monkeypatch.setenv('GRAPPOLO_B200_AUTOTUNE', '0')
        louvain.run_multiphase_csr(g, mode=_lib.GLV_MODE_FAST)  # warm
        base = [louvain.run_multiphase_csr(g, mode=_lib.GLV_MODE_FAST)[1] for _ in range(3)]
        monkeypatch.setenv('GRAPPOLO_B200_AUTOTUNE', '1')
        first = louvain.run_multiphase_csr(g, mode=_lib.GLV_MODE_FAST)[1]
        tuned = [louvain.run_multiphase_csr(g, mode=_lib.GLV_MODE_FAST)[1] for _ in range(3)]
    finally:
        _lib.lib().glv_set_profiling(0)
    assert first['tuned_block_max'] > 0  # tuned now, or cached by an earlier test
    for st in tuned:
        assert st['tuned_from_cache'] == 1
        assert (st['tuned_block_max'], st['tuned_hub_chunk']) == \
            (first['tuned_block_max'], first['tuned_hub_chunk'])
        assert lo - 1e-3 <= st['final_modularity'] <= hi + 1e-3
    t_base = sorted(s['sweep_kernel_time'] / s['total_iterations'] for s in base)[1]
    t_tuned = sorted(s['sweep_kernel_time'] / s['total_iterations'] for s in tuned)[1]
    assert t_tuned <= 1.10 * t_base, (t_tuned, t_base, first['tuned_block_max'],
                                      first['tuned_hub_chunk'])
