"""Fast and learned mode against the reference's own modularity at benchmark shape.

Fast mode is not bit-exact (its colouring and accumulation are parallel, as
the reference's are on many threads), so its bar is the final modularity of
the reference itself: within 1e-3 (absolute) of what Grappolo's
runMultiPhaseColoring (Coloring/runMultiPhaseColoring.cpp:51-238, printed at
:216) reaches on the same graph.  The reference's many-thread result moves
with the thread count, so the anchor is the range it covers at 1, 2, 4 and 8
OpenMP threads (tests/golden/fast_pins.json, made by make_fast_pins.py from
the reference compiled from its sources), widened by a run of the reference
at all host cores made here on the smallest graph.

Graphs: R-MAT scale 18 and 20 (the R-MAT benchmark's generator, a/b/c =
0.57/0.19/0.19, edge factor 16, FP64 weights in (0, 1]) and the planted
power-law graph at 1M vertices (the learned-vs-plain benchmark's generator).
"""
import json
import os
import sys

import numpy as np
import pytest

from grappolo_b200 import _lib, gate, louvain

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, 'golden'))
from make_fast_pins import graph_digest, make_graph  # noqa: E402

FAST_Q_TOL = 1e-3  # |Q_gpu - Q_reference| (absolute), against the reference's thread range
MODES = {'fast': _lib.GLV_MODE_FAST, 'learned': _lib.GLV_MODE_LEARNED}


def _pins():
    with open(os.path.join(HERE, 'golden', 'fast_pins.json')) as f:
        return json.load(f)


_graphs = {}


def _graph(name):
    if name not in _graphs:
        _graphs.clear()  # one graph at a time (the 1M-vertex cases hold ~1 GB)
        g = make_graph(name)
        assert graph_digest(g) == _pins()[name]['graph_sha256'], 'generator output changed'
        _graphs[name] = g
    return _graphs[name]


def _within(q, lo, hi):
    return lo - FAST_Q_TOL <= q <= hi + FAST_Q_TOL


CASES = [('rmat18', 'fast'), ('rmat18', 'learned'), ('rmat20', 'fast'), ('rmat20', 'learned'),
         ('powerlaw1m', 'fast'), ('powerlaw1m', 'learned')]


@pytest.mark.parametrize('name,mode', CASES)
def test_final_modularity_within_reference_range(name, mode, oracle):
    pin = _pins()[name]
    g = _graph(name)
    if mode == 'learned':
        params, tau = gate.load_default()  # the shipped, GPU-trained network
        gate.set_gate(params, tau)
    C, st = louvain.run_multiphase_csr(g, coloring=True, mode=MODES[mode])
    lo, hi = pin['printed_range']
    q = st['final_modularity']
    assert _within(q, lo, hi), (name, mode, q, lo, hi)
    # isolated vertices belong to no community (Coloring/runMultiPhaseColoring.cpp:141)
    deg = np.diff(g.ptr)
    assert np.all(C[deg == 0] == -1) and np.all(C[deg > 0] >= 0)
    # the modularity of the returned community array over the input graph,
    # against the same quantity of the reference's runs
    q_c = oracle.modularity(g, C)
    lo, hi = pin['restated_range']
    assert _within(q_c, lo, hi), (name, mode, q_c, lo, hi)


def test_rmat18_against_reference_at_all_host_cores(oracle):
    """The reference run here, on every host core, as a further anchor."""
    from oracle import Reference
    g = _graph('rmat18')
    pin = _pins()['rmat18']
    nt = os.cpu_count() or 1
    C_ref, s_ref, _ = Reference(fast=True).run_multiphase_coloring(g, nthreads=nt)
    lo = min(pin['printed_range'][0], s_ref['final_mod'])
    hi = max(pin['printed_range'][1], s_ref['final_mod'])
    _, st = louvain.run_multiphase_csr(g, coloring=True, mode=_lib.GLV_MODE_FAST)
    assert _within(st['final_modularity'], lo, hi), (st['final_modularity'], lo, hi, nt)
    assert np.all(C_ref >= -1)
