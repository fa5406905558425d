"""Fast-mode anchors: the reference's own runMultiPhaseColoring on benchmark-shaped graphs.

Run from the repository root after ``make -C oracle``:

    python tests/golden/make_fast_pins.py [--cases rmat18,rmat20,powerlaw1m] [--threads 1,2,4,8]

Parallel colour-class Louvain depends on the colouring, and the reference's
many-thread colouring is racy, so fast mode has no bit-exact target.  What it
must meet is the final modularity of the reference itself: for each graph
this script runs Grappolo's runMultiPhaseColoring
(Coloring/runMultiPhaseColoring.cpp:51-238, coloring = 1, threshold 1e-6,
C_thresh 1e-4, minGraphSize 1000) built from its sources with its shipped
flags (oracle/_ref/libgrappolo_ref_fast.so) at several OpenMP thread counts,
and with the strict parity build at one thread, and records

  * the printed "Final modularity" (Coloring/runMultiPhaseColoring.cpp:216),
  * the modularity of the returned community array over the input graph
    (the oracle's restated formula; the reference's computeModularity is a stub),
  * phases, iterations, clusters and the printed TOTAL TIME,

in ``fast_pins.json``, with a digest of the generated graph so a test can
check it rebuilt the same input.  The graphs are the seeded generators of
grappolo_b200.graphs at the shapes of the R-MAT and planted power-law
benchmark configurations, scaled down so the one-thread run ends in minutes.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from grappolo_b200 import graphs  # noqa: E402

OUT = os.path.join(HERE, 'fast_pins.json')


def make_graph(name: str):
    """The seeded graph of one anchor case (also used by the GPU tests)."""
    if name.startswith('rmat'):
        return graphs.rmat(int(name[4:]), seed=1)
    if name == 'powerlaw1m':
        return graphs.planted_powerlaw(1_000_000, seed=1)
    raise KeyError(name)


def graph_digest(g) -> str:
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.ptr, dtype='<i8').tobytes())
    h.update(np.ascontiguousarray(g.tail, dtype='<i8').tobytes())
    h.update(np.ascontiguousarray(g.weight, dtype='<f8').tobytes())
    return h.hexdigest()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument('--cases', default='rmat18,rmat20,powerlaw1m')
    ap.add_argument('--threads', default='1,2,4,8')
    args = ap.parse_args()
    from oracle import COracle, Reference
    ref_fast = Reference(fast=True)
    ref_strict = Reference(fast=False)
    orc = COracle()
    pins = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            pins = json.load(f)
    for name in args.cases.split(','):
        g = make_graph(name)
        entry = {'num_vertices': int(g.num_vertices), 'nnz': int(g.nnz),
                 'graph_sha256': graph_digest(g), 'runs': []}
        arms = [('strict', 1)] + [('shipped', int(t)) for t in args.threads.split(',')]
        for build, nt in arms:
            ref = ref_strict if build == 'strict' else ref_fast
            t0 = time.time()
            C, s, _ = ref.run_multiphase_coloring(g, nthreads=nt)
            wall = time.time() - t0
            q = orc.modularity(g, C)
            run = {'build': build, 'threads': nt, 'final_mod_printed': s.get('final_mod'),
                   'q_restated': q, 'phases': s.get('phases'),
                   'total_iterations': s.get('total_iterations'),
                   'final_clusters': s.get('final_clusters'),
                   'total_time_s': s.get('total_time'), 'wall_s': round(wall, 3)}
            entry['runs'].append(run)
            print(name, run, flush=True)
        printed = [r['final_mod_printed'] for r in entry['runs']]
        restated = [r['q_restated'] for r in entry['runs']]
        entry['printed_range'] = [min(printed), max(printed)]
        entry['restated_range'] = [min(restated), max(restated)]
        pins[name] = entry
        with open(OUT, 'w') as f:
            json.dump(pins, f, indent=1)


if __name__ == '__main__':
    main()
