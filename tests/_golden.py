"""Loading the golden fixtures made by tests/golden/make_golden.py."""
import json
import os

import numpy as np

from grappolo_b200.graphs import CSRGraph

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
CASES = ['karate', 'pp1000', 'pp1000_w', 'rmat10', 'pair', 'loops_isolated', 'cycle4_ties',
         'hubs', 'hubs_w']


def load(name):
    z = dict(np.load(os.path.join(GOLDEN, f'{name}.npz')))
    g = CSRGraph(z['ptr'], z['tail'], z['weight'])
    return g, z


def pins():
    with open(os.path.join(GOLDEN, 'pins.json')) as f:
        return json.load(f)


def mhash_cases():
    """(name, graph, numColors, expected) for every case of mhash.npz: the
    incomplete colouring (coloring = 3) of the reference at one thread, its
    rand() seeded by srand(seed) before each call."""
    z = np.load(os.path.join(GOLDEN, 'mhash.npz'))
    seed = int(z['seed'])
    out = []
    for name in map(str, z['names']):
        if f'{name}_ptr' in z.files:
            g = CSRGraph(z[f'{name}_ptr'], z[f'{name}_tail'].astype(np.int64),
                         np.ones(len(z[f'{name}_tail'])))
        else:
            g, _ = load(name)
        for nc in map(int, z['colors']):
            p = f'{name}_{nc}_'
            exp = {k[len(p):]: z[k] for k in z.files if k.startswith(p)}
            exp['seed'] = seed
            out.append((f'{name}-{nc}', g, nc, exp))
    return out


def srand(seed):
    """Seed the C library's rand(), which the multi-hash colouring draws from."""
    import ctypes as ct
    ct.CDLL(None).srand(seed)


def csr_cases():
    """(name, expected) for every edge list of csr_build.npz: the reference's
    removeEdges, SortEdgesUndirected and SortNodeEdgesByIndex outputs."""
    z = np.load(os.path.join(GOLDEN, 'csr_build.npz'))
    out = []
    for name in map(str, z['names']):
        p = f'{name}_'
        exp = {k[len(p):]: z[k] for k in z.files if k.startswith(p)}
        for k in list(exp):
            if exp[k].dtype == np.int32:
                exp[k] = exp[k].astype(np.float64 if k.endswith('weight') else np.int64)
        exp['nv'] = int(exp['nv'])
        exp['nge'] = int(exp['nge'])
        out.append((name, exp))
    return out


def compare_cases():
    """(name, C1, C2, expected) of compare.npz (computeCommunityComparisons
    as the reference printed it, and the arrays it left relabelled)."""
    z = np.load(os.path.join(GOLDEN, 'compare.npz'))
    out = []
    for name in map(str, z['names']):
        p = f'{name}_'
        exp = {k[len(p):]: z[k] for k in z.files if k.startswith(p)}
        out.append((name, exp.pop('C1').astype(np.int64), exp.pop('C2').astype(np.int64), exp))
    return out


def gini_cases():
    z = np.load(os.path.join(GOLDEN, 'compare.npz'))
    return [(z[f'gini{k}_sizes'], float(z[f'gini{k}_value']), z[f'gini{k}_sorted'])
            for k in range(int(z['ngini']))]


COMPARE_INTS = ('same_same', 'same_diff', 'diff_same', 'num_communities1', 'num_communities2')
COMPARE_FLOATS = ('precision', 'recall', 'f_score', 'gini1', 'gini2')


def vbase_cases():
    """(name, graph, input colouring, colour count, {type: expected colours},
    expected multiphase run or None) for every case of vbase.npz: the
    reference's vBaseRedistribution and its coloring = 2 multiphase run, one
    thread, built with the function's missing return added."""
    z = np.load(os.path.join(GOLDEN, 'vbase.npz'))
    out = []
    for name in map(str, z['names']):
        tail = z[f'{name}_tail'].astype(np.int64)
        w = z[f'{name}_weight'] if f'{name}_weight' in z.files else np.ones(len(tail))
        g = CSRGraph(z[f'{name}_ptr'], tail, w)
        exp = {int(t): z[f'{name}_t{t}'] for t in z[f'{name}_types']}
        mp = None
        if f'{name}_mp_C' in z.files:
            mp = dict(C=z[f'{name}_mp_C'], phases=int(z[f'{name}_mp_phases']),
                      total_iterations=int(z[f'{name}_mp_itr']),
                      final_clusters=int(z[f'{name}_mp_clusters']),
                      final_mod=float(z[f'{name}_mp_mod']))
        out.append((name, g, z[f'{name}_color'], int(z[f'{name}_ncolors']), exp, mp))
    return out
