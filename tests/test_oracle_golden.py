"""The C oracle against the golden fixtures generated by the reference itself."""
import hashlib
import os

import numpy as np
import pytest

from grappolo_b200 import graphs
from _golden import (CASES, COMPARE_FLOATS, COMPARE_INTS, compare_cases, csr_cases, gini_cases,
                     load, mhash_cases, pins, srand)


@pytest.mark.parametrize('name', CASES)
def test_coloring(oracle, name):
    g, z = load(name)
    col, mc = oracle.color_greedy(g)
    assert mc == z['max_color']
    assert np.array_equal(col, z['color'])


@pytest.mark.parametrize('name', CASES)
def test_coloring_phase(oracle, name):
    g, z = load(name)
    q, C, itr, _ = oracle.coloring_phase(g, z['color'], int(z['max_color']) + 1, -1.0, 1e-4)
    assert itr == z['cphase_itr']
    assert q == z['cphase_mod']
    assert np.array_equal(C, z['cphase_C'])


@pytest.mark.parametrize('name', CASES)
def test_basic_phase(oracle, name):
    g, z = load(name)
    q, C, itr, _ = oracle.basic_phase(g, -1.0, 1e-6)
    assert itr == z['bphase_itr']
    assert q == z['bphase_mod']
    assert np.array_equal(C, z['bphase_C'])


@pytest.mark.parametrize('name', CASES)
def test_renumber_and_coarsen(oracle, name):
    g, z = load(name)
    Cr, n = oracle.renumber(z['cphase_C'])
    assert n == z['renum_n']
    assert np.array_equal(Cr, z['renum_C'])
    cg, ne = oracle.build_next_level(g, Cr, n)
    assert ne == z['coarse_ne']
    assert np.array_equal(cg.ptr, z['coarse_ptr'])
    assert np.array_equal(cg.tail, z['coarse_tail'])
    assert np.array_equal(cg.weight, z['coarse_weight'])  # bit-exact FP64


@pytest.mark.parametrize('name', CASES)
def test_decisions(oracle, name):
    g, z = load(name)
    verts = np.arange(g.num_vertices)
    tg = oracle.decide_batch(g, z['state_C'], z['state_vdeg'], z['state_cdeg'], z['state_csize'],
                             float(z['state_const']), verts)
    assert np.array_equal(tg, z['state_targets'])


@pytest.mark.parametrize('name', CASES)
def test_multiphase(oracle, name):
    g, z = load(name)
    C, s, _ = oracle.run_multiphase_coloring(g, 1000, 1e-6, 1e-4)
    assert np.array_equal(C, z['mpc_C'])
    assert (s['phases'], s['total_iterations'], s['final_clusters']) == \
        (z['mpc_phases'], z['mpc_itr'], z['mpc_clusters'])
    assert abs(s['final_mod'] - z['mpc_mod']) <= 5e-7  # printed with %lf
    C, s, _ = oracle.run_multiphase_basic(g, 1e-6)
    assert np.array_equal(C, z['mpb_C'])
    assert (s['phases'], s['total_iterations'], s['final_clusters']) == \
        (z['mpb_phases'], z['mpb_itr'], z['mpb_clusters'])
    assert abs(s['final_mod'] - z['mpb_mod']) <= 5e-7


@pytest.mark.parametrize('name', ['planted_100k', 'planted_100k_w'])
def test_pinned_100k(oracle, name):
    g = graphs.planted_partition()
    if name.endswith('_w'):
        g = graphs.random_weights(g)
    pin = pins()[name]
    C, s, recs = oracle.run_multiphase_coloring(g, 1000, 1e-6, 1e-4)
    assert hashlib.sha256(C.astype('<i8').tobytes()).hexdigest() == pin['c_orig_sha256']
    assert s['phases'] == pin['phases'] and s['total_iterations'] == pin['total_iterations']
    assert s['final_clusters'] == pin['final_clusters']
    assert abs(s['final_mod'] - pin['final_mod']) <= 5e-7
    assert [r.num_colors for r in recs if r.colored] == pin['colors']
    assert [r.clusters for r in recs] == pin['clusters']


def _vf_cases():
    z = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'vf.npz'))
    for name in z['names']:
        name = str(name)
        g = graphs.CSRGraph(z[f'{name}_ptr'], z[f'{name}_tail'], z[f'{name}_weight'])
        yield name, g, {k[len(name) + 1:]: z[k] for k in z.files if k.startswith(name + '_')}


@pytest.mark.parametrize('name,g,ref', list(_vf_cases()), ids=lambda x: x if isinstance(x, str) else '')
def test_vertex_following_golden(oracle, name, g, ref):
    """Utility/vertexFollowing.cpp at one thread: follow map, count, and the
    vertex-following graph (integer-cast weights, no zero self-loops)."""
    C, n = oracle.vertex_following(g)
    assert n == int(ref['num']) and np.array_equal(C, ref['C'])
    cg, ne = oracle.build_new_graph_vf(g, ref['renum'], int(ref['ncl']))
    assert ne == int(ref['ne'])
    assert np.array_equal(cg.ptr, ref['cptr']) and np.array_equal(cg.tail, ref['ctail'])
    assert np.array_equal(cg.weight, ref['cweight'])


@pytest.mark.parametrize('case', mhash_cases(), ids=lambda c: c[0])
def test_multihash_coloring_golden(oracle, case):
    """Coloring/coloringMultiHashMaxMin.cpp at one thread: colours, maxColor."""
    _, g, nc, exp = case
    srand(exp['seed'])
    col, mc = oracle.color_mhash(g, nc)
    assert mc == int(exp['max_color'])
    assert np.array_equal(col, exp['color'])


@pytest.mark.parametrize('case', mhash_cases(), ids=lambda c: c[0])
def test_multiphase_multihash_golden(oracle, case):
    """runMultiPhaseColoring with coloring = 3: C_orig and the summary."""
    _, g, nc, exp = case
    srand(exp['seed'])
    C, s, _ = oracle.run_multiphase_coloring(g, coloring=3, num_colors=nc)
    assert np.array_equal(C, exp['C'])
    assert s['phases'] == int(exp['phases'])
    assert s['total_iterations'] == int(exp['itr'])
    assert s['final_clusters'] == int(exp['clusters'])
    assert abs(s['final_mod'] - float(exp['mod'])) <= 5e-7  # the reference prints %lf


@pytest.mark.parametrize('case', csr_cases(), ids=lambda c: c[0])
def test_edge_list_preprocessing_golden(oracle, case):
    """removeEdges, SortEdgesUndirected and SortNodeEdgesByIndex
    (Utility/utilityFunctions.cpp:416-531) on raw edge lists."""
    _, e = case
    nv = e['nv']
    h, t, w, nge = oracle.remove_edges(nv, e['head'], e['tail'], e['weight'])
    assert nge == e['nge']
    assert np.array_equal(h, e['rm_head']) and np.array_equal(t, e['rm_tail'])
    assert np.array_equal(w, e['rm_weight'])
    ptrs, sh, st, sw = oracle.sort_edges_undirected(nv, h[:nge], t[:nge], w[:nge])
    assert np.array_equal(ptrs, e['ptrs'])
    assert np.array_equal(st, e['rows_tail']) and np.array_equal(sw, e['rows_weight'])
    _, ot, ow = oracle.sort_node_edges(nv, ptrs, sh, st, sw)
    assert np.array_equal(ot, e['sorted_tail']) and np.array_equal(ow, e['sorted_weight'])
    rp, _, rt, rw = oracle.sort_edges_undirected(nv, e['head'], e['tail'], e['weight'])
    assert np.array_equal(rp, e['raw_ptrs'])
    assert np.array_equal(rt, e['raw_tail']) and np.array_equal(rw, e['raw_weight'])


def test_binary_file_golden(tmp_path):
    """karate.bin was written by the reference's writeGraphBinaryFormatNew:
    the Python reader gets karate back and the writer gives the same bytes."""
    path = os.path.join(os.path.dirname(__file__), 'golden', 'karate.bin')
    g, z = load('karate')
    r = graphs.read_binary(path)
    assert np.array_equal(r.ptr, z['ptr']) and np.array_equal(r.tail, z['tail'])
    assert np.array_equal(r.weight, z['weight'])
    out = tmp_path / 'k.bin'
    graphs.write_binary(g, str(out))
    assert out.read_bytes() == open(path, 'rb').read()


@pytest.mark.parametrize('case', compare_cases(), ids=lambda c: c[0])
def test_community_comparison_golden(oracle, case):
    """computeCommunityComparisons: pair counts exact, rates to the printed
    six decimals, the relabelled arrays as the reference leaves them."""
    _, C1, C2, exp = case
    st, a, b = oracle.compare(C1, C2)
    for k in COMPARE_INTS:
        assert st[k] == int(exp[k]), k
    for k in COMPARE_FLOATS:
        assert abs(st[k] - float(exp[k])) <= 5e-7, k
    assert np.array_equal(a, exp['C1_after']) and np.array_equal(b, exp['C2_after'])


@pytest.mark.parametrize('k', range(4))
def test_gini_golden(oracle, k):
    sizes, value, srt = gini_cases()[k]
    g, s = oracle.gini(sizes)
    assert g == value and np.array_equal(s, srt)


def test_colour_count_is_checked(oracle):
    """color_greedy returns the largest colour; a colouring phase or a
    redistribution given that as the colour count is refused before the C
    routines index their per-colour arrays with it."""
    g, _ = load('karate')
    col, mc = oracle.color_greedy(g)
    with pytest.raises(ValueError):
        oracle.coloring_phase(g, col, mc)
    with pytest.raises(ValueError):
        oracle.vbase(g, col, mc)
    q, C, itr, _ = oracle.coloring_phase(g, col, mc + 1)
    assert itr >= 1 and C.shape == (g.num_vertices,)
