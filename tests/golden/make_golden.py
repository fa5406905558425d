"""Generate the golden fixtures from Grappolo's own code (oracle/_ref, one thread).

Run from the repository root after ``make -C oracle``:

    python tests/golden/make_golden.py [/path/to/grappolo]
    python tests/golden/make_golden.py --vf     # only vf.npz (vertex following)
    python tests/golden/make_golden.py --mhash  # only mhash.npz (coloring = 3)
    python tests/golden/make_golden.py --csr    # only csr_build.npz and karate.bin
    python tests/golden/make_golden.py --compare  # only compare.npz
    python tests/golden/make_golden.py --vbase    # only vbase.npz (coloring = 2)

Each fixture ``<case>.npz`` holds an input CSR and what the reference's
functions return for it at OMP_NUM_THREADS=1: the distance-1 colouring, one
colour phase, one Jacobi phase, renumbering, the next-level graph, the move
decisions of a seeded state, and both multiphase drivers (C_orig plus the
printed summary).  ``pins.json`` records the 100k-vertex planted-partition
run (too large to store) as a digest of C_orig and its summary.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from grappolo_b200 import graphs  # noqa: E402
from oracle import Reference  # noqa: E402


def edge_cases():
    cases = {}
    cases['pair'] = graphs.from_edges(2, [(0, 1)])
    cases['loops_isolated'] = graphs.from_edges(
        9, [(0, 1), (1, 2), (2, 0), (2, 2), (3, 4), (4, 4), (5, 6), (6, 7), (7, 5), (0, 0)],
        weights=[1, 2, 1, 3, 1, 2, 1, 1, 1, 0.5])
    cases['cycle4_ties'] = graphs.from_edges(4, [(0, 1), (1, 2), (2, 3), (3, 0)])
    rng = np.random.default_rng(11)
    # hub of degree 5000 (global-table bin) and one of degree 400 (block bin)
    nv = 5402
    e = [(0, i) for i in range(1, 5001)] + [(5001, 5001 + i) for i in range(1, 401)]
    e += [tuple(x) for x in rng.integers(1, 5001, size=(3000, 2))]
    e += [(0, 5001)]
    cases['hubs'] = graphs.from_edges(nv, e)
    cases['hubs_w'] = graphs.random_weights(cases['hubs'], seed=5)
    return cases


def all_cases(ref_root):
    cases = {}
    cases['karate'] = Reference().load_metis(os.path.join(ref_root, 'karate.graph'))
    cases['pp1000'] = graphs.planted_partition(num_blocks=20, block_size=50, intra_degree=10,
                                               inter_degree=3, seed=2)
    cases['pp1000_w'] = graphs.random_weights(cases['pp1000'], seed=3)
    cases['rmat10'] = graphs.rmat(10, seed=4)
    cases.update(edge_cases())
    return cases


def seeded_state(g, rng):
    """A community state reachable by moves: random merges of neighbours."""
    nv = g.num_vertices
    C = np.arange(nv, dtype=np.int64)
    heads = g.heads()
    pick = rng.random(g.nnz) < 0.3
    for h, t in zip(heads[pick], g.tail[pick]):
        C[t] = C[h]
    vdeg = np.array([g.weight[g.ptr[i]:g.ptr[i + 1]].sum() for i in range(nv)])
    cdeg = np.zeros(nv)
    csize = np.zeros(nv, dtype=np.int64)
    for i in range(nv):
        cdeg[C[i]] += vdeg[i]
        csize[C[i]] += 1
    return C, vdeg, cdeg, csize


def make_case(R, g, rng):
    out = dict(ptr=g.ptr, tail=g.tail, weight=g.weight)
    col, mc, _ = R.color(g)
    out.update(color=col, max_color=mc)
    q, C, itr, _ = R.coloring_phase(g, col, mc + 1, -1.0, 1e-4)
    out.update(cphase_mod=q, cphase_C=C, cphase_itr=itr)
    q, Cb, itr, _ = R.basic_phase(g, -1.0, 1e-6)
    out.update(bphase_mod=q, bphase_C=Cb, bphase_itr=itr)
    Cr, ncl = R.renumber(C)
    out.update(renum_C=Cr, renum_n=ncl)
    cg, ne = R.build_next_level(g, Cr, ncl)
    out.update(coarse_ptr=cg.ptr, coarse_tail=cg.tail, coarse_weight=cg.weight, coarse_ne=ne)
    Cs, vdeg, cdeg, csize = seeded_state(g, rng)
    _, const = R.vertex_degrees(g)
    verts = np.arange(g.num_vertices, dtype=np.int64)
    tg = R.decide_batch(g, Cs, vdeg, cdeg, csize, const, verts)
    out.update(state_C=Cs, state_vdeg=vdeg, state_cdeg=cdeg, state_csize=csize,
               state_const=const, state_targets=tg)
    Co, s, _ = R.run_multiphase_coloring(g, 1000, 1e-6, 1e-4)
    out.update(mpc_C=Co, mpc_phases=s['phases'], mpc_itr=s['total_iterations'],
               mpc_clusters=s['final_clusters'], mpc_mod=s['final_mod'])
    Cb2, s2, _ = R.run_multiphase_basic(g, 1e-6)
    out.update(mpb_C=Cb2, mpb_phases=s2['phases'], mpb_itr=s2['total_iterations'],
               mpb_clusters=s2['final_clusters'], mpb_mod=s2['final_mod'])
    return out


def with_leaves(seed=0):
    """A random core with degree-one leaves, isolated pairs and isolated
    vertices; weights in (0.2, 3.7), so the integer cast of buildNewGraphVF
    matters."""
    rng = np.random.default_rng(seed)
    nv = 300
    e = [tuple(x) for x in rng.integers(0, 200, size=(400, 2))]
    e += [(200 + k, int(rng.integers(0, 200))) for k in range(60)]
    e += [(260 + 2 * k, 261 + 2 * k) for k in range(15)]
    w = rng.uniform(0.2, 3.7, len(e))
    return graphs.from_edges(nv, e, w)


def make_vf(R, ref_root):
    """vf.npz: vertexFollowing, renumbering and buildNewGraphVF at one thread."""
    cases = {k: v for k, v in all_cases(ref_root).items()
             if k in ('karate', 'pp1000_w', 'loops_isolated', 'hubs_w')}
    cases['leaves'] = with_leaves(0)
    out = {}
    for name, g in cases.items():
        C, num = R.vertex_following(g)
        Cr, ncl = R.renumber(C)
        cg, ne = R.build_new_graph_vf(g, Cr, ncl)
        out.update({f'{name}_ptr': g.ptr, f'{name}_tail': g.tail, f'{name}_weight': g.weight,
                    f'{name}_C': C, f'{name}_num': num, f'{name}_renum': Cr, f'{name}_ncl': ncl,
                    f'{name}_cptr': cg.ptr, f'{name}_ctail': cg.tail, f'{name}_cweight': cg.weight,
                    f'{name}_ne': ne})
    np.savez_compressed(os.path.join(HERE, 'vf.npz'), names=np.array(list(cases)), **out)
    print('wrote vf', list(cases))


MHASH_SEED = 1  # srand() seed drawn before each multi-hash call
MHASH_COLORS = (4, 16)


def make_mhash(R, ref_root):
    """mhash.npz: the incomplete multi-hash max/min colouring (coloring = 3)
    alone and inside runMultiPhaseColoring, at one thread, with the C
    library's rand() seeded by srand(MHASH_SEED) before each call.  Inputs are
    those of the <case>.npz fixtures, plus an unweighted 6000-vertex planted
    partition stored here."""
    import ctypes as ct
    libc = ct.CDLL(None)
    cases = {k: v for k, v in all_cases(ref_root).items()
             if k in ('karate', 'pp1000', 'pp1000_w', 'rmat10', 'loops_isolated', 'hubs')}
    cases['pp6k'] = graphs.planted_partition_mixed(6000, 40, 0.3, 8.0, seed=3)
    out = {}
    for name, g in cases.items():
        if name == 'pp6k':  # the others are the inputs of <name>.npz
            out.update({f'{name}_ptr': g.ptr, f'{name}_tail': g.tail.astype(np.int32)})
        for nc in MHASH_COLORS:
            libc.srand(MHASH_SEED)
            col, mc = R.color_mhash(g, nc)
            libc.srand(MHASH_SEED)
            Co, s, _ = R.run_multiphase_coloring(g, 1000, 1e-6, 1e-4, coloring=3, num_colors=nc)
            out.update({f'{name}_{nc}_color': col.astype(np.int16), f'{name}_{nc}_max_color': mc,
                        f'{name}_{nc}_C': Co.astype(np.int32), f'{name}_{nc}_phases': s['phases'],
                        f'{name}_{nc}_itr': s['total_iterations'],
                        f'{name}_{nc}_clusters': s['final_clusters'],
                        f'{name}_{nc}_mod': s['final_mod']})
    np.savez_compressed(os.path.join(HERE, 'mhash.npz'), names=np.array(list(cases)),
                        colors=np.array(MHASH_COLORS), seed=MHASH_SEED, **out)
    print('wrote mhash', list(cases))


def edge_list_cases(seed=17):
    """Edge lists with repeated pairs, pairs listed both ways round and
    self-loops, as raw inputs of removeEdges and the loaders' CSR build.
    Weights are integral (stored as int32)."""
    rng = np.random.default_rng(seed)
    out = {}
    for name, nv, ne, dup, wkind in [('tiny', 10, 60, 0.3, 'id'),
                                     ('mid', 200, 1500, 0.2, 'int'),
                                     ('wide', 1000, 2500, 0.1, 'id')]:
        h = rng.integers(0, nv, ne)
        t = rng.integers(0, nv, ne)
        k = int(ne * dup)
        src, dst = rng.integers(0, ne, k), rng.integers(0, ne, k)
        h[dst], t[dst] = h[src], t[src]
        flip = rng.random(ne) < 0.25
        h, t = np.where(flip, t, h), np.where(flip, h, t)
        # 'id': weight i + 1 names edge i, so every output weight shows which
        # input edge it came from
        w = np.arange(1.0, ne + 1) if wkind == 'id' else rng.integers(1, 6, ne) * 1.0
        out[name] = (nv, h.astype(np.int64), t.astype(np.int64), w)
    return out


def make_csr(R, ref_root):
    """csr_build.npz: removeEdges, SortEdgesUndirected and SortNodeEdgesByIndex
    of the reference on raw edge lists; karate.bin: karate written by the
    reference's writeGraphBinaryFormatNew."""
    out = {}
    cases = edge_list_cases()
    for name, (nv, h, t, w) in cases.items():
        rh, rt, rw, nge = R.remove_edges(nv, h, t, w)
        ptrs, sh, st, sw = R.sort_edges_undirected(nv, rh[:nge], rt[:nge], rw[:nge])
        oh, ot, ow = R.sort_node_edges(nv, ptrs, sh, st, sw)
        rptrs, _, rawt, raww = R.sort_edges_undirected(nv, h, t, w)
        i32 = lambda a: np.asarray(a).astype(np.int32)  # noqa: E731
        out.update({f'{name}_nv': nv, f'{name}_head': i32(h), f'{name}_tail': i32(t),
                    f'{name}_weight': i32(w), f'{name}_rm_head': i32(rh),
                    f'{name}_rm_tail': i32(rt), f'{name}_rm_weight': i32(rw), f'{name}_nge': nge,
                    f'{name}_ptrs': ptrs, f'{name}_rows_tail': i32(st),
                    f'{name}_rows_weight': i32(sw), f'{name}_sorted_tail': i32(ot),
                    f'{name}_sorted_weight': i32(ow), f'{name}_raw_ptrs': rptrs,
                    f'{name}_raw_tail': i32(rawt), f'{name}_raw_weight': i32(raww)})
    np.savez_compressed(os.path.join(HERE, 'csr_build.npz'), names=np.array(list(cases)), **out)
    g = all_cases(ref_root)['karate']
    R.write_binary(g, os.path.join(HERE, 'karate.bin'))
    print('wrote csr_build', list(cases), 'and karate.bin')


def comparison_cases(ref_root):
    """(truth, output) label pairs: planted blocks against the reference's
    own Louvain result, and random labellings with -1 entries, 0- and
    1-based ids."""
    z = np.load(os.path.join(HERE, 'pp1000.npz'))
    out = {'pp1000': (np.arange(1000) // 50, z['mpc_C'])}
    rng = np.random.default_rng(23)
    for name, n, k1, k2, b1, b2, m1, m2 in [('rand0', 3000, 40, 25, 0, 0, 0, 0),
                                             ('rand_neg', 4000, 60, 30, 1, 0, 40, 25),
                                             ('rand_one', 2500, 7, 300, 1, 1, 5, 50)]:
        C1 = rng.integers(0, k1, n) + b1
        C2 = rng.integers(0, k2, n) + b2
        C1[rng.integers(0, n, m1)] = -1
        C2[rng.integers(0, n, m2)] = -1
        out[name] = (C1, C2)
    return out


def make_compare(R, ref_root):
    """compare.npz: computeCommunityComparisons (printed statistics and the
    relabelled arrays) and computeGiniCoefficient of the reference."""
    out = {}
    cases = comparison_cases(ref_root)
    for name, (C1, C2) in cases.items():
        st, a, b = R.compare(C1, C2)
        out.update({f'{name}_C1': C1.astype(np.int32), f'{name}_C2': C2.astype(np.int32),
                    f'{name}_C1_after': a.astype(np.int32), f'{name}_C2_after': b.astype(np.int32)})
        out.update({f'{name}_{k}': v for k, v in st.items()})
    rng = np.random.default_rng(29)
    sizes = [rng.integers(0, 1000, 77), np.array([5]), rng.integers(0, 3, 500),
             np.arange(1, 4097)]
    for k, sz in enumerate(sizes):
        g, srt = R.gini(sz)
        out.update({f'gini{k}_sizes': sz, f'gini{k}_value': g, f'gini{k}_sorted': srt})
    np.savez_compressed(os.path.join(HERE, 'compare.npz'), names=np.array(list(cases)),
                        ngini=len(sizes), **out)
    print('wrote compare', list(cases))


def stars_and_clique(nv, nstars, clique, seed, paths=0, weighted=False):
    """Stars of 2-11 leaves and paths of 3-7 vertices on randomly permuted ids,
    isolated vertices, and a clique on the `clique` highest ids.  The clique
    sets the colour count; only colour 0 (the isolated vertices) is
    oversized, and the clique's colour-0 member comes last in vertex order, so
    a colour qualifies for every vertex vBaseRedistribution moves and its
    first-fit scan (Coloring/vBase.cpp:113-116) stays inside its arrays."""
    rng = np.random.default_rng(seed)
    e, v = [], 0
    for _ in range(nstars):
        k = int(rng.integers(2, 12))
        e += [(v, v + j) for j in range(1, k + 1)]
        v += k + 1
    for _ in range(paths):
        k = int(rng.integers(3, 8))
        e += [(v + j, v + j + 1) for j in range(k - 1)]
        v += k
    assert v <= nv - clique
    perm = rng.permutation(nv - clique)
    e = [(int(perm[a]), int(perm[b])) for a, b in e]
    c0 = nv - clique
    e += [(c0 + a, c0 + b) for a in range(clique) for b in range(a + 1, clique)]
    g = graphs.from_edges(nv, e)
    return graphs.random_weights(g, seed=seed) if weighted else g


def vbase_cases(ref_root):
    """(graph, types stored for the single call, multiphase stored) per case."""
    cases = {
        'pp1000': (all_cases(ref_root)['pp1000'], (1,), False),
        'rmat12': (graphs.rmat(12, seed=4), (1,), False),
        'star': (graphs.from_edges(60, [(0, i) for i in range(1, 60)] + [(1, 2), (3, 4)]),
                 (1,), False),
    }
    for nv, ns, kc, paths, seed in [(3000, 60, 10, 0, 0), (6000, 200, 12, 20, 1),
                                    (12000, 400, 16, 50, 2), (30000, 800, 20, 100, 1)]:
        cases[f'sc{nv}'] = (stars_and_clique(nv, ns, kc, seed, paths, weighted=seed == 1),
                            (0, 1), True)
    return cases


def make_vbase(ref_root):
    """vbase.npz: vBaseRedistribution (Coloring/vBase.cpp:6-168) and the
    coloring = 2 multiphase run (runMultiPhaseColoring.cpp:67-74,180-186) of
    the reference built with the function's missing return added
    (oracle/ref_vbase.cpp), one thread.  The input colouring is the
    reference's distance-1 colouring.  Type 0 and the multiphase run (which
    calls type 0) are stored only where the oracle finds a qualifying colour
    for every vertex that moves: elsewhere the reference reads past its
    frequency array and its result is not defined."""
    from oracle import COracle
    R = Reference(patched_vbase=True)
    O = COracle()
    out, names = {}, []
    for name, (g, types, mp) in vbase_cases(ref_root).items():
        col, mc, _ = R.color(g)
        nc = mc + 1
        out.update({f'{name}_ptr': g.ptr, f'{name}_tail': g.tail.astype(np.int32),
                    f'{name}_color': col.astype(np.int32), f'{name}_ncolors': nc})
        if mp:  # the single call reads no weights
            out[f'{name}_weight'] = g.weight
        for t in types:
            if t == 0:
                assert O.vbase(g, col, nc, 0)[2] == 0, name
            out[f'{name}_t{t}'] = R.vbase(g, col, nc, t)
        out[f'{name}_types'] = np.array(types)
        if mp:
            _, so, _ = O.run_multiphase_coloring(g, coloring=2)
            assert so['vbase_stuck'] == 0, name
            C, s, _ = R.run_multiphase_coloring(g, coloring=2)
            out.update({f'{name}_mp_C': C, f'{name}_mp_phases': s['phases'],
                        f'{name}_mp_itr': s['total_iterations'],
                        f'{name}_mp_clusters': s['final_clusters'],
                        f'{name}_mp_mod': s['final_mod']})
        names.append(name)
        print('vbase', name, g.num_vertices, g.nnz, 'colours', nc, 'types', types, 'multiphase', mp)
    np.savez_compressed(os.path.join(HERE, 'vbase.npz'), names=np.array(names), **out)


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 and not sys.argv[1].startswith('--') \
        else os.environ.get('GRAPPOLO_REFERENCE', '/root/reference')
    R = Reference()
    if '--vf' in sys.argv:
        make_vf(R, ref_root)
        return
    if '--mhash' in sys.argv:
        make_mhash(R, ref_root)
        return
    if '--csr' in sys.argv:
        make_csr(R, ref_root)
        return
    if '--compare' in sys.argv:
        make_compare(R, ref_root)
        return
    if '--vbase' in sys.argv:
        make_vbase(ref_root)
        return
    rng = np.random.default_rng(2024)
    for name, g in all_cases(ref_root).items():
        np.savez_compressed(os.path.join(HERE, f'{name}.npz'), **make_case(R, g, rng))
        print('wrote', name, g.num_vertices, g.nnz)
    pins = {}
    for name, g in [('planted_100k', graphs.planted_partition()),
                    ('planted_100k_w', graphs.random_weights(graphs.planted_partition()))]:
        Co, s, _ = R.run_multiphase_coloring(g, 1000, 1e-6, 1e-4)
        pins[name] = dict(c_orig_sha256=hashlib.sha256(Co.astype('<i8').tobytes()).hexdigest(),
                          phases=s['phases'], total_iterations=s['total_iterations'],
                          final_clusters=s['final_clusters'], final_mod=s['final_mod'],
                          colors=s['colors_per_phase'], clusters=s['clusters_per_phase'])
        print('pinned', name, pins[name])
    with open(os.path.join(HERE, 'pins.json'), 'w') as f:
        json.dump(pins, f, indent=1)


if __name__ == '__main__':
    main()
