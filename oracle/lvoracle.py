"""ctypes wrappers for the two CPU checkers (test infrastructure only)."""
from __future__ import annotations

import ctypes as ct
import dataclasses
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_c_long_p = ct.POINTER(ct.c_long)
_c_double_p = ct.POINTER(ct.c_double)
_c_int_p = ct.POINTER(ct.c_int)


def build(ref: str | None = None) -> None:
    """Compile liblvoracle.so and, when the reference tree is present, _ref/."""
    cmd = ['make', '-s', '-C', HERE, '-j8', 'all']
    if ref:
        cmd.append(f'REF={ref}')
    subprocess.run(cmd, check=True)


def _lp(a: np.ndarray):
    return a.ctypes.data_as(_c_long_p)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_c_double_p)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(_c_int_p)


def _csr(g):
    return (np.ascontiguousarray(g.ptr, dtype=np.int64),
            np.ascontiguousarray(g.tail, dtype=np.int64),
            np.ascontiguousarray(g.weight, dtype=np.float64))


class _PhaseC(ct.Structure):
    _fields_ = [('nv', ct.c_long), ('nnz', ct.c_long), ('colored', ct.c_int),
                ('recolored', ct.c_int), ('num_colors', ct.c_int), ('iterations', ct.c_int),
                ('mod', ct.c_double), ('clusters', ct.c_long)]


class _SummaryC(ct.Structure):
    _fields_ = [('phases', ct.c_int), ('total_iterations', ct.c_int),
                ('final_clusters', ct.c_long), ('final_mod', ct.c_double), ('nrec', ct.c_int)]


@dataclasses.dataclass
class PhaseRecord:
    nv: int
    nnz: int
    colored: bool
    recolored: bool
    num_colors: int
    iterations: int
    mod: float
    clusters: int


class COracle:
    """The C restatement of the reference's one-thread semantics."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, 'liblvoracle.so')
        if not os.path.exists(path):
            build()
        L = ct.CDLL(path)
        self.L = L
        L.lvo_vertex_degrees.restype = ct.c_double
        L.lvo_color_greedy.restype = ct.c_int
        L.lvo_color_mhash.restype = ct.c_int
        L.lvo_vbase.restype = ct.c_long
        L.lvo_last_vbase_stuck.restype = ct.c_long
        L.lvo_gini.restype = ct.c_double
        L.lvo_compare_communities.restype = ct.c_int
        L.lvo_remove_edges.restype = ct.c_long
        L.lvo_coloring_phase.restype = ct.c_double
        L.lvo_basic_phase.restype = ct.c_double
        L.lvo_renumber.restype = ct.c_long
        L.lvo_build_next_level.restype = ct.c_long
        L.lvo_vertex_following.restype = ct.c_long
        L.lvo_build_new_graph_vf.restype = ct.c_long
        L.lvo_modularity.restype = ct.c_double
        L.lvo_run_multiphase_coloring.restype = ct.c_int
        L.lvo_run_multiphase_basic.restype = ct.c_int

    def vertex_degrees(self, g):
        p, t, w = _csr(g)
        vd = np.zeros(g.num_vertices)
        c = self.L.lvo_vertex_degrees(ct.c_long(g.num_vertices), _lp(p), _dp(w), _dp(vd))
        return vd, c

    def color_greedy(self, g):
        p, t, w = _csr(g)
        col = np.full(g.num_vertices, -1, dtype=np.int32)
        mc = self.L.lvo_color_greedy(ct.c_long(g.num_vertices), _lp(p), _lp(t), _ip(col))
        return col, mc

    def coloring_phase(self, g, colors, num_colors, lower=-1.0, thresh=1e-4, trace_cap=256):
        p, t, w = _csr(g)
        C = np.zeros(g.num_vertices, dtype=np.int64)
        col = np.ascontiguousarray(colors, dtype=np.int32)
        # the C routine sizes its per-colour arrays by num_colors (one more
        # than the largest colour, as color_greedy's second result is the
        # largest colour): check before it writes past them
        if col.size and (col.min() < 0 or col.max() >= num_colors):
            raise ValueError('colours must lie in [0, num_colors)')
        itr = ct.c_int(0)
        tq = np.zeros(trace_cap)
        q = self.L.lvo_coloring_phase(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                      _ip(col), ct.c_int(num_colors), ct.c_double(lower),
                                      ct.c_double(thresh), ct.byref(itr), _dp(tq),
                                      ct.c_int(trace_cap))
        return q, C, itr.value, tq[:min(itr.value, trace_cap)].copy()

    def basic_phase(self, g, lower=-1.0, thresh=1e-6, trace_cap=256):
        p, t, w = _csr(g)
        C = np.zeros(g.num_vertices, dtype=np.int64)
        itr = ct.c_int(0)
        tq = np.zeros(trace_cap)
        q = self.L.lvo_basic_phase(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                   ct.c_double(lower), ct.c_double(thresh), ct.byref(itr),
                                   _dp(tq), ct.c_int(trace_cap))
        return q, C, itr.value, tq[:min(itr.value, trace_cap)].copy()

    def renumber(self, C):
        C = np.array(C, dtype=np.int64, copy=True)
        n = self.L.lvo_renumber(_lp(C), ct.c_long(C.shape[0]))
        return C, n

    def build_next_level(self, g, C, ncl):
        from grappolo_b200.graphs import CSRGraph
        p, t, w = _csr(g)
        C = np.ascontiguousarray(C, dtype=np.int64)
        op, ot, ow = _c_long_p(), _c_long_p(), _c_double_p()
        ne = ct.c_long(0)
        onnz = self.L.lvo_build_next_level(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w),
                                           _lp(C), ct.c_long(ncl), ct.byref(op), ct.byref(ot),
                                           ct.byref(ow), ct.byref(ne))
        out = CSRGraph(np.ctypeslib.as_array(op, (ncl + 1,)).copy(),
                       np.ctypeslib.as_array(ot, (max(onnz, 1),))[:onnz].copy(),
                       np.ctypeslib.as_array(ow, (max(onnz, 1),))[:onnz].copy())
        for a in (op, ot, ow):
            self.L.lvo_free(a)
        return out, ne.value

    def vertex_following(self, g):
        """(C, numVtxToFix) of Utility/vertexFollowing.cpp:46 (restated)."""
        p, t, _ = _csr(g)
        C = np.empty(g.num_vertices, dtype=np.int64)
        n = self.L.lvo_vertex_following(ct.c_long(g.num_vertices), _lp(p), _lp(t), _lp(C))
        return C, n

    def build_new_graph_vf(self, g, C, ncl):
        """(CSRGraph, numEdges) of Utility/vertexFollowing.cpp:91 (restated)."""
        from grappolo_b200.graphs import CSRGraph
        p, t, w = _csr(g)
        C = np.ascontiguousarray(C, dtype=np.int64)
        op, ot, ow = _c_long_p(), _c_long_p(), _c_double_p()
        ne = ct.c_long(0)
        onnz = self.L.lvo_build_new_graph_vf(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w),
                                             _lp(C), ct.c_long(ncl), ct.byref(op), ct.byref(ot),
                                             ct.byref(ow), ct.byref(ne))
        out = CSRGraph(np.ctypeslib.as_array(op, (ncl + 1,)).copy(),
                       np.ctypeslib.as_array(ot, (max(onnz, 1),))[:onnz].copy(),
                       np.ctypeslib.as_array(ow, (max(onnz, 1),))[:onnz].copy())
        for a in (op, ot, ow):
            self.L.lvo_free(a)
        return out, ne.value

    def remove_edges(self, nv, head, tail, w):
        """removeEdges on copies of the SoA arrays: (head, tail, w, NGE)."""
        h, t = np.array(head, dtype=np.int64), np.array(tail, dtype=np.int64)
        ww = np.array(w, dtype=np.float64)
        n = self.L.lvo_remove_edges(ct.c_long(nv), ct.c_long(len(h)), _lp(h), _lp(t), _dp(ww))
        return h, t, ww, n

    def sort_edges_undirected(self, nv, head, tail, w):
        """SortEdgesUndirected: (ptrs[NV+2], head, tail, w) of the 2*NE entries."""
        h, t = np.ascontiguousarray(head, dtype=np.int64), np.ascontiguousarray(tail, dtype=np.int64)
        ww = np.ascontiguousarray(w, dtype=np.float64)
        ne = len(h)
        ptrs = np.zeros(nv + 2, dtype=np.int64)
        oh, ot = np.zeros(2 * ne, dtype=np.int64), np.zeros(2 * ne, dtype=np.int64)
        ow = np.zeros(2 * ne)
        self.L.lvo_sort_edges_undirected(ct.c_long(nv), ct.c_long(ne), _lp(h), _lp(t), _dp(ww),
                                             _lp(ptrs), _lp(oh), _lp(ot), _dp(ow))
        return ptrs, oh, ot, ow

    def sort_node_edges(self, nv, ptrs, head, tail, w):
        """SortNodeEdgesByIndex on copies: (head, tail, w)."""
        p = np.ascontiguousarray(ptrs, dtype=np.int64)
        h, t = np.array(head, dtype=np.int64), np.array(tail, dtype=np.int64)
        ww = np.array(w, dtype=np.float64)
        self.L.lvo_sort_node_edges(ct.c_long(nv), _lp(p), _lp(h), _lp(t), _dp(ww))
        return h, t, ww

    def compare(self, C1, C2):
        """computeCommunityComparisons on copies: (stats dict, C1', C2')."""
        a, b = np.array(C1, dtype=np.int64), np.array(C2, dtype=np.int64)
        res, dres = np.zeros(5, dtype=np.int64), np.zeros(5)
        rc = self.L.lvo_compare_communities(_lp(a), _lp(b), ct.c_long(len(a)), _lp(res),
                                            _dp(dres))
        if rc != 0:
            raise ValueError('a community id below -1')
        return dict(same_same=int(res[0]), same_diff=int(res[1]), diff_same=int(res[2]),
                    num_communities1=int(res[3]), num_communities2=int(res[4]),
                    precision=dres[0], recall=dres[1], f_score=dres[2], gini1=dres[3],
                    gini2=dres[4]), a, b

    def gini(self, sizes):
        s = np.array(sizes, dtype=np.int64)
        return self.L.lvo_gini(_lp(s), ct.c_int(len(s))), s

    def vbase(self, g, color, ncolors, vtype=0):
        """vBaseRedistribution on a copy: (colours, moves, vertices for which
        no colour qualified -- where type 0 of the reference is undefined)."""
        p, t, _ = _csr(g)
        col = np.array(color, dtype=np.int32)
        if col.size and (col.min() < 0 or col.max() >= ncolors):
            raise ValueError('colours must lie in [0, ncolors)')
        stuck = ct.c_long(0)
        n = self.L.lvo_vbase(ct.c_long(g.num_vertices), _lp(p), _lp(t), _ip(col),
                             ct.c_int(ncolors), ct.c_int(vtype), ct.byref(stuck))
        return col, n, stuck.value

    def decide_batch(self, g, C, vdeg, cdeg, csize, constant, verts):
        p, t, w = _csr(g)
        C = np.ascontiguousarray(C, dtype=np.int64)
        vd = np.ascontiguousarray(vdeg, dtype=np.float64)
        cd = np.ascontiguousarray(cdeg, dtype=np.float64)
        cs = np.ascontiguousarray(csize, dtype=np.int64)
        vs = np.ascontiguousarray(verts, dtype=np.int64)
        out = np.zeros(vs.shape[0], dtype=np.int64)
        self.L.lvo_decide_batch(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                _dp(vd), _dp(cd), _lp(cs), ct.c_double(constant),
                                ct.c_long(vs.shape[0]), _lp(vs), _lp(out))
        return out

    def modularity(self, g, C):
        p, t, w = _csr(g)
        C = np.ascontiguousarray(C, dtype=np.int64)
        return self.L.lvo_modularity(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C))

    def _records(self, recs, n):
        return [PhaseRecord(r.nv, r.nnz, bool(r.colored), bool(r.recolored), r.num_colors,
                            r.iterations, r.mod, r.clusters) for r in recs[:n]]

    def color_mhash(self, g, num_colors=16):
        """Multi-hash max/min colouring; draws from the C library's rand()."""
        p, t, _ = _csr(g)
        col = np.empty(g.num_vertices, dtype=np.int32)
        mc = self.L.lvo_color_mhash(ct.c_long(g.num_vertices), _lp(p), _lp(t), ct.c_int(2),
                                    ct.c_int(max(1, num_colors // 4)), _ip(col))
        return col, mc

    def run_multiphase_coloring(self, g, min_graph_size=1000, threshold=1e-6, c_threshold=1e-4,
                                coloring=1, num_colors=16):
        p, t, w = _csr(g)
        C = np.full(g.num_vertices, -1, dtype=np.int64)
        s = _SummaryC()
        recs = (_PhaseC * 256)()
        rc = self.L.lvo_run_multiphase_coloring(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w),
                                                _lp(C), ct.c_int(coloring), ct.c_int(num_colors),
                                                ct.c_long(min_graph_size),
                                                ct.c_double(threshold), ct.c_double(c_threshold),
                                                ct.byref(s), recs, ct.c_int(256))
        if rc != 0:
            raise RuntimeError('oracle: colour count reached the 4096 cap')
        return C, dict(phases=s.phases, total_iterations=s.total_iterations,
                       final_clusters=s.final_clusters, final_mod=s.final_mod,
                       vbase_stuck=self.L.lvo_last_vbase_stuck()), \
            self._records(recs, min(s.nrec, 256))

    def run_multiphase_basic(self, g, threshold=1e-6):
        p, t, w = _csr(g)
        C = np.full(g.num_vertices, -1, dtype=np.int64)
        s = _SummaryC()
        recs = (_PhaseC * 256)()
        self.L.lvo_run_multiphase_basic(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                        ct.c_double(threshold), ct.byref(s), recs, ct.c_int(256))
        return C, dict(phases=s.phases, total_iterations=s.total_iterations,
                       final_clusters=s.final_clusters, final_mod=s.final_mod), \
            self._records(recs, min(s.nrec, 256))


_SUMMARY_KEYS = {
    'phases': r'Total number of phases\s*:\s*(\d+)',
    'total_iterations': r'Total number of iterations\s*:\s*(\d+)',
    'final_clusters': r'Final number of clusters\s*:\s*(\d+)',
    'final_mod': r'Final modularity\s*:\s*(-?[\d.]+)',
    'total_time': r'TOTAL TIME\s*:\s*([\d.]+)',
    'time_clustering': r'Total time for clustering\s*:\s*([\d.]+)',
    'time_building': r'Total time for building phases\s*:\s*([\d.]+)',
    'time_coloring': r'Total time for coloring\s*:\s*([\d.]+)',
}


def parse_reference_log(text: str) -> dict:
    out = {}
    for k, pat in _SUMMARY_KEYS.items():
        m = re.search(pat, text)
        if m:
            out[k] = float(m.group(1)) if '.' in m.group(1) else int(m.group(1))
    out['clusters_per_phase'] = [int(x) for x in re.findall(r'Number of unique clusters: (\d+)', text)]
    out['colors_per_phase'] = [int(x) for x in
                               re.findall(r'Within algoLouvainWithDistOneColoring\(#colors= (\d+)\)', text)]
    return out


def parse_comparison_log(text: str) -> dict:
    """The statistics block computeCommunityComparisons prints."""
    pats = {'num_communities1': r'Num communities in C1\s*:\s*(\d+)',
            'num_communities2': r'Num communities in C2\s*:\s*(\d+)',
            'same_same': r'Same-Same \(True positive\)\s*:\s*(\d+)',
            'same_diff': r'Same-Diff \(False negative\)\s*:\s*(\d+)',
            'diff_same': r'Diff-Same \(False positive\)\s*:\s*(\d+)',
            'precision': r'Precision\s*:\s*([-\d.naif]+)',
            'recall': r'Recall\s*:\s*([-\d.naif]+)',
            'f_score': r'F-score\s*:\s*([-\d.naif]+)',
            'gini1': r'Gini coefficient, C1\s*:\s*([-\d.naif]+)',
            'gini2': r'Gini coefficient, C2\s*:\s*([-\d.naif]+)'}
    out = {}
    for k, p in pats.items():
        m = re.search(p, text)
        if m:
            out[k] = int(m.group(1)) if p.endswith(r'(\d+)') else float(m.group(1))
    return out


class Reference:
    """Grappolo's own functions, compiled from its sources (oracle/_ref)."""

    def __init__(self, fast: bool = False, quiet: bool = True, patched_vbase: bool = False):
        """patched_vbase loads the build whose vBaseRedistribution gains its missing
        return (oracle/ref_vbase.cpp), so coloring = 2 runs; its type 0 is defined
        only where the oracle reports no stuck vertex."""
        name = 'libgrappolo_ref_fast.so' if fast else 'libgrappolo_ref.so'
        if patched_vbase:
            name = 'libgrappolo_ref_vbase.so'
        path = os.path.join(HERE, '_ref', name)
        if not os.path.exists(path):
            build()
        L = ct.CDLL(path)
        self.L = L
        L.ref_color.restype = ct.c_int
        L.ref_color_mhash.restype = ct.c_int
        L.ref_gini.restype = ct.c_double
        L.ref_compare.restype = ct.c_long
        L.ref_remove_edges.restype = ct.c_long
        L.ref_load_binary.restype = ct.c_long
        L.ref_coloring_phase.restype = ct.c_double
        L.ref_basic_phase.restype = ct.c_double
        L.ref_renumber.restype = ct.c_long
        L.ref_build_next_level.restype = ct.c_long
        L.ref_vertex_following.restype = ct.c_long
        L.ref_build_new_graph_vf.restype = ct.c_long
        L.ref_vertex_degrees.restype = ct.c_double
        L.ref_run_multiphase_coloring.restype = ct.c_long
        L.ref_run_multiphase_basic.restype = ct.c_long
        L.ref_load_metis.restype = ct.c_long
        L.ref_graph_create.restype = ct.c_void_p
        L.ref_graph_free.argtypes = [ct.c_void_p]
        L.ref_color_g.restype = ct.c_int
        L.ref_color_g.argtypes = [ct.c_void_p, _c_int_p, ct.c_int, _c_double_p]
        L.ref_coloring_phase_g.restype = ct.c_double
        L.ref_coloring_phase_g.argtypes = [ct.c_void_p, _c_long_p, _c_int_p, ct.c_int,
                                           ct.c_double, ct.c_double, ct.c_int, _c_int_p,
                                           _c_double_p]
        L.ref_set_quiet(ct.c_int(1 if quiet else 0))

    def color(self, g, nthreads=1):
        p, t, w = _csr(g)
        col = np.full(g.num_vertices, -1, dtype=np.int32)
        tt = ct.c_double(0)
        mc = self.L.ref_color(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _ip(col),
                              ct.c_int(nthreads), ct.byref(tt))
        return col, mc, tt.value

    def color_mhash(self, g, num_colors=16, nthreads=1):
        """The reference's multi-hash max/min colouring (rand() values)."""
        p, t, w = _csr(g)
        col = np.empty(g.num_vertices, dtype=np.int32)
        mc = self.L.ref_color_mhash(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w),
                                    ct.c_int(2), ct.c_int(max(1, num_colors // 4)), _ip(col),
                                    ct.c_int(nthreads))
        return col, mc

    def coloring_phase(self, g, colors, num_colors, lower=-1.0, thresh=1e-4, nthreads=1):
        p, t, w = _csr(g)
        C = np.zeros(g.num_vertices, dtype=np.int64)
        col = np.array(colors, dtype=np.int32, copy=True)
        itr, tt = ct.c_int(0), ct.c_double(0)
        q = self.L.ref_coloring_phase(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                      _ip(col), ct.c_int(num_colors), ct.c_double(lower),
                                      ct.c_double(thresh), ct.c_int(nthreads), ct.byref(itr),
                                      ct.byref(tt))
        return q, C, itr.value, tt.value

    def basic_phase(self, g, lower=-1.0, thresh=1e-6, nthreads=1):
        p, t, w = _csr(g)
        C = np.zeros(g.num_vertices, dtype=np.int64)
        itr, tt = ct.c_int(0), ct.c_double(0)
        q = self.L.ref_basic_phase(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                   ct.c_double(lower), ct.c_double(thresh), ct.c_int(nthreads),
                                   ct.byref(itr), ct.byref(tt))
        return q, C, itr.value, tt.value

    def renumber(self, C):
        C = np.array(C, dtype=np.int64, copy=True)
        n = self.L.ref_renumber(_lp(C), ct.c_long(C.shape[0]))
        return C, n

    def build_next_level(self, g, C, ncl, nthreads=1):
        from grappolo_b200.graphs import CSRGraph
        p, t, w = _csr(g)
        C = np.array(C, dtype=np.int64, copy=True)
        op, ot, ow = _c_long_p(), _c_long_p(), _c_double_p()
        ne = ct.c_long(0)
        onnz = self.L.ref_build_next_level(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w),
                                           _lp(C), ct.c_long(ncl), ct.c_int(nthreads),
                                           ct.byref(op), ct.byref(ot), ct.byref(ow), ct.byref(ne))
        if onnz < 0:
            raise RuntimeError('reference coarse graph has a head/row mismatch')
        out = CSRGraph(np.ctypeslib.as_array(op, (ncl + 1,)).copy(),
                       np.ctypeslib.as_array(ot, (max(onnz, 1),))[:onnz].copy(),
                       np.ctypeslib.as_array(ow, (max(onnz, 1),))[:onnz].copy())
        for a in (op, ot, ow):
            self.L.ref_free(a)
        return out, ne.value

    def vertex_following(self, g, nthreads=1):
        """(C, numVtxToFix) of the reference's vertexFollowing."""
        p, t, w = _csr(g)
        C = np.empty(g.num_vertices, dtype=np.int64)
        n = self.L.ref_vertex_following(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                        ct.c_int(nthreads))
        return C, n

    def build_new_graph_vf(self, g, C, ncl, nthreads=1):
        """(CSRGraph, numEdges) of the reference's buildNewGraphVF."""
        from grappolo_b200.graphs import CSRGraph
        p, t, w = _csr(g)
        C = np.array(C, dtype=np.int64, copy=True)
        op, ot, ow = _c_long_p(), _c_long_p(), _c_double_p()
        ne = ct.c_long(0)
        onnz = self.L.ref_build_new_graph_vf(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w),
                                             _lp(C), ct.c_long(ncl), ct.c_int(nthreads),
                                             ct.byref(op), ct.byref(ot), ct.byref(ow),
                                             ct.byref(ne))
        if onnz < 0:
            raise RuntimeError('reference VF graph has a head/row mismatch')
        out = CSRGraph(np.ctypeslib.as_array(op, (ncl + 1,)).copy(),
                       np.ctypeslib.as_array(ot, (max(onnz, 1),))[:onnz].copy(),
                       np.ctypeslib.as_array(ow, (max(onnz, 1),))[:onnz].copy())
        for a in (op, ot, ow):
            self.L.ref_free(a)
        return out, ne.value

    def remove_edges(self, nv, head, tail, w):
        """removeEdges on copies of the SoA arrays: (head, tail, w, NGE)."""
        h, t = np.array(head, dtype=np.int64), np.array(tail, dtype=np.int64)
        ww = np.array(w, dtype=np.float64)
        n = self.L.ref_remove_edges(ct.c_long(nv), ct.c_long(len(h)), _lp(h), _lp(t), _dp(ww))
        return h, t, ww, n

    def sort_edges_undirected(self, nv, head, tail, w):
        """SortEdgesUndirected: (ptrs[NV+2], head, tail, w) of the 2*NE entries."""
        h, t = np.ascontiguousarray(head, dtype=np.int64), np.ascontiguousarray(tail, dtype=np.int64)
        ww = np.ascontiguousarray(w, dtype=np.float64)
        ne = len(h)
        ptrs = np.zeros(nv + 2, dtype=np.int64)
        oh, ot = np.zeros(2 * ne, dtype=np.int64), np.zeros(2 * ne, dtype=np.int64)
        ow = np.zeros(2 * ne)
        self.L.ref_sort_edges_undirected(ct.c_long(nv), ct.c_long(ne), _lp(h), _lp(t), _dp(ww),
                                             _lp(ptrs), _lp(oh), _lp(ot), _dp(ow))
        return ptrs, oh, ot, ow

    def sort_node_edges(self, nv, ptrs, head, tail, w):
        """SortNodeEdgesByIndex on copies: (head, tail, w)."""
        p = np.ascontiguousarray(ptrs, dtype=np.int64)
        h, t = np.array(head, dtype=np.int64), np.array(tail, dtype=np.int64)
        ww = np.array(w, dtype=np.float64)
        self.L.ref_sort_node_edges(ct.c_long(nv), _lp(p), _lp(h), _lp(t), _dp(ww))
        return h, t, ww

    def write_binary(self, g, path, num_edges=None, weighted=1):
        """writeGraphBinaryFormatNew of a CSR graph."""
        p, t, w = _csr(g)
        ne = g.nnz // 2 if num_edges is None else num_edges
        self.L.ref_write_binary(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), ct.c_long(ne),
                                ct.c_long(weighted), str(path).encode())

    def load_binary(self, path):
        """parse_EdgeListBinaryNew: (ptr, head, tail, w, numEdges)."""
        op, oh, ot, ow = _c_long_p(), _c_long_p(), _c_long_p(), _c_double_p()
        ne = ct.c_long(0)
        nv = self.L.ref_load_binary(str(path).encode(), ct.byref(op), ct.byref(oh), ct.byref(ot),
                                    ct.byref(ow), ct.byref(ne))
        nnz = 2 * ne.value
        ptr = np.ctypeslib.as_array(op, (nv + 1,)).copy()
        arr = [np.ctypeslib.as_array(a, (max(nnz, 1),))[:nnz].copy() for a in (oh, ot, ow)]
        for a in (op, oh, ot, ow):
            self.L.ref_free(a)
        return ptr, arr[0], arr[1], arr[2], ne.value

    def compare(self, C1, C2, nthreads=1):
        """computeCommunityComparisons: (parsed statistics, C1', C2')."""
        a, b = np.array(C1, dtype=np.int64), np.array(C2, dtype=np.int64)
        buf = ct.create_string_buffer(1 << 16)
        self.L.ref_compare(_lp(a), _lp(b), ct.c_long(len(a)), ct.c_int(nthreads), buf,
                           ct.c_long(1 << 16))
        return parse_comparison_log(buf.value.decode(errors='replace')), a, b

    def gini(self, sizes):
        s = np.array(sizes, dtype=np.int64)
        return self.L.ref_gini(_lp(s), ct.c_int(len(s))), s

    def decide_batch(self, g, C, vdeg, cdeg, csize, constant, verts):
        p, t, w = _csr(g)
        C = np.ascontiguousarray(C, dtype=np.int64)
        vd = np.ascontiguousarray(vdeg, dtype=np.float64)
        cd = np.ascontiguousarray(cdeg, dtype=np.float64)
        cs = np.ascontiguousarray(csize, dtype=np.int64)
        vs = np.ascontiguousarray(verts, dtype=np.int64)
        out = np.zeros(vs.shape[0], dtype=np.int64)
        self.L.ref_decide_batch(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                _dp(vd), _dp(cd), _lp(cs), ct.c_double(constant),
                                ct.c_long(vs.shape[0]), _lp(vs), _lp(out))
        return out

    def vertex_degrees(self, g):
        p, t, w = _csr(g)
        vd = np.zeros(g.num_vertices)
        c = self.L.ref_vertex_degrees(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _dp(vd))
        return vd, c

    def run_multiphase_coloring(self, g, min_graph_size=1000, threshold=1e-6, c_threshold=1e-4,
                                nthreads=1, coloring=1, num_colors=16, replace_map=0):
        p, t, w = _csr(g)
        C = np.full(g.num_vertices, -1, dtype=np.int64)
        buf = ct.create_string_buffer(1 << 22)
        self.L.ref_run_multiphase_coloring(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w),
                                           _lp(C), ct.c_int(coloring), ct.c_int(num_colors),
                                           ct.c_int(replace_map), ct.c_long(min_graph_size),
                                           ct.c_double(threshold), ct.c_double(c_threshold),
                                           ct.c_int(nthreads), buf, ct.c_long(1 << 22))
        text = buf.value.decode(errors='replace')
        return C, parse_reference_log(text), text

    def run_multiphase_basic(self, g, threshold=1e-6, nthreads=1, basic_opt=0,
                             min_graph_size=1000, c_threshold=1e-4):
        p, t, w = _csr(g)
        C = np.full(g.num_vertices, -1, dtype=np.int64)
        buf = ct.create_string_buffer(1 << 22)
        self.L.ref_run_multiphase_basic(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                        ct.c_int(basic_opt), ct.c_long(min_graph_size),
                                        ct.c_double(threshold), ct.c_double(c_threshold),
                                        ct.c_int(nthreads), buf, ct.c_long(1 << 22))
        text = buf.value.decode(errors='replace')
        return C, parse_reference_log(text), text

    def run_multiphase_sync(self, g, sync_type=3, threshold=1e-6, nthreads=1,
                            min_graph_size=1000, c_threshold=1e-4):
        """runMultiPhaseSyncType (FullSyncOptimization/runMultiPhaseSyncType.cpp:48);
        sync_type 3 is the early-termination Louvain
        (parallelLouvainMethodEarlyTerminate.cpp:116-195)."""
        p, t, w = _csr(g)
        C = np.full(g.num_vertices, -1, dtype=np.int64)
        buf = ct.create_string_buffer(1 << 22)
        self.L.ref_run_multiphase_sync(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _lp(C),
                                       ct.c_int(sync_type), ct.c_long(min_graph_size),
                                       ct.c_double(threshold), ct.c_double(c_threshold),
                                       ct.c_int(nthreads), buf, ct.c_long(1 << 22))
        text = buf.value.decode(errors='replace')
        return C, parse_reference_log(text), text

    def vbase(self, g, color, ncolors, vtype=0):
        """vBaseRedistribution (Coloring/vBase.cpp:6-168) from the copy with its missing
        return added (oracle/ref_vbase.cpp); one thread.  Type 0 reads past its
        frequency array when no colour qualifies: callers keep only cases the
        oracle reports as never stuck."""
        path = os.path.join(HERE, '_ref', 'libgrappolo_ref_vbase.so')
        if not os.path.exists(path):
            build()
        L = self.L if self.L._name == path else ct.CDLL(path)
        p, t, w = _csr(g)
        col = np.ascontiguousarray(color, dtype=np.int32).copy()
        L.ref_vbase(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w), _ip(col),
                    ct.c_int(ncolors), ct.c_int(vtype))
        return col

    def graph(self, g):
        """A persistent reference `graph` (AoS) for repeated calls; free with free_graph."""
        p, t, w = _csr(g)
        return self.L.ref_graph_create(ct.c_long(g.num_vertices), _lp(p), _lp(t), _dp(w))

    def free_graph(self, handle):
        self.L.ref_graph_free(handle)

    def color_g(self, handle, nv, nthreads):
        col = np.full(nv, -1, dtype=np.int32)
        tt = ct.c_double(0)
        mc = self.L.ref_color_g(handle, _ip(col), ct.c_int(nthreads), ct.byref(tt))
        return col, mc, tt.value

    def coloring_phase_g(self, handle, nv, colors, num_colors, lower, thresh, nthreads):
        C = np.zeros(nv, dtype=np.int64)
        col = np.array(colors, dtype=np.int32, copy=True)
        itr, tt = ct.c_int(0), ct.c_double(0)
        q = self.L.ref_coloring_phase_g(handle, _lp(C), _ip(col), ct.c_int(num_colors),
                                        ct.c_double(lower), ct.c_double(thresh),
                                        ct.c_int(nthreads), ct.byref(itr), ct.byref(tt))
        return q, C, itr.value, tt.value

    def load_metis(self, path):
        from grappolo_b200.graphs import CSRGraph
        op, ot, ow = _c_long_p(), _c_long_p(), _c_double_p()
        nv = self.L.ref_load_metis(path.encode(), ct.byref(op), ct.byref(ot), ct.byref(ow))
        ptr = np.ctypeslib.as_array(op, (nv + 1,)).copy()
        nnz = int(ptr[-1])
        out = CSRGraph(ptr, np.ctypeslib.as_array(ot, (max(nnz, 1),))[:nnz].copy(),
                       np.ctypeslib.as_array(ow, (max(nnz, 1),))[:nnz].copy())
        for a in (op, ot, ow):
            self.L.ref_free(a)
        return out
