"""Host-side mirror of Grappolo's clustering API over the B200 engine.

Function names, argument meaning and return conventions follow the reference
(DefineStructure/color_comm.h, basic_comm.h, coloring.h, basic_util.h); the
work runs in libgrappolo_b200.so on the GPU.  Differences that a Python
caller sees:

* ``graph`` arguments are :class:`grappolo_b200.graphs.CSRGraph` (or
  :class:`Graph`), not freed by the call;
* results the reference returns through pointers are returned as values;
* ``nThreads`` selects the schedule: 1 -> verify mode (the reference's
  one-thread results, bit for bit), >1 -> fast mode (parallel colouring and
  atomic accumulation).  ``GRAPPOLO_B200_MODE=verify|fast`` overrides it.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

from . import _lib
from .graphs import CSRGraph

_P = ct.POINTER


def _mode(n_threads: int) -> int:
    env = os.environ.get('GRAPPOLO_B200_MODE', '').lower()
    if env == 'verify':
        return _lib.GLV_MODE_VERIFY
    if env == 'fast':
        return _lib.GLV_MODE_FAST
    return _lib.GLV_MODE_VERIFY if n_threads <= 1 else _lib.GLV_MODE_FAST


class Graph:
    """A ``graph`` struct (DefineStructure/defs.h:85-92) backed by numpy arrays."""

    EDGE = np.dtype([('head', '<i8'), ('tail', '<i8'), ('weight', '<f8')])

    def __init__(self, g: CSRGraph):
        self.csr = g
        self.ptr = np.ascontiguousarray(g.ptr, dtype=np.int64)
        self.edges = np.empty(g.nnz, dtype=self.EDGE)
        self.edges['head'] = g.heads()
        self.edges['tail'] = g.tail
        self.edges['weight'] = g.weight
        self.struct = _lib.GlvGraph(g.num_vertices, g.num_vertices, g.num_edges,
                                    self.ptr.ctypes.data_as(_P(ct.c_long)),
                                    self.edges.ctypes.data_as(_P(_lib.GlvEdge)))

    @property
    def numVertices(self) -> int:
        return self.csr.num_vertices


def _as_graph(g) -> Graph:
    return g if isinstance(g, Graph) else Graph(g)


def runMultiPhaseColoring(G, C_orig=None, coloring=1, numColors=16, replaceMap=0,
                          minGraphSize=1000, threshold=1e-6, C_threshold=1e-4, numThreads=1,
                          threadsOpt=1, stats: bool = False):
    """Coloring/runMultiPhaseColoring.cpp:51 — returns C_orig (int64[NV]); with
    ``stats`` also the run statistics (phases, iterations, "Final modularity"...)."""
    G = _as_graph(G)
    nv = G.numVertices
    if C_orig is None:
        C_orig = np.full(nv, -1, dtype=np.int64)
    st = _lib.GlvRunStats()
    _lib.check(_lib.lib().glv_run_multiphase_coloring(
        ct.byref(G.struct), C_orig.ctypes.data_as(_P(ct.c_long)), coloring, numColors,
        replaceMap, minGraphSize, threshold, C_threshold, _mode(numThreads), ct.byref(st)))
    return (C_orig, st.to_dict()) if stats else C_orig


def runMultiPhaseBasic(G, C_orig=None, basicOpt=0, minGraphSize=1000, threshold=1e-6,
                       C_threshold=1e-4, numThreads=1, threadsOpt=1, stats: bool = False):
    """BasicCommunitiesDetection/runMultiPhaseBasic.cpp:52."""
    G = _as_graph(G)
    nv = G.numVertices
    if C_orig is None:
        C_orig = np.full(nv, -1, dtype=np.int64)
    st = _lib.GlvRunStats()
    _lib.check(_lib.lib().glv_run_multiphase_basic(
        ct.byref(G.struct), C_orig.ctypes.data_as(_P(ct.c_long)), basicOpt, minGraphSize,
        threshold, C_threshold, _mode(numThreads), ct.byref(st)))
    return (C_orig, st.to_dict()) if stats else C_orig


def algoLouvainWithDistOneColoring(G, color, numColor, Lower=-1.0, thresh=1e-4, nThreads=1):
    """Coloring/parallelLouvainWithColoring.cpp:47 — returns (prevMod, C, numItr, totTime)."""
    G = _as_graph(G)
    C = np.zeros(G.numVertices, dtype=np.int64)
    col = np.ascontiguousarray(color, dtype=np.int32)
    q, itr, tt = ct.c_double(0), ct.c_int(0), ct.c_double(0)
    _lib.check(_lib.lib().glv_louvain_coloring_phase(
        ct.byref(G.struct), C.ctypes.data_as(_P(ct.c_long)), col.ctypes.data_as(_P(ct.c_int)),
        numColor, Lower, thresh, _mode(nThreads), ct.byref(q), ct.byref(itr), ct.byref(tt)))
    return q.value, C, itr.value, tt.value


def parallelLouvianMethod(G, Lower=-1.0, thresh=1e-6, nThreads=1):
    """BasicCommunitiesDetection/parallelLouvainMethod.cpp:65 — (prevMod, C, numItr, totTime)."""
    G = _as_graph(G)
    C = np.zeros(G.numVertices, dtype=np.int64)
    q, itr, tt = ct.c_double(0), ct.c_int(0), ct.c_double(0)
    _lib.check(_lib.lib().glv_louvain_basic_phase(
        ct.byref(G.struct), C.ctypes.data_as(_P(ct.c_long)), Lower, thresh, _mode(nThreads),
        ct.byref(q), ct.byref(itr), ct.byref(tt)))
    return q.value, C, itr.value, tt.value


def algoDistanceOneVertexColoringOpt(G, nThreads=1):
    """Coloring/coloringDistanceOne.cpp:50 — returns (vtxColor int32[NV], maxColor, totTime)."""
    G = _as_graph(G)
    col = np.full(G.numVertices, -1, dtype=np.int32)
    mc, tt = ct.c_int(0), ct.c_double(0)
    _lib.check(_lib.lib().glv_distance_one_coloring(
        ct.byref(G.struct), col.ctypes.data_as(_P(ct.c_int)), _mode(nThreads), ct.byref(mc),
        ct.byref(tt)))
    return col, mc.value, tt.value


def vBaseRedistribution(G, vtxColor, ncolors, type=0):
    """Coloring/vBase.cpp:6 — returns (rebalanced colours int32[NV], vertices moved)."""
    G = _as_graph(G)
    col = np.array(vtxColor, dtype=np.int32, copy=True)
    n = ct.c_long(0)
    _lib.check(_lib.lib().glv_vbase_redistribution(
        ct.byref(G.struct), col.ctypes.data_as(_P(ct.c_int)), ncolors, type, ct.byref(n)))
    return col, n.value


def algoColoringMultiHashMaxMin(G, nThreads=1, nHash=2, nItrs=4):
    """Coloring/coloringMultiHashMaxMin.cpp:59 — returns (vtxColor int32[NV],
    maxColor, totTime).  Random values come from the C library's rand()."""
    G = _as_graph(G)
    col = np.full(G.numVertices, -1, dtype=np.int32)
    mc, tt = ct.c_int(0), ct.c_double(0)
    _lib.check(_lib.lib().glv_color_multihash(
        ct.byref(G.struct), col.ctypes.data_as(_P(ct.c_int)), nHash, nItrs, ct.byref(mc),
        ct.byref(tt)))
    return col, mc.value, tt.value


def renumberClustersContiguously(C):
    """Utility/buildNextPhase.cpp:48 — returns (renumbered C, numUniqueClusters)."""
    C = np.array(C, dtype=np.int64, copy=True)
    n = ct.c_long(0)
    _lib.check(_lib.lib().glv_renumber_clusters(C.ctypes.data_as(_P(ct.c_long)), C.shape[0],
                                                ct.byref(n)))
    return C, n.value


def buildNextLevelGraphOpt(G, C, numUniqueClusters, nThreads=1):
    """Utility/buildNextPhase.cpp:83 — returns (CSRGraph of the next level, numEdges)."""
    G = _as_graph(G)
    C = np.ascontiguousarray(C, dtype=np.int64)
    out = _lib.GlvGraph()
    tt = ct.c_double(0)
    L = _lib.lib()
    _lib.check(L.glv_build_next_level(ct.byref(G.struct), ct.byref(out),
                                      C.ctypes.data_as(_P(ct.c_long)), numUniqueClusters,
                                      _mode(nThreads), ct.byref(tt)))
    return _take_graph(out)


def vertexFollowing(G):
    """Utility/vertexFollowing.cpp:46 — returns (C int64[NV], numVtxToFix)."""
    G = _as_graph(G)
    C = np.empty(G.numVertices, dtype=np.int64)
    n = ct.c_long(0)
    _lib.check(_lib.lib().glv_vertex_following(ct.byref(G.struct),
                                               C.ctypes.data_as(_P(ct.c_long)), ct.byref(n)))
    return C, n.value


def buildNewGraphVF(G, C, numUniqueClusters):
    """Utility/vertexFollowing.cpp:91 — returns (CSRGraph, numEdges) of the
    vertex-following graph (no zero self-loops, weights cast to integers)."""
    G = _as_graph(G)
    C = np.ascontiguousarray(C, dtype=np.int64)
    out = _lib.GlvGraph()
    tt = ct.c_double(0)
    _lib.check(_lib.lib().glv_build_new_graph_vf(ct.byref(G.struct), ct.byref(out),
                                                 C.ctypes.data_as(_P(ct.c_long)),
                                                 numUniqueClusters, ct.byref(tt)))
    return _take_graph(out)


def _edges(head, tail, weight=None):
    """A contiguous glv_edge array (Graph.EDGE records) from three arrays."""
    head = np.asarray(head, dtype=np.int64)
    e = np.empty(head.shape[0], dtype=Graph.EDGE)
    e['head'] = head
    e['tail'] = np.asarray(tail, dtype=np.int64)
    e['weight'] = 1.0 if weight is None else np.asarray(weight, dtype=np.float64)
    return e


def _ep(e):
    return e.ctypes.data_as(_P(_lib.GlvEdge))


def removeEdges(NV, edgeList):
    """Utility/utilityFunctions.cpp:416 — on a copy of ``edgeList`` (Graph.EDGE
    records): returns (edges, NGE); the first NGE records are the kept edges in
    the reference's order, the rest as they were."""
    e = np.array(edgeList, dtype=Graph.EDGE, copy=True)
    n = ct.c_long(0)
    _lib.check(_lib.lib().glv_remove_edges(NV, e.shape[0], _ep(e), ct.byref(n)))
    return e, n.value


def SortEdgesUndirected(NV, list1):
    """Utility/utilityFunctions.cpp:463 — returns (ptrs int64[NV+2], list2 of
    2*NE records: every edge in the rows of both ends, in list order)."""
    e = np.ascontiguousarray(list1, dtype=Graph.EDGE)
    out = np.empty(2 * e.shape[0], dtype=Graph.EDGE)
    ptrs = np.zeros(NV + 2, dtype=np.int64)
    _lib.check(_lib.lib().glv_sort_edges_undirected(NV, e.shape[0], _ep(e), _ep(out),
                                                    ptrs.ctypes.data_as(_P(ct.c_long))))
    return ptrs, out


def SortNodeEdgesByIndex(NV, list1, ptrs):
    """Utility/utilityFunctions.cpp:501 — returns a copy of ``list1`` with each
    row sorted by tail (equal tails: later entry first, as the reference)."""
    e = np.array(list1, dtype=Graph.EDGE, copy=True)
    p = np.ascontiguousarray(ptrs, dtype=np.int64)
    _lib.check(_lib.lib().glv_sort_node_edges_by_index(NV, _ep(e), None,
                                                       p.ctypes.data_as(_P(ct.c_long))))
    return e


def build_csr(NV, head, tail, weight=None, remove_edges=True, sort_rows=False):
    """Edge list to CSR on the GPU as the reference's loaders build it
    (glv_build_csr): optional removeEdges, both directions of every edge in list
    order, optional per-row sort.  Returns (CSRGraph, numEdges)."""
    e = _edges(head, tail, weight)
    flags = (_lib.GLV_CSR_REMOVE_EDGES if remove_edges else 0) | \
        (_lib.GLV_CSR_SORT_ROWS if sort_rows else 0)
    out = _lib.GlvGraph()
    _lib.check(_lib.lib().glv_build_csr(NV, e.shape[0], _ep(e), flags, ct.byref(out)))
    return _take_graph(out)


def build_csr_device(NV, d_head, d_tail, d_weight=None, remove_edges=True, sort_rows=False,
                     device='cuda'):
    """Device form (glv_dev_build_csr) on torch tensors: int64 heads / tails,
    float64 weights or None.  Returns (ptr int64[NV+1], tail int32, weight
    float64) tensors holding exactly the built entries."""
    import torch
    ne = int(d_head.shape[0])
    ptr = torch.empty(NV + 1, dtype=torch.int64, device=device)
    tail = torch.empty(max(2 * ne, 1), dtype=torch.int32, device=device)
    w = torch.empty(max(2 * ne, 1), dtype=torch.float64, device=device)
    flags = (_lib.GLV_CSR_REMOVE_EDGES if remove_edges else 0) | \
        (_lib.GLV_CSR_SORT_ROWS if sort_rows else 0)
    nnz = ct.c_long(0)
    stream = torch.cuda.current_stream(device).cuda_stream
    _lib.check(_lib.lib().glv_dev_build_csr(
        NV, ne, d_head.data_ptr(), d_tail.data_ptr(),
        d_weight.data_ptr() if d_weight is not None else None, flags, ptr.data_ptr(),
        tail.data_ptr(), w.data_ptr(), ct.byref(nnz), stream or None))
    return ptr, tail[:nnz.value], w[:nnz.value]


def parse_EdgeListBinaryNew(fileName):
    """InputsOutput/loadBinary.cpp:6 — returns (CSRGraph, numEdges)."""
    out = _lib.GlvGraph()
    _lib.check(_lib.lib().glv_load_binary(os.fsencode(fileName), ct.byref(out)))
    return _take_graph(out)


def writeGraphBinaryFormatNew(G, filename, weighted=1):
    """InputsOutput/writeBinary.cpp:2 — writes ``G`` (numEdges = nnz / 2 records
    pairs, as the reference stores 2*numEdges entries)."""
    G = _as_graph(G)
    st = _lib.GlvGraph(G.struct.numVertices, G.struct.sVertices, G.csr.nnz // 2,
                       G.struct.edgeListPtrs, G.struct.edgeList)
    _lib.check(_lib.lib().glv_write_binary(ct.byref(st), os.fsencode(filename), weighted))


def load_binary_device(fileName, device='cuda'):
    """Streams a binary graph file into device memory (glv_dev_load_binary).
    Returns (ptr int64[NV+1], tail int32[2*NE], weight float64[2*NE]) tensors."""
    import torch
    nv, ne, wt = ct.c_long(0), ct.c_long(0), ct.c_long(0)
    path = os.fsencode(fileName)
    L = _lib.lib()
    _lib.check(L.glv_binary_header(path, ct.byref(nv), ct.byref(ne), ct.byref(wt)))
    nnz = 2 * ne.value
    ptr = torch.empty(nv.value + 1, dtype=torch.int64, device=device)
    tail = torch.empty(max(nnz, 1), dtype=torch.int32, device=device)
    w = torch.empty(max(nnz, 1), dtype=torch.float64, device=device)
    stream = torch.cuda.current_stream(device).cuda_stream
    _lib.check(L.glv_dev_load_binary(path, nv.value, nnz, ptr.data_ptr(), tail.data_ptr(),
                                     w.data_ptr(), stream or None))
    return ptr, tail[:nnz], w[:nnz]


def computeCommunityComparisons(C1, C2):
    """Utility/utilityClusterComparisonMetrics.cpp:50 — C1 is the truth.
    Returns (statistics dict, C1', C2'): the pair counts (same_same,
    same_diff, diff_same), precision, recall, f_score, the Gini coefficients
    and the label arrays relabelled as the reference leaves them."""
    a = np.array(C1, dtype=np.int64, copy=True)
    b = np.array(C2, dtype=np.int64, copy=True)
    r = _lib.GlvComparison()
    lp = lambda x: x.ctypes.data_as(_P(ct.c_long))  # noqa: E731
    _lib.check(_lib.lib().glv_compare_communities(lp(a), a.shape[0], lp(b), b.shape[0],
                                                  ct.byref(r)))
    return r.to_dict(), a, b


def compare_communities_device(d_C1, d_C2, stream=0):
    """glv_dev_compare_communities on int64 torch tensors (relabelled in place)."""
    r = _lib.GlvComparison()
    _lib.check(_lib.lib().glv_dev_compare_communities(d_C1.numel(), d_C1.data_ptr(),
                                                      d_C2.data_ptr(), ct.byref(r),
                                                      stream or None))
    return r.to_dict()


def computeGiniCoefficient(colorSize):
    """utilityClusterComparisonMetrics.cpp:310 — returns (Gini coefficient,
    sizes sorted ascending)."""
    s = np.array(colorSize, dtype=np.int64, copy=True)
    g = ct.c_double(0)
    _lib.check(_lib.lib().glv_gini_coefficient(s.ctypes.data_as(_P(ct.c_long)), s.shape[0],
                                               ct.byref(g)))
    return g.value, s


def _take_graph(out):
    """CSRGraph + numEdges from a glv_graph whose arrays the library malloc'd
    (released here)."""
    nv = out.numVertices
    ptr = np.ctypeslib.as_array(out.edgeListPtrs, (nv + 1,)).copy()
    nnz = int(ptr[-1])
    libc = ct.CDLL(None)
    if nnz:
        raw = np.ctypeslib.as_array(ct.cast(out.edgeList, _P(ct.c_char)), (nnz * 24,))
        rec = np.frombuffer(raw.tobytes(), dtype=Graph.EDGE)
        heads = rec['head'].copy()
        tail = rec['tail'].copy()
        w = rec['weight'].copy()
    else:
        heads = tail = np.zeros(0, dtype=np.int64)
        w = np.zeros(0)
    libc.free(ct.cast(out.edgeListPtrs, ct.c_void_p))
    libc.free(ct.cast(out.edgeList, ct.c_void_p))
    expect = np.repeat(np.arange(nv, dtype=np.int64), np.diff(ptr))
    if not np.array_equal(heads, expect):
        raise RuntimeError('coarse graph head/row mismatch')
    return CSRGraph(ptr, tail, w), out.numEdges


def modularity(G, C) -> float:
    """Q of an assignment, the formula of Coloring/parallelLouvainWithColoring.cpp:226-249
    (the reference's computeModularity is an unimplemented stub)."""
    G = _as_graph(G)
    C = np.ascontiguousarray(C, dtype=np.int64)
    q = ct.c_double(0)
    _lib.check(_lib.lib().glv_modularity(ct.byref(G.struct), C.ctypes.data_as(_P(ct.c_long)),
                                         ct.byref(q)))
    return q.value


def decide_batch(g: CSRGraph, C, vDeg, cDeg, cSize, constant, verts):
    """Move decisions for `verts` against one fixed state (buildLocalMapCounter + max,
    Utility/utilityClusteringFunctions.cpp:172-194,226-259)."""
    p = np.ascontiguousarray(g.ptr, dtype=np.int64)
    t = np.ascontiguousarray(g.tail, dtype=np.int64)
    w = np.ascontiguousarray(g.weight, dtype=np.float64)
    C = np.ascontiguousarray(C, dtype=np.int64)
    vd = np.ascontiguousarray(vDeg, dtype=np.float64)
    cd = np.ascontiguousarray(cDeg, dtype=np.float64)
    cs = np.ascontiguousarray(cSize, dtype=np.int64)
    vs = np.ascontiguousarray(verts, dtype=np.int64)
    out = np.zeros(vs.shape[0], dtype=np.int64)
    lp = lambda a: a.ctypes.data_as(_P(ct.c_long))  # noqa: E731
    dp = lambda a: a.ctypes.data_as(_P(ct.c_double))  # noqa: E731
    _lib.check(_lib.lib().glv_decide_batch(g.num_vertices, lp(p), lp(t), dp(w), lp(C), dp(vd),
                                           dp(cd), lp(cs), constant, vs.shape[0], lp(vs),
                                           lp(out)))
    return out


def run_multiphase_csr(g: CSRGraph, coloring: bool = True, minGraphSize=1000, threshold=1e-6,
                       C_threshold=1e-4, mode: int = _lib.GLV_MODE_VERIFY):
    """SoA host entry (glv_run_multiphase_*_csr): returns (C_orig, stats dict)."""
    p = np.ascontiguousarray(g.ptr, dtype=np.int64)
    t = np.ascontiguousarray(g.tail, dtype=np.int64)
    w = np.ascontiguousarray(g.weight, dtype=np.float64)
    C = np.full(g.num_vertices, -1, dtype=np.int64)
    st = _lib.GlvRunStats()
    L = _lib.lib()
    lp = lambda a: a.ctypes.data_as(_P(ct.c_long))  # noqa: E731
    if coloring:
        rc = L.glv_run_multiphase_coloring_csr(g.num_vertices, lp(p), lp(t),
                                               w.ctypes.data_as(_P(ct.c_double)), lp(C),
                                               minGraphSize, threshold, C_threshold, mode,
                                               ct.byref(st))
    else:
        rc = L.glv_run_multiphase_basic_csr(g.num_vertices, lp(p), lp(t),
                                            w.ctypes.data_as(_P(ct.c_double)), lp(C), threshold,
                                            mode, ct.byref(st))
    _lib.check(rc)
    return C, st.to_dict()


def run_multiphase_device(nv, d_ptr, d_tail, d_weight, d_C_orig, coloring=True,
                          minGraphSize=1000, threshold=1e-6, C_threshold=1e-4,
                          mode: int = _lib.GLV_MODE_FAST, stream=0):
    """Device-resident entry (glv_dev_run_multiphase): pointers are ints (e.g.
    torch ``tensor.data_ptr()``): ptr int64[nv+1], tail int32, weight f64, C_orig int32."""
    st = _lib.GlvRunStats()
    _lib.check(_lib.lib().glv_dev_run_multiphase(nv, d_ptr, d_tail, d_weight, d_C_orig,
                                                 1 if coloring else 0, minGraphSize, threshold,
                                                 C_threshold, mode, stream or None,
                                                 ct.byref(st)))
    return st.to_dict()


def _batch_stats(G):
    """A glv_batch_stats with its per-graph arrays (kept alive by the dict)."""
    arrs = {'final_modularity': np.zeros(G), 'phases': np.zeros(G, dtype=np.int32),
            'iterations': np.zeros(G, dtype=np.int32), 'clusters': np.zeros(G, dtype=np.int64),
            'done_seconds': np.zeros(G)}
    st = _lib.GlvBatchStats()
    st.final_modularity = arrs['final_modularity'].ctypes.data_as(_P(ct.c_double))
    st.phases = arrs['phases'].ctypes.data_as(_P(ct.c_int))
    st.iterations = arrs['iterations'].ctypes.data_as(_P(ct.c_int))
    st.clusters = arrs['clusters'].ctypes.data_as(_P(ct.c_long))
    st.done_seconds = arrs['done_seconds'].ctypes.data_as(_P(ct.c_double))
    return st, arrs


def _batch_dict(st, arrs):
    d = {k: getattr(st, k) for k in ('rounds', 'time_total', 'time_clustering', 'time_coloring',
                                     'time_building', 'time_transfer', 'edges_swept',
                                     'kernel_launches')}
    d.update({k: v.copy() for k, v in arrs.items()})
    return d


def union(graphs):
    """Lay graphs end to end as one CSR (tails shifted to global ids).
    Returns (vertex_offsets int64[G+1], CSRGraph)."""
    voff = np.zeros(len(graphs) + 1, dtype=np.int64)
    np.cumsum([g.num_vertices for g in graphs], out=voff[1:])
    eoff = np.zeros(len(graphs) + 1, dtype=np.int64)
    np.cumsum([g.nnz for g in graphs], out=eoff[1:])
    ptr = np.empty(voff[-1] + 1, dtype=np.int64)
    tail = np.empty(eoff[-1], dtype=np.int64)
    w = np.empty(eoff[-1], dtype=np.float64)
    for k, g in enumerate(graphs):
        ptr[voff[k]:voff[k + 1]] = g.ptr[:-1] + eoff[k]
        tail[eoff[k]:eoff[k + 1]] = g.tail + voff[k]
        w[eoff[k]:eoff[k + 1]] = g.weight
    ptr[-1] = eoff[-1]
    return voff, CSRGraph(ptr, tail, w)


def run_batch(graphs, coloring: bool = True, minGraphSize=1000, threshold=1e-6,
              C_threshold=1e-4, mode: int = _lib.GLV_MODE_FAST):
    """Many independent graphs in one batched run (glv_run_batch_csr).

    Returns (list of per-graph community arrays in graph-local ids, stats dict
    with per-graph arrays final_modularity/phases/iterations/clusters/done_seconds)."""
    voff, u = union(graphs)
    C = np.full(u.num_vertices, -1, dtype=np.int64)
    st, arrs = _batch_stats(len(graphs))
    lp = lambda a: a.ctypes.data_as(_P(ct.c_long))  # noqa: E731
    _lib.check(_lib.lib().glv_run_batch_csr(
        len(graphs), lp(voff), lp(u.ptr), lp(np.ascontiguousarray(u.tail, dtype=np.int64)),
        u.weight.ctypes.data_as(_P(ct.c_double)), lp(C), 1 if coloring else 0, minGraphSize,
        threshold, C_threshold, mode, ct.byref(st)))
    return [C[voff[k]:voff[k + 1]] for k in range(len(graphs))], _batch_dict(st, arrs)


def run_batch_device(vertex_offsets, d_ptr, d_tail, d_weight, d_C, coloring=True,
                     minGraphSize=1000, threshold=1e-6, C_threshold=1e-4,
                     mode: int = _lib.GLV_MODE_FAST, stream=0):
    """Device-resident batch (glv_dev_run_batch); vertex_offsets is a host int64 array."""
    voff = np.ascontiguousarray(vertex_offsets, dtype=np.int64)
    st, arrs = _batch_stats(len(voff) - 1)
    _lib.check(_lib.lib().glv_dev_run_batch(
        len(voff) - 1, voff.ctypes.data_as(_P(ct.c_long)), d_ptr, d_tail, d_weight, d_C,
        1 if coloring else 0, minGraphSize, threshold, C_threshold, mode, stream or None,
        ct.byref(st)))
    return _batch_dict(st, arrs)
