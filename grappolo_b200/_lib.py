"""ctypes binding of libgrappolo_b200.so (the C ABI in include/grappolo_b200.h).

The library is built in-tree by ``grappolo_b200.build`` (or
``__graft_entry__.build()``).  There is no CPU fallback: if the shared library
is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as ct
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libgrappolo_b200.so')

GLV_OK = 0
GLV_CSR_REMOVE_EDGES = 1
GLV_CSR_SORT_ROWS = 2
GLV_MODE_VERIFY = 0
GLV_MODE_FAST = 1
GLV_MODE_LEARNED = 2
GLV_GATE_PARAMS = 4673
GLV_GATE_FEATURES = 6
GLV_MAX_PHASES = 256
GLV_KERNEL_SLOTS = 11

ERRORS = {
    1: 'invalid argument', 2: 'CUDA error', 3: 'out of memory',
    4: 'colouring needs more than 4096 colours', 5: 'numVertices >= 2^31',
    6: 'unsupported option', 7: 'no CUDA device', 8: 'size exceeds a fixed limit',
}


class GlvEdge(ct.Structure):
    _fields_ = [('head', ct.c_long), ('tail', ct.c_long), ('weight', ct.c_double)]


class GlvGraph(ct.Structure):
    _fields_ = [('numVertices', ct.c_long), ('sVertices', ct.c_long), ('numEdges', ct.c_long),
                ('edgeListPtrs', ct.POINTER(ct.c_long)), ('edgeList', ct.POINTER(GlvEdge))]


class GlvComparison(ct.Structure):
    _fields_ = [('n1', ct.c_long), ('n2', ct.c_long), ('num_communities1', ct.c_long),
                ('num_communities2', ct.c_long), ('same_same', ct.c_long),
                ('same_diff', ct.c_long), ('diff_same', ct.c_long), ('precision', ct.c_double),
                ('recall', ct.c_double), ('f_score', ct.c_double), ('gini1', ct.c_double),
                ('gini2', ct.c_double)]

    def to_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class GlvPhaseStats(ct.Structure):
    _fields_ = [('num_vertices', ct.c_long), ('nnz', ct.c_long), ('colored', ct.c_int),
                ('recolored', ct.c_int), ('num_colors', ct.c_int), ('iterations', ct.c_int),
                ('modularity', ct.c_double), ('clusters', ct.c_long),
                ('time_sweep', ct.c_double), ('time_color', ct.c_double),
                ('time_coarsen', ct.c_double), ('edges_swept', ct.c_double)]


class GlvRunStats(ct.Structure):
    _fields_ = [('phases', ct.c_int), ('total_iterations', ct.c_int),
                ('final_clusters', ct.c_long), ('final_modularity', ct.c_double),
                ('time_total', ct.c_double), ('time_clustering', ct.c_double),
                ('time_coloring', ct.c_double), ('time_building', ct.c_double),
                ('time_transfer', ct.c_double), ('edges_swept', ct.c_double),
                ('kernel_launches', ct.c_long), ('sweep_kernel_time', ct.c_double),
                ('sweep_bytes', ct.c_double), ('sweep_steps', ct.c_long),
                ('kernel_time', ct.c_double * GLV_KERNEL_SLOTS), ('nphase', ct.c_int),
                ('phase', GlvPhaseStats * GLV_MAX_PHASES), ('tuned_block_max', ct.c_int),
                ('tuned_hub_chunk', ct.c_int), ('tuned_from_cache', ct.c_int),
                ('hub_cluster', ct.c_int)]

    def to_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ('phase', 'kernel_time')}
        d['kernel_time'] = list(self.kernel_time)
        d['phase'] = [{k: getattr(p, k) for k, _ in GlvPhaseStats._fields_}
                      for p in self.phase[:self.nphase]]
        return d


class GlvBatchStats(ct.Structure):
    _fields_ = [('final_modularity', ct.POINTER(ct.c_double)), ('phases', ct.POINTER(ct.c_int)),
                ('iterations', ct.POINTER(ct.c_int)), ('clusters', ct.POINTER(ct.c_long)),
                ('done_seconds', ct.POINTER(ct.c_double)), ('rounds', ct.c_int),
                ('time_total', ct.c_double), ('time_clustering', ct.c_double),
                ('time_coloring', ct.c_double), ('time_building', ct.c_double),
                ('time_transfer', ct.c_double), ('edges_swept', ct.c_double),
                ('kernel_launches', ct.c_long)]


class GrappoloError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f'grappolo_b200 error {code} ({ERRORS.get(code, "?")}): {msg}')
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f'{LIB_PATH} is missing: build it with grappolo_b200.build.build()')
    L = ct.CDLL(LIB_PATH)
    P = ct.POINTER
    L.glv_version.restype = ct.c_char_p
    L.glv_last_error.restype = ct.c_char_p
    L.glv_kernel_launch_count.restype = ct.c_long
    L.glv_set_profiling.argtypes = [ct.c_int]
    for name in ('glv_run_multiphase_coloring', 'glv_run_multiphase_basic',
                 'glv_run_multiphase_coloring_csr', 'glv_run_multiphase_basic_csr',
                 'glv_dev_run_multiphase', 'glv_louvain_coloring_phase',
                 'glv_louvain_basic_phase', 'glv_distance_one_coloring', 'glv_color_multihash',
                 'glv_renumber_clusters', 'glv_build_next_level', 'glv_modularity',
                 'glv_decide_batch', 'glv_dev_modularity_static', 'glv_gate_set',
                 'glv_gate_infer', 'glv_gate_grad', 'glv_gate_train', 'glv_trace_begin',
                 'glv_trace_end', 'glv_run_batch_csr', 'glv_dev_run_batch',
                 'glv_vertex_following', 'glv_build_new_graph_vf', 'glv_remove_edges',
                 'glv_sort_edges_undirected', 'glv_sort_node_edges_by_index', 'glv_build_csr',
                 'glv_dev_build_csr', 'glv_binary_header', 'glv_load_binary', 'glv_write_binary',
                 'glv_dev_load_binary', 'glv_compare_communities',
                 'glv_dev_compare_communities', 'glv_gini_coefficient',
                 'glv_vbase_redistribution'):
        getattr(L, name).restype = ct.c_int
    L.glv_run_multiphase_coloring.argtypes = [P(GlvGraph), P(ct.c_long), ct.c_int, ct.c_int,
                                              ct.c_int, ct.c_long, ct.c_double, ct.c_double,
                                              ct.c_int, P(GlvRunStats)]
    L.glv_run_multiphase_basic.argtypes = [P(GlvGraph), P(ct.c_long), ct.c_int, ct.c_long,
                                           ct.c_double, ct.c_double, ct.c_int, P(GlvRunStats)]
    L.glv_run_multiphase_coloring_csr.argtypes = [ct.c_long, P(ct.c_long), P(ct.c_long),
                                                  P(ct.c_double), P(ct.c_long), ct.c_long,
                                                  ct.c_double, ct.c_double, ct.c_int,
                                                  P(GlvRunStats)]
    L.glv_run_multiphase_basic_csr.argtypes = [ct.c_long, P(ct.c_long), P(ct.c_long),
                                               P(ct.c_double), P(ct.c_long), ct.c_double,
                                               ct.c_int, P(GlvRunStats)]
    L.glv_dev_run_multiphase.argtypes = [ct.c_long, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                         ct.c_void_p, ct.c_int, ct.c_long, ct.c_double,
                                         ct.c_double, ct.c_int, ct.c_void_p, P(GlvRunStats)]
    L.glv_louvain_coloring_phase.argtypes = [P(GlvGraph), P(ct.c_long), P(ct.c_int), ct.c_int,
                                             ct.c_double, ct.c_double, ct.c_int,
                                             P(ct.c_double), P(ct.c_int), P(ct.c_double)]
    L.glv_louvain_basic_phase.argtypes = [P(GlvGraph), P(ct.c_long), ct.c_double, ct.c_double,
                                          ct.c_int, P(ct.c_double), P(ct.c_int),
                                          P(ct.c_double)]
    L.glv_distance_one_coloring.argtypes = [P(GlvGraph), P(ct.c_int), ct.c_int, P(ct.c_int),
                                            P(ct.c_double)]
    L.glv_color_multihash.argtypes = [P(GlvGraph), P(ct.c_int), ct.c_int, ct.c_int, P(ct.c_int),
                                      P(ct.c_double)]
    L.glv_remove_edges.argtypes = [ct.c_long, ct.c_long, P(GlvEdge), P(ct.c_long)]
    L.glv_sort_edges_undirected.argtypes = [ct.c_long, ct.c_long, P(GlvEdge), P(GlvEdge),
                                            P(ct.c_long)]
    L.glv_sort_node_edges_by_index.argtypes = [ct.c_long, P(GlvEdge), P(GlvEdge), P(ct.c_long)]
    L.glv_build_csr.argtypes = [ct.c_long, ct.c_long, P(GlvEdge), ct.c_int, P(GlvGraph)]
    L.glv_dev_build_csr.argtypes = [ct.c_long, ct.c_long, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                    ct.c_int, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                    P(ct.c_long), ct.c_void_p]
    L.glv_binary_header.argtypes = [ct.c_char_p, P(ct.c_long), P(ct.c_long), P(ct.c_long)]
    L.glv_load_binary.argtypes = [ct.c_char_p, P(GlvGraph)]
    L.glv_write_binary.argtypes = [P(GlvGraph), ct.c_char_p, ct.c_long]
    L.glv_dev_load_binary.argtypes = [ct.c_char_p, ct.c_long, ct.c_long, ct.c_void_p, ct.c_void_p,
                                      ct.c_void_p, ct.c_void_p]
    L.glv_compare_communities.argtypes = [P(ct.c_long), ct.c_long, P(ct.c_long), ct.c_long,
                                          P(GlvComparison)]
    L.glv_dev_compare_communities.argtypes = [ct.c_long, ct.c_void_p, ct.c_void_p,
                                              P(GlvComparison), ct.c_void_p]
    L.glv_gini_coefficient.argtypes = [P(ct.c_long), ct.c_int, P(ct.c_double)]
    L.glv_vbase_redistribution.argtypes = [P(GlvGraph), P(ct.c_int), ct.c_int, ct.c_int,
                                           P(ct.c_long)]
    L.glv_renumber_clusters.argtypes = [P(ct.c_long), ct.c_long, P(ct.c_long)]
    L.glv_build_next_level.argtypes = [P(GlvGraph), P(GlvGraph), P(ct.c_long), ct.c_long,
                                       ct.c_int, P(ct.c_double)]
    L.glv_modularity.argtypes = [P(GlvGraph), P(ct.c_long), P(ct.c_double)]
    L.glv_vertex_following.argtypes = [P(GlvGraph), P(ct.c_long), P(ct.c_long)]
    L.glv_build_new_graph_vf.argtypes = [P(GlvGraph), P(GlvGraph), P(ct.c_long), ct.c_long,
                                         P(ct.c_double)]
    L.glv_decide_batch.argtypes = [ct.c_long, P(ct.c_long), P(ct.c_long), P(ct.c_double),
                                   P(ct.c_long), P(ct.c_double), P(ct.c_double), P(ct.c_long),
                                   ct.c_double, ct.c_long, P(ct.c_long), P(ct.c_long)]
    L.glv_dev_modularity_static.argtypes = [ct.c_long, ct.c_void_p, ct.c_void_p, ct.c_void_p,
                                            ct.c_void_p, ct.c_void_p, ct.c_double, ct.c_void_p,
                                            ct.c_void_p]
    L.glv_run_batch_csr.argtypes = [ct.c_int, P(ct.c_long), P(ct.c_long), P(ct.c_long),
                                    P(ct.c_double), P(ct.c_long), ct.c_int, ct.c_long,
                                    ct.c_double, ct.c_double, ct.c_int, P(GlvBatchStats)]
    L.glv_dev_run_batch.argtypes = [ct.c_int, P(ct.c_long), ct.c_void_p, ct.c_void_p,
                                    ct.c_void_p, ct.c_void_p, ct.c_int, ct.c_long, ct.c_double,
                                    ct.c_double, ct.c_int, ct.c_void_p, P(GlvBatchStats)]
    fp = P(ct.c_float)
    L.glv_gate_set.argtypes = [fp, ct.c_float]
    L.glv_gate_infer.argtypes = [ct.c_long, ct.c_void_p, ct.c_void_p, ct.c_void_p]
    L.glv_gate_grad.argtypes = [ct.c_long, fp, fp, fp, fp, fp, P(ct.c_double)]
    L.glv_gate_train.argtypes = [ct.c_long, fp, fp, fp, ct.c_int, ct.c_long, ct.c_float,
                                 ct.c_uint, fp, P(ct.c_double)]
    L.glv_trace_begin.argtypes = [ct.c_long, ct.c_double]
    L.glv_trace_fetch.restype = ct.c_long
    L.glv_trace_fetch.argtypes = [fp, fp, ct.c_long]
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != GLV_OK:
        raise GrappoloError(rc, lib().glv_last_error().decode(errors='replace'))
