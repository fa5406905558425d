#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace glv {

// Batches of independent graphs in one level.
//
// The graphs of a batch are laid end to end as one level (their disjoint
// union): graph g owns the vertex range [voff[g], voff[g+1]).  No edge joins
// two graphs, so colour classes, communities, renumbering and coarsening never
// mix them, and one persistent launch per iteration sweeps every graph that is
// still moving.  What is per graph: the modularity constant 1/(2m_g) used by
// the gains, the modularity sums, the phase loop's tests and its state
// (Coloring/runMultiPhaseColoring.cpp:51-238 run graph by graph).  A graph
// that converges inside a phase is skipped whole (its vertices stay), a graph
// whose run has finished drops out of the next level.
//
// Kernels of batch levels; the Engine's batch loop is in batch.cuh.

// skip[v] = 1 when v's graph is not sweeping.
__global__ void k_graph_skip(int64_t nv, const int32_t *gid, const uint8_t *act, uint8_t *skip) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    skip[v] = act[gid[v]] ? 0 : 1;
}

// past <- curr <- target for the graphs still sweeping (Jacobi phases).
__global__ void k_rotate_active(int64_t nv, const int32_t *gid, const uint8_t *act,
                                int32_t *past, int32_t *curr, const int32_t *tgt) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    if (!act[gid[v]]) continue;
    past[v] = curr[v];
    curr[v] = tgt[v];
  }
}

// gid[v] = g for v in [voff[g], voff[g+1]); one block row per graph.
__global__ void k_fill_gid(int G, const int64_t *voff, int32_t *gid) {
  for (int g = blockIdx.x; g < G; g += gridDim.x)
    for (int64_t v = voff[g] + threadIdx.x; v < voff[g + 1]; v += blockDim.x) gid[v] = g;
}

// Per-graph sums of vertex degrees: contiguous vertex ranges per block, a
// running sum per thread added to its graph's slot when the graph changes.
__global__ void k_graph_degsum(int64_t nv, const int32_t *gid, const double *vDeg, double *gsum) {
  const int64_t b = nv * blockIdx.x / gridDim.x, e = nv * (blockIdx.x + 1) / gridDim.x;
  int32_t cur = -1;
  double acc = 0.0;
  for (int64_t v = b + threadIdx.x; v < e; v += blockDim.x) {
    const int32_t g = gid[v];
    if (g != cur) {
      if (cur >= 0 && acc != 0.0) atomicAdd(&gsum[cur], acc);
      cur = g;
      acc = 0.0;
    }
    acc = __dadd_rn(acc, vDeg[v]);
  }
  if (cur >= 0 && acc != 0.0) atomicAdd(&gsum[cur], acc);
}

// 1/(2m_g) (Utility/utilityClusteringFunctions.cpp:89-96, graph by graph).
__global__ void k_graph_cst(int G, const double *gsum, double *gcst) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x)
    gcst[g] = 1.0 / gsum[g];
}

// cl_end[g] = 1 + the largest renumbered community id in graph g.
__global__ void k_graph_cluster_end(int64_t nv, const int32_t *gid, const int32_t *C,
                                    int32_t *cl_end) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = C[v];
    if (c >= 0) atomicMax(&cl_end[gid[v]], c + 1);
  }
}

// C_orig of every graph that took part in the phase, in graph-local ids
// (k_compose graph by graph; a graph still in its first phase has never been
// coarsened, so its level vertices are its original ones).
__global__ void k_compose_batch(int64_t n_orig, const int32_t *gid_orig, const int64_t *orig_off,
                                const int64_t *lvl_off, const int32_t *cl_off,
                                const uint8_t *took_part, const uint8_t *first, const int32_t *C,
                                int32_t *C_orig) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n_orig;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t g = gid_orig[v];
    if (!took_part[g]) continue;
    int64_t u;
    if (first[g]) {
      u = lvl_off[g] + (v - orig_off[g]);
    } else {
      const int32_t y = C_orig[v];
      if (y < 0) continue;
      u = lvl_off[g] + y;
    }
    const int32_t x = C[u];
    C_orig[v] = (x < 0) ? -1 : x - cl_off[g];
  }
}

enum NextKind : uint8_t { NEXT_DONE = 0, NEXT_COARSEN = 1, NEXT_SAME = 2 };

// Community ids for building the next level: coarsening graphs map to their
// renumbered clusters, graphs that repeat the level (the switch to Jacobi
// phases) to themselves, finished graphs to -1 (they drop out).
__global__ void k_next_ids(int64_t nv, const int32_t *gid, const uint8_t *kind,
                           const int64_t *lvl_off, const int64_t *new_off, const int32_t *cl_off,
                           const int32_t *C, int32_t *C_next) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t g = gid[v];
    int32_t x = -1;
    if (kind[g] == NEXT_COARSEN) {
      const int32_t c = C[v];
      x = (c < 0) ? -1 : (int32_t)(new_off[g] + (c - cl_off[g]));
    } else if (kind[g] == NEXT_SAME) {
      x = (int32_t)(new_off[g] + (v - lvl_off[g]));
    }
    C_next[v] = x;
  }
}

// Colours of the next level: graphs recoloured keep color (already written),
// graphs on stale colours take the first entries of their previous range
// (Coloring/runMultiPhaseColoring.cpp:173), all others get colour 0.
__global__ void k_stale_colors(int64_t nv, const int32_t *gid, const uint8_t *how,
                               const int64_t *new_off, const int64_t *old_off,
                               const int32_t *old_color, int32_t *color) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t g = gid[v];
    if (how[g] == 1) continue;  // fresh colouring
    color[v] = (how[g] == 2) ? old_color[old_off[g] + (v - new_off[g])] : 0;
  }
}

// C[v] = saved[v] for the graphs flagged in `grp` (merges the colour-phase
// graphs' results back after the Jacobi graphs' phase reset the level).
__global__ void k_merge_group(int64_t nv, const int32_t *gid, const uint8_t *grp,
                              const int32_t *saved, int32_t *C) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    if (grp[gid[v]]) C[v] = saved[v];
}

// out[k] = ptr[idx[k]].
__global__ void k_gather_i64(int64_t n, const int64_t *idx, const int64_t *ptr, int64_t *out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    out[k] = ptr[idx[k]];
}

// A tail outside its row's graph sets *bad (input check of a batch).
__global__ void k_check_batch_tails(int64_t nv, const int64_t *ptr, const int32_t *tail,
                                    const int32_t *gid, const int64_t *voff, int32_t *bad) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t g = gid[v];
    const int64_t lo = voff[g], hi = voff[g + 1];
    for (int64_t j = ptr[v]; j < ptr[v + 1]; ++j) {
      const int32_t t = tail[j];
      if (t < lo || t >= hi) { atomicOr(bad, 1); break; }
    }
  }
}

}  // namespace glv
