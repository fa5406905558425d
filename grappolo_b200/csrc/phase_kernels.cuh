// Per-phase kernels around the sweep: degrees, modularity, colouring, the
// colour/bin schedule, community-total updates, renumbering and coarsening.
#pragma once

#include <cooperative_groups.h>

#include "glv_common.cuh"

namespace glv {

namespace cg = cooperative_groups;

// ---------------------------------------------------------------------------
// Phase init: vDeg = CSR-order row sums (Utility/utilityClusteringFunctions.cpp:70-87),
// cInfo = {1, vDeg}, C = identity (initCommAss, :98-104).  One thread per row
// keeps the reference's summation order.
__global__ void k_init_phase(int64_t nv, const int64_t *ptr, const double *w, double *vDeg,
                             double *cDeg, int32_t *cSize, int32_t *C, int32_t *C2) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    const int64_t e = ptr[v + 1];
    for (int64_t j = ptr[v]; j < e; ++j) s = __dadd_rn(s, w[j]);
    vDeg[v] = s;
    cDeg[v] = s;
    cSize[v] = 1;
    C[v] = (int32_t)v;
    if (C2) C2[v] = (int32_t)v;
  }
}

// Same results when every summation order is exact (integral weights) or when
// bit-exactness is not asked for: one warp per row (levels of long rows; see
// k_row_sums_tiles for levels of short ones).
__global__ void k_init_phase_warp(int64_t nv, const int64_t *ptr, const double *w, double *vDeg,
                                  double *cDeg, int32_t *cSize, int32_t *C, int32_t *C2) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = wid; v < nv; v += nw) {
    double s = 0.0;
    const int64_t e = ptr[v + 1];
    for (int64_t j = ptr[v] + lane; j < e; j += 32) s = __dadd_rn(s, w[j]);
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s = __dadd_rn(s, __shfl_xor_sync(FULL, s, off));
    if (lane == 0) {
      vDeg[v] = s;
      cDeg[v] = s;
      cSize[v] = 1;
      C[v] = (int32_t)v;
      if (C2) C2[v] = (int32_t)v;
    }
  }
}

// 1 / sequential sum (calConstantForSecondTerm, :89-96 at one thread).
__global__ void k_constant_sequential(int64_t n, const double *x, double *out) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s = __dadd_rn(s, x[i]);
  out[0] = __ddiv_rn(1.0, s);
  out[1] = s;
}

// Deterministic two-level reductions: blocks write partials, one block folds
// them in index order.
template <int BS>
__device__ __forceinline__ double block_sum(double x, double *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) x = __dadd_rn(x, __shfl_xor_sync(FULL, x, off));
  if (lane == 0) sh[warp] = x;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < BS / 32; ++k) r = __dadd_rn(r, sh[k]);
  __syncthreads();
  return r;  // valid in thread 0
}

__global__ void __launch_bounds__(256) k_sum_partials(int64_t n, const double *x, double *part) {
  __shared__ double sh[8];
  double s = 0.0;
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t b = (int64_t)blockIdx.x * per, e = min(n, b + per);
  for (int64_t i = b + threadIdx.x; i < e; i += blockDim.x) s = __dadd_rn(s, x[i]);
  s = block_sum<256>(s, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void k_constant_from_partials(int nparts, const double *part, double *out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < nparts; ++i) s = __dadd_rn(s, part[i]);
  out[0] = __ddiv_rn(1.0, s);
  out[1] = s;
}

// ---------------------------------------------------------------------------
// Modularity: e_xx = sum_i cWI[i], a2_x = sum_i cDeg[i]^2, Q = e_xx*c - a2_x*c*c
// (Coloring/parallelLouvainWithColoring.cpp:226-249,
//  BasicCommunitiesDetection/parallelLouvainMethod.cpp:247-255).
// Colour phases compute cWI[i] = sum_{j: C[tail]==C[i]} w here; Jacobi phases
// pass the per-vertex Counter[own] their sweep produced (own_w).
// Each block takes 256 consecutive vertices and walks their edges
// edge-parallel, so hub rows do not serialise one lane.
constexpr int kModVB = 256;

__global__ void __launch_bounds__(256) k_modularity_part(int64_t nv, const int64_t *ptr,
                                                         const int32_t *tail, const double *w,
                                                         const int32_t *C, const double *own_w,
                                                         const double *cDeg, double *part_e,
                                                         double *part_a) {
  __shared__ int64_t s_ptr[kModVB + 1];
  __shared__ int32_t s_c[kModVB];
  __shared__ double sh[8];
  const int64_t v0 = (int64_t)blockIdx.x * kModVB;
  const int64_t v1 = min(nv, v0 + kModVB);
  const int nvb = (int)(v1 - v0);
  double a2 = 0.0, ex = 0.0;
  if (threadIdx.x < nvb) {
    const double d = cDeg[v0 + threadIdx.x];
    a2 = __dmul_rn(d, d);
  }
  if (own_w) {
    if (threadIdx.x < nvb) ex = own_w[v0 + threadIdx.x];
  } else {
    for (int k = threadIdx.x; k <= nvb; k += blockDim.x) s_ptr[k] = ptr[v0 + k];
    for (int k = threadIdx.x; k < nvb; k += blockDim.x) s_c[k] = C[v0 + k];
    __syncthreads();
    const int64_t eb = s_ptr[0], ee = s_ptr[nvb];
    int h = 0;
    for (int64_t e = eb + threadIdx.x; e < ee; e += blockDim.x) {
      while (s_ptr[h + 1] <= e) ++h;
      // a vertex labelled -1 belongs to no community: its entries add nothing
      if (s_c[h] >= 0 && C[tail[e]] == s_c[h]) ex = __dadd_rn(ex, w[e]);
    }
  }
  ex = block_sum<256>(ex, sh);
  a2 = block_sum<256>(a2, sh);
  if (threadIdx.x == 0) { part_e[blockIdx.x] = ex; part_a[blockIdx.x] = a2; }
}

// Merge-path tiles.  The items of a level are its rows' entries interleaved
// with one "row end" per row (row i's entries come before its end), nv + nnz
// items in all; a tile is kMergeTile consecutive items.  A hub row is cut over
// many tiles and a run of empty rows costs one item each, so every tile has
// the same work whatever the degree distribution.
constexpr int kMergeTile = 4096;

__host__ __device__ inline int64_t merge_tiles(int64_t nv, int64_t nnz) {
  return (nv + nnz + kMergeTile - 1) / kMergeTile;
}

// split_row[t] = rows ended before item t * kMergeTile: the largest i in
// [0, nv] with ptr[i] + i <= d (ptr[i] + i is strictly increasing in i).
__global__ void k_merge_splits(int64_t nv, int64_t nnz, const int64_t *ptr, int64_t ntiles,
                               int64_t *split_row) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t d = min(t * (int64_t)kMergeTile, nv + nnz);
    int64_t lo = max((int64_t)0, d - nnz), hi = min(d, nv);
    while (lo < hi) {
      const int64_t mid = (lo + hi + 1) >> 1;
      if (ptr[mid] + mid <= d) lo = mid; else hi = mid - 1;
    }
    split_row[t] = lo;
  }
}

// Shared memory of one merge tile: row starts relative to the tile's first
// entry (clamped to [0, kMergeTile + 1]) and the rows' communities.
struct MergeSmem {
  int32_t off[kMergeTile + 2];
  int32_t comm[kMergeTile + 1];
};

// Row sums of w (vertex degrees) over merge-path tiles, for the parallel
// modes (any order of a row's additions): every entry is read once, with
// coalesced loads, instead of a warp walking each row.  A tile sums its
// entries per row (a segmented scan over each warp's entries, then one
// shared add per row and warp); a row wholly inside the tile is stored, a row that
// spans tiles gets each tile's part with an atomic add (vDeg must be zero on
// entry).  Launched with kRowSumThreads threads and sizeof(RowSumSmem) bytes.
constexpr int kRowSumThreads = 256;
struct RowSumSmem {
  double acc[kMergeTile + 1];
  int32_t off[kMergeTile + 2];
};

__global__ void __launch_bounds__(kRowSumThreads) k_row_sums_tiles(int64_t nv, int64_t nnz,
                                                                   const int64_t *ptr,
                                                                   const double *w,
                                                                   const int64_t *split_row,
                                                                   double *vDeg) {
  extern __shared__ unsigned char smem_raw[];
  RowSumSmem &sm = *reinterpret_cast<RowSumSmem *>(smem_raw);
  const int lane = threadIdx.x & 31;
  const int64_t ntiles = merge_tiles(nv, nnz);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t d0 = tile * (int64_t)kMergeTile;
    const int64_t d1 = min(d0 + (int64_t)kMergeTile, nv + nnz);
    const int64_t i0 = split_row[tile], i1 = split_row[tile + 1];
    const int64_t j0 = d0 - i0, j1 = d1 - i1;
    if (j1 <= j0) continue;  // only row ends: those rows are complete or zero (tile-uniform)
    // rows holding entries j0..j1-1: i0 .. ih
    const int64_t ih = min(i1, nv - 1);
    const int nr = (int)(ih - i0 + 1);
    for (int k = threadIdx.x; k <= nr; k += kRowSumThreads) {
      const int64_t r = ptr[i0 + k] - j0;
      sm.off[k] = (int32_t)max((int64_t)0, min(r, (int64_t)kMergeTile + 1));
      if (k < nr) sm.acc[k] = 0.0;
    }
    __syncthreads();
    const int ne = (int)(j1 - j0);
    for (int q0 = 0; q0 < ne; q0 += kRowSumThreads) {  // ne is the tile's: warp-uniform
      const int q = q0 + (int)threadIdx.x;
      const bool has = q < ne;
      int lo = 0;
      double x = 0.0;
      if (has) {
        int hi = nr - 1;  // the last row starting at or before q
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sm.off[mid] <= q) lo = mid; else hi = mid - 1;
        }
        x = w[j0 + q];
      }
      // the warp's entries come in row order: a segmented inclusive scan
      // leaves each row's warp sum in its last lane
      const int key = has ? lo : -1 - lane;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const double y = __shfl_up_sync(FULL, x, off);
        const int ky = __shfl_up_sync(FULL, key, off);
        if (lane >= off && ky == key) x += y;
      }
      const int knext = __shfl_down_sync(FULL, key, 1);
      if (has && (lane == 31 || knext != key)) atomicAdd(&sm.acc[lo], x);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nr; k += kRowSumThreads) {
      const int64_t i = i0 + k;
      const bool whole = ptr[i] >= j0 && i < i1;  // starts and ends in this tile
      if (whole) vDeg[i] = sm.acc[k];
      else if (sm.acc[k] != 0.0) atomicAdd(&vDeg[i], sm.acc[k]);
    }
    __syncthreads();  // the next tile reuses the shared arrays
  }
}

// The singleton state of a phase from the degrees in vDeg.
__global__ void k_init_phase_fill(int64_t nv, const double *vDeg, double *cDeg, int32_t *cSize,
                                  int32_t *C, int32_t *C2) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    cDeg[v] = vDeg[v];
    cSize[v] = 1;
    C[v] = (int32_t)v;
    if (C2) C2[v] = (int32_t)v;
  }
}

// Modularity partials of merge tile `tile` added to (ex, a2): a2 over the rows
// that end in the tile, ex over its entries whose two ends share a community
// (colour phases) or the rows' own_w (Jacobi phases).  All NT threads call.
template <int NT>
__device__ __forceinline__ void modularity_merge_tile(int64_t tile, int64_t nv, int64_t nnz,
                                                      const int64_t *ptr, const int32_t *tail,
                                                      const double *w, const int32_t *C,
                                                      const double *own_w, const double *cDeg,
                                                      const int64_t *split_row, MergeSmem *sm,
                                                      double &ex, double &a2) {
  const int64_t d0 = tile * (int64_t)kMergeTile;
  const int64_t d1 = min(d0 + (int64_t)kMergeTile, nv + nnz);
  const int64_t i0 = split_row[tile], i1 = split_row[tile + 1];
  const int64_t j0 = d0 - i0, j1 = d1 - i1;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += NT) {
    const double dg = cDeg[i];
    a2 = __dadd_rn(a2, __dmul_rn(dg, dg));
    if (own_w) ex = __dadd_rn(ex, own_w[i]);
  }
  if (own_w || j1 <= j0) return;  // tile-uniform
  // rows holding entries j0..j1-1: i0 .. ih
  const int64_t ih = min(i1, nv - 1);
  const int nr = (int)(ih - i0 + 1);
  __syncthreads();  // the previous tile's readers are done
  for (int k = threadIdx.x; k <= nr; k += NT) {
    const int64_t r = ptr[i0 + k] - j0;
    sm->off[k] = (int32_t)max((int64_t)0, min(r, (int64_t)kMergeTile + 1));
  }
  for (int k = threadIdx.x; k < nr; k += NT) sm->comm[k] = C[i0 + k];
  __syncthreads();
  const int ne = (int)(j1 - j0);
#pragma unroll 4
  for (int q = threadIdx.x; q < ne; q += NT) {
    int lo = 0, hi = nr - 1;  // the last row starting at or before q
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sm->off[mid] <= q) lo = mid; else hi = mid - 1;
    }
    const int64_t e = j0 + q;
    if (C[tail[e]] == sm->comm[lo]) ex = __dadd_rn(ex, w[e]);
  }
}

// Batches of graphs: per-graph modularity sums {e_xx, a2_x} in gacc[2g],
// gacc[2g + 1].  A thread keeps one running pair and adds it to its graph's
// slots when the graph changes, so a contiguous tile range costs a few atomics
// per thread.
struct GraphAcc {
  int32_t g = -1;
  double e = 0.0, a = 0.0;
};

__device__ __forceinline__ void graph_acc_flush(GraphAcc &acc, double *gacc) {
  if (acc.g >= 0) {
    if (acc.e != 0.0) atomicAdd(&gacc[2 * acc.g], acc.e);
    if (acc.a != 0.0) atomicAdd(&gacc[2 * acc.g + 1], acc.a);
  }
  acc.e = 0.0;
  acc.a = 0.0;
}

__device__ __forceinline__ void graph_acc_add(GraphAcc &acc, int32_t g, double e, double a,
                                              double *gacc) {
  if (g != acc.g) {
    graph_acc_flush(acc, gacc);
    acc.g = g;
  }
  acc.e = __dadd_rn(acc.e, e);
  acc.a = __dadd_rn(acc.a, a);
}

template <int NT>
__device__ __forceinline__ void modularity_merge_tile_graphs(
    int64_t tile, int64_t nv, int64_t nnz, const int64_t *ptr, const int32_t *tail,
    const double *w, const int32_t *C, const double *own_w, const double *cDeg,
    const int64_t *split_row, const int32_t *gid, double *gacc, MergeSmem *sm, GraphAcc &acc) {
  const int64_t d0 = tile * (int64_t)kMergeTile;
  const int64_t d1 = min(d0 + (int64_t)kMergeTile, nv + nnz);
  const int64_t i0 = split_row[tile], i1 = split_row[tile + 1];
  const int64_t j0 = d0 - i0, j1 = d1 - i1;
  for (int64_t i = i0 + threadIdx.x; i < i1; i += NT) {
    const double dg = cDeg[i];
    graph_acc_add(acc, gid[i], own_w ? own_w[i] : 0.0, __dmul_rn(dg, dg), gacc);
  }
  if (own_w || j1 <= j0) return;  // tile-uniform
  const int64_t ih = min(i1, nv - 1);
  const int nr = (int)(ih - i0 + 1);
  __syncthreads();
  for (int k = threadIdx.x; k <= nr; k += NT) {
    const int64_t r = ptr[i0 + k] - j0;
    sm->off[k] = (int32_t)max((int64_t)0, min(r, (int64_t)kMergeTile + 1));
  }
  for (int k = threadIdx.x; k < nr; k += NT) sm->comm[k] = C[i0 + k];
  __syncthreads();
  const int ne = (int)(j1 - j0);
  for (int q = threadIdx.x; q < ne; q += NT) {
    int lo = 0, hi = nr - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sm->off[mid] <= q) lo = mid; else hi = mid - 1;
    }
    const int64_t e = j0 + q;
    if (C[tail[e]] == sm->comm[lo]) graph_acc_add(acc, gid[i0 + lo], w[e], 0.0, gacc);
  }
}

// Graph-of-launches form: each block folds the tiles blockIdx.x + k*gridDim.x
// and writes one partial pair.
__global__ void __launch_bounds__(256) k_modularity_merge(int64_t nv, int64_t nnz,
                                                          const int64_t *ptr, const int32_t *tail,
                                                          const double *w, const int32_t *C,
                                                          const double *own_w, const double *cDeg,
                                                          const int64_t *split_row,
                                                          double *part_e, double *part_a) {
  __shared__ MergeSmem sm;
  __shared__ double sh[8];
  double ex = 0.0, a2 = 0.0;
  const int64_t ntiles = merge_tiles(nv, nnz);
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x)
    modularity_merge_tile<256>(t, nv, nnz, ptr, tail, w, C, own_w, cDeg, split_row, &sm, ex, a2);
  ex = block_sum<256>(ex, sh);
  a2 = block_sum<256>(a2, sh);
  if (threadIdx.x == 0) { part_e[blockIdx.x] = ex; part_a[blockIdx.x] = a2; }
}

// The CSR entries (i -> t, i != t) whose two ends run in the same relaxed
// sweep step (step_of[i] == step_of[t] and relaxed[step_of[i]]), as member
// slots (pos_of) and weight, appended at *count up to `cap` (count keeps
// growing past cap, so the caller sees an overflow).  Merge-path tiles: hub
// rows spread over many blocks.
__global__ void __launch_bounds__(256) k_step_pairs(int64_t nv, int64_t nnz, const int64_t *ptr,
                                                    const int32_t *tail, const double *w,
                                                    const int32_t *step_of,
                                                    const uint8_t *relaxed,
                                                    const int32_t *pos_of,
                                                    const int64_t *split_row, int64_t cap,
                                                    int32_t *pu, int32_t *pt, double *pw,
                                                    unsigned long long *count) {
  __shared__ MergeSmem sm;
  const int64_t ntiles = merge_tiles(nv, nnz);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t d0 = tile * (int64_t)kMergeTile;
    const int64_t d1 = min(d0 + (int64_t)kMergeTile, nv + nnz);
    const int64_t i0 = split_row[tile], i1 = split_row[tile + 1];
    const int64_t j0 = d0 - i0, j1 = d1 - i1;
    if (j1 <= j0) continue;  // tile-uniform
    const int64_t ih = min(i1, nv - 1);
    const int nr = (int)(ih - i0 + 1);
    __syncthreads();
    for (int k = threadIdx.x; k <= nr; k += blockDim.x) {
      const int64_t r = ptr[i0 + k] - j0;
      sm.off[k] = (int32_t)max((int64_t)0, min(r, (int64_t)kMergeTile + 1));
    }
    // the row's step, or -1 when the step is an independent set
    for (int k = threadIdx.x; k < nr; k += blockDim.x) {
      const int32_t st = step_of[i0 + k];
      sm.comm[k] = (st >= 0 && relaxed[st]) ? st : -1;
    }
    __syncthreads();
    const int ne = (int)(j1 - j0);
    for (int q = threadIdx.x; q < ne; q += blockDim.x) {
      int lo = 0, hi = nr - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sm.off[mid] <= q) lo = mid; else hi = mid - 1;
      }
      const int32_t st = sm.comm[lo];
      if (st < 0) continue;
      const int64_t e = j0 + q;
      const int32_t t = tail[e];
      const int64_t i = i0 + lo;
      if (t == (int32_t)i || step_of[t] != st) continue;
      const unsigned long long k = atomicAdd(count, 1ull);
      if ((int64_t)k < cap) {
        pu[k] = pos_of[i];
        pt[k] = pos_of[t];
        pw[k] = w[e];
      }
    }
  }
}

// step_of[members[pos]] = the step (class) holding pos, pos_of[members[pos]] = pos.
__global__ void k_member_steps(int64_t nmem, const int32_t *members, int nclass,
                               const int64_t *cls_begin, int32_t *step_of, int32_t *pos_of) {
  for (int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < nmem;
       pos += (int64_t)gridDim.x * blockDim.x) {
    int lo = 0, hi = nclass - 1;  // last class starting at or before pos
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cls_begin[mid] <= pos) lo = mid; else hi = mid - 1;
    }
    const int32_t v = members[pos];
    step_of[v] = lo;
    pos_of[v] = (int32_t)pos;
  }
}

// out[0] = Q, out[1] = e_xx, out[2] = a2_x.  `cst` = {constant, 2m}.
__global__ void __launch_bounds__(256) k_modularity_final(int nparts, const double *part_e,
                                                          const double *part_a, const double *cst,
                                                          double *out) {
  __shared__ double sh[8];
  double e = 0.0, a = 0.0;
  const int per = (nparts + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per, en = min(nparts, b + per);
  for (int i = b; i < en; ++i) { e = __dadd_rn(e, part_e[i]); a = __dadd_rn(a, part_a[i]); }
  e = block_sum<256>(e, sh);
  a = block_sum<256>(a, sh);
  if (threadIdx.x == 0) {
    const double c = cst[0];
    out[0] = __dsub_rn(__dmul_rn(e, c), __dmul_rn(__dmul_rn(a, c), c));
    out[1] = e;
    out[2] = a;
  }
}

// ---------------------------------------------------------------------------
// Distance-1 colouring by priority order (Jones-Plassmann).  A vertex takes
// the smallest colour not used by its higher-priority neighbours once they are
// all coloured.  With priority "lower id first" this is exactly the
// sequential first-fit pass of Coloring/coloringDistanceOne.cpp:137-150 at one
// thread; with hashed priorities it is the parallel independent-set form.
// With `key` given, priority is (key, id): the iterated-greedy recolouring
// orders vertices by their previous colour class.
__device__ __forceinline__ bool prio_before(int32_t u, int32_t v, int hashed, uint32_t seed,
                                            const int32_t *key = nullptr) {
  if (key) {
    const int32_t ku = key[u], kv = key[v];
    return (ku < kv) || (ku == kv && u < v);
  }
  if (!hashed) return u < v;
  const uint32_t hu = mix32((uint32_t)u ^ seed), hv = mix32((uint32_t)v ^ seed);
  return (hu < hv) || (hu == hv && u < v);
}

__global__ void k_color_init(int64_t nv, const int64_t *ptr, const int32_t *tail, int hashed,
                             uint32_t seed, int32_t *pending, int32_t *color, int32_t *frontier,
                             int32_t *fcount, const int32_t *key) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    int32_t cnt = 0;
    for (int64_t j = ptr[v]; j < ptr[v + 1]; ++j) {
      const int32_t u = tail[j];
      if (u != (int32_t)v && prio_before(u, (int32_t)v, hashed, seed, key)) ++cnt;
    }
    pending[v] = cnt;
    color[v] = -1;
    if (cnt == 0) frontier[atomicAdd(fcount, 1)] = (int32_t)v;
  }
}

// Persistent cooperative kernel: one grid-wide barrier per round.  fcount has
// three counters used round-robin (read / push / reset).  Each round colours
// at least one vertex, so the loop ends after at most nv rounds.
__global__ void __launch_bounds__(256) k_color_rounds(int64_t nv, const int64_t *ptr,
                                                      const int32_t *tail, int hashed,
                                                      uint32_t seed, int32_t *pending,
                                                      int32_t *color, int32_t *front0,
                                                      int32_t *front1, int32_t *fcount,
                                                      int32_t *status, const int32_t *key) {
  cg::grid_group grid = cg::this_grid();
  __shared__ uint32_t bm[8][kMaxColors / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  uint32_t *mybm = bm[warp];
  for (int64_t round = 0; round <= nv; ++round) {
    int32_t *cur = (round & 1) ? front1 : front0;
    int32_t *nxt = (round & 1) ? front0 : front1;
    const int32_t n = *((volatile int32_t *)&fcount[round % 3]);
    if (n == 0) break;
    if (blockIdx.x == 0 && threadIdx.x == 0) fcount[(round + 2) % 3] = 0;
    for (int64_t k = wid; k < n; k += nw) {
      const int32_t v = cur[k];
      const int64_t rb = ptr[v], re = ptr[v + 1];
      const int64_t deg = re - rb;
      const int words = (int)((deg + 32) / 32 < kMaxColors / 32 ? (deg + 32) / 32 : kMaxColors / 32);
      for (int q = lane; q < words; q += 32) mybm[q] = 0u;
      __syncwarp();
      for (int64_t j = rb + lane; j < re; j += 32) {
        const int32_t u = tail[j];
        if (u != v && prio_before(u, v, hashed, seed, key)) {
          const int32_t cu = color[u];
          if (cu >= 0 && cu < words * 32) atomicOr(&mybm[cu >> 5], 1u << (cu & 31));
        }
      }
      __syncwarp();
      int first = INT32_MAX;
      for (int q = lane; q < words; q += 32) {
        const uint32_t free_bits = ~mybm[q];
        if (free_bits) { first = q * 32 + __ffs(free_bits) - 1; break; }
      }
      first = __reduce_min_sync(FULL, first);
      if (first == INT32_MAX) first = words * 32;  // all marked: next colour
      if (first >= kMaxColors) {
        if (lane == 0) atomicExch(status, 1);
        first = kMaxColors - 1;
      }
      if (lane == 0) color[v] = first;
      __syncwarp();
      for (int64_t j = rb + lane; j < re; j += 32) {
        const int32_t u = tail[j];
        if (u != v && prio_before(v, u, hashed, seed, key)) {
          if (atomicSub(&pending[u], 1) == 1) nxt[atomicAdd(&fcount[(round + 1) % 3], 1)] = u;
        }
      }
    }
    grid.sync();
  }
}

// Coloring/coloringMultiHashMaxMin.cpp:124-160: one (iteration, hash) pass of
// the incomplete max/min colouring.  An uncoloured vertex (colour maxColor)
// takes `cur` when its random value beats every neighbour not coloured in an
// earlier pass, `cur` + 1 when it is below all of them.  A neighbour coloured
// in this pass still compares (its colour is >= cur), so the outcome does not
// depend on the order of the vertices.  One warp per vertex.
__global__ void k_mhash_pass(int64_t nv, const int64_t *ptr, const int32_t *tail,
                             const double *rnd, int32_t *col, int32_t maxColor, int32_t cur,
                             unsigned long long *count) {
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t v = wid; v < nv; v += nw) {
    if (col[v] != maxColor) continue;  // warp-uniform
    const double rv = rnd[v];
    bool isMax = true, isMin = true;
    for (int64_t j = ptr[v] + lane; j < ptr[v + 1]; j += 32) {
      const int32_t u = tail[j];
      if (u == (int32_t)v) continue;
      if (col[u] < cur) continue;
      const double ru = rnd[u];
      if (rv <= ru) isMax = false;
      if (rv >= ru) isMin = false;
    }
    isMax = __all_sync(FULL, isMax);
    isMin = __all_sync(FULL, isMin);
    if (lane == 0 && (isMax || isMin)) {
      col[v] = isMax ? cur : cur + 1;
      atomicAdd(count, 1ull);
    }
  }
}

// key[v] = ncolors - 1 - color[v]: recolour the last class first (Culberson's
// reverse-class order; a greedy pass over whole classes never adds colours).
__global__ void k_reverse_class_key(int64_t nv, const int32_t *color, int32_t ncolors,
                                    int32_t *key) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    key[v] = ncolors - 1 - color[v];
}

// key[v] = map[color[v]]: colour classes relabelled as the sweep steps that
// run them (several classes may share a step).
__global__ void k_remap_colors(int64_t nv, const int32_t *color, const int32_t *map,
                               int32_t *key) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    key[v] = map[color[v]];
}

__global__ void k_max_color(int64_t nv, const int32_t *color, int32_t *out) {
  int32_t m = -1;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    m = max(m, color[v]);
  m = __reduce_max_sync(FULL, (unsigned)(m + 1)) - 1;
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

// ---------------------------------------------------------------------------
// Schedule: vertices sorted by key = (colour*nsub + sublevel)*NBINS + bin;
// a stable sort keeps ascending ids inside every (class, bin) segment.
__global__ void k_schedule_keys(int64_t nv, const int64_t *ptr, const int32_t *color,
                                const int32_t *sub, int nsub, BinLimits lim, int32_t *keys,
                                int32_t *vals, int32_t *hist) {
  // every lane of a warp takes each round, so equal keys of a round share one
  // histogram update (a few keys take most vertices)
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t v0 = (int64_t)blockIdx.x * blockDim.x; v0 < nv; v0 += stride) {
    const int64_t v = v0 + threadIdx.x;
    int k = -1;
    if (v < nv) {
      const int64_t deg = ptr[v + 1] - ptr[v];
      const int c = color ? color[v] : 0;
      const int s = sub ? sub[v] : 0;
      k = (c * nsub + s) * NBINS + degree_bin(deg, lim);
      keys[v] = k;
      vals[v] = (int32_t)v;
    }
    const unsigned m = __match_any_sync(FULL, k);
    if (k >= 0 && lane == __ffs(m) - 1) atomicAdd(&hist[k], __popc(m));
  }
}

// Per-member hub table offsets: prefix over table capacities within a class.
__global__ void k_hub_caps(int64_t n, const int32_t *members, const int64_t *ptr, int64_t *cap) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = members[k];
    cap[k] = table_cap(ptr[v + 1] - ptr[v]);
  }
}

// ---------------------------------------------------------------------------
// Community totals after a class (cInfo += cUpdate,
// parallelLouvainWithColoring.cpp:213-217).  Atomic form: the sweep already
// summed the deltas into dDeg/dSize; the first thread to claim a community's
// delta adds it to the totals and clears it.
__global__ void k_apply_deltas(int64_t begin, int64_t end, const int32_t *move_old,
                               const int32_t *move_new, double *dDeg, int32_t *dSize,
                               double *cDeg, int32_t *cSize) {
  for (int64_t pos = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < end;
       pos += (int64_t)gridDim.x * blockDim.x) {
    const int32_t o = move_old[pos];
    if (o < 0) continue;
    const int32_t cs[2] = {move_new[pos], o};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int32_t c = cs[k];
      // Each field is claimed separately, so exactly one thread writes it.
      const unsigned long long bits = atomicExch((unsigned long long *)&dDeg[c], 0ull);
      if (bits != 0ull) cDeg[c] = __dadd_rn(cDeg[c], __longlong_as_double((long long)bits));
      const int32_t s = atomicExch(&dSize[c], 0);
      if (s != 0) cSize[c] += s;
    }
  }
}

// Ordered form: one record per (community, vertex) delta, sorted by
// (community, vertex id), folded from 0.0 in member order as the reference's
// one-thread loop accumulates cUpdate.
struct DeltaRec {
  double d;
  int32_t s;
  int32_t pad;
};

__global__ void k_delta_records(int64_t begin, int64_t end, const int32_t *members,
                                const int32_t *move_old, const int32_t *move_new,
                                const double *vDeg, uint64_t sentinel, uint64_t *keys,
                                DeltaRec *recs) {
  for (int64_t pos = begin + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < end;
       pos += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = 2 * (pos - begin);
    const int32_t o = move_old[pos];
    if (o < 0) {
      keys[k] = sentinel; keys[k + 1] = sentinel;
      recs[k] = DeltaRec{0.0, 0, 0}; recs[k + 1] = DeltaRec{0.0, 0, 0};
      continue;
    }
    const int32_t v = members[pos];
    const int32_t n = move_new[pos];
    const double d = vDeg[v];
    keys[k] = ((uint64_t)(uint32_t)n << 32) | (uint32_t)v;
    recs[k] = DeltaRec{d, 1, 0};
    keys[k + 1] = ((uint64_t)(uint32_t)o << 32) | (uint32_t)v;
    recs[k + 1] = DeltaRec{-d, -1, 0};
  }
}

__global__ void k_fold_deltas(int64_t n, const uint64_t *keys, const DeltaRec *recs,
                              uint64_t sentinel, double *cDeg, int32_t *cSize) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t ki = keys[i];
    if (ki >= sentinel) continue;
    const uint32_t c = (uint32_t)(ki >> 32);
    if (i > 0 && (uint32_t)(keys[i - 1] >> 32) == c) continue;
    double s = 0.0;
    int32_t cnt = 0;
    for (int64_t j = i; j < n && keys[j] < sentinel && (uint32_t)(keys[j] >> 32) == c; ++j) {
      s = __dadd_rn(s, recs[j].d);
      cnt += recs[j].s;
    }
    cDeg[c] = __dadd_rn(cDeg[c], s);
    cSize[c] += cnt;
  }
}

// ---------------------------------------------------------------------------
// Renumbering by first occurrence (Utility/buildNextPhase.cpp:48-79):
// first[c] = min{i : C[i] = c}; position i opens a new id iff first[C[i]] == i;
// new ids are the exclusive prefix count of openings.
__global__ void k_fill_i32(int64_t n, int32_t *x, int32_t val) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = val;
}

__global__ void k_first_occurrence(int64_t n, const int32_t *C, int32_t *first) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = C[i];
    if (c >= 0) atomicMin(&first[c], (int32_t)i);
  }
}

__global__ void k_open_flags(int64_t n, const int32_t *C, const int32_t *first, int32_t *flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = C[i];
    flag[i] = (c >= 0 && first[c] == (int32_t)i) ? 1 : 0;
  }
}

__global__ void k_apply_renumber(int64_t n, int32_t *C, const int32_t *first,
                                 const int32_t *scan) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = C[i];
    if (c >= 0) C[i] = scan[first[c]];
  }
}

// C_orig composition (runMultiPhaseColoring.cpp:132-144).
__global__ void k_compose(int64_t n, int32_t *C_orig, const int32_t *C, int first_phase) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (first_phase) C_orig[i] = C[i];
    else if (C_orig[i] >= 0) C_orig[i] = C[C_orig[i]];
  }
}

// ---------------------------------------------------------------------------
// Coarsening (Utility/buildNextPhase.cpp:83-255).  Records: one seed (a, a,
// 0.0) per cluster, then one per CSR entry i->t with a = C[i] >= b = C[t] >= 0,
// in (i, j) order.  A stable radix sort by (a << nb) | b groups each pair with
// its entries still in (i, j) order.  The records are written in two passes
// over the merge tiles: k_coarse_tile_counts counts each tile's records, an
// exclusive scan places the tiles, and k_coarse_records_compact writes each
// tile's records at its place in entry order (the sort then moves about half
// as many records as one slot per entry would).
template <bool WRITE>
__device__ __forceinline__ void coarse_tile(int64_t tile, int64_t nv, int64_t nnz,
                                            const int64_t *ptr, const int32_t *tail,
                                            const double *w, const int32_t *C, int nb,
                                            const int64_t *split_row, MergeSmem *sm,
                                            int32_t *s_warp, uint64_t *keys, double *vals,
                                            int64_t base, int64_t *count) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  const int64_t d0 = tile * (int64_t)kMergeTile;
  const int64_t d1 = min(d0 + (int64_t)kMergeTile, nv + nnz);
  const int64_t i0 = split_row[tile], i1 = split_row[tile + 1];
  const int64_t j0 = d0 - i0, j1 = d1 - i1;
  int64_t kept = 0;
  if (j1 > j0) {  // tile-uniform
    const int64_t ih = min(i1, nv - 1);
    const int nr = (int)(ih - i0 + 1);
    __syncthreads();
    for (int k = threadIdx.x; k <= nr; k += blockDim.x) {
      const int64_t r = ptr[i0 + k] - j0;
      sm->off[k] = (int32_t)max((int64_t)0, min(r, (int64_t)kMergeTile + 1));
    }
    for (int k = threadIdx.x; k < nr; k += blockDim.x) sm->comm[k] = C[i0 + k];
    __syncthreads();
    const int ne = (int)(j1 - j0);
    for (int q0 = 0; q0 < ne; q0 += blockDim.x) {  // block-uniform rounds
      const int q = q0 + (int)threadIdx.x;
      bool keep = false;
      uint64_t key = 0;
      int64_t e = 0;
      if (q < ne) {
        int lo = 0, hi = nr - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sm->off[mid] <= q) lo = mid; else hi = mid - 1;
        }
        e = j0 + q;
        const int32_t a = sm->comm[lo];
        const int32_t b = C[tail[e]];
        keep = a >= b && b >= 0;
        key = ((uint64_t)a << nb) | (uint64_t)(uint32_t)b;
      }
      const unsigned m = __ballot_sync(FULL, keep);
      if (WRITE) {
        // place of this round's records: warps in order, lanes in order
        if (lane == 0) s_warp[warp] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
        for (int k = 0; k < nwb; ++k) {
          const int c = s_warp[k];
          if (k < warp) before += c;
          total += c;
        }
        if (keep) {
          const int64_t at = base + kept + before + __popc(m & ((1u << lane) - 1u));
          keys[at] = key;
          vals[at] = w[e];
        }
        kept += total;
        __syncthreads();
      } else {
        kept += __popc(m);  // per warp; summed over warps below
      }
    }
  }
  if (!WRITE) {
    if (lane == 0) s_warp[warp] = (int32_t)kept;
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t t = 0;
      for (int k = 0; k < nwb; ++k) t += s_warp[k];
      count[tile] = t;
    }
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_coarse_tile_counts(
    int64_t nv, int64_t nnz, const int64_t *ptr, const int32_t *tail, const int32_t *C, int nb,
    const int64_t *split_row, int64_t *count) {
  __shared__ MergeSmem sm;
  __shared__ int32_t s_warp[32];
  const int64_t ntiles = merge_tiles(nv, nnz);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    coarse_tile<false>(tile, nv, nnz, ptr, tail, nullptr, C, nb, split_row, &sm, s_warp, nullptr,
                       nullptr, 0, count);
}

// Seeds (a, a, 0.0) in slots 0..ncl-1, then every tile's records from
// ncl + tile_off[tile].
__global__ void __launch_bounds__(256) k_coarse_records_compact(
    int64_t nv, int64_t nnz, const int64_t *ptr, const int32_t *tail, const double *w,
    const int32_t *C, int64_t ncl, int nb, const int64_t *split_row, const int64_t *tile_off,
    uint64_t *keys, double *vals) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < ncl;
       a += (int64_t)gridDim.x * blockDim.x) {
    keys[a] = ((uint64_t)a << nb) | (uint64_t)a;
    vals[a] = 0.0;
  }
  __shared__ MergeSmem sm;
  __shared__ int32_t s_warp[32];
  const int64_t ntiles = merge_tiles(nv, nnz);
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
    coarse_tile<true>(tile, nv, nnz, ptr, tail, w, C, nb, split_row, &sm, s_warp, keys, vals,
                      ncl + tile_off[tile], nullptr);
}

// Segment heads of the sorted records -> flags (1 at the first record of each
// distinct key, sentinel excluded).
__global__ void k_segment_heads(int64_t n, const uint64_t *keys, uint64_t sentinel,
                                int32_t *flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    flag[i] = (k < sentinel && (i == 0 || keys[i - 1] != k)) ? 1 : 0;
  }
}

// Fold each pair's records in order (one thread per pair): the reference's
// map entry starts at the first weight (or 0.0 for the self seed) and adds
// the rest in (i, j) order.
__global__ void k_fold_pairs(int64_t n, const uint64_t *keys, const double *vals,
                             const int32_t *flag, const int64_t *uidx, uint64_t sentinel,
                             uint64_t *ukeys, double *uvals) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    const uint64_t k = keys[i];
    double s = vals[i];
    for (int64_t j = i + 1; j < n && keys[j] == k; ++j) s = __dadd_rn(s, vals[j]);
    const int64_t u = uidx[i];
    ukeys[u] = k;
    uvals[u] = s;
  }
}

// Atomic form for FAST mode: every record adds into its pair's slot.
__global__ void k_scatter_pairs(int64_t n, const uint64_t *keys, const double *vals,
                                const int32_t *flag, const int64_t *uidx, uint64_t sentinel,
                                uint64_t *ukeys, double *uvals) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    if (k >= sentinel) continue;
    const int64_t u = uidx[i] - (flag[i] ? 0 : 1);
    if (flag[i]) ukeys[u] = k;
    atomicAdd(&uvals[u], vals[i]);
  }
}

// Row sizes of the coarse CSR: pair (a, b) counts once in row a and, when
// a > b, once more in row b (buildNextPhase.cpp:157-170).
__global__ void k_row_counts(int64_t np, const uint64_t *ukeys, int nb, int64_t *lower_cnt,
                             int64_t *upper_cnt, int64_t *ne_off) {
  const uint64_t mask = (1ull << nb) - 1;
  const int lane = threadIdx.x & 31;
  unsigned long long off_diag = 0;  // this thread's pairs with a > b
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = (int64_t)(ukeys[p] >> nb), b = (int64_t)(ukeys[p] & mask);
    atomicAdd((unsigned long long *)&lower_cnt[a], 1ull);
    if (a > b) {
      atomicAdd((unsigned long long *)&upper_cnt[b], 1ull);
      ++off_diag;
    }
  }
  // one counter update per warp (a single counter for every pair serialised them)
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) off_diag += __shfl_xor_sync(FULL, off_diag, off);
  if (lane == 0 && off_diag) atomicAdd((unsigned long long *)ne_off, off_diag);
}

// Lower part of each row: pairs (a, b <= a) in ascending b.  Pairs are sorted
// by (a, b), so a pair's rank inside row a is p - first pair of a; also emits
// the transposed key (b << nb) | a of every off-diagonal pair for the mirror.
// The transposed keys come in ascending a for each b, so a stable sort of
// their b bits alone orders them by (b, a).
__global__ void k_emit_lower(int64_t np, const uint64_t *ukeys, const double *uvals, int nb,
                             const int64_t *row_ptr, const int64_t *lower_first,
                             int32_t *otail, double *ow, uint64_t *tkeys, double *tvals,
                             uint64_t sentinel) {
  const uint64_t mask = (1ull << nb) - 1;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = (int64_t)(ukeys[p] >> nb), b = (int64_t)(ukeys[p] & mask);
    const int64_t at = row_ptr[a] + (p - lower_first[a]);
    otail[at] = (int32_t)b;
    ow[at] = uvals[p];
    if (a > b) {
      tkeys[p] = ((uint64_t)b << nb) | (uint64_t)a;
      tvals[p] = uvals[p];
    } else {
      tkeys[p] = sentinel;
      tvals[p] = 0.0;
    }
  }
}

// Mirrored part: transposed pairs sorted by (b, a) land after row b's lower
// part, in ascending a (the order cluster a emits them at one thread,
// buildNextPhase.cpp:205-223).
__global__ void k_emit_upper(int64_t np, const uint64_t *tkeys, const double *tvals, int nb,
                             const int64_t *row_ptr, const int64_t *lower_cnt,
                             const int64_t *upper_first, int32_t *otail, double *ow,
                             uint64_t sentinel) {
  const uint64_t mask = (1ull << nb) - 1;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < np;
       q += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = tkeys[q];
    if (k >= sentinel) continue;
    const int64_t b = (int64_t)(k >> nb), a = (int64_t)(k & mask);
    const int64_t at = row_ptr[b] + lower_cnt[b] + (q - upper_first[b]);
    otail[at] = (int32_t)a;
    ow[at] = tvals[q];
  }
}

// first index of each row's run in a sorted key array (keys >> shift = row).
__global__ void k_run_first(int64_t n, const uint64_t *keys, int shift, uint64_t sentinel,
                            int64_t *first) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    if (k >= sentinel) continue;
    const uint64_t r = k >> shift;
    if (i == 0 || (keys[i - 1] >> shift) != r) first[r] = i;
  }
}

}  // namespace glv

namespace glv {

// ---------------------------------------------------------------------------
// Fast-mode colouring: speculative first-fit with priority conflict
// resolution (the parallel form of Coloring/coloringDistanceOne.cpp:129-188,
// with hashed priorities in place of its RngStream values).  Each round every
// uncoloured vertex takes the smallest colour not seen on its neighbours;
// then a vertex that shares its colour with a higher-priority neighbour gives
// it up and joins the next round.  The highest-priority vertex of every
// conflict keeps its colour, so each round colours at least one vertex.

// First free colour over the neighbours of v (self-loops skipped); `bm` is a
// bitmap of kMaxColors bits shared by the `team` threads calling this.
template <int TEAM>
__device__ __forceinline__ int first_free_color(const int64_t *ptr, const int32_t *tail,
                                                const int32_t *color, int32_t v, uint32_t *bm,
                                                int tid) {
  const int64_t rb = ptr[v], re = ptr[v + 1];
  const int64_t deg = re - rb;
  const int words = (int)((deg + 32) / 32 < kMaxColors / 32 ? (deg + 32) / 32 : kMaxColors / 32);
  for (int q = tid; q < words; q += TEAM) bm[q] = 0u;
  if (TEAM == 32) __syncwarp(); else __syncthreads();
  for (int64_t j = rb + tid; j < re; j += TEAM) {
    const int32_t u = tail[j];
    if (u != v) {
      const int32_t cu = color[u];
      if (cu >= 0 && cu < words * 32) atomicOr(&bm[cu >> 5], 1u << (cu & 31));
    }
  }
  if (TEAM == 32) __syncwarp(); else __syncthreads();
  int first = INT32_MAX;
  for (int q = tid; q < words; q += TEAM) {
    const uint32_t free_bits = ~bm[q];
    if (free_bits) { first = q * 32 + __ffs(free_bits) - 1; break; }
  }
  return first;  // per-thread candidate; caller reduces (min)
}

// Warp per vertex (rows below kSpecBlockDeg entries).
// List lengths come from device counters, so rounds run back to back without
// the host reading them.
__global__ void __launch_bounds__(256) k_spec_assign_warp(const int32_t *count,
                                                          const int32_t *list,
                                                          const int64_t *ptr, const int32_t *tail,
                                                          int32_t *color, int32_t *status) {
  __shared__ uint32_t bm[8][kMaxColors / 32];
  const int64_t n = *count;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = wid; k < n; k += nw) {
    const int32_t v = list[k];
    int first = first_free_color<32>(ptr, tail, color, v, bm[warp], lane);
    first = __reduce_min_sync(FULL, first);
    if (first == INT32_MAX) {
      const int64_t deg = ptr[v + 1] - ptr[v];
      first = (int)((deg + 32) / 32 < kMaxColors / 32 ? (deg + 32) / 32 : kMaxColors / 32) * 32;
    }
    if (first >= kMaxColors) {
      if (lane == 0) atomicExch(status, 1);
      first = kMaxColors - 1;
    }
    if (lane == 0) color[v] = first;
    __syncwarp();
  }
}

// Block per vertex (hubs).
__global__ void __launch_bounds__(512) k_spec_assign_block(const int32_t *count,
                                                           const int32_t *list,
                                                           const int64_t *ptr,
                                                           const int32_t *tail, int32_t *color,
                                                           int32_t *status) {
  __shared__ uint32_t bm[kMaxColors / 32];
  __shared__ int s_min[16];
  const int64_t n = *count;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t k = blockIdx.x; k < n; k += gridDim.x) {
    const int32_t v = list[k];
    int first = first_free_color<512>(ptr, tail, color, v, bm, threadIdx.x);
    first = __reduce_min_sync(FULL, first);
    if (lane == 0) s_min[warp] = first;
    __syncthreads();
    if (threadIdx.x == 0) {
      int f = s_min[0];
      for (int q = 1; q < 16; ++q) f = min(f, s_min[q]);
      if (f == INT32_MAX) {
        const int64_t deg = ptr[v + 1] - ptr[v];
        f = (int)((deg + 32) / 32 < kMaxColors / 32 ? (deg + 32) / 32 : kMaxColors / 32) * 32;
      }
      if (f >= kMaxColors) { atomicExch(status, 1); f = kMaxColors - 1; }
      color[v] = f;
    }
    __syncthreads();
  }
}

// Conflict priority of the speculative colouring: larger degree first (the
// dense core of a skewed graph settles early, which keeps the colour count
// near the largest-first greedy one), then a hash of the id, then the id.
__device__ __forceinline__ bool spec_wins(int32_t u, int32_t v, const int64_t *ptr,
                                          uint32_t seed) {
  const int64_t du = ptr[u + 1] - ptr[u], dv = ptr[v + 1] - ptr[v];
  if (du != dv) return du > dv;
  return prio_before(v, u, 1, seed);
}

// A vertex that shares its colour with a higher-priority neighbour resets
// and goes to the next round's list.  Warp per vertex.
__global__ void __launch_bounds__(256) k_spec_conflicts(const int32_t *count, const int32_t *list,
                                                        const int64_t *ptr, const int32_t *tail,
                                                        uint32_t seed, int32_t *color,
                                                        int32_t *next, int32_t *next_count) {
  const int lane = threadIdx.x & 31;
  const int64_t n = *count;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = wid; k < n; k += nw) {
    const int32_t v = list[k];
    const int32_t cv = color[v];
    bool lose = false;
    for (int64_t j = ptr[v] + lane; j < ptr[v + 1] && !lose; j += 32) {
      const int32_t u = tail[j];
      if (u != v && color[u] == cv && spec_wins(u, v, ptr, seed)) lose = true;
    }
    if (__any_sync(FULL, lose) && lane == 0) {
      color[v] = -1;
      next[atomicAdd(next_count, 1)] = v;
    }
  }
}

// Same, one block per vertex (rows of at least kSpecBlockDeg entries).
__global__ void __launch_bounds__(512) k_spec_conflicts_block(const int32_t *count,
                                                              const int32_t *list,
                                                              const int64_t *ptr,
                                                              const int32_t *tail, uint32_t seed,
                                                              int32_t *color, int32_t *next,
                                                              int32_t *next_count) {
  __shared__ int s_lose;
  const int64_t n = *count;
  for (int64_t k = blockIdx.x; k < n; k += gridDim.x) {
    const int32_t v = list[k];
    if (threadIdx.x == 0) s_lose = 0;
    __syncthreads();
    const int32_t cv = color[v];
    for (int64_t j = ptr[v] + threadIdx.x; j < ptr[v + 1]; j += blockDim.x) {
      if (*((volatile int *)&s_lose)) break;
      const int32_t u = tail[j];
      if (u != v && color[u] == cv && spec_wins(u, v, ptr, seed)) s_lose = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0 && s_lose) {
      color[v] = -1;
      next[atomicAdd(next_count, 1)] = v;
    }
    __syncthreads();
  }
}

// Initial lists: rows with no neighbour but themselves take colour 0; the
// rest go to the warp or block list by degree.  Rows of at least `core_deg`
// entries (the core, swept in batches) take kCoreColor and stay out of the
// lists: no other vertex sees them (their colour is negative), so the
// colouring covers only the graph without the core.
constexpr int32_t kCoreColor = -2;
__global__ void k_spec_init(int64_t nv, const int64_t *ptr, const int32_t *tail,
                            int64_t block_deg, int64_t core_deg, int32_t *color, int32_t *wl,
                            int32_t *wcount, int32_t *bl, int32_t *bcount,
                            unsigned long long *ncore) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int64_t rb = ptr[v], re = ptr[v + 1];
    if (re - rb >= core_deg) {
      color[v] = kCoreColor;
      atomicAdd(ncore, 1ull);
      continue;
    }
    bool any = false;
    for (int64_t j = rb; j < re && !any; ++j) any = tail[j] != (int32_t)v;
    color[v] = any ? -1 : 0;
    if (!any) continue;
    if (re - rb >= block_deg) bl[atomicAdd(bcount, 1)] = (int32_t)v;
    else wl[atomicAdd(wcount, 1)] = (int32_t)v;
  }
}

// Core vertices join one of `nbatch` classes after the `base` colours of the
// rest, by a hash of the id (balanced in expectation, the same on every run).
__global__ void k_core_batches(int64_t nv, int32_t base, int32_t nbatch, int32_t *color) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    if (color[v] == kCoreColor) color[v] = base + (int32_t)(mix32((uint32_t)v) % (uint32_t)nbatch);
}

// Split a list by degree (next round's lists).
__global__ void k_spec_split(const int32_t *count, const int32_t *list, const int64_t *ptr,
                             int64_t block_deg, int32_t *wl, int32_t *wcount, int32_t *bl,
                             int32_t *bcount) {
  const int64_t n = *count;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = list[k];
    if (ptr[v + 1] - ptr[v] >= block_deg) bl[atomicAdd(bcount, 1)] = v;
    else wl[atomicAdd(wcount, 1)] = v;
  }
}

// ---------------------------------------------------------------------------
// Chunked coarsening (large levels outside verify mode): every CSR entry
// i -> t with a = C[i] in [a0, a1) and b = C[t] >= 0 becomes one record
// ((a - a0) << nb | b, w), plus a seed (a, a, 0.0) per community.  Sorting
// and summing the records of a chunk gives its coarse rows whole (both
// directions come from the symmetric input), in (a, b) order, so the chunks'
// outputs laid end to end are the coarse CSR.  Equal to the two-sort path in
// exact arithmetic (integral weights); the order of additions differs.

// cnt[a] = 1 (its seed) + the entries of the rows in community a.
__global__ void k_comm_entry_counts(int64_t nv, const int64_t *ptr, const int32_t *C,
                                    int64_t *cnt) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t a = C[v];
    const int64_t d = ptr[v + 1] - ptr[v];
    if (a >= 0 && d > 0) atomicAdd((unsigned long long *)&cnt[a], (unsigned long long)d);
  }
}

__global__ void k_fill_i64(int64_t n, int64_t *x, int64_t val) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] = val;
}

// bounds[k] = the first community whose record prefix reaches k * total / K.
__global__ void k_chunk_bounds(int64_t ncl, const int64_t *prefix, int K, int64_t *bounds) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > K) return;
  const int64_t total = prefix[ncl];
  const int64_t target = (int64_t)((double)total * k / K);
  int64_t lo = 0, hi = ncl;  // smallest a with prefix[a] >= target
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (prefix[mid] >= target) hi = mid; else lo = mid + 1;
  }
  bounds[k] = (k == K) ? ncl : lo;
}

// Shared memory of one tile of the community-ordered rows: row starts
// relative to the tile's first entry, the rows' communities and their first
// entries in the CSR.
struct PermTileSmem {
  int32_t off[kMergeTile + 2];
  int32_t comm[kMergeTile + 1];
  int64_t base[kMergeTile + 1];
};

// Records of the chunk [a0, a1) (merge-path tiles, warp-aggregated slots).
// The tiles run over the level's rows in community order: row r of that
// order is vertex perm[r], its entries start at pptr[r] in the order's
// numbering and at ptr[perm[r]] in the CSR, so the rows of a chunk are a
// contiguous run of tiles.  Only tiles [t0, t1) are read (the chunk's run, or
// a slice of it when its records exceed the buffer); seeds come with the
// slice that has `seeds` set; records past `cap` are counted but not written
// (the caller then cuts the slice finer).  Dynamic shared memory:
// sizeof(PermTileSmem).
__global__ void __launch_bounds__(256) k_chunk_records(
    int64_t nv, int64_t nnz, const int64_t *ptr, const int32_t *tail, const double *w,
    const int32_t *C, const int32_t *perm, const int64_t *pptr, const int64_t *split_row,
    int32_t a0, int32_t a1, int nb, int64_t t0, int64_t t1, int seeds, int trunc,
    unsigned long long cap, unsigned long long *counter, uint64_t *keys, double *vals) {
  extern __shared__ unsigned char dsm_raw[];
  PermTileSmem &sm = *reinterpret_cast<PermTileSmem *>(dsm_raw);
  const int lane = threadIdx.x & 31;
  if (seeds) {
    for (int64_t a = a0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < a1;
         a += (int64_t)gridDim.x * blockDim.x) {
      const unsigned long long s = atomicAdd(counter, 1ull);
      if (s < cap) {
        keys[s] = ((uint64_t)(a - a0) << nb) | (uint64_t)a;
        vals[s] = 0.0;
      }
    }
  }
  for (int64_t tile = t0 + blockIdx.x; tile < t1; tile += gridDim.x) {
    const int64_t d0 = tile * (int64_t)kMergeTile;
    const int64_t d1 = min(d0 + (int64_t)kMergeTile, nv + nnz);
    const int64_t i0 = split_row[tile], i1 = split_row[tile + 1];
    const int64_t j0 = d0 - i0, j1 = d1 - i1;
    if (j1 <= j0) continue;  // tile-uniform
    const int64_t ih = min(i1, nv - 1);
    const int nr = (int)(ih - i0 + 1);
    __syncthreads();
    for (int k = threadIdx.x; k <= nr; k += blockDim.x) {
      const int64_t r = pptr[i0 + k] - j0;
      sm.off[k] = (int32_t)max((int64_t)0, min(r, (int64_t)kMergeTile + 1));
    }
    for (int k = threadIdx.x; k < nr; k += blockDim.x) {
      const int32_t v = perm[i0 + k];
      sm.comm[k] = C[v];
      sm.base[k] = ptr[v] - pptr[i0 + k];
    }
    __syncthreads();
    const int ne = (int)(j1 - j0);
    // every lane of a warp runs the same trip count, so the ballot sees them all
    const int trips = (ne + blockDim.x - 1) / blockDim.x;
    for (int it = 0; it < trips; ++it) {
      const int q = it * blockDim.x + threadIdx.x;
      bool take = false;
      uint64_t key = 0;
      double val = 0.0;
      if (q < ne) {
        int lo = 0, hi = nr - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sm.off[mid] <= q) lo = mid; else hi = mid - 1;
        }
        const int32_t a = sm.comm[lo];
        if (a >= a0 && a < a1) {
          const int64_t e = j0 + q + sm.base[lo];  // the entry's place in the CSR
          const int32_t b = C[tail[e]];
          if (b >= 0) {
            take = true;
            key = ((uint64_t)(a - a0) << nb) | (uint64_t)b;
            val = trunc ? (double)(long long)w[e] : w[e];
          }
        }
      }
      const unsigned m = __ballot_sync(FULL, take);
      if (!m) continue;
      unsigned long long base = 0;
      if (lane == __ffs(m) - 1) base = atomicAdd(counter, (unsigned long long)__popc(m));
      base = __shfl_sync(FULL, base, __ffs(m) - 1);
      if (take) {
        const unsigned long long s = base + __popc(m & ((1u << lane) - 1u));
        if (s < cap) {
          keys[s] = key;
          vals[s] = val;
        }
      }
    }
  }
}

// Community order of the rows: degrees of the rows in that order (for the
// order's row starts).
__global__ void k_perm_degrees(int64_t nv, const int32_t *perm, const int64_t *ptr,
                               int64_t *deg) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nv;
       r += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = perm[r];
    deg[r] = ptr[v + 1] - ptr[v];
  }
}

// Sort keys of the community order: C as unsigned (a vertex without a
// community, -1, sorts last) and the vertex id.
__global__ void k_comm_order_keys(int64_t nv, const int32_t *C, uint32_t *keys, int32_t *ids) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    keys[v] = (uint32_t)C[v];
    ids[v] = (int32_t)v;
  }
}

// Tile run of each chunk [bounds[k], bounds[k+1]): the first row of the
// community order with C >= bounds[k] (binary search in the sorted keys),
// turned into a merge-path coordinate and a tile index (first tile that
// reaches it for a start, past it for an end).
__global__ void k_chunk_tiles(int K, const int64_t *bounds, int64_t nv, const uint32_t *skeys,
                              const int64_t *pptr, int64_t *tiles) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > K) return;
  const uint32_t a = (uint32_t)bounds[k];
  int64_t lo = 0, hi = nv;  // first r with skeys[r] >= a
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (skeys[mid] >= a) hi = mid; else lo = mid + 1;
  }
  const int64_t d = pptr[lo] + lo;  // merge coordinate where the chunk's rows start
  tiles[k] = (k == 0) ? 0 : d / kMergeTile;
}

// Row counts and the chunk's tails of its unique (a, b) pairs.
// (ndiag counts the diagonal pairs)
__global__ void k_chunk_emit(int64_t np, const uint64_t *ukeys, int nb, int32_t a0,
                             int64_t *rowc, int32_t *otail, unsigned long long *ndiag) {
  const uint64_t mask = (1ull << nb) - 1;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = ukeys[p];
    const int64_t a = a0 + (int64_t)(k >> nb), b = (int64_t)(k & mask);
    atomicAdd((unsigned long long *)&rowc[a], 1ull);
    otail[p] = (int32_t)b;
    if (a == b) atomicAdd(ndiag, 1ull);
  }
}

// Utility/vertexFollowing.cpp:46-88: C[i] = i, -1 when isolated, its only
// neighbour t when i has degree one and t has degree > 1 or i > t.
__global__ void k_vertex_following(int64_t nv, const int64_t *ptr, const int32_t *tail,
                                   int32_t *C, unsigned long long *num) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t d = ptr[i + 1] - ptr[i];
    int32_t c = (int32_t)i;
    if (d == 0) {
      c = -1;
      atomicAdd(num, 1ull);
    } else if (d == 1) {
      const int32_t t = tail[ptr[i]];
      if (ptr[t + 1] - ptr[t] > 1 || i > t) {
        c = t;
        atomicAdd(num, 1ull);
      }
    }
    C[i] = c;
  }
}

}  // namespace glv
