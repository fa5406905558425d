// Local-moving sweep kernels (one launch per colour class and degree bin).
//
// Per vertex v with community own = C[v] and weighted degree k = vDeg[v] the
// kernels compute what Grappolo's buildLocalMapCounter + max compute
// (Utility/utilityClusteringFunctions.cpp:172-194, 226-259):
//   Counter[c] = sum of w(v,t) over neighbours t with C[t] = c, in CSR order,
//   selfLoop   = sum of w(v,v) entries,
//   eix = Counter[own] - selfLoop,  ax = cDeg[own] - k,
//   gain(c) = 2*(Counter[c] - eix) - 2*k*(cDeg[c] - ax)*constant  (c != own),
// and move to the strictly positive best gain (ties: lower id), with the
// reference's swap protection for two singletons.  Every per-community sum is
// folded in CSR order (leader lanes add their group's weights lane by lane,
// chunks in row order), so the sums are bit-identical to the reference's.
#pragma once

#include <cooperative_groups.h>

#include "glv_common.cuh"

namespace glv {

struct SweepArgs {
  const int64_t *ptr;
  const int32_t *tail;
  const double *w;
  int32_t *C;            // communities read; colour phases also write decisions here
  int32_t *target;       // Jacobi phases: decisions (nullptr in colour phases)
  double *own_w;         // Jacobi phases: Counter[own] per vertex (cluster weight internal)
  const double *vDeg;
  const double *cDeg;
  const int32_t *cSize;
  double constant;
  const int32_t *members;  // vertices ordered by (colour, bin, id)
  int32_t *move_old;       // per member slot: old community if it moved, else -1
  int32_t *move_new;       // per member slot: decision
  double *dDeg;            // community-degree deltas (atomic accumulation)
  int32_t *dSize;
  int atomic_deltas;       // 1: accumulate deltas here; 0: ordered fold after the class
  int32_t *hub_keys;       // BIN_HUB global tables
  double *hub_vals;
  const int64_t *hub_off;  // per member slot: table offset
  // learned gating (colour phases of the persistent path; nullptr = off)
  const uint8_t *skip;     // per vertex: 1 = not evaluated this sweep (stays)
  double *rec_own;         // per vertex: Counter[own] of its last evaluation
  float *rec_gain;         // per vertex: best positive gain of its last evaluation
  int32_t *last_move;      // per vertex: iteration of its last move
  int32_t iter;            // this sweep's iteration number within the phase
  // batches of graphs (one level holds many graphs; nullptr = one graph)
  const int32_t *gid;      // per vertex: its graph
  const double *gcst;      // per graph: 1 / (2m) of that graph
  // per block: sum over the moves of 2 (e_iy - e_ix), the change each move
  // makes to the modularity's internal-weight term (nullptr = not tracked)
  double *exx_delta;
  // colour phases whose classes include batches of the core: decisions reach
  // C only after their step (the apply stage), so every member of a step
  // decides against the communities its step started from
  int defer_c;
};

__device__ __forceinline__ bool skipped(const SweepArgs &a, int32_t v) {
  return a.skip && a.skip[v];
}

// The modularity constant that vertex v's gains use: its own graph's.
__device__ __forceinline__ double cst_of(const SweepArgs &a, int32_t v) {
  return a.gid ? a.gcst[a.gid[v]] : a.constant;
}

// A vertex the gate left out keeps its community and moves nothing.
__device__ __forceinline__ void emit_stay(const SweepArgs &a, int64_t pos, int32_t v,
                                          int32_t own) {
  if (a.target) a.target[v] = own;
  a.move_old[pos] = -1;
  a.move_new[pos] = own;
}

// Writes the decision of vertex v (member slot pos) and its delta records.
__device__ __forceinline__ void emit_decision(const SweepArgs &a, int64_t pos, int32_t v,
                                              int32_t own, int32_t target, double degree,
                                              double own_w, double best_g = 0.0) {
  if (a.rec_own) {
    a.rec_own[v] = own_w;
    a.rec_gain[v] = (float)best_g;
  }
  if (a.target) {
    a.target[v] = target;
    if (a.own_w) a.own_w[v] = own_w;
  } else if (!a.defer_c) {
    a.C[v] = target;
  }
  bool moved = (target != own) && (target != -1);
  a.move_old[pos] = moved ? own : -1;
  a.move_new[pos] = target;
  if (moved && a.exx_delta) {
    // the move's gain is t1 - t2 with t1 = 2 (e_iy - e_ix) (louvain_gain):
    // recover t1 from it and t2, computed as the gain computed it
    const double ax = __dsub_rn(a.cDeg[own], degree);
    const double t2 = __dmul_rn(__dmul_rn(__dmul_rn(2.0, degree), __dsub_rn(a.cDeg[target], ax)),
                                cst_of(a, v));
    atomicAdd(&a.exx_delta[blockIdx.x], __dadd_rn(best_g, t2));
  }
  if (moved && a.last_move) a.last_move[v] = a.iter;
  if (moved && a.atomic_deltas) {
    atomicAdd(&a.dDeg[target], degree);
    atomicAdd(&a.dDeg[own], -degree);
    atomicAdd(&a.dSize[target], 1);
    atomicAdd(&a.dSize[own], -1);
  }
}

// Final choice: best strictly positive gain or stay; swap protection
// (utilityClusteringFunctions.cpp:254-256).
__device__ __forceinline__ int32_t finish_choice(const SweepArgs &a, int32_t own, double best_g,
                                                 int32_t best_c) {
  int32_t t = (best_g > 0.0) ? best_c : own;
  if (t != own && a.cSize[t] == 1 && a.cSize[own] == 1 && t > own) t = own;
  return t;
}

// The same with cSize[own] loaded by the caller ahead of time: only a move
// out of a singleton reads the target's size.
__device__ __forceinline__ int32_t finish_choice(const SweepArgs &a, int32_t own, int32_t own_size,
                                                 double best_g, int32_t best_c) {
  int32_t t = (best_g > 0.0) ? best_c : own;
  if (t != own && own_size == 1 && t > own && a.cSize[t] == 1) t = own;
  return t;
}

// ---------------------------------------------------------------------------
// Rows of at most G entries: G lanes per vertex, one entry per lane, no table.
// One warp handles the 32/G member slots starting at `base` (all lanes call).
template <int G>
__device__ __forceinline__ void small_item(const SweepArgs &a, int64_t base, int64_t end) {
  const int lane = threadIdx.x & 31;
  const int grp = lane / G;
  const int gl = lane & (G - 1);
  const unsigned gmask = (G == 32) ? FULL : (((1u << G) - 1u) << (grp * G));
  const int64_t pos = base + grp;
  const bool valid = pos < end;
  const int32_t v = valid ? a.members[pos] : 0;
  const int64_t rb = valid ? a.ptr[v] : 0;
  const int deg = valid ? (int)(a.ptr[v + 1] - rb) : 0;
  const int32_t own = (valid && deg > 0) ? a.C[v] : -1;
  const bool skip = valid && deg > 0 && skipped(a, v);
  const bool has = !skip && gl < deg;
  const int32_t t = has ? __ldcs(&a.tail[rb + gl]) : -1;
  const double wt = has ? __ldcs(&a.w[rb + gl]) : 0.0;
  const int32_t c = has ? a.C[t] : -1;
  const unsigned long long key =
      has ? (((unsigned long long)grp << 32) | (uint32_t)c) : (0xFFFFFFFF00000000ull | lane);
  const unsigned m = __match_any_sync(FULL, key);
  const bool leader = has && (lane == __ffs(m) - 1);
  // Ordered fold of each community group (lane order == CSR order).
  unsigned rem = leader ? m : 0u;
  const int rounds = __reduce_max_sync(FULL, (unsigned)__popc(rem));
  double sum = 0.0;
  for (int it = 0; it < rounds; ++it) {
    const int src = rem ? __ffs(rem) - 1 : lane;
    const double x = __shfl_sync(FULL, wt, src);
    if (rem) { sum = __dadd_rn(sum, x); rem &= rem - 1; }
  }
  // Self-loop weight, in CSR order.
  unsigned sm = __ballot_sync(FULL, has && t == v) & gmask;
  const int srounds = __reduce_max_sync(FULL, (unsigned)__popc(sm));
  double self_loop = 0.0;
  for (int it = 0; it < srounds; ++it) {
    const int src = sm ? __ffs(sm) - 1 : lane;
    const double x = __shfl_sync(FULL, wt, src);
    if (sm) { self_loop = __dadd_rn(self_loop, x); sm &= sm - 1; }
  }
  // Counter[own]
  const unsigned om = __ballot_sync(FULL, leader && c == own) & gmask;
  const double osum = __shfl_sync(FULL, sum, om ? __ffs(om) - 1 : lane);
  const double own_w = om ? osum : 0.0;
  const double degree = (valid && deg > 0) ? a.vDeg[v] : 0.0;
  double g = 0.0;
  int32_t bc = INT32_MAX;
  if (leader && c != own) {
    const double eix = __dsub_rn(own_w, self_loop);
    const double ax = __dsub_rn(a.cDeg[own], degree);
    const double gain = louvain_gain(sum, eix, degree, a.cDeg[c], ax, cst_of(a, v));
    if (gain > 0.0) { g = gain; bc = c; }
  }
#pragma unroll
  for (int off = G / 2; off >= 1; off >>= 1) {
    const double og = __shfl_xor_sync(FULL, g, off);
    const int32_t oc = __shfl_xor_sync(FULL, bc, off);
    if (better(og, oc, g, bc)) { g = og; bc = oc; }
  }
  if (valid && gl == 0) {
    if (skip) {
      emit_stay(a, pos, v, own);
    } else {
      const int32_t tgt = (deg == 0) ? -1 : finish_choice(a, own, g, bc);
      emit_decision(a, pos, v, own, tgt, degree, own_w, g);
    }
  }

}

template <int G>
__global__ void __launch_bounds__(256) k_sweep_small(SweepArgs a, int64_t begin, int64_t end) {
  constexpr int VPW = 32 / G;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = begin + wid * VPW; base < end; base += nw * VPW) small_item<G>(a, base, end);
}

// ---------------------------------------------------------------------------
// Shared/global open-addressing table helpers.  Keys are community ids (>= 0),
// -1 marks an empty slot; values start at 0.0.

// Find or insert `key`, returning its slot.  Safe under concurrent inserts.
__device__ __forceinline__ uint32_t table_slot(int32_t *keys, uint32_t mask, int32_t key) {
  uint32_t s = hash_slot(key, mask);
  while (true) {
    int32_t k = keys[s];
    if (k == key) return s;
    if (k == -1) {
      int32_t old = atomicCAS(&keys[s], -1, key);
      if (old == -1 || old == key) return s;
    }
    s = (s + 1) & mask;
  }
}

// table_slot that also tells whether this call inserted the key.
__device__ __forceinline__ uint32_t table_slot_new(int32_t *keys, uint32_t mask, int32_t key,
                                                   bool &fresh) {
  uint32_t s = hash_slot(key, mask);
  fresh = false;
  while (true) {
    int32_t k = keys[s];
    if (k == key) return s;
    if (k == -1) {
      int32_t old = atomicCAS(&keys[s], -1, key);
      if (old == -1) { fresh = true; return s; }
      if (old == key) return s;
    }
    s = (s + 1) & mask;
  }
}

__device__ __forceinline__ uint32_t table_find(const int32_t *keys, uint32_t mask, int32_t key) {
  uint32_t s = hash_slot(key, mask);
  while (keys[s] != key) s = (s + 1) & mask;
  return s;
}

// One warp accumulates row [rb, re) into the table in CSR order.  Leaders
// fold their group's weights starting from the table value, so each
// community's sum is the sequential CSR-order sum.  Returns the self-loop sum
// (same value in every lane).  With `atomic_add` the group sums are added with
// atomics instead (used when several warps share one table).  With `fill`
// every slot this call fills first is appended to fill[] (count in *nfill).
__device__ __forceinline__ double warp_accumulate(const SweepArgs &a, int32_t v, int64_t rb,
                                                  int64_t re, int64_t stride, int32_t *keys,
                                                  double *vals, uint32_t mask, bool atomic_add,
                                                  int32_t *fill = nullptr, int *nfill = nullptr) {
  const int lane = threadIdx.x & 31;
  double self_loop = 0.0;
  // Software pipeline, two rounds deep: while this round is folded, the next
  // round's communities are gathered and the round after's entries load.
  // Neighbours' communities do not change during the sweep of one step.  The
  // row's entries are read once per sweep: streaming loads (evict-first in
  // L1 and L2) keep them from pushing the gathered per-vertex arrays out of L2.
  const int64_t j0 = rb + lane, j1 = j0 + stride;
  int32_t t_cur = (j0 < re) ? __ldcs(&a.tail[j0]) : -1;
  double w_cur = (j0 < re) ? __ldcs(&a.w[j0]) : 0.0;
  int32_t t_next = (j1 < re) ? __ldcs(&a.tail[j1]) : -1;
  double w_next = (j1 < re) ? __ldcs(&a.w[j1]) : 0.0;
  int32_t c_cur = (j0 < re) ? a.C[t_cur] : -1;
  for (int64_t base = rb; base < re; base += stride) {
    const int64_t j = base + lane;
    const bool has = j < re;
    const int32_t t = t_cur;
    const double wt = w_cur;
    const int32_t c = c_cur;
    const int64_t jn = j + stride, jnn = j + 2 * stride;
    c_cur = (jn < re) ? a.C[t_next] : -1;
    t_cur = t_next;
    w_cur = w_next;
    t_next = (jnn < re) ? __ldcs(&a.tail[jnn]) : -1;
    w_next = (jnn < re) ? __ldcs(&a.w[jnn]) : 0.0;
    const uint32_t key = has ? (uint32_t)c : (0x80000000u | lane);
    const unsigned m = __match_any_sync(FULL, key);
    const bool leader = has && (lane == __ffs(m) - 1);
    uint32_t slot = 0;
    double acc = 0.0;
    if (leader) {
      if (fill) {
        bool fresh;
        slot = table_slot_new(keys, mask, c, fresh);
        if (fresh) fill[atomicAdd(nfill, 1)] = (int32_t)slot;
      } else {
        slot = table_slot(keys, mask, c);
      }
      if (!atomic_add) acc = vals[slot];
    }
    unsigned rem = leader ? m : 0u;
    const int rounds = __reduce_max_sync(FULL, (unsigned)__popc(rem));
    for (int it = 0; it < rounds; ++it) {
      const int src = rem ? __ffs(rem) - 1 : lane;
      const double x = __shfl_sync(FULL, wt, src);
      if (rem) { acc = __dadd_rn(acc, x); rem &= rem - 1; }
    }
    if (leader) {
      if (atomic_add) atomicAdd(&vals[slot], acc);
      else vals[slot] = acc;
    }
    unsigned sm = __ballot_sync(FULL, has && t == v);
    while (sm) {  // warp-uniform
      const int src = __ffs(sm) - 1;
      self_loop = __dadd_rn(self_loop, __shfl_sync(FULL, wt, src));
      sm &= sm - 1;
    }
    __syncwarp();
  }
  return self_loop;
}

// Best (gain, id) over table slots [first, cap) with stride.
__device__ __forceinline__ void scan_table(const SweepArgs &a, const int32_t *keys,
                                           const double *vals, uint32_t first, uint32_t cap,
                                           uint32_t stride, int32_t own, double eix, double ax,
                                           double degree, double cst, double &g, int32_t &bc) {
  // four slots per thread in flight: their cDeg gathers overlap
  for (uint32_t s0 = first; s0 < cap; s0 += 4 * stride) {
    int32_t k[4];
    double cd[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t s = s0 + q * stride;
      k[q] = (s < cap) ? keys[s] : -1;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) cd[q] = (k[q] >= 0 && k[q] != own) ? a.cDeg[k[q]] : 0.0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (k[q] < 0 || k[q] == own) continue;
      const double gain =
          louvain_gain(vals[s0 + q * stride], eix, degree, cd[q], ax, cst);
      if (gain > 0.0 && better(gain, k[q], g, bc)) { g = gain; bc = k[q]; }
    }
  }
}

__device__ __forceinline__ void warp_argmax(double &g, int32_t &bc) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    const double og = __shfl_xor_sync(FULL, g, off);
    const int32_t oc = __shfl_xor_sync(FULL, bc, off);
    if (better(og, oc, g, bc)) { g = og; bc = oc; }
  }
}

// ---------------------------------------------------------------------------
// Rows of 33..warp_max entries: one warp per vertex, table (capacity <= 256)
// in the warp's slice of shared memory.
__device__ __forceinline__ void warp_table_vertex(const SweepArgs &a, int64_t pos, int32_t *keys,
                                                  double *vals) {
  const int lane = threadIdx.x & 31;
  const int32_t v = a.members[pos];
  if (skipped(a, v)) {
    if (lane == 0) emit_stay(a, pos, v, a.C[v]);
    return;
  }
  const int64_t rb = a.ptr[v], re = a.ptr[v + 1];
  const int32_t own = a.C[v];
  const double degree = a.vDeg[v];
  const double cdeg_own = a.cDeg[own];
  const int32_t own_size = (lane == 0) ? a.cSize[own] : 0;
  const uint32_t cap = table_cap(re - rb);
  const uint32_t mask = cap - 1;
  for (uint32_t s = lane; s < cap; s += 32) { keys[s] = -1; vals[s] = 0.0; }
  __syncwarp();
  if (lane == 0) keys[hash_slot(own, mask)] = own;
  __syncwarp();
  const double self_loop = warp_accumulate(a, v, rb, re, 32, keys, vals, mask, false);
  const double own_w = vals[hash_slot(own, mask)];
  const double eix = __dsub_rn(own_w, self_loop);
  const double ax = __dsub_rn(cdeg_own, degree);
  double g = 0.0;
  int32_t bc = INT32_MAX;
  scan_table(a, keys, vals, lane, cap, 32, own, eix, ax, degree, cst_of(a, v), g, bc);
  warp_argmax(g, bc);
  if (lane == 0)
    emit_decision(a, pos, v, own, finish_choice(a, own, own_size, g, bc), degree, own_w, g);
  __syncwarp();
}

template <int CAP>
__global__ void __launch_bounds__(256) k_sweep_warp(SweepArgs a, int64_t begin, int64_t end) {
  extern __shared__ unsigned char smem_raw[];
  const int warp = threadIdx.x >> 5;
  const int nwb = blockDim.x >> 5;
  double *vals = reinterpret_cast<double *>(smem_raw) + (size_t)warp * CAP;
  int32_t *keys = reinterpret_cast<int32_t *>(reinterpret_cast<double *>(smem_raw) + (size_t)nwb * CAP) +
                  (size_t)warp * CAP;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t pos = begin + wid; pos < end; pos += nw) warp_table_vertex(a, pos, keys, vals);
}

// ---------------------------------------------------------------------------
// Large rows: one block per vertex; the table is `keys`/`vals` (shared memory
// or a global region).  ordered = 1: warp 0 walks the whole row in CSR order
// (bit-exact sums); ordered = 0: all warps take chunks and add group sums with
// atomics.  `red` is block scratch of 3 x 32 words.  All threads call.
__device__ __forceinline__ void block_vertex(const SweepArgs &a, int64_t pos, int32_t *keys,
                                             double *vals, int ordered, double *s_self,
                                             double *s_g, int32_t *s_c) {
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nwb = blockDim.x >> 5;
  const int32_t v = a.members[pos];
  const int64_t rb = a.ptr[v], re = a.ptr[v + 1];
  const uint32_t cap = table_cap(re - rb);
  const uint32_t mask = cap - 1;
  for (uint32_t s = threadIdx.x; s < cap; s += blockDim.x) { keys[s] = -1; vals[s] = 0.0; }
  __syncthreads();
  const int32_t own = a.C[v];
  if (threadIdx.x == 0) keys[hash_slot(own, mask)] = own;
  __syncthreads();
  double self_loop;
  if (ordered) {
    if (warp == 0) {
      double sl = warp_accumulate(a, v, rb, re, 32, keys, vals, mask, false);
      if (lane == 0) s_self[0] = sl;
    }
    __syncthreads();
    self_loop = s_self[0];
  } else {
    double sl = warp_accumulate(a, v, rb + 32 * warp, re, 32 * nwb, keys, vals, mask, true);
    if (lane == 0) s_self[warp] = sl;
    __syncthreads();
    self_loop = 0.0;
    for (int k = 0; k < nwb; ++k) self_loop = __dadd_rn(self_loop, s_self[k]);
  }
  const double degree = a.vDeg[v];
  const double own_w = vals[hash_slot(own, mask)];
  const double eix = __dsub_rn(own_w, self_loop);
  const double ax = __dsub_rn(a.cDeg[own], degree);
  double g = 0.0;
  int32_t bc = INT32_MAX;
  scan_table(a, keys, vals, threadIdx.x, cap, blockDim.x, own, eix, ax, degree, cst_of(a, v), g, bc);
  warp_argmax(g, bc);
  if (lane == 0) { s_g[warp] = g; s_c[warp] = bc; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < nwb; ++k)
      if (better(s_g[k], s_c[k], g, bc)) { g = s_g[k]; bc = s_c[k]; }
    emit_decision(a, pos, v, own, finish_choice(a, own, g, bc), degree, own_w, g);
  }
  __syncthreads();
}

// Team of T threads (T/32 warps; T == blockDim.x or a named-barrier slice of
// the block) handles one row with the table in `keys`/`vals`; parallel
// accumulation only.  `red` arrays have one entry per warp of the team.
template <int T>
__device__ __forceinline__ void team_sync(int team) {
  if (T == 512) __syncthreads();
  else asm volatile("bar.sync %0, %1;" ::"r"(team + 1), "r"(T) : "memory");
}

template <int T>
__device__ __forceinline__ void team_vertex(const SweepArgs &a, int64_t pos, int32_t *keys,
                                            double *vals, int team, double *s_self, double *s_g,
                                            int32_t *s_c) {
  constexpr int NW = T / 32;
  const int tt = threadIdx.x % T;
  const int lane = tt & 31, tw = tt >> 5;
  const int32_t v = a.members[pos];
  if (skipped(a, v)) {  // team-uniform
    if (tt == 0) emit_stay(a, pos, v, a.C[v]);
    return;
  }
  // the row's bounds and the vertex's own values load together, and the
  // community totals of its own community right after: they arrive while
  // the table is cleared and the row accumulates
  const int64_t rb = a.ptr[v], re = a.ptr[v + 1];
  const int32_t own = a.C[v];
  const double degree = a.vDeg[v];
  const double cdeg_own = a.cDeg[own];
  const int32_t own_size = (tt == 0) ? a.cSize[own] : 0;
  const uint32_t cap = table_cap(re - rb);
  const uint32_t mask = cap - 1;
  for (uint32_t s = tt; s < cap; s += T) { keys[s] = -1; vals[s] = 0.0; }
  team_sync<T>(team);
  if (tt == 0) keys[hash_slot(own, mask)] = own;
  team_sync<T>(team);
  const double sl = warp_accumulate(a, v, rb + 32 * tw, re, 32 * NW, keys, vals, mask, true);
  if (lane == 0) s_self[tw] = sl;
  team_sync<T>(team);
  double self_loop = 0.0;
  for (int k = 0; k < NW; ++k) self_loop = __dadd_rn(self_loop, s_self[k]);
  const double own_w = vals[hash_slot(own, mask)];
  const double eix = __dsub_rn(own_w, self_loop);
  const double ax = __dsub_rn(cdeg_own, degree);
  double g = 0.0;
  int32_t bc = INT32_MAX;
  scan_table(a, keys, vals, tt, cap, T, own, eix, ax, degree, cst_of(a, v), g, bc);
  warp_argmax(g, bc);
  if (lane == 0) { s_g[tw] = g; s_c[tw] = bc; }
  team_sync<T>(team);
  if (tt == 0) {
    for (int k = 1; k < NW; ++k)
      if (better(s_g[k], s_c[k], g, bc)) { g = s_g[k]; bc = s_c[k]; }
    emit_decision(a, pos, v, own, finish_choice(a, own, own_size, g, bc), degree, own_w, g);
  }
  team_sync<T>(team);
}

// BIN_T128/T256/BLOCK keep the table in shared memory (capacity up to 8192),
// BIN_HUB in global scratch at hub_off.
__global__ void __launch_bounds__(512) k_sweep_block(SweepArgs a, int64_t begin, int64_t end,
                                                     int hub, int ordered) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ double s_self[32];
  __shared__ double s_g[32];
  __shared__ int32_t s_c[32];
  for (int64_t pos = begin + blockIdx.x; pos < end; pos += gridDim.x) {
    int32_t *keys;
    double *vals;
    if (hub) {
      keys = a.hub_keys + a.hub_off[pos];
      vals = a.hub_vals + a.hub_off[pos];
    } else {
      const int32_t v = a.members[pos];
      const uint32_t cap = table_cap(a.ptr[v + 1] - a.ptr[v]);
      vals = reinterpret_cast<double *>(smem_raw);
      keys = reinterpret_cast<int32_t *>(vals + cap);
    }
    block_vertex(a, pos, keys, vals, ordered, s_self, s_g, s_c);
  }
}

// ---------------------------------------------------------------------------
// Hubs in the parallel-accumulation modes: each hub's row is cut into chunks
// that all blocks share (hub_accum_chunk), its table is scanned in segments of
// the slots that were filled (hub_scan_segment), and one warp per hub folds
// the segments' partial arg-maxes (hub_final).  Every table is left empty
// again by the scan, so tables are cleared only when allocated.
struct HubWork {
  int32_t *keys;            // tables (keys -1 = empty)
  double *vals;
  const int64_t *tab_off;   // per member slot: table offset
  int32_t *occ;             // filled-slot lists
  const int64_t *occ_off;   // per member slot: list offset
  int32_t *cnt;             // per member slot: filled slots
  double *self_w;           // per member slot: self-loop weight
  double *own_w;            // per member slot: Counter[own]
  const int32_t *chunk_pos; // chunk -> member slot
  const int64_t *chunk_beg, *chunk_end;  // CSR range
  const int32_t *seg_pos;   // segment -> member slot
  const int64_t *seg_beg, *seg_end;      // range in the filled-slot list
  double *part_g;           // per segment: best gain
  int32_t *part_c;          //              and its community
  const int64_t *hub_seg_beg, *hub_seg_end;  // per member slot: its segments
  int32_t *chunks_left;     // per member slot: chunks still accumulating
  int32_t *big;             // per member slot: 1 = decided by the segment scan
  int32_t *step_big;        // per step: some hub of the step is big (unused by the persistent kernel)
  // persistent kernel: segments are tasks of their step that wait for the
  // hub's chunks; the last segment to finish decides the hub
  int32_t *segs_left;       // per member slot: segments not yet scanned
  uint32_t *state;          // per member slot: 4 * epoch + 1 decided, + 2 segments needed
  uint32_t epoch;           // this launch (0: the launch-per-kernel path, big[] instead)
  int32_t *err;             // set when a segment's wait gives up
  int chunk;                // CSR entries per accumulation chunk (<= kHubChunk)
  // persistent kernel on thread-block clusters (cluster_row_tasks): the hub
  // rows' tasks, one per (row, community partition); a partitioned row's
  // partial bests are ct_g/ct_c[task] and segs_left[member slot] counts its
  // partitions not yet done
  const int32_t *ct_pos;    // task -> member slot
  const int32_t *ct_part;   // task -> partition index
  const int32_t *ct_nparts; // task -> partitions of its row (a power of two)
  double *ct_g;             // task -> best gain of its partition
  int32_t *ct_c;            //         and its community
};

constexpr int kHubChunk = 2048;      // most CSR entries per accumulation work item
constexpr int kHubSeg = 8192;        // filled slots per scan work item
constexpr int kHubStageCap = 4096;   // block-local staging table of one chunk
constexpr int kHubInlineCap = 4096;  // filled slots the last chunk's block scans itself
constexpr int kHubBatch = 4;         // table slots a thread has in flight at once
static_assert(kHubChunk < kHubStageCap, "a chunk's distinct keys must fit the staging table");
// staging values, the filled-slot list and staging keys of one chunk
constexpr int kHubStageSmem = kHubStageCap * (int)(sizeof(double) + 2 * sizeof(int32_t));

// Best (gain, id) over the filled slots occ[k0..k1) of a hub table; the slots
// are emptied for the table's next use.  kHubBatch slots per thread are
// loaded before any is used, so the occ -> key -> cDeg chains overlap.
__device__ __forceinline__ void hub_scan_slots(const SweepArgs &a, int32_t *keys, double *vals,
                                               const int32_t *occ, int64_t k0, int64_t k1,
                                               int32_t own, double eix, double ax, double degree,
                                               double cst, double &g, int32_t &bc) {
  for (int64_t kb = k0 + threadIdx.x; kb < k1; kb += (int64_t)kHubBatch * blockDim.x) {
    int32_t s[kHubBatch], c[kHubBatch];
    double val[kHubBatch], cd[kHubBatch];
#pragma unroll
    for (int j = 0; j < kHubBatch; ++j) {
      const int64_t k = kb + (int64_t)j * blockDim.x;
      s[j] = (k < k1) ? __ldcg(&occ[k]) : -1;
    }
#pragma unroll
    for (int j = 0; j < kHubBatch; ++j) {
      c[j] = (s[j] >= 0) ? __ldcg(&keys[s[j]]) : -1;
      val[j] = (s[j] >= 0) ? __ldcg(&vals[s[j]]) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < kHubBatch; ++j) cd[j] = (c[j] >= 0 && c[j] != own) ? a.cDeg[c[j]] : 0.0;
#pragma unroll
    for (int j = 0; j < kHubBatch; ++j) {
      if (s[j] < 0) continue;
      if (c[j] != own) {
        const double gain = louvain_gain(val[j], eix, degree, cd[j], ax, cst);
        if (gain > 0.0 && better(gain, c[j], g, bc)) { g = gain; bc = c[j]; }
      }
      keys[s[j]] = -1;
      vals[s[j]] = 0.0;
    }
  }
}

// All threads of the block call.  The chunk is first folded into a
// block-local shared table (`skeys`/`svals`, kHubStageCap slots; at most
// kHubChunk distinct keys), then each distinct community is added to the
// hub's global table once — a hub's neighbours concentrate on a few
// communities, and per-warp global atomics on those slots would serialise.
__device__ __forceinline__ void hub_accum_chunk(const SweepArgs &a, const HubWork &h, int64_t ci,
                                                int32_t *skeys, double *svals, double *s_self,
                                                double *s_g, int32_t *s_c, int *s_flag, int step) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  const int32_t pos = h.chunk_pos[ci];
  const int64_t eb = h.chunk_beg[ci], ee = h.chunk_end[ci];
  const int32_t v = a.members[pos];
  const bool skip = skipped(a, v);  // block-uniform
  const uint32_t smask = kHubStageCap - 1;
  // the staging slots in the order they were first filled (s_flag[0] of them)
  int32_t *sfill = reinterpret_cast<int32_t *>(svals + kHubStageCap);
  if (!skip) {
  for (uint32_t q = threadIdx.x; q < kHubStageCap; q += blockDim.x) { skeys[q] = -1; svals[q] = 0.0; }
  if (threadIdx.x == 0) { s_self[0] = 0.0; s_flag[0] = 0; }
  __syncthreads();
  double sl = warp_accumulate(a, v, eb + 32 * warp, ee, 32 * nwb, skeys, svals, smask, true, sfill,
                              s_flag);
  if (lane == 0 && sl != 0.0) atomicAdd(&s_self[0], sl);
  __syncthreads();
  const int nfill = s_flag[0];
  const uint32_t mask = table_cap(a.ptr[v + 1] - a.ptr[v]) - 1;
  int32_t *keys = h.keys + h.tab_off[pos];
  double *vals = h.vals + h.tab_off[pos];
  int32_t *occ = h.occ + h.occ_off[pos];
  const int32_t own = a.C[v];
  // Each thread inserts kHubBatch staged keys at once: the probes of one
  // round are independent CASes in flight together.  Only the filled staging
  // slots are visited (at most kHubChunk: one round of 4 x 512 keys).
  for (int q0 = 0; q0 < nfill; q0 += kHubBatch * (int)blockDim.x) {
    // nfill is the block's: a block-uniform loop
    int32_t c[kHubBatch];
    double val[kHubBatch];
    uint32_t s[kHubBatch];
    bool pend[kHubBatch], ins[kHubBatch];
#pragma unroll
    for (int j = 0; j < kHubBatch; ++j) {
      const int q = q0 + j * (int)blockDim.x + (int)threadIdx.x;
      const int32_t sl = (q < nfill) ? sfill[q] : -1;
      c[j] = (sl >= 0) ? skeys[sl] : -1;
      val[j] = (sl >= 0) ? svals[sl] : 0.0;
      pend[j] = c[j] >= 0;
      ins[j] = false;
      s[j] = pend[j] ? hash_slot(c[j], mask) : 0u;
    }
    bool more = pend[0] || pend[1] || pend[2] || pend[3];
    while (more) {  // per thread; no warp-synchronous work inside
      int32_t old[kHubBatch];
#pragma unroll
      for (int j = 0; j < kHubBatch; ++j) old[j] = pend[j] ? atomicCAS(&keys[s[j]], -1, c[j]) : 0;
      more = false;
#pragma unroll
      for (int j = 0; j < kHubBatch; ++j) {
        if (!pend[j]) continue;
        if (old[j] == -1) { ins[j] = true; pend[j] = false; }
        else if (old[j] == c[j]) pend[j] = false;
        else { s[j] = (s[j] + 1) & mask; more = true; }
      }
    }
    // filled-slot list: one counter update per warp
    int nins = 0;
#pragma unroll
    for (int j = 0; j < kHubBatch; ++j) nins += ins[j] ? 1 : 0;
    int incl = nins;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, off);
      if (lane >= off) incl += y;
    }
    const int total = __shfl_sync(FULL, incl, 31);
    int obase = 0;
    if (lane == 31 && total > 0) obase = atomicAdd(&h.cnt[pos], total);
    obase = __shfl_sync(FULL, obase, 31) + incl - nins;
#pragma unroll
    for (int j = 0; j < kHubBatch; ++j)
      if (ins[j]) occ[obase++] = (int32_t)s[j];
#pragma unroll
    for (int j = 0; j < kHubBatch; ++j) {
      if (c[j] < 0) continue;
      atomicAdd(&vals[s[j]], val[j]);
      if (c[j] == own) atomicAdd(&h.own_w[pos], val[j]);
    }
  }
  if (threadIdx.x == 0 && s_self[0] != 0.0) atomicAdd(&h.self_w[pos], s_self[0]);
  }  // !skip
  // The block that finishes a hub's last chunk decides it when the hub has
  // few distinct communities; otherwise it marks the hub for the segment scan.
  // Every thread publishes its table and list writes before the countdown.
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_flag[0] = (atomicSub(&h.chunks_left[pos], 1) == 1) ? 1 : 0;
  __syncthreads();
  if (!s_flag[0]) return;
  __threadfence();
  if (skip) {
    if (threadIdx.x == 0) {
      emit_stay(a, pos, v, a.C[v]);
      h.chunks_left[pos] = (int32_t)((a.ptr[v + 1] - a.ptr[v] + h.chunk - 1) / h.chunk);
      if (h.epoch) {
        __threadfence();
        atomicExch(&h.state[pos], 4u * h.epoch + 1u);
      }
    }
    __syncthreads();
    return;
  }
  const uint32_t mask = table_cap(a.ptr[v + 1] - a.ptr[v]) - 1;
  int32_t *keys = h.keys + h.tab_off[pos];
  double *vals = h.vals + h.tab_off[pos];
  int32_t *occ = h.occ + h.occ_off[pos];
  const int32_t own = a.C[v];
  const int32_t nfill = __ldcg(&h.cnt[pos]);
  if (nfill > kHubInlineCap) {
    if (threadIdx.x == 0) {
      if (h.epoch) {
        atomicExch(&h.state[pos], 4u * h.epoch + 2u);  // its segment tasks decide it
      } else {
        h.big[pos] = 1;
        if (step >= 0) atomicOr(&h.step_big[step], 1);
      }
    }
    __syncthreads();
    return;
  }
  const double degree = a.vDeg[v];
  const double own_w = __ldcg(&h.own_w[pos]);
  const double eix = __dsub_rn(own_w, __ldcg(&h.self_w[pos]));
  const double ax = __dsub_rn(a.cDeg[own], degree);
  double g = 0.0;
  int32_t bc = INT32_MAX;
  hub_scan_slots(a, keys, vals, occ, 0, nfill, own, eix, ax, degree, cst_of(a, v), g, bc);
  warp_argmax(g, bc);
  if (lane == 0) { s_g[warp] = g; s_c[warp] = bc; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < nwb; ++k)
      if (better(s_g[k], s_c[k], g, bc)) { g = s_g[k]; bc = s_c[k]; }
    emit_decision(a, pos, v, own, finish_choice(a, own, g, bc), degree, own_w, g);
    h.cnt[pos] = 0;
    h.self_w[pos] = 0.0;
    h.own_w[pos] = 0.0;
    h.chunks_left[pos] = (int32_t)((a.ptr[v + 1] - a.ptr[v] + h.chunk - 1) / h.chunk);
    if (h.epoch) {
      __threadfence();
      atomicExch(&h.state[pos], 4u * h.epoch + 1u);
    }
  }
  __syncthreads();
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

constexpr uint32_t kSpinLimit = 1u << 22;  // polls of a segment's wait (x >= 128 ns)

// Persistent kernel: one scan segment of a hub as a block task (all threads
// call).  Segments are queued after every chunk of their step and a chunk
// never waits, so the wait ends once the hub's chunks are folded.  The last
// segment to finish folds the partial arg-maxes and decides the hub.
__device__ __forceinline__ void hub_segment_task(const SweepArgs &a, const HubWork &h, int64_t si,
                                                 double *s_g, int32_t *s_c, uint32_t *s_word) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  const int32_t pos = h.seg_pos[si];
  const uint32_t decided = 4u * h.epoch + 1u;
  if (threadIdx.x == 0) {
    uint32_t st, it = 0;
    while ((st = ld_acquire(&h.state[pos])) < decided) {
      if (++it > kSpinLimit) {
        atomicExch(h.err, 1);
        st = 0;
        break;
      }
      __nanosleep(128);
    }
    s_word[0] = st;
  }
  __syncthreads();
  const uint32_t st = s_word[0];
  __syncthreads();
  if (st != decided + 1u) return;  // decided by its last chunk (block-uniform)
  const int32_t v = a.members[pos];
  const int32_t own = a.C[v];
  const double degree = a.vDeg[v];
  const double own_w = __ldcg(&h.own_w[pos]);
  const double eix = __dsub_rn(own_w, __ldcg(&h.self_w[pos]));
  const double ax = __dsub_rn(a.cDeg[own], degree);
  int32_t *keys = h.keys + h.tab_off[pos];
  double *vals = h.vals + h.tab_off[pos];
  const int32_t *occ = h.occ + h.occ_off[pos];
  const int64_t ob = h.seg_beg[si];
  const int64_t oe = min(h.seg_end[si], (int64_t)__ldcg(&h.cnt[pos]));
  double g = 0.0;
  int32_t bc = INT32_MAX;
  if (ob < oe) hub_scan_slots(a, keys, vals, occ, ob, oe, own, eix, ax, degree, cst_of(a, v), g, bc);
  warp_argmax(g, bc);
  if (lane == 0) { s_g[warp] = g; s_c[warp] = bc; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < nwb; ++k)
      if (better(s_g[k], s_c[k], g, bc)) { g = s_g[k]; bc = s_c[k]; }
    h.part_g[si] = g;
    h.part_c[si] = bc;
    __threadfence();
    s_word[0] = (atomicSub(&h.segs_left[pos], 1) == 1) ? 1u : 0u;
  }
  __syncthreads();
  const bool last = s_word[0] != 0;
  __syncthreads();
  if (!last || warp != 0) return;
  __threadfence();
  g = 0.0;
  bc = INT32_MAX;
  for (int64_t k = h.hub_seg_beg[pos] + lane; k < h.hub_seg_end[pos]; k += 32) {
    const double pg = __ldcg(&h.part_g[k]);
    const int32_t pc = __ldcg(&h.part_c[k]);
    if (better(pg, pc, g, bc)) { g = pg; bc = pc; }
  }
  warp_argmax(g, bc);
  if (lane == 0) {
    emit_decision(a, pos, v, own, finish_choice(a, own, g, bc), degree, own_w, g);
    h.cnt[pos] = 0;
    h.self_w[pos] = 0.0;
    h.own_w[pos] = 0.0;
    h.chunks_left[pos] = (int32_t)((a.ptr[v + 1] - a.ptr[v] + h.chunk - 1) / h.chunk);
    h.segs_left[pos] = (int32_t)(h.hub_seg_end[pos] - h.hub_seg_beg[pos]);
  }
}

// All threads of the block call; s_g/s_c are 32-entry block scratch.
__device__ __forceinline__ void hub_scan_segment(const SweepArgs &a, const HubWork &h, int64_t si,
                                                 double *s_g, int32_t *s_c) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  const int32_t pos = h.seg_pos[si];
  if (!h.big[pos]) return;  // decided when its last chunk finished (block-uniform)
  const int32_t v = a.members[pos];
  const int32_t own = a.C[v];
  const double degree = a.vDeg[v];
  const double eix = __dsub_rn(h.own_w[pos], h.self_w[pos]);
  const double ax = __dsub_rn(a.cDeg[own], degree);
  int32_t *keys = h.keys + h.tab_off[pos];
  double *vals = h.vals + h.tab_off[pos];
  const int32_t *occ = h.occ + h.occ_off[pos];
  const int64_t ob = h.seg_beg[si];
  const int64_t oe = min(h.seg_end[si], (int64_t)h.cnt[pos]);
  double g = 0.0;
  int32_t bc = INT32_MAX;
  hub_scan_slots(a, keys, vals, occ, ob, oe, own, eix, ax, degree, cst_of(a, v), g, bc);
  warp_argmax(g, bc);
  if (lane == 0) { s_g[warp] = g; s_c[warp] = bc; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < nwb; ++k)
      if (better(s_g[k], s_c[k], g, bc)) { g = s_g[k]; bc = s_c[k]; }
    h.part_g[si] = g;
    h.part_c[si] = bc;
  }
  __syncthreads();
}

// One warp per hub (all lanes call).
__device__ __forceinline__ void hub_final(const SweepArgs &a, const HubWork &h, int64_t pos) {
  const int lane = threadIdx.x & 31;
  if (!h.big[pos]) return;
  double g = 0.0;
  int32_t bc = INT32_MAX;
  for (int64_t si = h.hub_seg_beg[pos] + lane; si < h.hub_seg_end[pos]; si += 32)
    if (better(h.part_g[si], h.part_c[si], g, bc)) { g = h.part_g[si]; bc = h.part_c[si]; }
  warp_argmax(g, bc);
  if (lane == 0) {
    const int32_t v = a.members[pos];
    const int32_t own = a.C[v];
    emit_decision(a, pos, v, own, finish_choice(a, own, g, bc), a.vDeg[v], h.own_w[pos], g);
    h.cnt[pos] = 0;
    h.self_w[pos] = 0.0;
    h.own_w[pos] = 0.0;
    h.big[pos] = 0;
    h.chunks_left[pos] = (int32_t)((a.ptr[v + 1] - a.ptr[v] + h.chunk - 1) / h.chunk);
  }
}

// ---------------------------------------------------------------------------
// Hub rows on thread-block clusters (persistent kernel, parallel modes).  The
// CL blocks of a cluster hold one open-addressing table in their shared
// memory, reached through distributed shared memory: slot s lives in block
// s mod CL at local slot s / CL, up to CL x kClusterBlockSlots slots.  A row
// whose table would need more is split by community: partition p of P takes
// the neighbours whose community c has mix32(c) mod P = p, each partition a
// separate task that reads the whole row; the partitions' best moves are
// folded by the last one to finish.  Nothing of a hub table touches HBM.

constexpr int kClusterBlockSlots = 8192;  // table slots in one block's shared region
constexpr int kClusterMax = 16;           // largest cluster the tasks support
constexpr int kClusterMaxParts = 2;       // most partitions of a cluster row (each reads the row)

// Per-block scratch of the cluster tasks; rank 0's copy is the one read.
struct ClusterShared {
  double acc[2][2];              // by task parity: the row's self-loop weight, Counter[own]
  double g[kClusterMax];         // per block: best gain
  int32_t c[kClusterMax];        //            and its community
  int64_t next;                  // next task of the step (set by rank 0)
};

// Partitions of a row of `deg` entries on a cluster of `cl` blocks, and the
// slots of each partition's table (both powers of two).
__host__ __device__ inline void cluster_row_shape(int64_t deg, int cl, uint32_t *nparts,
                                                  uint32_t *cap) {
  const uint32_t need = table_cap(deg);
  const uint32_t full = (uint32_t)cl * kClusterBlockSlots;
  *nparts = need > full ? need / full : 1u;
  *cap = need / *nparts;
}

// Find or insert `key` in the cluster table; returns the slot, or UINT32_MAX
// when every slot holds another key (a partition far above its expected
// load; the caller raises the error flag).
__device__ __forceinline__ uint32_t cluster_table_slot(cooperative_groups::cluster_group &cl,
                                                       int32_t *keys, uint32_t mask,
                                                       unsigned cl_bits, int32_t key) {
  uint32_t s = hash_slot(key, mask);
  const uint32_t rank_mask = (1u << cl_bits) - 1u;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    int32_t *k = cl.map_shared_rank(keys, s & rank_mask) + (s >> cl_bits);
    const int32_t old = atomicCAS(k, -1, key);
    if (old == -1 || old == key) return s;
    s = (s + 1) & mask;
  }
  return UINT32_MAX;
}

// Warp gw of the cluster's nw warps adds its entries of row [rb, rb + deg) that
// fall in partition `part` to the cluster table, and sums (per lane) the row's
// self-loop weight and the weight to the row's own community.
__device__ __forceinline__ void cluster_accumulate(const SweepArgs &a,
                                                   cooperative_groups::cluster_group &cl,
                                                   int32_t v, int32_t own, int64_t rb, int64_t re,
                                                   int64_t gw, int64_t nw, int32_t *keys,
                                                   double *vals, uint32_t mask, unsigned cl_bits,
                                                   uint32_t part, uint32_t part_mask,
                                                   double &self_w, double &own_w, bool &overflow) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = 32 * nw;
  const uint32_t rank_mask = (1u << cl_bits) - 1u;
  // two rounds in flight, as in warp_accumulate
  const int64_t j0 = rb + 32 * gw + lane, j1 = j0 + stride;
  int32_t t_cur = (j0 < re) ? __ldcs(&a.tail[j0]) : -1;
  double w_cur = (j0 < re) ? __ldcs(&a.w[j0]) : 0.0;
  int32_t t_next = (j1 < re) ? __ldcs(&a.tail[j1]) : -1;
  double w_next = (j1 < re) ? __ldcs(&a.w[j1]) : 0.0;
  int32_t c_cur = (j0 < re) ? a.C[t_cur] : -1;
  for (int64_t base = rb + 32 * gw; base < re; base += stride) {
    const int64_t j = base + lane;
    const bool has = j < re;
    const int32_t t = t_cur;
    const double wt = w_cur;
    const int32_t c = c_cur;
    const int64_t jn = j + stride, jnn = j + 2 * stride;
    c_cur = (jn < re) ? a.C[t_next] : -1;
    t_cur = t_next;
    w_cur = w_next;
    t_next = (jnn < re) ? __ldcs(&a.tail[jnn]) : -1;
    w_next = (jnn < re) ? __ldcs(&a.w[jnn]) : 0.0;
    if (has && t == v) self_w += wt;
    if (has && c == own) own_w += wt;
    const bool mine = has && (mix32((uint32_t)c) & part_mask) == part;
    const uint32_t key = mine ? (uint32_t)c : (0x80000000u | lane);
    const unsigned m = __match_any_sync(FULL, key);
    const bool leader = mine && (lane == __ffs(m) - 1);
    double acc = 0.0;
    unsigned rem = leader ? m : 0u;
    const int rounds = __reduce_max_sync(FULL, (unsigned)__popc(rem));
    for (int it = 0; it < rounds; ++it) {
      const int src = rem ? __ffs(rem) - 1 : lane;
      const double x = __shfl_sync(FULL, wt, src);
      if (rem) { acc += x; rem &= rem - 1; }
    }
    if (leader) {
      const uint32_t s = cluster_table_slot(cl, keys, mask, cl_bits, c);
      if (s == UINT32_MAX) overflow = true;
      else atomicAdd(cl.map_shared_rank(vals, s & rank_mask) + (s >> cl_bits), acc);
    }
  }
}

// The hub tasks [tb, tb + ntask) of one step, run by every thread of every
// block of the cluster.  `keys`/`vals` are this block's table region (at
// least kClusterBlockSlots slots), `cs` its ClusterShared, `red` 32 doubles
// and `redc` 32 ints of block scratch (every block of the cluster calls with
// the same tb, ntask and ctr).  Two cluster barriers per task: after
// the inserts (row sums complete), and after the scan (every block's best in
// rank 0, its own slots cleared again, the next task published).  The row
// sums alternate between two slots by task parity, so rank 0 clears one pair
// while the blocks may already add to the other.
__device__ __forceinline__ void cluster_row_tasks(const SweepArgs &a, const HubWork &h, int64_t tb,
                                               int64_t ntask, int64_t *ctr, int32_t *keys,
                                               double *vals, ClusterShared *cs, double *red,
                                               int32_t *redc) {
  namespace cgx = cooperative_groups;
  cgx::cluster_group cl = cgx::this_cluster();
  const unsigned ncl = cl.num_blocks(), rank = cl.block_rank();
  const unsigned cl_bits = __ffs(ncl) - 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  ClusterShared *cs0 = cl.map_shared_rank(cs, 0);
  for (uint32_t q = threadIdx.x; q < kClusterBlockSlots; q += blockDim.x) {
    keys[q] = -1;
    vals[q] = 0.0;
  }
  if (rank == 0 && threadIdx.x == 0) {
    cs->next = (int64_t)atomicAdd((unsigned long long *)ctr, 1ull);
    cs->acc[0][0] = cs->acc[0][1] = cs->acc[1][0] = cs->acc[1][1] = 0.0;
  }
  cl.sync();
  for (unsigned it = 0;; ++it) {
    const int64_t t = cs0->next;
    if (t >= ntask) break;
    const int64_t ti = tb + t;
    const int32_t pos = h.ct_pos[ti];
    const uint32_t part = (uint32_t)h.ct_part[ti], nparts = (uint32_t)h.ct_nparts[ti];
    const int32_t v = a.members[pos];
    const int32_t own = a.C[v];
    if (skipped(a, v)) {  // cluster-uniform
      if (rank == 0 && threadIdx.x == 0 && part == 0) emit_stay(a, pos, v, own);
      cl.sync();  // every block has read `next`
      if (rank == 0 && threadIdx.x == 0)
        cs->next = (int64_t)atomicAdd((unsigned long long *)ctr, 1ull);
      cl.sync();
      continue;
    }
    double *acc = cs0->acc[it & 1];
    const int64_t rb = a.ptr[v], re = a.ptr[v + 1];
    uint32_t np, cap;
    cluster_row_shape(re - rb, (int)ncl, &np, &cap);
    const uint32_t local = cap >> cl_bits;  // this block's slots of the table
    double self_w = 0.0, own_w = 0.0;
    bool overflow = false;
    cluster_accumulate(a, cl, v, own, rb, re, (int64_t)rank * nwb + warp, (int64_t)ncl * nwb, keys,
                       vals, cap - 1, cl_bits, part, nparts - 1, self_w, own_w, overflow);
    if (overflow) atomicExch(h.err, 2);
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
      self_w += __shfl_xor_sync(FULL, self_w, off);
      own_w += __shfl_xor_sync(FULL, own_w, off);
    }
    if (lane == 0) {
      if (self_w != 0.0) atomicAdd(&acc[0], self_w);
      if (own_w != 0.0) atomicAdd(&acc[1], own_w);
    }
    cl.sync();  // every entry is in the table, the row sums are complete
    const double degree = a.vDeg[v];
    const double row_own = acc[1];
    const double eix = __dsub_rn(row_own, acc[0]);
    const double ax = __dsub_rn(a.cDeg[own], degree);
    double g = 0.0;
    int32_t bc = INT32_MAX;
    scan_table(a, keys, vals, threadIdx.x, local, blockDim.x, own, eix, ax, degree, cst_of(a, v),
               g, bc);
    warp_argmax(g, bc);
    if (lane == 0) { red[warp] = g; redc[warp] = bc; }
    __syncthreads();  // the block's scan is done: its slots are cleared below
    if (threadIdx.x == 0) {
      for (int k = 1; k < nwb; ++k)
        if (better(red[k], redc[k], g, bc)) { g = red[k]; bc = redc[k]; }
      cs0->g[rank] = g;
      cs0->c[rank] = bc;
      if (rank == 0) cs->next = (int64_t)atomicAdd((unsigned long long *)ctr, 1ull);
    }
    for (uint32_t q = threadIdx.x; q < local; q += blockDim.x) {
      keys[q] = -1;
      vals[q] = 0.0;
    }
    cl.sync();  // bests in rank 0, tables clear, next task published
    if (rank == 0 && threadIdx.x == 0) {
      g = cs->g[0];
      bc = cs->c[0];
      for (unsigned k = 1; k < ncl; ++k)
        if (better(cs->g[k], cs->c[k], g, bc)) { g = cs->g[k]; bc = cs->c[k]; }
      cs->acc[it & 1][0] = 0.0;  // read by every block before the barrier above
      cs->acc[it & 1][1] = 0.0;
      bool decide = true;
      if (nparts > 1) {
        // the last partition of the row to finish folds the others' bests
        h.ct_g[ti] = g;
        h.ct_c[ti] = bc;
        __threadfence();
        decide = atomicSub(&h.segs_left[pos], 1) == 1;
        if (decide) {
          __threadfence();
          const int64_t t0 = ti - part;
          for (uint32_t k = 0; k < nparts; ++k) {
            const double pg = __ldcg(&h.ct_g[t0 + k]);
            const int32_t pc = __ldcg(&h.ct_c[t0 + k]);
            if (better(pg, pc, g, bc)) { g = pg; bc = pc; }
          }
          h.segs_left[pos] = (int32_t)nparts;
        }
      }
      if (decide) emit_decision(a, pos, v, own, finish_choice(a, own, g, bc), degree, row_own, g);
    }
  }
}

__global__ void __launch_bounds__(512) k_hub_accum(SweepArgs a, HubWork h, int64_t cb,
                                                   int64_t ce) {
  extern __shared__ unsigned char smem_raw[];
  __shared__ double s_self[1], s_g[32];
  __shared__ int32_t s_c[32];
  __shared__ int s_flag[1];
  // staging values, the filled-slot list, staging keys (kHubStageSmem bytes)
  double *svals = reinterpret_cast<double *>(smem_raw);
  int32_t *skeys = reinterpret_cast<int32_t *>(svals + kHubStageCap) + kHubStageCap;
  for (int64_t ci = cb + blockIdx.x; ci < ce; ci += gridDim.x)
    hub_accum_chunk(a, h, ci, skeys, svals, s_self, s_g, s_c, s_flag, -1);
}

__global__ void __launch_bounds__(256) k_hub_scan(SweepArgs a, HubWork h, int64_t sb,
                                                  int64_t se) {
  __shared__ double s_g[32];
  __shared__ int32_t s_c[32];
  for (int64_t si = sb + blockIdx.x; si < se; si += gridDim.x) hub_scan_segment(a, h, si, s_g, s_c);
}

__global__ void __launch_bounds__(256) k_hub_final(SweepArgs a, HubWork h, int64_t b,
                                                   int64_t e) {
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t pos = b + wid; pos < e; pos += nw) hub_final(a, h, pos);
}

}  // namespace glv
