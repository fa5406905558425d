// Iterated greedy recolouring (Culberson): the vertices of each colour class
// of an existing proper colouring are recoloured first-fit, class after class,
// against the new colours of the classes already done.  A class is an
// independent set, so all its vertices are recoloured at once; a pass can only
// keep or lower the number of colours.  One cooperative persistent launch per
// pass, one step per class, with the sweep's schedule (members sorted by class
// and degree bin, hub rows cut into chunks).
#pragma once

#include <cooperative_groups.h>
#include <cstdint>

#include "glv_common.cuh"
#include "persist.cuh"

namespace glv {

struct RecolorArgs {
  const int64_t *ptr;
  const int32_t *tail;
  const int32_t *members;      // vertices ordered by (class, degree bin, id)
  int32_t *newc;               // new colours (-1 until recoloured)
  const StepDesc *steps;       // one step per class
  int nsteps;
  int64_t *task_ctr;           // per step (zero at launch)
  const int32_t *chunk_pos;    // hub rows: chunk -> member slot
  const int64_t *chunk_beg, *chunk_end;
  const int64_t *hub_off;      // per member slot: offset of its hub table region
  int32_t *hub_words;          // hub table regions, used as all-ones bitmaps here
  int32_t *chunks_left;        // per member slot: chunks not yet folded
  int chunk;                   // CSR entries per hub chunk
};

constexpr int kRecolorThreads = 512;
constexpr int kColorWords = kMaxColors / 32;

// First zero bit of the `words`-word bitmap (bit set = colour used).
__device__ __forceinline__ int warp_first_free(const uint32_t *bm, int words) {
  const int lane = threadIdx.x & 31;
  int first = INT32_MAX;
  for (int q = lane; q < words; q += 32) {
    const uint32_t fr = ~bm[q];
    if (fr) { first = q * 32 + __ffs(fr) - 1; break; }
  }
  first = __reduce_min_sync(FULL, first);
  return first == INT32_MAX ? words * 32 : first;
}

// Rows of at most G entries, 32/G vertices per warp: the used colours below
// G+1 fit a 64-bit mask reduced across the group.
template <int G>
__device__ __forceinline__ void recolor_small(const RecolorArgs &r, int64_t base, int64_t end) {
  const int lane = threadIdx.x & 31, grp = lane / G, gl = lane & (G - 1);
  const int64_t pos = base + grp;
  const bool valid = pos < end;
  const int32_t v = valid ? r.members[pos] : 0;
  const int64_t rb = valid ? r.ptr[v] : 0;
  const int deg = valid ? (int)(r.ptr[v + 1] - rb) : 0;
  uint64_t used = 0;
  if (gl < deg) {
    const int32_t u = r.tail[rb + gl];
    const int32_t cu = (u != v) ? r.newc[u] : -1;
    if (cu >= 0 && cu < 64) used = 1ull << cu;
  }
#pragma unroll
  for (int off = G / 2; off >= 1; off >>= 1) {
    const uint32_t lo = __shfl_xor_sync(FULL, (uint32_t)used, off);
    const uint32_t hi = __shfl_xor_sync(FULL, (uint32_t)(used >> 32), off);
    used |= ((uint64_t)hi << 32) | lo;
  }
  if (valid && gl == 0) r.newc[v] = __ffsll((long long)~used) - 1;
}

// One warp per vertex, bitmap in the warp's shared words.
__device__ __forceinline__ void recolor_warp(const RecolorArgs &r, int64_t pos, uint32_t *bm) {
  const int lane = threadIdx.x & 31;
  const int32_t v = r.members[pos];
  const int64_t rb = r.ptr[v], re = r.ptr[v + 1];
  const int words = (int)min((re - rb + 32) / 32, (int64_t)kColorWords);
  for (int q = lane; q < words; q += 32) bm[q] = 0u;
  __syncwarp();
  for (int64_t j = rb + lane; j < re; j += 32) {
    const int32_t u = r.tail[j];
    const int32_t cu = (u != v) ? r.newc[u] : -1;
    if (cu >= 0 && cu < words * 32) atomicOr(&bm[cu >> 5], 1u << (cu & 31));
  }
  __syncwarp();
  const int c = warp_first_free(bm, words);
  if (lane == 0) r.newc[v] = c;
  __syncwarp();
}

// One block per vertex (rows up to the block bin), bitmap in shared memory.
__device__ __forceinline__ void recolor_block(const RecolorArgs &r, int64_t pos, uint32_t *bm) {
  const int32_t v = r.members[pos];
  const int64_t rb = r.ptr[v], re = r.ptr[v + 1];
  const int words = (int)min((re - rb + 32) / 32, (int64_t)kColorWords);
  for (int q = threadIdx.x; q < words; q += blockDim.x) bm[q] = 0u;
  __syncthreads();
  for (int64_t j = rb + threadIdx.x; j < re; j += blockDim.x) {
    const int32_t u = r.tail[j];
    const int32_t cu = (u != v) ? r.newc[u] : -1;
    if (cu >= 0 && cu < words * 32) atomicOr(&bm[cu >> 5], 1u << (cu & 31));
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int c = warp_first_free(bm, words);
    if (threadIdx.x == 0) r.newc[v] = c;
  }
  __syncthreads();
}

// One chunk of a hub row: fold its colours into a shared bitmap, clear them in
// the hub's global all-ones bitmap; the block finishing the hub's last chunk
// takes the first colour still set and restores the words to all ones.
__device__ __forceinline__ void recolor_hub_chunk(const RecolorArgs &r, int64_t ci, uint32_t *bm,
                                                  int *s_flag) {
  const int32_t pos = r.chunk_pos[ci];
  const int32_t v = r.members[pos];
  uint32_t *gw = reinterpret_cast<uint32_t *>(r.hub_words + r.hub_off[pos]);
  for (int q = threadIdx.x; q < kColorWords; q += blockDim.x) bm[q] = 0u;
  __syncthreads();
  for (int64_t j = r.chunk_beg[ci] + threadIdx.x; j < r.chunk_end[ci]; j += blockDim.x) {
    const int32_t u = r.tail[j];
    const int32_t cu = (u != v) ? r.newc[u] : -1;
    if (cu >= 0 && cu < kMaxColors) atomicOr(&bm[cu >> 5], 1u << (cu & 31));
  }
  __syncthreads();
  for (int q = threadIdx.x; q < kColorWords; q += blockDim.x)
    if (bm[q]) atomicAnd(&gw[q], ~bm[q]);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_flag[0] = (atomicSub(&r.chunks_left[pos], 1) == 1) ? 1 : 0;
  __syncthreads();
  if (!s_flag[0]) return;  // block-uniform
  __threadfence();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    int first = INT32_MAX;
    for (int q = lane; q < kColorWords; q += 32) {
      const uint32_t fr = __ldcg(&gw[q]);
      if (fr) { first = q * 32 + __ffs(fr) - 1; break; }
    }
    first = __reduce_min_sync(FULL, first);
    for (int q = lane; q < kColorWords; q += 32) gw[q] = 0xffffffffu;
    if (lane == 0) {
      r.newc[v] = (first == INT32_MAX) ? kMaxColors - 1 : first;
      r.chunks_left[pos] = (int32_t)((r.ptr[v + 1] - r.ptr[v] + r.chunk - 1) / r.chunk);
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kRecolorThreads) k_recolor_pass(RecolorArgs r) {
  cg::grid_group grid = cg::this_grid();
  constexpr int NW = kRecolorThreads / 32;
  __shared__ uint32_t s_bm[NW][kColorWords / 4];  // warp bitmaps: rows below 1024 entries
  __shared__ uint32_t s_block[kColorWords];
  __shared__ int64_t s_task;
  __shared__ int s_flag;
  const int warp = threadIdx.x >> 5;
  for (int s = 0; s < r.nsteps; ++s) {
    const StepDesc &st = r.steps[s];
    const int64_t t_hub = st.hub_chunk[1] - st.hub_chunk[0];
    const int64_t t_blk = st.seg[BIN_BLOCK + 1] - st.seg[BIN_BLOCK];
    const int64_t n8 = st.seg[2] - st.seg[0];              // degree <= 8: 4 per warp
    const int64_t n32 = st.seg[4] - st.seg[2];             // 9..32: one warp each
    const int64_t nw = st.seg[BIN_BLOCK] - st.seg[4];      // 33..1023: one warp each
    const int64_t witems = (n8 + 3) / 4 + n32 + nw;
    const int64_t t_w = (witems + NW - 1) / NW;
    const int64_t ntask = t_hub + t_blk + t_w;
    while (true) {
      if (threadIdx.x == 0) s_task = atomicAdd((unsigned long long *)&r.task_ctr[s], 1ull);
      __syncthreads();
      int64_t t = s_task;
      __syncthreads();
      if (t >= ntask) break;
      if (t < t_hub) {
        recolor_hub_chunk(r, st.hub_chunk[0] + t, s_block, &s_flag);
        continue;
      }
      t -= t_hub;
      if (t < t_blk) {
        recolor_block(r, st.seg[BIN_BLOCK] + t, s_block);
        continue;
      }
      t -= t_blk;
      int64_t k = t * NW + warp;
      if (k >= witems) continue;
      const int64_t i8 = (n8 + 3) / 4;
      if (k < i8) { recolor_small<8>(r, st.seg[0] + 4 * k, st.seg[2]); continue; }
      k -= i8;
      if (k < n32) { recolor_small<32>(r, st.seg[2] + k, st.seg[4]); continue; }
      k -= n32;
      recolor_warp(r, st.seg[4] + k, s_bm[warp]);
    }
    grid.sync();
  }
}

}  // namespace glv
