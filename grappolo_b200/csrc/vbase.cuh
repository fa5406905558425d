// Balanced recolouring (Coloring/vBase.cpp:6-168, vBaseRedistribution), the
// `coloring = 2` option of runMultiPhaseColoring.
//
// avg = ceil(NV / ncolors); classes holding more than avg vertices are
// oversized.  In vertex order, a vertex of an oversized class whose class
// still holds more than avg moves to a colour that no neighbour has, that
// holds fewer than avg vertices and that was not oversized: the first such
// colour (type 0) or the least used, lowest on ties (type 1).  Where no colour
// qualifies the vertex stays.  At one thread the reference makes exactly
// these moves, one vertex at a time against the current colours, so its
// conflict pass never fires; the result is a proper colouring whatever the
// mode.  Every decision depends on the frequencies left by all earlier ones,
// so the moves run in one block in vertex order: the block's threads share
// each candidate's neighbour scan, the colour frequencies and the bitmaps of
// open colours live in shared memory, and the loop ends as soon as no colour
// is open.  Only vertices of oversized classes are visited.

namespace glv {

constexpr int kVbaseThreads = 1024;
constexpr int kVbaseWords = kMaxColors / 32;

__global__ void k_color_hist(int64_t nv, const int32_t *color, int32_t *freq) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(&freq[color[v]], 1);
}

__global__ void k_vbase_flags(int64_t nv, const int32_t *color, const int32_t *freq, int64_t avg,
                              int32_t *flag) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    flag[v] = freq[color[v]] > avg ? 1 : 0;
}

__global__ void __launch_bounds__(kVbaseThreads)
    k_vbase(const int64_t *ptr, const int32_t *tail, int32_t *color, const int32_t *cand,
            const int64_t *ncand_p, const int32_t *freq0, int ncolors, int64_t avg, int type,
            unsigned long long *moves) {
  __shared__ int32_t freq[kMaxColors];
  __shared__ uint32_t open[kVbaseWords], mark[kVbaseWords];
  __shared__ int s_open, s_pick;
  __shared__ unsigned long long s_best;
  const int tid = threadIdx.x;
  const int words = (ncolors + 31) / 32;
  for (int c = tid; c < kMaxColors; c += blockDim.x) freq[c] = c < ncolors ? freq0[c] : 0;
  if (tid == 0) s_open = 0;
  __syncthreads();
  for (int q = tid; q < kVbaseWords; q += blockDim.x) {
    uint32_t bits = 0;
    for (int b = 0; b < 32; ++b) {
      const int c = q * 32 + b;
      // open: not oversized at the start and below avg (vBase.cpp:84-90, 113-126)
      if (c < ncolors && freq[c] < avg) bits |= 1u << b;
    }
    open[q] = bits;
    if (bits) atomicAdd(&s_open, __popc(bits));
  }
  __syncthreads();
  const int64_t ncand = *ncand_p;
  unsigned long long moved = 0;
  for (int64_t k = 0; k < ncand; ++k) {
    if (s_open == 0) break;  // no colour can take a vertex any more
    const int32_t v = cand[k];
    const int32_t c0 = color[v];
    if (freq[c0] <= avg) continue;  // its class is down to avg (block-uniform)
    for (int q = tid; q < words; q += blockDim.x) mark[q] = 0u;
    if (tid == 0) {
      s_pick = -1;
      s_best = ~0ull;
    }
    __syncthreads();
    for (int64_t j = ptr[v] + tid; j < ptr[v + 1]; j += blockDim.x) {
      const int32_t u = tail[j];
      if (u == v) continue;
      const int32_t cu = color[u];
      if (cu >= 0 && cu < ncolors) atomicOr(&mark[cu >> 5], 1u << (cu & 31));
    }
    __syncthreads();
    if (type == 0) {
      if (tid < 32) {
        int first = INT32_MAX;
        for (int q = tid; q < words; q += 32) {
          const uint32_t ok = open[q] & ~mark[q];
          if (ok) {
            first = q * 32 + __ffs(ok) - 1;
            break;
          }
        }
        first = __reduce_min_sync(FULL, first);
        if (tid == 0 && first != INT32_MAX) s_pick = first;
      }
    } else {
      for (int q = tid; q < words; q += blockDim.x) {
        uint32_t ok = open[q] & ~mark[q];
        while (ok) {
          const int c = q * 32 + __ffs(ok) - 1;
          ok &= ok - 1;
          atomicMin(&s_best, ((unsigned long long)(uint32_t)freq[c] << 32) | (uint32_t)c);
        }
      }
      __syncthreads();
      if (tid == 0 && s_best != ~0ull) s_pick = (int)(s_best & 0xffffffffu);
    }
    __syncthreads();
    if (tid == 0 && s_pick >= 0) {
      const int c = s_pick;
      freq[c] += 1;
      freq[c0] -= 1;
      color[v] = c;
      if (freq[c] >= avg) {
        open[c >> 5] &= ~(1u << (c & 31));
        s_open -= 1;
      }
      ++moved;
    }
    __syncthreads();
  }
  if (tid == 0) *moves = moved;
}

}  // namespace glv
