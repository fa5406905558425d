// Coarsening without sorts (fast and learned modes).
//
// Builds the next level the reference's buildNextLevelGraphOpt builds
// (Utility/buildNextPhase.cpp:83-255): one row per community a holding, for
// every community b adjacent to it, the sum of the weights of the entries
// i -> t with C[i] = a and C[t] = b (the internal entries, self-loops
// included, summed into (a, a)), and an (a, a) entry in every row.  The
// reference visits the rows in order and keeps a map per community; the
// verify-mode path (Engine::coarsen's sorts) reproduces its entry order and
// its sums' order bit for bit.  Here, where neither order is part of the
// result, the entries of each community's members are folded on chip:
//
//   1. members: the vertices with a community and at least one entry, sorted
//      by community (radix sort on the community bits); mptr[m] = offset of
//      member m's first entry in the community-ordered entry sequence;
//   2. block tasks of at most kHashTile entries of that sequence, each
//      folded into a shared table keyed by (a, b) (warp groups of equal
//      keys pre-summed): a window task takes every small community (at most
//      kHashWindow entries) whose first entry lies in one kHashWindow-entry
//      window of the sequence -- they are contiguous and span at most
//      2 kHashWindow entries -- and writes their rows directly; a big
//      community is cut into kHashTile-entry chunks whose sums are added
//      into a global table of its own, one atomic per distinct b per chunk;
//   3. the big tables are emitted in 8192-slot chunks;
//   4. row lengths are scanned and every row is copied into place, with an
//      (a, a, 0.0) entry added where the community had no internal entry.
//
// With few communities (dense mode, ncl <= kDenseCoarseMax) step 2 adds every
// (a, b) sum into an ncl x ncl matrix with a presence bit instead, and the
// rows are read off the matrix in ascending b.
//
// The order of each sum's additions is not fixed (shared and global
// atomics; the hash tables also leave the entry order inside a row open), so
// a row's sum for b and row b's sum for a may differ in the last bit;
// integral weights give exact sums.
#pragma once

#include "glv_common.cuh"

namespace glv {

constexpr int kHashTile = 1024;             // entries folded by one block task
constexpr int kHashWindow = kHashTile / 2;  // small communities: at most this many entries
constexpr int kHashTileSlots = 2048;        // its (a, b) table
constexpr int kHashThreads = 256;
constexpr int kHashPer = kHashTile / kHashThreads;  // entries per thread
constexpr int kBigChunk = 8192;             // table slots per emission task
constexpr uint64_t kEmptyPair = ~0ull;
constexpr int64_t kDenseCoarseMax = 16384;  // dense output: at most 2 GB of sums

// key = community (members) or ncl (vertices left out: no community or no
// entries); value = the vertex.
__global__ void k_hc_member_keys(int64_t nv, const int32_t *Cm, const int64_t *ptr, int64_t ncl,
                                 uint32_t *keys, int32_t *verts) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = Cm[v];
    keys[v] = (c >= 0 && ptr[v + 1] > ptr[v]) ? (uint32_t)c : (uint32_t)ncl;
    verts[v] = (int32_t)v;
  }
}

// Member degrees (in community order) and the member count.
__global__ void k_hc_member_degrees(int64_t nv, const uint32_t *keys, const int32_t *verts,
                                    const int64_t *ptr, int64_t ncl, int64_t *mdeg,
                                    int64_t *nmem) {
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nv;
       m += (int64_t)gridDim.x * blockDim.x) {
    const bool in = keys[m] < (uint32_t)ncl;
    const int32_t v = verts[m];
    mdeg[m] = in ? ptr[v + 1] - ptr[v] : 0;
    if (in && (m + 1 == nv || keys[m + 1] >= (uint32_t)ncl)) *nmem = m + 1;
  }
}

// Entry range [cE0[a], cE1[a]) of every community with members.
__global__ void k_hc_community_ranges(int64_t nmem, const uint32_t *keys, const int64_t *mptr,
                                      int64_t *cE0, int64_t *cE1) {
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < nmem;
       m += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t a = keys[m];
    if (m == 0 || keys[m - 1] != a) cE0[a] = mptr[m];
    if (m + 1 == nmem || keys[m + 1] != a) cE1[a] = mptr[m + 1];
  }
}

__device__ __forceinline__ bool hc_big(int64_t e0, int64_t e1) { return e1 - e0 > kHashWindow; }

// Window tasks: [tE0[w], tE1[w]) spans the small communities whose first
// entry lies in window w (tE0 starts at ~0, tE1 at 0: tE1 <= tE0 = no task).
// Big chunks: their task count per community.
__global__ void k_hc_windows(int64_t ncl, const int64_t *cE0, const int64_t *cE1,
                             unsigned long long *tE0, unsigned long long *tE1, int64_t *nbch) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < ncl;
       a += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e0 = cE0[a], e1 = cE1[a];
    int64_t nb = 0;
    if (e1 > e0) {
      if (hc_big(e0, e1)) {
        nb = (e1 - e0 + kHashTile - 1) / kHashTile;
      } else {
        const int64_t w = e0 / kHashWindow;
        atomicMin(&tE0[w], (unsigned long long)e0);
        atomicMax(&tE1[w], (unsigned long long)e1);
      }
    }
    nbch[a] = nb;
  }
}

// Big-community chunk tasks after the nwin window tasks.
__global__ void k_hc_big_tasks(int64_t ncl, int64_t nwin, const int64_t *cE0, const int64_t *cE1,
                               const int64_t *nbch_off, unsigned long long *tE0,
                               unsigned long long *tE1) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < ncl;
       a += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e0 = cE0[a], e1 = cE1[a];
    for (int64_t k = nbch_off[a]; k < nbch_off[a + 1]; ++k) {
      const int64_t x0 = e0 + (k - nbch_off[a]) * kHashTile;
      tE0[nwin + k] = (unsigned long long)x0;
      tE1[nwin + k] = (unsigned long long)min(x0 + kHashTile, e1);
    }
  }
}

// Global table slots of every big community (0 for the others): distinct
// neighbours <= min(entries, ncl), at most half full.  Chunks of kBigChunk
// slots for the emission.
__global__ void k_hc_big_caps(int64_t ncl, const int64_t *cE0, const int64_t *cE1, int64_t *cap,
                              int64_t *nchunk) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < ncl;
       a += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = 0;
    if (hc_big(cE0[a], cE1[a])) {
      const int64_t d = min(cE1[a] - cE0[a], ncl);
      c = 8;
      while (c < 2 * d + 2) c <<= 1;
    }
    cap[a] = c;
    nchunk[a] = (c + kBigChunk - 1) / kBigChunk;
  }
}

__global__ void k_hc_chunk_list(int64_t ncl, const int64_t *nchunk_off, int32_t *chunk_comm) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < ncl;
       a += (int64_t)gridDim.x * blockDim.x)
    for (int64_t k = nchunk_off[a]; k < nchunk_off[a + 1]; ++k) chunk_comm[k] = (int32_t)a;
}

__device__ __forceinline__ uint32_t pair_slot(uint64_t key) {
  const uint32_t a = (uint32_t)(key >> 32), b = (uint32_t)key;
  const uint32_t h = a * 0x9E3779B1u ^ b * 0x85EBCA77u;
  return (h ^ (h >> 15)) & (kHashTileSlots - 1);
}

__device__ __forceinline__ int64_t hc_member_of(const int64_t *mptr, int64_t nmem, int64_t e) {
  int64_t lo = 0, hi = nmem - 1;  // last member starting at or before e
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) >> 1;
    if (mptr[mid] <= e) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// First and last member of every task, one binary search per thread (ahead
// of the task kernel, so no block waits on a chain of dependent loads).
__global__ void k_hc_tile_members(int64_t ntask, const unsigned long long *tE0,
                                  const unsigned long long *tE1, const int64_t *mptr,
                                  int64_t nmem, int64_t *mlo, int64_t *mhi) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntask;
       t += (int64_t)gridDim.x * blockDim.x) {
    if (tE1[t] <= tE0[t]) continue;  // an empty window: tE0 = ~0, tE1 = 0 (unsigned)
    mlo[t] = hc_member_of(mptr, nmem, (int64_t)tE0[t]);
    mhi[t] = hc_member_of(mptr, nmem, (int64_t)tE1[t] - 1);
  }
}

struct HashTileArgs {
  int64_t ntask, nwin;          // tasks: nwin windows, then the big chunks
  int64_t nmem, ncl;
  const int64_t *mptr;          // nmem + 1
  const unsigned long long *tE0, *tE1;  // per task: entry range (empty window: tE1 <= tE0)
  const int64_t *mlo, *mhi;     // per task: first and last member
  const uint32_t *keys;         // member -> community
  const int32_t *verts;         // member -> vertex
  const int64_t *ptr;
  const int32_t *tail;
  const double *w;
  const int32_t *Cm;
  const int64_t *cE0;           // community -> first entry (its row's output offset)
  const int64_t *gtoff;         // big community -> table offset (cap = gtoff[a+1] - gtoff[a])
  int32_t *gkeys;               // big tables: neighbour community (-1 empty)
  double *gvals;
  int32_t *out_b;               // community a's row at [cE0[a], cE0[a] + cnt[a])
  double *out_w;
  int64_t *cnt;
  uint8_t *has_self;            // 1: the row has its (a, a) entry
  int32_t *err;                 // a global table that filled up (cannot happen: half full)
  // dense output (few communities): every (a, b) sum goes to dense[a * ncl + b]
  // and its presence bit, instead of the rows and tables above
  double *dense;
  uint32_t *dense_bits;
};

struct HashTileSmem {
  uint64_t key[kHashTileSlots];
  double val[kHashTileSlots];
  int64_t rdelta[kHashTile];    // member's CSR index minus its entry offset
  int64_t c0[kHashTile];        // member's community's first entry
  int32_t mofs[kHashTile + 1];  // member entry offsets relative to the task start (clamped)
  uint32_t comm[kHashTile];     // member's community (non-decreasing)
  int32_t cnt[kHashTile];       // at a community's first member: entries written
};

__global__ void __launch_bounds__(kHashThreads) k_hc_tiles(HashTileArgs p) {
  extern __shared__ unsigned char smem_raw[];
  HashTileSmem &sm = *reinterpret_cast<HashTileSmem *>(smem_raw);
  const int lane = threadIdx.x & 31;
  for (int64_t task = blockIdx.x; task < p.ntask; task += gridDim.x) {
    if (p.tE1[task] <= p.tE0[task]) continue;  // an empty window (unsigned; block-uniform)
    const int64_t e0 = (int64_t)p.tE0[task], e1 = (int64_t)p.tE1[task];
    const bool window = task < p.nwin;
    for (int s = threadIdx.x; s < kHashTileSlots; s += kHashThreads) {
      sm.key[s] = kEmptyPair;
      sm.val[s] = 0.0;
    }
    const int64_t m_lo = p.mlo[task];
    const int nm = (int)(p.mhi[task] - m_lo + 1);  // <= kHashTile: every member has an entry
    for (int k = threadIdx.x; k <= nm; k += kHashThreads) {
      const int64_t m = m_lo + k;
      sm.mofs[k] = (int32_t)max((int64_t)-1, min(p.mptr[m] - e0, (int64_t)kHashTile + 1));
      if (k < nm) {
        const int32_t v = p.verts[m];
        const uint32_t c = p.keys[m];
        sm.rdelta[k] = p.ptr[v] - p.mptr[m];
        sm.comm[k] = c;
        sm.cnt[k] = 0;
        sm.c0[k] = (window && !p.dense) ? p.cE0[c] : 0;
      }
    }
    __syncthreads();
    // entries: all loads of a thread's kHashPer entries issue before any use
    int32_t t[kHashPer], b[kHashPer];
    uint32_t a[kHashPer];
    double wt[kHashPer];
#pragma unroll
    for (int q = 0; q < kHashPer; ++q) {
      const int r = q * kHashThreads + threadIdx.x;
      const int64_t e = e0 + r;
      t[q] = -1;
      a[q] = 0;
      wt[q] = 0.0;
      if (e < e1) {
        int lo = 0, hi = nm - 1;
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (sm.mofs[mid] <= r) lo = mid; else hi = mid - 1;
        }
        const int64_t j = e + sm.rdelta[lo];
        t[q] = __ldcs(&p.tail[j]);
        wt[q] = __ldcs(&p.w[j]);
        a[q] = sm.comm[lo];
      }
    }
#pragma unroll
    for (int q = 0; q < kHashPer; ++q) b[q] = (t[q] >= 0) ? p.Cm[t[q]] : -1;
#pragma unroll
    for (int q = 0; q < kHashPer; ++q) {
      const bool has = b[q] >= 0;
      const uint64_t key = has ? (((uint64_t)a[q] << 32) | (uint32_t)b[q]) : (kEmptyPair - lane);
      const unsigned m = __match_any_sync(FULL, key);
      const bool leader = has && lane == __ffs(m) - 1;
      double acc = 0.0;
      unsigned rem = leader ? m : 0u;
      const int rounds = __reduce_max_sync(FULL, (unsigned)__popc(rem));
      for (int it = 0; it < rounds; ++it) {
        const int src = rem ? __ffs(rem) - 1 : lane;
        const double x = __shfl_sync(FULL, wt[q], src);
        if (rem) { acc += x; rem &= rem - 1; }
      }
      if (leader) {
        uint32_t s = pair_slot(key);
        while (true) {  // at most kHashTile keys in kHashTileSlots slots: a slot is found
          const uint64_t old = atomicCAS((unsigned long long *)&sm.key[s],
                                         (unsigned long long)kEmptyPair, (unsigned long long)key);
          if (old == kEmptyPair || old == key) break;
          s = (s + 1) & (kHashTileSlots - 1);
        }
        atomicAdd(&sm.val[s], acc);
      }
    }
    __syncthreads();
    // flush: a window's communities are final here; a big chunk's sums go to
    // its community's table; dense mode adds everything into the matrix
    for (int s = threadIdx.x; s < kHashTileSlots; s += kHashThreads) {
      const uint64_t key = sm.key[s];
      if (key == kEmptyPair) continue;
      const uint32_t ca = (uint32_t)(key >> 32);
      const int32_t cb = (int32_t)(uint32_t)key;
      const double val = sm.val[s];
      if (p.dense) {
        const int64_t cell = (int64_t)ca * p.ncl + cb;
        atomicAdd(&p.dense[cell], val);
        atomicOr(&p.dense_bits[cell >> 5], 1u << (cell & 31));
      } else if (window) {
        int lo = 0, hi = nm - 1;  // the community's first member in the task
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (sm.comm[mid] < ca) lo = mid + 1; else hi = mid;
        }
        const int64_t c0 = sm.c0[lo];
        const int k = atomicAdd(&sm.cnt[lo], 1);
        p.out_b[c0 + k] = cb;
        p.out_w[c0 + k] = val;
        if (cb == (int32_t)ca) p.has_self[ca] = 1;
      } else {
        const int64_t off = p.gtoff[ca];
        const uint32_t mask = (uint32_t)(p.gtoff[ca + 1] - off - 1);
        uint32_t g = hash_slot(cb, mask);
        bool done = false;
        for (uint32_t probe = 0; probe <= mask; ++probe) {
          const int32_t old = atomicCAS(&p.gkeys[off + g], -1, cb);
          if (old == -1 || old == cb) { done = true; break; }
          g = (g + 1) & mask;
        }
        if (done) atomicAdd(&p.gvals[off + g], val);
        else atomicExch(p.err, 1);
      }
    }
    __syncthreads();
    // row lengths of the window's communities (members come in community
    // order, so a community's first member in the window is its first)
    if (window && !p.dense)
      for (int k = threadIdx.x; k < nm; k += kHashThreads) {
        const uint32_t ca = sm.comm[k];
        if (k == 0 || sm.comm[k - 1] != ca) p.cnt[ca] = sm.cnt[k];
      }
    __syncthreads();  // the next task reuses the shared arrays
  }
}

// The big communities' tables, kBigChunk slots per block task: filled slots
// are appended to the community's row (one counter update per block).
// Launched with 256 threads.
__global__ void __launch_bounds__(256) k_hc_big_emit(int64_t nchunks, const int32_t *chunk_comm,
                                                     const int64_t *nchunk_off,
                                                     const int64_t *gtoff, const int32_t *gkeys,
                                                     const double *gvals, const int64_t *cE0,
                                                     int32_t *out_b, double *out_w, int64_t *cnt,
                                                     uint8_t *has_self) {
  __shared__ int s_n[8];
  __shared__ int64_t s_base;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t ch = blockIdx.x; ch < nchunks; ch += gridDim.x) {
    const int32_t ca = chunk_comm[ch];
    const int64_t off = gtoff[ca], cap = gtoff[ca + 1] - off;
    const int64_t s0 = (ch - nchunk_off[ca]) * kBigChunk, s1 = min(s0 + kBigChunk, cap);
    // count, then write at a block-wide offset
    int mine = 0;
    for (int64_t s = s0 + threadIdx.x; s < s1; s += blockDim.x) mine += (gkeys[off + s] >= 0);
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_n[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) { const int x = s_n[k]; s_n[k] = tot; tot += x; }
      s_base = tot ? (int64_t)atomicAdd((unsigned long long *)&cnt[ca], (unsigned long long)tot) : 0;
    }
    __syncthreads();
    int64_t o = cE0[ca] + s_base + s_n[warp] + incl - mine;
    for (int64_t s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
      const int32_t cb = gkeys[off + s];
      if (cb < 0) continue;
      out_b[o] = cb;
      out_w[o] = gvals[off + s];
      if (cb == ca) has_self[ca] = 1;
      ++o;
    }
    __syncthreads();
  }
}

// Row lengths: the emitted entries plus an (a, a) entry where none was.
__global__ void k_hc_row_lengths(int64_t ncl, const int64_t *cnt, const uint8_t *has_self,
                                 int64_t *rowc) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < ncl;
       a += (int64_t)gridDim.x * blockDim.x)
    rowc[a] = cnt[a] + (has_self[a] ? 0 : 1);
  if (blockIdx.x == 0 && threadIdx.x == 0) rowc[ncl] = 0;
}

// Dense output: row a's entries are the set presence bits of cells
// [a * ncl, (a + 1) * ncl), in ascending b; an (a, a) entry is added where
// its bit is clear.  One warp per row.
__global__ void k_hc_dense_counts(int64_t ncl, const uint32_t *bits, int64_t *rowc) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t a = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < ncl; a += warps) {
    int64_t n = 0;
    for (int64_t b = lane; b < ncl; b += 32) {
      const int64_t cell = a * ncl + b;
      n += (bits[cell >> 5] >> (cell & 31)) & 1u;
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) n += __shfl_xor_sync(FULL, n, off);
    const int64_t self = a * ncl + a;
    if (lane == 0) rowc[a] = n + (((bits[self >> 5] >> (self & 31)) & 1u) ? 0 : 1);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) rowc[ncl] = 0;
}

__global__ void k_hc_dense_emit(int64_t ncl, const uint32_t *bits, const double *dense,
                                const int64_t *optr, int32_t *otail, double *ow) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t a = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < ncl; a += warps) {
    int64_t o = optr[a];
    for (int64_t b0 = 0; b0 < ncl; b0 += 32) {
      const int64_t b = b0 + lane;
      const int64_t cell = a * ncl + b;
      const bool set = b < ncl && ((bits[cell >> 5] >> (cell & 31)) & 1u);
      const bool on = set || b == a;
      const unsigned m = __ballot_sync(FULL, on);
      if (on) {
        const int64_t q = o + __popc(m & ((1u << lane) - 1u));
        otail[q] = (int32_t)b;
        ow[q] = set ? dense[cell] : 0.0;
      }
      o += __popc(m);
    }
  }
}

constexpr int kCopyTile = 2048;

// First and last row of every output tile.
__global__ void k_hc_copy_rows(int64_t ntiles, int64_t ncl, const int64_t *optr, int64_t *alo,
                               int64_t *ahi) {
  const int64_t nnz = optr[ncl];
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < ntiles;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x0 = t * kCopyTile, x1 = min(x0 + kCopyTile, nnz) - 1;
    for (int side = 0; side < 2; ++side) {
      const int64_t x = side ? x1 : x0;
      int64_t lo = 0, hi = ncl - 1;  // last row starting at or before x
      while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (optr[mid] <= x) lo = mid; else hi = mid - 1;
      }
      (side ? ahi : alo)[t] = lo;
    }
  }
}

// Output positions in tiles of kCopyTile: each row is copied from its
// community's entry range, the missing (a, a, 0.0) entry first.
__global__ void __launch_bounds__(256) k_hc_compact(int64_t ncl, const int64_t *optr,
                                                    const int64_t *alo, const int64_t *ahi,
                                                    const int64_t *cE0, const uint8_t *has_self,
                                                    const int32_t *in_b, const double *in_w,
                                                    int32_t *otail, double *ow) {
  __shared__ int64_t s_ptr[kCopyTile + 1];
  __shared__ int64_t s_src[kCopyTile];
  __shared__ uint8_t s_seed[kCopyTile];
  const int64_t nnz = optr[ncl];
  const int64_t ntiles = (nnz + kCopyTile - 1) / kCopyTile;
  for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int64_t p0 = tile * kCopyTile, p1 = min(p0 + kCopyTile, nnz);
    const int64_t a0 = alo[tile];
    const int nr = (int)(ahi[tile] - a0 + 1);  // <= kCopyTile: every row has an entry
    for (int k = threadIdx.x; k <= nr; k += blockDim.x) {
      s_ptr[k] = optr[a0 + k];
      if (k < nr) {
        const uint8_t seed = has_self[a0 + k] ? 0 : 1;
        s_seed[k] = seed;
        s_src[k] = cE0[a0 + k] - seed;
      }
    }
    __syncthreads();
    for (int64_t q = p0 + threadIdx.x; q < p1; q += blockDim.x) {
      int lo = 0, hi = nr - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s_ptr[mid] <= q) lo = mid; else hi = mid - 1;
      }
      const int64_t k = q - s_ptr[lo];
      const bool seed = k == 0 && s_seed[lo];
      otail[q] = seed ? (int32_t)(a0 + lo) : in_b[s_src[lo] + k];
      ow[q] = seed ? 0.0 : in_w[s_src[lo] + k];
    }
    __syncthreads();
  }
}

}  // namespace glv
