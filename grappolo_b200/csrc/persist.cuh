// One Louvain iteration in one cooperative launch (parallel-accumulation modes).
//
// The colour classes of an iteration depend on each other (a class decides
// against the community totals left by the classes before it), and R-MAT-like
// graphs need hundreds of classes, most of them small and made of high-degree
// vertices.  Launching a few kernels per class leaves the GPU waiting on
// launches and on the single largest row of each class.  Here every block of
// a persistent grid takes part in every class:
//   stage 1  hub rows on thread-block clusters (one table over the shared
//            memory of a cluster's blocks) or, without clusters, hub chunks
//            (global tables); rows of 1024..4095 entries per
//            block; rows of 128..1023 entries per 128-thread team (shared
//            tables); then warp items (rows <= 32 entries, and 33..127-entry
//            rows with a per-warp shared table)                  -> grid barrier
//            (a hub with more filled slots than its last chunk's block
//            scans is decided by scan-segment tasks of the same queue)
//   stage 2  community totals += the class's deltas             -> grid barrier
// (stage 2 after the class's last sublevel), then the modularity pass of the
// iteration.
#pragma once

#include <cooperative_groups.h>

#include "phase_kernels.cuh"
#include "sweep.cuh"

namespace glv {

struct StepDesc {
  int64_t seg[NBINS + 1];  // member positions of each degree bin
  int64_t hub_chunk[2];    // hub accumulation work items
  int64_t hub_segs[2];     // hub scan work items
  int64_t apply[2];        // member range whose deltas are applied after this step
  int64_t cls;             // colour class of the step
  int64_t ctask[2];        // hub tasks on thread-block clusters (cluster_row_tasks)
};

struct IterArgs {
  SweepArgs a;
  HubWork h;
  const StepDesc *steps;
  int nsteps;
  int jacobi;              // 1: Q on the state before the moves, totals updated after
  int64_t nv;
  const int32_t *C_mod;    // communities the modularity pass compares (colour phases)
  const double *own_w_mod; // Jacobi phases: Counter[own] per vertex
  double *part_e, *part_a; // per 256-vertex tile partials
  const double *cst;       // {constant, 2m}
  double *mod_out;         // {Q, e_xx, a2_x}
  double *cDeg;
  int32_t *cSize;
  uint64_t *trace;         // optional: globaltimer at each barrier, 4 per step + 2
  int64_t *task_ctr;       // per step: next block, team and cluster task (zero at launch)
  const int32_t *class_kept;  // gated sweeps: vertices the gate kept per class (NULL = all)
  int64_t nnz;
  const int64_t *split_row;   // merge-path tile boundaries of the level
  // batches of graphs: per-graph modularity sums instead of one Q
  const int32_t *gid;
  double *gacc;
  // The internal-weight term e_xx: 0 = a full pass over the level (stored in
  // exx_state); 1 = exx_state plus this sweep's moves' changes (a.exx_delta),
  // with only sum cDeg^2 taken in full; 2 = both, Q from the carried value
  // and the full pass's e_xx in mod_out[3] (a self-check)
  int exx_mode;
  double *exx_state;
  // Carried e_xx with classes that are not independent sets (core batches):
  // the CSR entries (member slot of u, member slot of t, w) whose two ends
  // run in the same step.  Each move's change 2 (e_iy - e_ix) assumes its
  // neighbours stay; for such an entry whose two ends both moved the carried
  // sum is corrected by w ([y_u == y_t] + [x_u == x_t] - [y_u == x_t] - [x_u == y_t]).
  const int32_t *pair_u, *pair_t;
  const double *pair_w;
  int64_t npairs;
};

// Gated or batched sweeps: kept[c] = 1 when some member of colour class c is
// evaluated (kept must be zero on entry).  Member positions are strided over
// the grid; a position's class is found by binary search in cls_begin.
__global__ void k_class_kept(int nclass, const int64_t *cls_begin, int64_t nmem,
                             const int32_t *members, const uint8_t *skip, int32_t *kept) {
  for (int64_t pos = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < nmem;
       pos += (int64_t)gridDim.x * blockDim.x) {
    if (skip[members[pos]]) continue;
    int lo = 0, hi = nclass - 1;  // last class starting at or before pos
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (cls_begin[mid] <= pos) lo = mid; else hi = mid - 1;
    }
    if (kept[lo] == 0) kept[lo] = 1;
  }
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

#define GLV_TRACE(slot)                                                  \
  do {                                                                   \
    if (p.trace && blockIdx.x == 0 && threadIdx.x == 0) p.trace[slot] = global_ns(); \
  } while (0)

// Debug traces, 4 slots per step after the 4 per step + 2: the latest time
// over the grid at which a queue of step s ran dry (q = 0 block queue, 1 team
// queue, 2 warp items, 3 cluster tasks).
#define GLV_QTRACE(s, q, cond)                                                       \
  do {                                                                               \
    if (p.trace && (cond))                                                           \
      atomicMax((unsigned long long *)&p.trace[4 * p.nsteps + 2 + 4 * (s) + (q)],    \
                (unsigned long long)global_ns());                                    \
  } while (0)

constexpr int kPersistThreads = 512;
constexpr int kPersistTableCap = 8192;  // BIN_BLOCK rows: degree <= 4095
constexpr int kPersistWarpCap = 256;    // warp-table rows: degree <= 127
constexpr int kTeamThreads = 128;      // team of the 128..1023-entry rows
constexpr int kTeamCap = 2048;         // its table: table_cap(1023)
constexpr size_t kPersistSmem = (size_t)kPersistTableCap * (sizeof(double) + sizeof(int32_t));
static_assert(kPersistThreads / kTeamThreads * kTeamCap == kPersistTableCap,
              "team tables tile the block table");
static_assert(kTeamThreads / 32 * kPersistWarpCap <= kTeamCap,
              "warp tables tile their team's table");
static_assert(kPersistSmem >= sizeof(MergeSmem), "merge tiles must fit");
static_assert(kPersistTableCap >= kClusterBlockSlots, "a cluster table part must fit");
static_assert(kHubStageCap * (sizeof(double) + sizeof(int32_t)) <=
                  (size_t)kPersistTableCap * sizeof(double),
              "a hub chunk's staging values and filled-slot list sit below the table keys");
static_assert(kPersistSmem >= (size_t)(kPersistThreads / 32) * kPersistWarpCap *
                                  (sizeof(double) + sizeof(int32_t)),
              "warp tables must fit in the block-table region");

// Community totals += the deltas the sweep accumulated (see k_apply_deltas).
__device__ __forceinline__ void apply_deltas_range(const IterArgs &p, int64_t b, int64_t e,
                                                   int64_t gt, int64_t ngt) {
  for (int64_t pos = b + gt; pos < e; pos += ngt) {
    const int32_t o = p.a.move_old[pos];
    if (p.a.defer_c) {
      // deferred decisions: moves, and isolated vertices leaving every community
      const int32_t n = p.a.move_new[pos];
      if (o >= 0 || n < 0) p.a.C[p.a.members[pos]] = n;
    }
    if (o < 0) continue;
    const int32_t cs[2] = {p.a.move_new[pos], o};
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int32_t c = cs[k];
      const unsigned long long bits = atomicExch((unsigned long long *)&p.a.dDeg[c], 0ull);
      if (bits != 0ull) p.cDeg[c] = __dadd_rn(p.cDeg[c], __longlong_as_double((long long)bits));
      const int32_t s = atomicExch(&p.a.dSize[c], 0);
      if (s != 0) p.cSize[c] += s;
    }
  }
}

// Q from the per-block partials (block 0, all threads).
__device__ __forceinline__ void modularity_fold(const IterArgs &p, int64_t nparts, double *sh) {
  double e = 0.0, a = 0.0, d = 0.0;
  const int64_t per = (nparts + blockDim.x - 1) / blockDim.x;
  const int64_t b = threadIdx.x * per, en = min(nparts, b + per);
  for (int64_t i = b; i < en; ++i) {
    e = __dadd_rn(e, p.part_e[i]);
    a = __dadd_rn(a, p.part_a[i]);
    if (p.exx_mode == 2) d = __dadd_rn(d, p.a.exx_delta[i]);
  }
  e = block_sum<kPersistThreads>(e, sh);
  a = block_sum<kPersistThreads>(a, sh);
  if (p.exx_mode == 2) d = block_sum<kPersistThreads>(d, sh);
  if (threadIdx.x == 0) {
    const double c = p.cst[0];
    double exx = e;  // mode 0: the full pass
    if (p.exx_mode == 1) exx = __dadd_rn(p.exx_state[0], e);  // e holds the moves' changes
    if (p.exx_mode == 2) {
      exx = __dadd_rn(p.exx_state[0], d);
      p.mod_out[3] = e;
    }
    if (p.exx_state) p.exx_state[0] = exx;
    p.mod_out[0] = __dsub_rn(__dmul_rn(exx, c), __dmul_rn(__dmul_rn(a, c), c));
    p.mod_out[1] = exx;
    p.mod_out[2] = a;
  }
}

// kClusters: the instantiation launched with a cluster dimension, which runs
// the steps' cluster tasks; the other one leaves that code out entirely (its
// registers go to the other paths).
template <bool kClusters>
__global__ void __launch_bounds__(kPersistThreads, 2) k_sweep_iteration(IterArgs p) {
  cg::grid_group grid = cg::this_grid();
  extern __shared__ unsigned char smem_raw[];
  __shared__ double s_self[32], s_g[32], sh[32];
  __shared__ int32_t s_c[32];
  const int warp = threadIdx.x >> 5, nwb = blockDim.x >> 5;
  const int64_t ngw = (int64_t)gridDim.x * nwb;
  // warps numbered across blocks first: a step with few warp items spreads over SMs
  const int64_t gwi = (int64_t)warp * gridDim.x + blockIdx.x;
  const int64_t gt = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t ngt = (int64_t)gridDim.x * blockDim.x;
  // shared table region: one 8192-slot table (block tasks), four 2048-slot
  // team tables, or a 256-slot table per warp inside its team's table
  const int team = threadIdx.x / kTeamThreads, tt = threadIdx.x % kTeamThreads;
  double *tvals = reinterpret_cast<double *>(smem_raw);
  int32_t *tkeys = reinterpret_cast<int32_t *>(tvals + kPersistTableCap);
  double *team_vals = tvals + (size_t)team * kTeamCap;
  int32_t *team_keys = tkeys + (size_t)team * kTeamCap;
  double *wvals = team_vals + (size_t)(tt >> 5) * kPersistWarpCap;
  int32_t *wkeys = team_keys + (size_t)(tt >> 5) * kPersistWarpCap;
  GLV_TRACE(4 * p.nsteps);
  // next task of the block and team queues, by task parity: the following
  // task is fetched when a task starts and published after it ends
  __shared__ int64_t s_task[2];
  __shared__ int64_t s_team_task[kPersistThreads / kTeamThreads][2];
  __shared__ int s_flag;
  __shared__ uint32_t s_word;
  __shared__ ClusterShared s_cluster;
  // this block's slot of the moves' e_xx changes (only this block writes it)
  if (p.a.exx_delta && threadIdx.x == 0) p.a.exx_delta[blockIdx.x] = 0.0;
  for (int s = 0; s < p.nsteps; ++s) {
    const StepDesc &st = p.steps[s];
    // a class the gate emptied is skipped whole (no work, no barrier)
    if (p.class_kept && p.class_kept[st.cls] == 0) continue;
    // Stage 1 in three parts, each from its own queue: (A) hub chunks and
    // rows of 1024..4095 entries, whole blocks with an 8192-slot table;
    // (B) rows of 128..1023 entries, 128-thread teams (four per block, each
    // fetching its own rows, 2048-slot tables); (C) warp items (rows of up to
    // 32 entries, several per warp; rows of 33..127 entries, one per warp),
    // item t to warp t mod (warps of the grid), in the warp's slice of its
    // team's table region.
    const int64_t n4 = st.seg[1] - st.seg[0], n8 = st.seg[2] - st.seg[1];
    const int64_t n16 = st.seg[3] - st.seg[2], n32 = st.seg[4] - st.seg[3];
    const int64_t nw = st.seg[5] - st.seg[4];
    const int64_t i4 = (n4 + 7) / 8, i8 = (n8 + 3) / 4, i16 = (n16 + 1) / 2;
    const int64_t witems = i4 + i8 + i16 + n32 + nw;
    const int64_t t_hub = st.hub_chunk[1] - st.hub_chunk[0];
    const int64_t t_blk = st.seg[BIN_BLOCK + 1] - st.seg[BIN_BLOCK];
    const int64_t t_seg = st.hub_segs[1] - st.hub_segs[0];
    const int64_t n256 = st.seg[BIN_T256 + 1] - st.seg[BIN_T256];
    const int64_t n128 = st.seg[BIN_T128 + 1] - st.seg[BIN_T128];
    const int64_t t_ct = kClusters ? st.ctask[1] - st.ctask[0] : 0;
    if constexpr (kClusters) if (t_ct > 0) {
      // hub rows on clusters (launches with a cluster dimension): every block
      // of a cluster takes part in every task of its cluster
      cluster_row_tasks(p.a, p.h, st.ctask[0], t_ct, &p.task_ctr[3 * s + 2],
                        reinterpret_cast<int32_t *>(tvals + kPersistTableCap), tvals, &s_cluster,
                        s_g, s_c);
      GLV_QTRACE(s, 3, threadIdx.x == 0);
    }
    if (t_hub + t_blk + t_seg > 0) {
      // hub chunks, then block rows, then hub scan segments (which wait for
      // their hub's chunks: every chunk is handed out before any segment)
      unsigned long long *ctr = (unsigned long long *)&p.task_ctr[3 * s];
      if (threadIdx.x == 0) s_task[0] = (int64_t)atomicAdd(ctr, 1ull);
      __syncthreads();
      for (unsigned it = 0;; ++it) {
        const int64_t t = s_task[it & 1];
        if (t >= t_hub + t_blk + t_seg) break;
        const int64_t nxt = (threadIdx.x == 0) ? (int64_t)atomicAdd(ctr, 1ull) : 0;
        if (t < t_hub) {
          hub_accum_chunk(p.a, p.h, st.hub_chunk[0] + t,
                          reinterpret_cast<int32_t *>(tvals + kPersistTableCap), tvals, s_self,
                          s_g, s_c, &s_flag, s);
        } else if (t < t_hub + t_blk) {
          team_vertex<512>(p.a, st.seg[BIN_BLOCK] + (t - t_hub),
                           reinterpret_cast<int32_t *>(tvals + kPersistTableCap), tvals, 0, s_self,
                           s_g, s_c);
        } else {
          hub_segment_task(p.a, p.h, st.hub_segs[0] + (t - t_hub - t_blk), s_g, s_c, &s_word);
        }
        if (threadIdx.x == 0) s_task[(it + 1) & 1] = nxt;
        __syncthreads();
      }
      GLV_QTRACE(s, 0, threadIdx.x == 0);
    }
    if (n256 + n128 > 0) {
      unsigned long long *ctr = (unsigned long long *)&p.task_ctr[3 * s + 1];
      if (tt == 0) s_team_task[team][0] = (int64_t)atomicAdd(ctr, 1ull);
      team_sync<128>(team);
      for (unsigned it = 0;; ++it) {
        const int64_t t = s_team_task[team][it & 1];
        if (t >= n256 + n128) break;
        const int64_t nxt = (tt == 0) ? (int64_t)atomicAdd(ctr, 1ull) : 0;
        const int64_t pos = (t < n256) ? st.seg[BIN_T256] + t : st.seg[BIN_T128] + (t - n256);
        team_vertex<128>(p.a, pos, team_keys, team_vals, team, s_self + 4 * team,
                         s_g + 4 * team, s_c + 4 * team);
        if (tt == 0) s_team_task[team][(it + 1) & 1] = nxt;
        team_sync<128>(team);
      }
      GLV_QTRACE(s, 1, tt == 0);
    }
    for (int64_t k = gwi; k < witems; k += ngw) {
      int64_t q = k;
      if (q < i4) { small_item<4>(p.a, st.seg[0] + 8 * q, st.seg[1]); continue; }
      q -= i4;
      if (q < i8) { small_item<8>(p.a, st.seg[1] + 4 * q, st.seg[2]); continue; }
      q -= i8;
      if (q < i16) { small_item<16>(p.a, st.seg[2] + 2 * q, st.seg[3]); continue; }
      q -= i16;
      if (q < n32) { small_item<32>(p.a, st.seg[3] + q, st.seg[4]); continue; }
      q -= n32;
      warp_table_vertex(p.a, st.seg[4] + q, wkeys, wvals);
    }
    GLV_QTRACE(s, 2, (threadIdx.x & 31) == 0 && gwi < witems);
    grid.sync();
    GLV_TRACE(4 * s);
    if (!p.jacobi && st.apply[1] > st.apply[0]) {
      apply_deltas_range(p, st.apply[0], st.apply[1], gt, ngt);
      grid.sync();
      GLV_TRACE(4 * s + 3);
    }
  }
  {
    // merge-path tiles, one partial pair per block
    double ex = 0.0, a2 = 0.0;
    const int64_t ntiles = merge_tiles(p.nv, p.nnz);
    MergeSmem *msm = reinterpret_cast<MergeSmem *>(smem_raw);
    __syncthreads();  // stage-1 tables in the same shared memory are done
    if (p.exx_mode >= 1 && p.npairs > 0) {
      // same-step entries whose two ends both moved (see IterArgs::pair_u)
      double corr = 0.0;
      for (int64_t k = gt; k < p.npairs; k += ngt) {
        const int32_t pu = p.pair_u[k], pt = p.pair_t[k];
        const int32_t xu = p.a.move_old[pu], xt = p.a.move_old[pt];
        if (xu < 0 || xt < 0) continue;
        const int32_t yu = p.a.move_new[pu], yt = p.a.move_new[pt];
        const int f = (yu == yt) + (xu == xt) - (yu == xt) - (xu == yt);
        if (f != 0) corr = __dadd_rn(corr, __dmul_rn((double)f, p.pair_w[k]));
      }
      corr = block_sum<kPersistThreads>(corr, sh);
      if (threadIdx.x == 0 && corr != 0.0) p.a.exx_delta[blockIdx.x] += corr;
      __syncthreads();
    }
    if (p.exx_mode == 1) {
      // e_xx is carried: only a2 = sum of cDeg^2 over the level
      for (int64_t c = gt; c < p.nv; c += ngt) a2 = __dadd_rn(a2, __dmul_rn(p.cDeg[c], p.cDeg[c]));
      if (threadIdx.x == 0) ex = p.a.exx_delta[blockIdx.x];
    } else if (p.gid) {
      // contiguous tile ranges, so a thread's running pair changes graph rarely
      GraphAcc acc;
      const int64_t tb = ntiles * blockIdx.x / gridDim.x;
      const int64_t te = ntiles * (blockIdx.x + 1) / gridDim.x;
      for (int64_t tile = tb; tile < te; ++tile)
        modularity_merge_tile_graphs<kPersistThreads>(tile, p.nv, p.nnz, p.a.ptr, p.a.tail, p.a.w,
                                                      p.C_mod, p.own_w_mod, p.cDeg, p.split_row,
                                                      p.gid, p.gacc, msm, acc);
      graph_acc_flush(acc, p.gacc);
    } else {
      for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
        modularity_merge_tile<kPersistThreads>(tile, p.nv, p.nnz, p.a.ptr, p.a.tail, p.a.w,
                                               p.C_mod, p.own_w_mod, p.cDeg, p.split_row, msm, ex,
                                               a2);
    }
    ex = block_sum<kPersistThreads>(ex, sh);
    a2 = block_sum<kPersistThreads>(a2, sh);
    if (threadIdx.x == 0) { p.part_e[blockIdx.x] = ex; p.part_a[blockIdx.x] = a2; }
  }
  grid.sync();
  GLV_TRACE(4 * p.nsteps + 1);
  if (blockIdx.x == 0) {
    if (!p.gid) modularity_fold(p, gridDim.x, sh);
    if (threadIdx.x == 0) p.mod_out[4] = (double)__ldcg(p.h.err);
  }
  if (p.jacobi && p.nsteps > 0) {
    // Q above used the totals before the moves; now take the moves' deltas.
    apply_deltas_range(p, p.steps[0].apply[0], p.steps[p.nsteps - 1].apply[1], gt, ngt);
  }
}

}  // namespace glv
