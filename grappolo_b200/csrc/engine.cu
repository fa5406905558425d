// Host side of the B200 Louvain engine: device-resident levels, the colour /
// degree-bin schedule, CUDA-graph-captured sweep iterations, the multiphase
// drivers and the C ABI declared in include/grappolo_b200.h.
#include <algorithm>
#include <cmath>
#include <climits>
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <string>
#include <map>
#include <unordered_map>
#include <vector>

#include <functional>
#include <mutex>
#include <thread>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "batch_kernels.cuh"
#include "gate.cuh"
#include "persist.cuh"
#include "recolor.cuh"
#include "vbase.cuh"
#include "coarsen_hash.cuh"
#include "phase_kernels.cuh"
#include "sweep.cuh"

namespace glv {

static std::atomic<long> g_launches{0};

// Library-owned stream-ordered memory pool per device.  Freed blocks stay
// cached in the pool (release threshold = max), so the large per-phase buffers
// of one run (and of the next run) do not go back to the driver at every
// synchronisation; glv_release_cached_memory() returns them.
static std::mutex g_pool_mu;
constexpr int kMaxDevices = 128;  // device ordinals the per-device tables cover
static cudaMemPool_t g_pool[kMaxDevices];

static cudaMemPool_t engine_pool() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pool[dev] = p;
  }
  return g_pool[dev];
}
// One internal stream per device, created once.  Creating and destroying a
// stream per call made the first pool allocation of the next call wait
// (0.1-0.9 s) while the pool settled the blocks freed on the destroyed
// stream.  Calls from several host threads on one device share the stream,
// so their work is serialised (each call still waits only for its own
// results).
static std::mutex g_stream_mu;
static cudaStream_t g_stream[kMaxDevices];
static cudaError_t engine_stream(cudaStream_t *s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_stream_mu);
  if (!g_stream[dev]) {
    e = cudaStreamCreateWithFlags(&g_stream[dev], cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
  }
  *s = g_stream[dev];
  return cudaSuccess;
}

// Blocks the engine freed, kept by device and size class and handed to later
// allocations of the same class.  All engine work on a device runs on its one
// internal stream, so a block reused here is ordered after its last use.  In
// steady state (the same call repeated) no allocation reaches the driver: a
// pool allocation after a call's frees sometimes waited 0.1-0.9 s.  A failed
// pool allocation first returns the cached blocks; glv_release_cached_memory
// returns them too.
struct BlockCache {
  std::mutex mu;
  std::map<size_t, std::vector<void *>> free;  // by size class, ascending
  std::unordered_map<void *, size_t> live;
  std::unordered_map<void *, uint64_t> last_use;  // call generation of the block's last use
  uint64_t gen = 0;                                // calls finished on this device
};
static BlockCache g_cache[kMaxDevices];

// End of a call: blocks the call did not use go back to the pool, so a
// workload whose sizes change (the waves of a batch) does not hoard memory.
static void end_call_block_cache(int dev, cudaStream_t s) {
  if (dev < 0 || dev >= kMaxDevices) return;
  BlockCache &bc = g_cache[dev];
  std::lock_guard<std::mutex> lock(bc.mu);
  for (auto &kv : bc.free) {
    auto &v = kv.second;
    size_t keep = 0;
    for (size_t i = 0; i < v.size(); ++i) {
      auto it = bc.last_use.find(v[i]);
      if (it != bc.last_use.end() && it->second >= bc.gen) {
        v[keep++] = v[i];
      } else {
        if (it != bc.last_use.end()) bc.last_use.erase(it);
        cudaFreeAsync(v[i], s);
      }
    }
    v.resize(keep);
  }
  ++bc.gen;
}

static int current_device() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) d = 0;
  return d;
}

static void flush_block_cache(int dev, cudaStream_t s) {
  if (dev < 0 || dev >= kMaxDevices) return;
  BlockCache &bc = g_cache[dev];
  std::lock_guard<std::mutex> lock(bc.mu);
  for (auto &kv : bc.free)
    for (void *q : kv.second) {
      bc.last_use.erase(q);
      cudaFreeAsync(q, s);
    }
  bc.free.clear();
}

static std::atomic<int> g_profile{0};  // 0 off, 1 per-class sweep, 2 per launch

// Learned gate (process-wide): parameters and keep threshold.
static std::mutex g_gate_mu;
static std::vector<float> g_gate_params;
static float g_gate_tau = 0.5f;

// Trace capture for training: (features, moved) rows of plain colour sweeps.
struct TraceSink {
  bool on = false;
  double rate = 1.0;
  int64_t cap = 0;
  int device = -1;
  float *x = nullptr;      // [cap][6]
  float *y = nullptr;      // [cap]
  unsigned long long *n = nullptr;
};
static TraceSink g_trace;
static thread_local std::string g_err;

static int fail(int code, const char *msg) {
  g_err = msg;
  return code;
}
static int fail(int code, const std::string &msg) { return fail(code, msg.c_str()); }

#define CK(expr)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (expr);                                                             \
    if (e_ != cudaSuccess) {                                                             \
      g_err = std::string(#expr) + ": " + cudaGetErrorString(e_);                        \
      return e_ == cudaErrorMemoryAllocation ? GLV_ERR_OOM : GLV_ERR_CUDA;              \
    }                                                                                    \
  } while (0)

#define TRY(expr)                 \
  do {                            \
    int r_ = (expr);              \
    if (r_ != GLV_OK) return r_;  \
  } while (0)

#define LAUNCH(kernel, grid, block, smem, stream, ...)            \
  do {                                                            \
    kernel<<<(grid), (block), (smem), (stream)>>>(__VA_ARGS__);   \
    ++launches_;                                                  \
    CK(cudaGetLastError());                                       \
  } while (0)

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

static int bits_for(int64_t x) {  // bits to hold values 0..x
  int b = 1;
  while (b < 62 && (int64_t(1) << b) <= x) ++b;
  return b;
}

// A device level graph.
struct Level {
  int64_t nv = 0, nnz = 0;
  int64_t *ptr = nullptr;
  int32_t *tail = nullptr;
  double *w = nullptr;
  bool owned = false;
};

// One (class, sublevel) step: member positions of each degree bin.
struct Step {
  int64_t seg[NBINS + 1];
  int64_t hub_chunk[2] = {0, 0};  // k_hub_accum work items
  int64_t hub_segs[2] = {0, 0};   // k_hub_scan work items
};

struct ClassSched {
  int64_t begin = 0, end = 0;  // member positions of the whole class
  int color = 0;               // the key (colour) the class was built from
  bool relaxed = false;        // not an independent set (a core batch or merged classes)
  std::vector<Step> steps;
};

// CUDA-event pairs captured into the phase graph as event-record nodes.
// Level 1 brackets each class's sweep launches; level 2 brackets every launch
// (slots: degree bins, then apply, then modularity).
constexpr int kSlotApply = NBINS, kSlotModularity = NBINS + 1, kSlots = NBINS + 2;
static_assert(kSlots == GLV_KERNEL_SLOTS, "glv_run_stats.kernel_time must hold every slot");

struct Probes {
  int level = 0;
  std::vector<int> slot;
  std::vector<cudaEvent_t> b, e;
  double slot_s[kSlots] = {0};
  double sweep_s = 0;
  long sweep_pairs = 0;
  ~Probes() {
    for (auto x : b) cudaEventDestroy(x);
    for (auto x : e) cudaEventDestroy(x);
  }
  // Opens a pair for `sl` (-1: a whole class's sweep); returns its index or -1.
  int begin(int sl, int need_level, cudaStream_t s, int *idx) {
    *idx = -1;
    if (level < need_level) return GLV_OK;
    cudaEvent_t x, y;
    CK(cudaEventCreate(&x));
    CK(cudaEventCreate(&y));
    b.push_back(x);
    e.push_back(y);
    slot.push_back(sl);
    *idx = (int)b.size() - 1;
    // During capture only the External flag turns a record into a graph node.
    CK(cudaEventRecordWithFlags(x, s, cudaEventRecordExternal));
    return GLV_OK;
  }
  int end(int idx, cudaStream_t s) {
    if (idx >= 0) CK(cudaEventRecordWithFlags(e[idx], s, cudaEventRecordExternal));
    return GLV_OK;
  }
  // Adds one replay's elapsed times.
  void collect() {
    for (size_t k = 0; k < b.size(); ++k) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, b[k], e[k]) != cudaSuccess) {
        cudaGetLastError();  // keep a failed query from surfacing at the next launch
        continue;
      }
      const double t = ms * 1e-3;
      if (slot[k] < 0) { sweep_s += t; ++sweep_pairs; }
      else slot_s[slot[k]] += t;
    }
  }
};

// Per-graph control of a batch level (batch.cuh).  Graph g's vertices at the
// current level are [voff[g], voff[g+1]) (empty once its run has finished).
struct Batch {
  int G = 0;
  std::vector<int64_t> voff;   // level vertex offsets
  std::vector<int64_t> gnnz;   // CSR entries per graph at this level
  int32_t *gid = nullptr;      // device: graph of each level vertex
  double *gcst = nullptr;      // device: per-graph 1/(2m)
  double *gsum = nullptr;      // device: per-graph degree sums
  double *gacc = nullptr;      // device: per-graph {e_xx, a2_x}
  uint8_t *act = nullptr;      // device: graph still sweeping in this phase
  std::vector<uint8_t> h_act, in_phase, stale;
  std::vector<double> h_gcst, h_acc, lower, mod, done_s;
  std::vector<int> itr;
  double thresh = 0;
};

// Per-graph results of a batch run (caller-owned arrays of G entries).
struct BatchResult {
  double *final_modularity;
  int *phases;
  int *iterations;
  long *clusters;
  double *done_s;
  int rounds;
};

class Engine {
 public:
  explicit Engine(cudaStream_t s, int mode) : s_(s), mode_(mode) {}
  ~Engine() { release(); }

  int init(int64_t nv0, int64_t nnz0);
  int upload_check(const Level &L);
  int color(const Level &L, int *ncolors, double *secs, bool sweep = false);
  int coloring_phase(const Level &L, int ncolors, bool stale, double lower, double thresh,
                     double *mod, int *itr);
  int basic_phase(const Level &L, double lower, double thresh, double *mod, int *itr);
  int renumber(int32_t *C, int64_t n, int64_t *ncl);
  int coarsen(const Level &in, const int32_t *C, int64_t ncl, Level *out, int64_t *num_edges);
  int coarsen_hash(const Level &in, const int32_t *Cm, int64_t ncl, Level *out,
                   int64_t *num_edges, bool dense);
  int coarsen_chunked(const Level &in, const int32_t *C, int64_t ncl, Level *out,
                      int64_t *num_edges, int64_t budget, bool vf = false);
  int modularity_of(const Level &L, const int32_t *C, double *q);
  int decide(const Level &L, const int32_t *verts, int64_t nverts);
  int run_multiphase(const Level &L0, int32_t *d_C_orig, bool coloring, long min_graph_size,
                     double threshold, double c_threshold, glv_run_stats *st);
  int run_multiphase_batch(const Level &L0, const std::vector<int64_t> &voff0,
                           int32_t *d_C_orig, bool coloring, long min_graph_size,
                           double threshold, double c_threshold, BatchResult *res);
  int batch_level(Batch &b, const Level &L, const std::vector<int64_t> &voff);
  int sublevels_batch(const Level &L, const Batch &b, int32_t **d_sub, int *nsub);
  void free_level(Level &L);
  Batch *bt_ = nullptr;  // set while a batch runs
  // colouring of colour phases: 1 = distance-1 (the default), 2 = distance-1
  // then balanced (vBaseRedistribution, first fit), 3 = the incomplete
  // multi-hash max/min colouring with mhash_nhash_ hashes and mhash_itrs_
  // iterations
  int color_algo_ = 1;
  int mhash_nhash_ = 2, mhash_itrs_ = 4;
  int color_mhash(const Level &L, int *ncolors);
  // Balanced recolouring of a proper colouring (coloring = 2); *moves may be NULL
  int vbase(const Level &L, int ncolors, int type, long *moves);

  // state buffers (device)
  double *vDeg = nullptr, *cDeg = nullptr, *dDeg = nullptr, *own_w = nullptr;
  int32_t *cSize = nullptr, *dSize = nullptr;
  int32_t *C = nullptr, *Cpast = nullptr, *Ctgt = nullptr;
  int32_t *color_ = nullptr;
  const bool debug_ = getenv("GRAPPOLO_B200_DEBUG") != nullptr;
  int dev_ = current_device();
  double *cst = nullptr;  // {constant, 2m}
  long launches_ = 0;
  bool integral = false;
  double t_sweep = 0, t_color = 0, t_coarsen = 0;
  double edges_swept = 0;
  double sweep_kernel_s = 0, sweep_bytes = 0;
  long sweep_steps = 0;
  long gated_iterations_ = 0;
  double slot_s[kSlots] = {0};
  // learned gate state
  double *rec_own_ = nullptr;
  float *rec_gain_ = nullptr, *feat_ = nullptr, *gate_p_ = nullptr;
  int32_t *last_move_ = nullptr;
  uint8_t *skip_ = nullptr;
  unsigned long long *evald_ = nullptr;
  int phase_index_ = 0;
  bool learned() const { return mode_ == GLV_MODE_LEARNED; }
  int gate_init(int64_t nv, bool tracing);
  void gate_release();
  int64_t avail_bytes();

 public:  // the allocator (the C ABI helpers allocate level-0 arrays through it)
  // Requests above 1 MiB are rounded up to quarter-octave size classes so that
  // repeated runs, whose level sizes differ slightly, reuse the pool's blocks.
  static size_t size_class(size_t bytes) {
    if (bytes <= (1u << 20)) return bytes;
    int e = 63 - __builtin_clzll(bytes);
    const size_t step = (size_t(1) << e) >> 2;
    return (bytes + step - 1) / step * step;
  }
  template <class T>
  int alloc(T **p, size_t n) {
    if (!pool_) pool_ = engine_pool();
    if (!pool_) return fail(GLV_ERR_CUDA, "could not create the device memory pool");
    if (n * sizeof(T) >= (size_t(1) << 30) && getenv("GRAPPOLO_B200_DEBUG")) {
      uint64_t used = 0;
      cudaMemPoolGetAttribute(pool_, cudaMemPoolAttrUsedMemCurrent, &used);
      fprintf(stderr, "grappolo_b200: alloc %.2f GB (pool used %.2f GB)\n",
              n * sizeof(T) * 1e-9, used * 1e-9);
    }
    const size_t bytes = size_class(std::max<size_t>(n, 1) * sizeof(T));
    BlockCache &bc = g_cache[dev_];
    {
      // the smallest cached block of at least this class and at most twice it
      // (repeated calls whose sizes drift a little, like a batch's waves,
      // reuse each other's blocks)
      std::lock_guard<std::mutex> lock(bc.mu);
      for (auto it = bc.free.lower_bound(bytes); it != bc.free.end() && it->first <= 2 * bytes;
           ++it) {
        if (it->second.empty()) continue;
        *p = static_cast<T *>(it->second.back());
        it->second.pop_back();
        bc.live[(void *)*p] = it->first;
        bc.last_use[(void *)*p] = bc.gen;
        return GLV_OK;
      }
    }
    const double ta = debug_ ? now_s() : 0.0;
    cudaError_t e = cudaMallocFromPoolAsync((void **)p, bytes, pool_, s_);
    if (e == cudaErrorMemoryAllocation) {
      // hand the cached blocks to the pool and retry; then also return the
      // pool's unused memory to the device and retry once more
      cudaGetLastError();
      flush_block_cache(dev_, s_);
      cudaStreamSynchronize(s_);
      e = cudaMallocFromPoolAsync((void **)p, bytes, pool_, s_);
      if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        cudaMemPoolTrimTo(pool_, 0);
        if (debug_) fprintf(stderr, "grappolo_b200: pool trimmed after a failed allocation\n");
        e = cudaMallocFromPoolAsync((void **)p, bytes, pool_, s_);
      } else if (debug_) {
        fprintf(stderr, "grappolo_b200: block cache returned after a failed allocation\n");
      }
    }
    if (debug_ && now_s() - ta > 2e-3)
      fprintf(stderr, "grappolo_b200: slow allocation of %.3f GB: %.4f s\n", bytes * 1e-9,
              now_s() - ta);
    CK(e);
    std::lock_guard<std::mutex> lock(bc.mu);
    bc.live[(void *)*p] = bytes;
    bc.last_use[(void *)*p] = bc.gen;
    return GLV_OK;
  }
  template <class T>
  void dfree(T *&p) {
    if (!p) return;
    BlockCache &bc = g_cache[dev_];
    {
      std::lock_guard<std::mutex> lock(bc.mu);
      auto it = bc.live.find((void *)p);
      if (it != bc.live.end()) {
        bc.free[it->second].push_back((void *)p);
        bc.live.erase(it);
        p = nullptr;
        return;
      }
    }
    cudaFreeAsync(p, s_);
    p = nullptr;
  }
  int temp(size_t bytes) {
    if (bytes <= temp_bytes_) return GLV_OK;
    dfree(temp_);
    temp_bytes_ = bytes + (bytes >> 3) + 1024;
    return alloc(reinterpret_cast<unsigned char **>(&temp_), temp_bytes_);
  }
  void release();
  int phase_init(const Level &L, bool need_past);
  int merge_splits(const Level &L);
  int build_schedule(const Level &L, const int32_t *color, int ncolors, const int32_t *sub,
                     int nsub, std::vector<ClassSched> *sched, bool hubs = true);
  int hub_offsets(const Level &L, std::vector<ClassSched> &sched);
  int group_classes(const Level &L, int ncolors, std::vector<ClassSched> *sched);
  int sublevels(const Level &L, int ncolors, int32_t **d_sub, int *nsub);
  int launch_sweep(const Level &L, const Step &st, SweepArgs a, bool ordered, Probes *pr);
  int launch_apply(const ClassSched &cs, bool ordered);
  int launch_modularity(const Level &L, const int32_t *Cm, const double *ownw);
  int color_jp(const Level &L, int *ncolors, const int32_t *key = nullptr);
  int run_persistent(const Level &L, const std::vector<ClassSched> &sched, SweepArgs a,
                     bool jacobi, double lower, double thresh, double *mod, int *itr);
  bool persistent() const {
    const char *e = getenv("GRAPPOLO_B200_PERSISTENT");
    return !ordered() && !(e && e[0] == '0');
  }
  int color_spec(const Level &L, int *ncolors, int64_t core_deg = INT64_MAX, int core_batches = 0);
  int recolor(const Level &L, int *ncolors, int passes);
  int grow_hub(size_t entries);
  bool ordered() const { return mode_ == GLV_MODE_VERIFY && !integral; }
  void account(Probes &pr, const Level &L) {
    if (pr.b.empty()) return;
    const double s0 = pr.sweep_s;
    const long p0 = pr.sweep_pairs;
    double before[kSlots];
    for (int k = 0; k < kSlots; ++k) before[k] = pr.slot_s[k];
    pr.collect();
    sweep_kernel_s += pr.sweep_s - s0;
    sweep_steps += pr.sweep_pairs - p0;
    for (int k = 0; k < kSlots; ++k) slot_s[k] += pr.slot_s[k] - before[k];
    sweep_bytes += 16.0 * (double)L.nnz + 36.0 * (double)L.nv;
  }

  cudaStream_t s_;
  cudaMemPool_t pool_ = nullptr;
  int mode_;
  int nsm_ = 148;
  int64_t nv0_ = 0, nnz0_ = 0;
  BinLimits lim_{127, 4095};
  // schedule buffers
  int32_t *keys_ = nullptr, *keys2_ = nullptr, *members_ = nullptr, *vals_ = nullptr;
  int32_t *move_old_ = nullptr, *move_new_ = nullptr, *hist_ = nullptr;
  int64_t *hub_off_ = nullptr;
  int32_t *hub_keys_ = nullptr;
  double *hub_vals_ = nullptr;
  size_t hub_cap_ = 0;
  // parallel hub path (per member slot arrays, work lists, filled-slot lists)
  int64_t *hub_occ_off_ = nullptr, *hub_seg_beg_ = nullptr, *hub_seg_end_ = nullptr;
  int32_t *hub_cnt_ = nullptr, *hub_left_ = nullptr, *hub_big_ = nullptr, *step_big_ = nullptr;
  int32_t *hub_segs_left_ = nullptr, *hub_err_ = nullptr;
  uint32_t *hub_state_ = nullptr;
  uint32_t epoch_ = 0;  // persistent launches of this engine (hub states compare against it)
  int hub_chunk_ = kHubChunk;  // CSR entries per hub chunk (the autotuner may lower it)
  // trial launches of the autotuner: stop after this many iterations (0 = the
  // phase's own test) and keep the last launch's device time
  int max_iters_ = 0;
  double last_launch_s_ = 0.0;
  bool tune_cached_ = false;
  int tune_choice_[2] = {0, 0};  // block_max, hub chunk chosen for this run (0 = not tuned)
  int first_cluster_ = -1;       // cluster size of the run's first colour phase (-1 = none yet)
  int autotune(const Level &L, int ncolors, std::vector<ClassSched> *sched,
               const std::function<int(std::vector<ClassSched> *)> &make_sched, SweepArgs a,
               double lower, double thresh);
  double *hub_self_ = nullptr, *hub_ownw_ = nullptr;
  int32_t *hub_occ_ = nullptr;
  size_t hub_occ_cap_ = 0;
  int32_t *chunk_pos_ = nullptr, *seg_pos_ = nullptr, *part_c_ = nullptr;
  int64_t *chunk_beg_ = nullptr, *chunk_end_ = nullptr, *seg_beg_ = nullptr, *seg_end_ = nullptr;
  double *part_g_ = nullptr;
  size_t chunk_cap_ = 0, seg_cap_ = 0;
  // Hub rows of the persistent kernel on thread-block clusters of cluster_
  // blocks (0: all hubs as chunks over global tables).  A hub whose table
  // needs at most cluster_parts_ cluster-sized partitions is a cluster row
  // when the schedule is built for the persistent sweep (sweep_rows_);
  // hub_pos_h_/hub_deg_h_ are the cluster rows' member slots (ascending) and
  // row lengths.
  int cluster_ = 0;
  int cluster_parts_ = kClusterMaxParts;
  bool sweep_rows_ = false;
  int32_t *ct_pos_ = nullptr, *ct_part_ = nullptr, *ct_nparts_ = nullptr, *ct_c_ = nullptr;
  double *ct_g_ = nullptr;
  size_t ct_cap_ = 0;
  std::vector<int32_t> hub_pos_h_;
  std::vector<int64_t> hub_deg_h_;
  int cluster_grid(int cl);  // blocks of a cooperative launch with cl-block clusters
  int cluster_grid_[kClusterMax + 1] = {};
  bool hub_tables_clean_ = false;
  // The current colour phase runs some colour classes together in one step
  // (group_classes), so a step's members are not an independent set.
  bool relaxed_ = false;
  // Classes at and above this colour of colour_ are batches of the core (not
  // independent sets); INT32_MAX = every class is an independent set.
  int core_color_ = INT32_MAX;
  HubWork hub_work() const {
    return HubWork{hub_keys_, hub_vals_, hub_off_, hub_occ_, hub_occ_off_, hub_cnt_, hub_self_,
                   hub_ownw_, chunk_pos_, chunk_beg_, chunk_end_, seg_pos_, seg_beg_, seg_end_,
                   part_g_, part_c_, hub_seg_beg_, hub_seg_end_, hub_left_, hub_big_, step_big_,
                   hub_segs_left_, hub_state_, 0u, hub_err_, hub_chunk_, ct_pos_, ct_part_,
                   ct_nparts_, ct_g_, ct_c_};
  }
  int hist_cap_ = 0;
  // ordered-delta buffers
  uint64_t *dkeys_ = nullptr, *dkeys2_ = nullptr;
  DeltaRec *drecs_ = nullptr, *drecs2_ = nullptr;
  // modularity
  double *part_e_ = nullptr, *part_a_ = nullptr, *mod_out_ = nullptr;
  int64_t *split_row_ = nullptr;  // merge-path tiles of the current level
  int64_t split_cap_ = 0;
  double *h_mod_ = nullptr;  // pinned
  // misc
  unsigned char *temp_ = nullptr;
  size_t temp_bytes_ = 0;
  int64_t max_class_ = 0;
  // coarsening records, sized for level 0 and reused by every level
  uint64_t *ck1_ = nullptr, *ck2_ = nullptr;
  double *cv1_ = nullptr, *cv2_ = nullptr;
  int64_t crec_cap_ = 0;
};

constexpr int kConstParts = 1024;  // blocks of the constant's reduction

static int grid_for(int64_t n, int block, int cap) {
  int64_t g = (n + block - 1) / block;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, cap));
}

void Engine::release() {
  double **dp[] = {&vDeg, &cDeg, &dDeg, &own_w, &cst, &hub_vals_, &part_e_, &part_a_, &mod_out_};
  for (auto p : dp) dfree(*p);
  int32_t **ip[] = {&cSize, &dSize, &C, &Cpast, &Ctgt, &color_, &keys_, &keys2_, &members_,
                    &vals_, &move_old_, &move_new_, &hist_, &hub_keys_};
  for (auto p : ip) dfree(*p);
  dfree(hub_off_);
  dfree(hub_occ_off_); dfree(hub_seg_beg_); dfree(hub_seg_end_); dfree(hub_cnt_);
  dfree(hub_self_); dfree(hub_ownw_); dfree(hub_occ_); dfree(hub_left_); dfree(hub_big_);
  dfree(hub_segs_left_); dfree(hub_state_); dfree(hub_err_);
  dfree(step_big_); dfree(chunk_pos_); dfree(seg_pos_);
  dfree(ct_pos_); dfree(ct_part_); dfree(ct_nparts_); dfree(ct_g_); dfree(ct_c_);
  dfree(part_c_); dfree(chunk_beg_); dfree(chunk_end_); dfree(seg_beg_); dfree(seg_end_);
  dfree(part_g_);
  dfree(dkeys_); dfree(dkeys2_); dfree(drecs_); dfree(drecs2_);
  dfree(ck1_); dfree(ck2_); dfree(cv1_); dfree(cv2_);
  dfree(rec_own_); dfree(rec_gain_); dfree(feat_); dfree(gate_p_); dfree(last_move_);
  dfree(skip_); dfree(evald_);
  dfree(split_row_);
  split_cap_ = 0;
  dfree(temp_);
  if (h_mod_) cudaFreeHost(h_mod_);
  h_mod_ = nullptr;
  cudaStreamSynchronize(s_);
}

int Engine::init(int64_t nv0, int64_t nnz0) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm_, cudaDevAttrMultiProcessorCount, dev));
  nv0_ = nv0;
  nnz0_ = nnz0;
  const size_t n = (size_t)nv0 + 1;
  TRY(alloc(&vDeg, n)); TRY(alloc(&cDeg, n)); TRY(alloc(&dDeg, n)); TRY(alloc(&own_w, n));
  TRY(alloc(&cSize, n)); TRY(alloc(&dSize, n));
  TRY(alloc(&C, n)); TRY(alloc(&Cpast, n)); TRY(alloc(&Ctgt, n)); TRY(alloc(&color_, n));
  TRY(alloc(&keys_, n)); TRY(alloc(&keys2_, n)); TRY(alloc(&members_, n)); TRY(alloc(&vals_, n));
  TRY(alloc(&move_old_, n)); TRY(alloc(&move_new_, n)); TRY(alloc(&hub_off_, n));
  TRY(alloc(&hub_occ_off_, n)); TRY(alloc(&hub_seg_beg_, n)); TRY(alloc(&hub_seg_end_, n));
  TRY(alloc(&hub_cnt_, n)); TRY(alloc(&hub_self_, n)); TRY(alloc(&hub_ownw_, n));
  TRY(alloc(&hub_left_, n)); TRY(alloc(&hub_big_, n));
  TRY(alloc(&hub_segs_left_, n)); TRY(alloc(&hub_state_, n)); TRY(alloc(&hub_err_, 1));
  CK(cudaMemsetAsync(hub_state_, 0, n * sizeof(uint32_t), s_));
  CK(cudaMemsetAsync(hub_err_, 0, sizeof(int32_t), s_));
  CK(cudaMemsetAsync(hub_cnt_, 0, n * sizeof(int32_t), s_));
  CK(cudaMemsetAsync(hub_big_, 0, n * sizeof(int32_t), s_));
  CK(cudaMemsetAsync(hub_self_, 0, n * sizeof(double), s_));
  CK(cudaMemsetAsync(hub_ownw_, 0, n * sizeof(double), s_));
  if (const char *bm = getenv("GRAPPOLO_B200_BLOCK_MAX")) {
    const int v = atoi(bm);
    if (v >= lim_.warp_max && v <= 4095) lim_.block_max = v;
  }
  // hub rows on clusters of this many blocks (1, 2, 4, 8 or 16; 0 = global
  // tables, the default); the autotuner may change it
  cluster_ = 0;
  if (const char *cl = getenv("GRAPPOLO_B200_CLUSTER")) {
    const int v = atoi(cl);
    if (v == 0 || (v <= kClusterMax && (v & (v - 1)) == 0)) cluster_ = v;
  }
  if (cluster_ > 0 && cluster_grid(cluster_) < cluster_) cluster_ = 0;
  if (getenv("GRAPPOLO_B200_DEBUG"))
    fprintf(stderr, "grappolo_b200: hub clusters of %d blocks (grid %d)\n", cluster_,
            cluster_ > 0 ? cluster_grid(cluster_) : 0);
  if (const char *cp = getenv("GRAPPOLO_B200_CLUSTER_PARTS")) {
    const int v = atoi(cp);
    if (v >= 1 && (v & (v - 1)) == 0) cluster_parts_ = v;
  }
  TRY(alloc(&cst, 4));
  // partials of the modularity pass (one per 256 vertices) and of the
  // constant's reduction (kConstParts blocks) share these buffers
  const size_t nparts = std::max<size_t>((n + kModVB - 1) / kModVB, kConstParts) + 1;
  TRY(alloc(&part_e_, nparts)); TRY(alloc(&part_a_, nparts)); TRY(alloc(&mod_out_, 8));
  CK(cudaMallocHost((void **)&h_mod_, 8 * sizeof(double)));
  CK(cudaMemsetAsync(dDeg, 0, n * sizeof(double), s_));
  CK(cudaMemsetAsync(dSize, 0, n * sizeof(int32_t), s_));
  return GLV_OK;
}


// Integral-weight detection: every weight a non-negative integer and the total
// below 2^53 -> every sum in any order is exact.
__global__ void k_check_weights(int64_t nnz, const double *w, const int32_t *tail, int64_t nv,
                                int32_t *flags, double *total) {
  double s = 0.0;
  bool frac = false, bad = false;  // flags kept per thread: one update per warp at the end
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nnz;
       j += (int64_t)gridDim.x * blockDim.x) {
    const double x = w[j];
    frac = frac || !(x >= 0.0 && x == floor(x));
    const int32_t t = tail[j];
    bad = bad || t < 0 || t >= nv;
    s += x;
  }
  frac = __any_sync(FULL, frac);
  bad = __any_sync(FULL, bad);
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(FULL, s, off);
  if ((threadIdx.x & 31) == 0) {
    if (frac) atomicOr(&flags[0], 1);
    if (bad) atomicOr(&flags[1], 1);
    atomicAdd(total, s);
  }
}

int Engine::upload_check(const Level &L) {
  int32_t *flags;
  double *total;
  TRY(alloc(&flags, 2));
  TRY(alloc(&total, 1));
  CK(cudaMemsetAsync(flags, 0, 2 * sizeof(int32_t), s_));
  CK(cudaMemsetAsync(total, 0, sizeof(double), s_));
  LAUNCH(k_check_weights, grid_for(L.nnz, 256, nsm_ * 8), 256, 0, s_, L.nnz, L.w, L.tail, L.nv,
         flags, total);
  int32_t hf[2];
  double ht;
  CK(cudaMemcpyAsync(hf, flags, sizeof(hf), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(&ht, total, sizeof(double), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  dfree(flags);
  dfree(total);
  if (hf[1]) return fail(GLV_ERR_ARG, "edge tail out of range [0, numVertices)");
  integral = (hf[0] == 0) && (ht < 9007199254740992.0);
  return GLV_OK;
}

// split_row_ <- the merge-path tile boundaries of L.
int Engine::merge_splits(const Level &L) {
  const int64_t nt = merge_tiles(L.nv, L.nnz);
  if (nt + 1 > split_cap_) {
    dfree(split_row_);
    split_cap_ = nt + 1;
    TRY(alloc(&split_row_, split_cap_));
  }
  LAUNCH(k_merge_splits, grid_for(nt + 1, 256, nsm_ * 16), 256, 0, s_, L.nv, L.nnz, L.ptr, nt,
         split_row_);
  return GLV_OK;
}

int Engine::phase_init(const Level &L, bool need_past) {
  TRY(merge_splits(L));
  if (ordered()) {
    LAUNCH(k_init_phase, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, L.ptr, L.w, vDeg, cDeg,
           cSize, C, need_past ? Cpast : (int32_t *)nullptr);
  } else {
    if (L.nnz >= 64 * L.nv) {  // long rows: a warp per row reads them coalesced
      LAUNCH(k_init_phase_warp, grid_for(L.nv * 32, 256, nsm_ * 16), 256, 0, s_, L.nv, L.ptr,
             L.w, vDeg, cDeg, cSize, C, need_past ? Cpast : (int32_t *)nullptr);
    } else {  // short rows: merge-path tiles (split_row_ from merge_splits above)
      CK(cudaMemsetAsync(vDeg, 0, L.nv * sizeof(double), s_));
      const int64_t nt = merge_tiles(L.nv, L.nnz);
      if (L.nnz > 0)
        LAUNCH(k_row_sums_tiles, (int)std::max<int64_t>(1, std::min<int64_t>(nt, nsm_ * 8)),
               kRowSumThreads, sizeof(RowSumSmem), s_, L.nv, L.nnz, L.ptr, L.w, split_row_, vDeg);
      LAUNCH(k_init_phase_fill, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, vDeg, cDeg,
             cSize, C, need_past ? Cpast : (int32_t *)nullptr);
    }
  }
  if (ordered()) {
    LAUNCH(k_constant_sequential, 1, 1, 0, s_, L.nv, vDeg, cst);
  } else {
    LAUNCH(k_sum_partials, kConstParts, 256, 0, s_, L.nv, vDeg, part_e_);
    LAUNCH(k_constant_from_partials, 1, 32, 0, s_, kConstParts, part_e_, cst);
  }
  if (bt_) {
    // one constant per graph
    CK(cudaMemsetAsync(bt_->gsum, 0, bt_->G * sizeof(double), s_));
    LAUNCH(k_graph_degsum, grid_for(L.nv, 256, nsm_ * 8), 256, 0, s_, L.nv, bt_->gid, vDeg,
           bt_->gsum);
    LAUNCH(k_graph_cst, grid_for(bt_->G, 256, nsm_ * 4), 256, 0, s_, bt_->G, bt_->gsum,
           bt_->gcst);
    CK(cudaMemcpyAsync(bt_->h_gcst.data(), bt_->gcst, bt_->G * sizeof(double),
                       cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
  }
  return GLV_OK;
}

// ----------------------------------------------------------------- colouring
// Fast-mode colour phases sweep the core (rows in degree bin
// GRAPPOLO_B200_CORE_BIN and above, default the 128..511 bin) apart from the
// colour classes: the colouring covers the rest of the graph, and the core
// vertices run in GRAPPOLO_B200_CORE_BATCHES classes (default 32) that each
// decide against one snapshot of their members' communities.  Skewed graphs
// need hundreds of colours for their dense core, each a grid-wide step with a
// few long rows; a core vertex has most of its weight outside its batch, so
// deciding a batch together changes little of what each decision sees.
static void core_settings(int *core_bin, int *batches) {
  *core_bin = BIN_T128;
  *batches = 32;
  if (const char *e = getenv("GRAPPOLO_B200_CORE_BIN")) *core_bin = atoi(e);
  if (const char *e = getenv("GRAPPOLO_B200_CORE_BATCHES")) *batches = atoi(e);
}

int Engine::color(const Level &L, int *ncolors, double *secs, bool sweep) {
  const double t0 = now_s();
  core_color_ = INT32_MAX;
  if (L.nv == 0 && color_algo_ != 3) {
    *ncolors = 0;
    return GLV_OK;
  }
  // GRAPPOLO_B200_COLORING overrides the mode's colouring: spec (speculative
  // largest-degree-first), jp (Jones-Plassmann, hashed priorities in fast
  // mode), id (Jones-Plassmann in vertex-id order, verify mode's colouring)
  const char *cm = getenv("GRAPPOLO_B200_COLORING");
  bool spec = mode_ != GLV_MODE_VERIFY;
  if (cm && (!strcmp(cm, "jp") || !strcmp(cm, "id"))) spec = false;
  if (cm && !strcmp(cm, "spec")) spec = true;
  const bool dbg = getenv("GRAPPOLO_B200_DEBUG") != nullptr;
  double td = now_s();
  if (color_algo_ == 3) {
    TRY(color_mhash(L, ncolors));
    if (secs) *secs = now_s() - t0;
    return GLV_OK;
  }
  int core_bin = NBINS, nbatch = 0;
  if (sweep && spec && color_algo_ == 1 && mode_ != GLV_MODE_VERIFY && !bt_)
    core_settings(&core_bin, &nbatch);
  const int64_t core_deg = (core_bin > BIN_G4 && core_bin < NBINS && nbatch > 0)
                               ? first_degree_of_bin(core_bin, lim_)
                               : INT64_MAX;
  TRY(spec ? color_spec(L, ncolors, core_deg, nbatch) : color_jp(L, ncolors));
  if (dbg) {
    cudaStreamSynchronize(s_);
    fprintf(stderr, "grappolo_b200: colouring %.4f s (%d colours)\n", now_s() - td, *ncolors);
    td = now_s();
  }
  // Outside verify mode, iterated greedy (Culberson): recolour whole classes,
  // last class first; such a pass never needs more colours, and on power-law
  // graphs it removes many.  Every class is a step of every sweep, so fewer
  // classes mean fewer barriers and shorter latency chains.  Passes stop when
  // one removes no colour (GRAPPOLO_B200_RECOLOR sets the maximum, 0 = off).
  // Only colourings with many classes are worth a pass, which costs about one
  // colouring (GRAPPOLO_B200_RECOLOR_MIN: the class count that triggers it).
  if (mode_ != GLV_MODE_VERIFY && core_color_ == INT32_MAX) {
    const char *rp = getenv("GRAPPOLO_B200_RECOLOR");
    const char *rm = getenv("GRAPPOLO_B200_RECOLOR_MIN");
    if (*ncolors > (rm ? atoi(rm) : 64)) TRY(recolor(L, ncolors, rp ? atoi(rp) : 2));
    if (dbg) {
      cudaStreamSynchronize(s_);
      fprintf(stderr, "grappolo_b200: recolour %.4f s (%d colours)\n", now_s() - td, *ncolors);
    }
  }
  // coloring = 2: runMultiPhaseColoring.cpp:67-74, 180-186
  if (color_algo_ == 2) TRY(vbase(L, *ncolors, 0, nullptr));
  if (secs) *secs = now_s() - t0;
  return GLV_OK;
}

int Engine::vbase(const Level &L, int ncolors, int type, long *moves) {
  if (L.nv == 0 || ncolors <= 0) {
    if (moves) *moves = 0;
    return GLV_OK;
  }
  if (ncolors > kMaxColors) return fail(GLV_ERR_COLORS, "more colours than the 4096 cap");
  const int64_t nv = L.nv;
  const int64_t avg = (int64_t)ceil((double)nv / (double)ncolors);  // vBase.cpp:80
  int32_t *freq, *flag, *cand;
  int64_t *ncand;
  unsigned long long *dmoves;
  TRY(alloc(&freq, ncolors));
  TRY(alloc(&flag, nv));
  TRY(alloc(&cand, nv));
  TRY(alloc(&ncand, 1));
  TRY(alloc(&dmoves, 1));
  CK(cudaMemsetAsync(freq, 0, ncolors * sizeof(int32_t), s_));
  LAUNCH(k_color_hist, grid_for(nv, 256, nsm_ * 16), 256, 0, s_, nv, color_, freq);
  LAUNCH(k_vbase_flags, grid_for(nv, 256, nsm_ * 16), 256, 0, s_, nv, color_, freq, avg, flag);
  size_t tb = 0;
  CK(cub::DeviceSelect::Flagged(nullptr, tb, thrust::counting_iterator<int32_t>(0), flag, cand,
                                ncand, nv, s_));
  char *temp;
  TRY(alloc(&temp, (int64_t)tb));
  CK(cub::DeviceSelect::Flagged(temp, tb, thrust::counting_iterator<int32_t>(0), flag, cand,
                                ncand, nv, s_));
  LAUNCH(k_vbase, 1, kVbaseThreads, 0, s_, L.ptr, L.tail, color_, cand, ncand, freq, ncolors,
         avg, type, dmoves);
  unsigned long long hm = 0;
  CK(cudaMemcpyAsync(&hm, dmoves, sizeof(hm), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  dfree(temp);
  dfree(freq);
  dfree(flag);
  dfree(cand);
  dfree(ncand);
  dfree(dmoves);
  if (moves) *moves = (long)hm;
  return GLV_OK;
}

// Verify mode: Jones-Plassmann in vertex-id priority = the reference's
// one-thread sequential first-fit.
int Engine::color_jp(const Level &L, int *ncolors, const int32_t *key) {
  int32_t *pending, *f0, *f1, *fcount, *status, *maxc;
  TRY(alloc(&pending, L.nv)); TRY(alloc(&f0, L.nv)); TRY(alloc(&f1, L.nv));
  TRY(alloc(&fcount, 3)); TRY(alloc(&status, 2)); TRY(alloc(&maxc, 1));
  CK(cudaMemsetAsync(fcount, 0, 3 * sizeof(int32_t), s_));
  CK(cudaMemsetAsync(status, 0, 2 * sizeof(int32_t), s_));
  CK(cudaMemsetAsync(maxc, 0xff, sizeof(int32_t), s_));
  // fast mode hashes the priorities (independent sets of random order);
  // GRAPPOLO_B200_COLORING=id keeps the vertex-id order of verify mode
  const char *cm = getenv("GRAPPOLO_B200_COLORING");
  const int hashed = (mode_ != GLV_MODE_VERIFY && !(cm && !strcmp(cm, "id"))) ? 1 : 0;
  const uint32_t seed = 0x5bd1e995u;
  LAUNCH(k_color_init, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, L.ptr, L.tail, hashed,
         seed, pending, color_, f0, fcount, key);
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_color_rounds, 256, 0));
  int grid = std::max(1, per_sm) * nsm_;
  int64_t nv = L.nv;
  const int64_t *ptr = L.ptr;
  const int32_t *tail = L.tail;
  int32_t *color = color_;
  void *args[] = {&nv, (void *)&ptr, (void *)&tail, (void *)&hashed, (void *)&seed, &pending,
                  &color, &f0, &f1, &fcount, &status, (void *)&key};
  CK(cudaLaunchCooperativeKernel((void *)k_color_rounds, grid, 256, args, 0, s_));
  ++launches_;
  LAUNCH(k_max_color, grid_for(L.nv, 256, nsm_ * 8), 256, 0, s_, L.nv, color_, maxc);
  int32_t h[2], hm;
  CK(cudaMemcpyAsync(h, status, sizeof(h), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(&hm, maxc, sizeof(hm), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  dfree(pending); dfree(f0); dfree(f1); dfree(fcount); dfree(status); dfree(maxc);
  if (h[0]) return fail(GLV_ERR_COLORS, "colouring needs more than 4096 colours");
  *ncolors = hm + 1;
  return GLV_OK;
}

// Fast mode: speculative first-fit rounds with hashed-priority conflicts.
constexpr int64_t kSpecBlockDeg = 2048;

int Engine::color_spec(const Level &L, int *ncolors, int64_t core_deg, int core_batches) {
  int32_t *wl, *bl, *nx, *cnt, *status, *maxc;
  unsigned long long *ncore;
  TRY(alloc(&wl, L.nv)); TRY(alloc(&bl, L.nv)); TRY(alloc(&nx, L.nv));
  TRY(alloc(&cnt, 4)); TRY(alloc(&status, 1)); TRY(alloc(&maxc, 1)); TRY(alloc(&ncore, 1));
  CK(cudaMemsetAsync(cnt, 0, 4 * sizeof(int32_t), s_));
  CK(cudaMemsetAsync(status, 0, sizeof(int32_t), s_));
  CK(cudaMemsetAsync(maxc, 0xff, sizeof(int32_t), s_));
  CK(cudaMemsetAsync(ncore, 0, sizeof(unsigned long long), s_));
  const uint32_t seed = 0x5bd1e995u;
  if (core_batches <= 0) core_deg = INT64_MAX;
  LAUNCH(k_spec_init, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, L.ptr, L.tail,
         kSpecBlockDeg, core_deg, color_, wl, cnt, bl, cnt + 1, ncore);
  // Rounds run in groups without a host read: the kernels take the list
  // lengths from device counters, and a round after the last conflict is a
  // set of empty launches.  The host reads the counters once per group.
  constexpr int kSpecGroup = 8;
  const int gw = nsm_ * 16, gb = nsm_ * 4;
  int rounds = 0;
  while (true) {
    for (int r = 0; r < kSpecGroup; ++r, ++rounds) {
      LAUNCH(k_spec_assign_warp, gw, 256, 0, s_, cnt, wl, L.ptr, L.tail, color_, status);
      LAUNCH(k_spec_assign_block, gb, 512, 0, s_, cnt + 1, bl, L.ptr, L.tail, color_, status);
      CK(cudaMemsetAsync(cnt + 2, 0, sizeof(int32_t), s_));
      LAUNCH(k_spec_conflicts, gw, 256, 0, s_, cnt, wl, L.ptr, L.tail, seed, color_, nx, cnt + 2);
      LAUNCH(k_spec_conflicts_block, gb, 512, 0, s_, cnt + 1, bl, L.ptr, L.tail, seed, color_,
             nx, cnt + 2);
      CK(cudaMemsetAsync(cnt, 0, 2 * sizeof(int32_t), s_));
      LAUNCH(k_spec_split, gw, 256, 0, s_, cnt + 2, nx, L.ptr, kSpecBlockDeg, wl, cnt, bl,
             cnt + 1);
    }
    int32_t h[2];
    const double tw = debug_ ? now_s() : 0.0;
    CK(cudaMemcpyAsync(h, cnt, 2 * sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    if (debug_)
      fprintf(stderr, "grappolo_b200: spec rounds %d: wait %.4f s, lists %d + %d\n", rounds,
              now_s() - tw, h[0], h[1]);
    if (h[0] + h[1] == 0) break;
    if (rounds > 100000) return fail(GLV_ERR_CUDA, "speculative colouring did not settle");
  }
  if (getenv("GRAPPOLO_B200_DEBUG"))
    fprintf(stderr, "grappolo_b200: speculative colouring nv=%ld rounds=%d\n", (long)L.nv, rounds);
  LAUNCH(k_max_color, grid_for(L.nv, 256, nsm_ * 8), 256, 0, s_, L.nv, color_, maxc);
  int32_t hs, hm;
  unsigned long long hcore = 0;
  CK(cudaMemcpyAsync(&hs, status, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(&hm, maxc, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(&hcore, ncore, sizeof(hcore), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  if (hs) {
    dfree(wl); dfree(bl); dfree(nx); dfree(cnt); dfree(status); dfree(maxc); dfree(ncore);
    return fail(GLV_ERR_COLORS, "colouring needs more than 4096 colours");
  }
  *ncolors = hm + 1;
  if (hcore > 0) {
    // (fewer batches for small cores cost modularity on planted power-law
    // graphs and saved no time: every core keeps core_batches steps)
    const int nb = (int)std::min<unsigned long long>(hcore, (unsigned long long)core_batches);
    if (*ncolors + nb > kMaxColors) {
      dfree(wl); dfree(bl); dfree(nx); dfree(cnt); dfree(status); dfree(maxc); dfree(ncore);
      return fail(GLV_ERR_COLORS, "colouring needs more than 4096 colours");
    }
    LAUNCH(k_core_batches, grid_for(L.nv, 256, nsm_ * 8), 256, 0, s_, L.nv, (int32_t)*ncolors,
           (int32_t)nb, color_);
    core_color_ = *ncolors;
    *ncolors += nb;
    if (debug_)
      fprintf(stderr, "grappolo_b200: %d colours + %d batches of %llu core vertices\n",
              core_color_, nb, hcore);
  }
  dfree(wl); dfree(bl); dfree(nx); dfree(cnt); dfree(status); dfree(maxc); dfree(ncore);
  return GLV_OK;
}

template <class T>
static int upload(cudaStream_t s, T *dst, const std::vector<T> &src);

// Coloring/coloringMultiHashMaxMin.cpp:59-228.  The random values are the
// reference's: rand() of the C library, hash by hash, vertex by vertex
// (:45-57, :95-101), so a process that seeds it the same way gets the same
// colouring.  Vertices left uncoloured keep colour maxColor (an improper
// class); *ncolors = maxColor + 1, as runMultiPhaseColoring counts them.
int Engine::color_mhash(const Level &L, int *ncolors) {
  const int nHash = mhash_nhash_, nItrs = mhash_itrs_;
  const int64_t nv = L.nv;
  if (nv == 0) {  // the first iteration colours nothing and all are coloured (:160-168)
    *ncolors = 2 * (0 - 1) * nHash + 2 * nHash + 1 + 1;
    return GLV_OK;
  }
  std::vector<double> h((size_t)nHash * nv);
  for (int k = 0; k < nHash; ++k)
    for (int64_t v = 0; v < nv; ++v) h[(size_t)k * nv + v] = (double)rand();
  double *rnd;
  unsigned long long *count;
  TRY(alloc(&rnd, h.size()));
  TRY(alloc(&count, 1));
  TRY(upload(s_, rnd, h));
  int maxColor = 2 * nHash * nItrs;
  LAUNCH(k_fill_i32, grid_for(nv, 256, nsm_ * 16), 256, 0, s_, nv, color_, maxColor);
  long totalColored = 0;
  unsigned long long iterFreq = 0;
  for (int itr = 0; itr < nItrs; ++itr) {
    CK(cudaMemsetAsync(count, 0, sizeof(*count), s_));
    for (int ih = 0; ih < nHash; ++ih) {
      const int cur = 2 * itr * nHash + 2 * ih;
      LAUNCH(k_mhash_pass, grid_for(nv * 32, 256, nsm_ * 16), 256, 0, s_, nv, L.ptr, L.tail,
             rnd + (size_t)ih * nv, color_, (int32_t)(2 * nHash * nItrs), (int32_t)cur, count);
    }
    unsigned long long c = 0;
    CK(cudaMemcpyAsync(&c, count, sizeof(c), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    iterFreq += c;
    totalColored += (long)iterFreq;
    if (iterFreq == 0) {
      if (totalColored == nv) {
        maxColor = 2 * (itr - 1) * nHash + 2 * nHash + 1;
        break;
      }
    } else {
      iterFreq = 0;
    }
  }
  dfree(rnd);
  dfree(count);
  *ncolors = maxColor + 1;
  return GLV_OK;
}

// Improper (reused) colourings: split each class into sublevels so that a
// vertex comes after its same-colour lower-id neighbours — the order in which
// the reference's one-thread loop sees their in-place updates.
int Engine::sublevels(const Level &L, int ncolors, int32_t **d_sub, int *nsub) {
  std::vector<int64_t> ptr(L.nv + 1);
  std::vector<int32_t> tail(L.nnz), col(L.nv);
  CK(cudaMemcpyAsync(ptr.data(), L.ptr, (L.nv + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(tail.data(), L.tail, L.nnz * sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(col.data(), color_, L.nv * sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  std::vector<int32_t> sub(L.nv, 0);
  int mx = 0;
  for (int64_t v = 0; v < L.nv; ++v) {
    int d = 0;
    for (int64_t j = ptr[v]; j < ptr[v + 1]; ++j) {
      const int32_t u = tail[j];
      if (u < v && col[u] == col[v]) d = std::max(d, sub[u] + 1);
    }
    sub[v] = d;
    mx = std::max(mx, d);
  }
  *nsub = mx + 1;
  *d_sub = nullptr;
  if (mx == 0) return GLV_OK;
  TRY(alloc(d_sub, L.nv));
  CK(cudaMemcpyAsync(*d_sub, sub.data(), L.nv * sizeof(int32_t), cudaMemcpyHostToDevice, s_));
  CK(cudaStreamSynchronize(s_));
  return GLV_OK;
}

// ------------------------------------------------------------------ schedule
// `hubs`: also lay out the block-path hub tables and work lists (every path but
// the persistent sweep, which plans its long rows itself).
int Engine::build_schedule(const Level &L, const int32_t *color, int ncolors, const int32_t *sub,
                           int nsub, std::vector<ClassSched> *sched, bool hubs) {
  const bool debug = getenv("GRAPPOLO_B200_DEBUG") != nullptr;
  const double tsd = now_s();
  const int64_t nkeys = (int64_t)ncolors * nsub * NBINS;
  if (nkeys + 1 > hist_cap_) {
    dfree(hist_);
    hist_cap_ = (int)(nkeys + 1);
    TRY(alloc(&hist_, hist_cap_));
  }
  CK(cudaMemsetAsync(hist_, 0, (nkeys + 1) * sizeof(int32_t), s_));
  LAUNCH(k_schedule_keys, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, L.ptr, color, sub,
         nsub, lim_, keys_, vals_, hist_);
  const int end_bit = bits_for(nkeys);
  size_t tb = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys_, keys2_, vals_, members_, L.nv, 0,
                                     end_bit, s_));
  TRY(temp(tb));
  CK(cub::DeviceRadixSort::SortPairs(temp_, tb, keys_, keys2_, vals_, members_, L.nv, 0, end_bit,
                                     s_));
  std::vector<int32_t> hist(nkeys);
  CK(cudaMemcpyAsync(hist.data(), hist_, nkeys * sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  sched->clear();
  int64_t pos = 0;
  max_class_ = 0;
  for (int c = 0; c < ncolors; ++c) {
    ClassSched cs;
    cs.begin = pos;
    cs.color = c;
    for (int sl = 0; sl < nsub; ++sl) {
      Step st;
      int64_t cnt = 0;
      for (int b = 0; b < NBINS; ++b) {
        st.seg[b] = pos;
        pos += hist[((int64_t)c * nsub + sl) * NBINS + b];
        cnt += hist[((int64_t)c * nsub + sl) * NBINS + b];
      }
      st.seg[NBINS] = pos;
      if (cnt) cs.steps.push_back(st);
    }
    cs.end = pos;
    if (cs.end > cs.begin) {
      max_class_ = std::max(max_class_, cs.end - cs.begin);
      sched->push_back(cs);
    }
  }
  if (debug) fprintf(stderr, "grappolo_b200: schedule sort+hist %.4f s\n", now_s() - tsd);
  return hubs ? hub_offsets(L, *sched) : GLV_OK;
}

// Fast mode: colour classes whose members all have long rows (degree bin at
// least GRAPPOLO_B200_MERGE_BIN, default the hub bin) run in steps of up to
// GRAPPOLO_B200_MERGE_CLASSES classes (default 16; 0 or 1 = every class its
// own step).  Skewed graphs colour their dense core of high-degree vertices
// with hundreds of classes of a few vertices each, and every class is a
// grid-wide step; a vertex of such a class has almost all of its weight on
// vertices outside the core, so deciding a few core classes against one
// snapshot changes little of what each decision sees.  A group takes the
// place of its first class; the other classes keep their order.  Returns the
// schedule rebuilt over the groups (relaxed_ set) or leaves it unchanged.
int Engine::group_classes(const Level &L, int ncolors, std::vector<ClassSched> *sched) {
  relaxed_ = false;
  if (mode_ == GLV_MODE_VERIFY || bt_ || sched->size() < 2) return GLV_OK;
  int gmax = 16, min_bin = BIN_HUB;
  if (const char *e = getenv("GRAPPOLO_B200_MERGE_CLASSES")) gmax = atoi(e);
  if (const char *e = getenv("GRAPPOLO_B200_MERGE_BIN")) min_bin = atoi(e);
  if (gmax <= 1 || min_bin < 0 || min_bin >= NBINS) return GLV_OK;
  std::vector<int32_t> map(ncolors, 0);
  int ngroups = 0, open = -1, in_open = 0, merged = 0;
  for (const ClassSched &cs : *sched) {
    bool long_rows = cs.steps.size() == 1;
    for (const Step &st : cs.steps) long_rows = long_rows && st.seg[min_bin] == st.seg[0];
    if (!long_rows) {
      map[cs.color] = ngroups++;
      continue;
    }
    if (open < 0 || in_open >= gmax) {
      open = ngroups++;
      in_open = 0;
    } else {
      ++merged;
    }
    map[cs.color] = open;
    ++in_open;
  }
  if (merged == 0) return GLV_OK;
  // colours with no member keep a slot that no vertex uses
  int32_t *d_map, *key;
  TRY(alloc(&d_map, ncolors));
  TRY(alloc(&key, L.nv));
  TRY(upload(s_, d_map, map));
  LAUNCH(k_remap_colors, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, color_, d_map, key);
  const int rc = build_schedule(L, key, ngroups, nullptr, 1, sched);
  CK(cudaStreamSynchronize(s_));
  dfree(d_map);
  dfree(key);
  TRY(rc);
  relaxed_ = true;
  {
    std::vector<int> members_per_group(ngroups, 0);
    for (int c = 0; c < ncolors; ++c) ++members_per_group[map[c]];
    for (ClassSched &cs : *sched) cs.relaxed = cs.color < ngroups && members_per_group[cs.color] > 1;
  }
  if (getenv("GRAPPOLO_B200_DEBUG"))
    fprintf(stderr, "grappolo_b200: %d colour classes run in %zu steps (%d merged)\n",
            ngroups + merged, sched->size(), merged);
  return GLV_OK;
}

int Engine::grow_hub(size_t entries) {
  if (entries <= hub_cap_) return GLV_OK;
  dfree(hub_keys_);
  dfree(hub_vals_);
  hub_cap_ = entries;
  TRY(alloc(&hub_keys_, hub_cap_));
  TRY(alloc(&hub_vals_, hub_cap_));
  return GLV_OK;
}

__global__ void k_scatter_i64(int64_t n, const int32_t *pos, const int64_t *val, int64_t *out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    out[pos[k]] = val[k];
}

__global__ void k_hub_chunk_counts(int64_t n, const int32_t *pos, const int32_t *members,
                                   const int64_t *ptr, const int64_t *seg_beg,
                                   const int64_t *seg_end, int chunk, int32_t *left,
                                   int32_t *segs_left) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = members[pos[k]];
    left[pos[k]] = (int32_t)((ptr[v + 1] - ptr[v] + chunk - 1) / chunk);
    segs_left[pos[k]] = (int32_t)(seg_end[pos[k]] - seg_beg[pos[k]]);
  }
}

__global__ void k_row_bounds_at(int64_t n, const int32_t *pos, const int32_t *members,
                                const int64_t *ptr, int64_t *out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = members[pos[k]];
    out[2 * k] = ptr[v];
    out[2 * k + 1] = ptr[v + 1];
  }
}

template <class T>
static int upload(cudaStream_t s, T *dst, const std::vector<T> &src) {
  if (src.empty()) return GLV_OK;
  CK(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  return GLV_OK;
}

// Hub tables and work lists.  Ordered accumulation (verify mode, non-integral
// weights) walks each hub with one warp and reuses one table region per step;
// the parallel path gives every hub of the schedule a private table, cut its
// row into kHubChunk-entry chunks and its filled-slot list into kHubSeg
// segments.
constexpr size_t kHubStepSlots = size_t(1) << 28;  // hub table slots of one step (3 GB)

int Engine::hub_offsets(const Level &L, std::vector<ClassSched> &sched) {
  const bool parallel = !ordered();
  std::vector<int64_t> tab_off, occ_off, seg_b, seg_e;
  std::vector<int32_t> c_pos, s_pos;
  std::vector<int64_t> c_beg, c_end, s_beg, s_end;
  std::vector<int64_t> hub_pos_all;
  size_t need_tab = 0;
  // row bounds of every hub of the schedule, in one gather
  std::vector<int32_t> hpos;
  for (auto &cs : sched)
    for (auto &st : cs.steps)
      for (int64_t k = st.seg[BIN_HUB]; k < st.seg[BIN_HUB + 1]; ++k) hpos.push_back((int32_t)k);
  std::vector<int64_t> hb_all(2 * hpos.size());
  hub_pos_h_.clear();
  hub_deg_h_.clear();
  const bool cl_rows = parallel && sweep_rows_ && cluster_ > 0;
  if (!hpos.empty()) {
    int32_t *d_pos;
    int64_t *bounds;
    TRY(alloc(&d_pos, hpos.size()));
    TRY(alloc(&bounds, 2 * hpos.size()));
    TRY(upload(s_, d_pos, hpos));
    LAUNCH(k_row_bounds_at, grid_for((int64_t)hpos.size(), 256, nsm_ * 4), 256, 0, s_,
           (int64_t)hpos.size(), d_pos, members_, L.ptr, bounds);
    CK(cudaMemcpyAsync(hb_all.data(), bounds, hb_all.size() * sizeof(int64_t),
                       cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    dfree(d_pos);
    dfree(bounds);
  }
  // A step whose hubs' tables would pass kHubStepSlots is cut into several
  // steps of the same class (its other bins stay in the first): members of a
  // class are independent and its deltas are applied after its last step, so
  // the decisions do not change.
  if (!hpos.empty()) {
    size_t hc = 0;
    for (auto &cs : sched) {
      std::vector<Step> out;
      for (auto &st : cs.steps) {
        const int64_t b = st.seg[BIN_HUB], e = st.seg[BIN_HUB + 1];
        size_t acc = 0;
        int64_t cut = b;
        Step cur = st;
        for (int64_t k = b; k < e; ++k) {
          const int64_t deg = hb_all[2 * (hc + (k - b)) + 1] - hb_all[2 * (hc + (k - b))];
          const size_t cap = table_cap(deg);
          if (acc > 0 && acc + cap > kHubStepSlots) {
            cur.seg[BIN_HUB] = cut;
            for (int q = BIN_HUB + 1; q <= NBINS; ++q) cur.seg[q] = k;
            out.push_back(cur);
            Step nx;
            for (int q = 0; q <= BIN_HUB; ++q) nx.seg[q] = k;
            for (int q = BIN_HUB + 1; q <= NBINS; ++q) nx.seg[q] = e;
            cur = nx;
            cut = k;
            acc = 0;
          }
          acc += cap;
        }
        hc += (size_t)(e - b);
        out.push_back(cur);
      }
      cs.steps = out;
    }
  }
  size_t hcur = 0;
  size_t need_occ = 0;
  for (auto &cs : sched)
    for (auto &st : cs.steps) {
      const int64_t b = st.seg[BIN_HUB], e = st.seg[BIN_HUB + 1];
      st.hub_chunk[0] = st.hub_chunk[1] = (int64_t)c_pos.size();
      st.hub_segs[0] = st.hub_segs[1] = (int64_t)s_pos.size();
      if (e == b) continue;
      const int64_t *hb = hb_all.data() + 2 * hcur;
      hcur += (size_t)(e - b);
      // a step's tables and filled-slot lists are empty again when it ends
      // (the scan clears the slots it visits, the finalisation the counters),
      // so every step starts its regions at offset 0
      size_t step_tab = 0, step_occ = 0;
      for (int64_t k = 0; k < e - b; ++k) {
        const int64_t rb = hb[2 * k], re = hb[2 * k + 1], deg = re - rb;
        const int64_t pos = b + k;
        uint32_t np = 0, cap = 0;
        if (cl_rows) cluster_row_shape(deg, cluster_, &np, &cap);
        if (cl_rows && np <= (uint32_t)cluster_parts_) {
          // a cluster row: no global table, chunks or segments
          hub_pos_h_.push_back((int32_t)pos);
          hub_deg_h_.push_back(deg);
          tab_off.push_back(0);
          occ_off.push_back(0);
          seg_b.push_back((int64_t)s_pos.size());
          seg_e.push_back((int64_t)s_pos.size());
          continue;
        }
        tab_off.push_back((int64_t)step_tab);
        step_tab += table_cap(deg);
        if (!parallel) continue;
        occ_off.push_back((int64_t)step_occ);
        step_occ += (size_t)deg + 1;
        for (int64_t x = rb; x < re; x += hub_chunk_) {
          c_pos.push_back((int32_t)pos);
          c_beg.push_back(x);
          c_end.push_back(std::min<int64_t>(re, x + hub_chunk_));
        }
        seg_b.push_back((int64_t)s_pos.size());
        for (int64_t x = 0; x < deg + 1; x += kHubSeg) {
          s_pos.push_back((int32_t)pos);
          s_beg.push_back(x);
          s_end.push_back(std::min<int64_t>(deg + 1, x + kHubSeg));
        }
        seg_e.push_back((int64_t)s_pos.size());
      }
      need_tab = std::max(need_tab, step_tab);
      need_occ = std::max(need_occ, step_occ);
      st.hub_chunk[1] = (int64_t)c_pos.size();
      st.hub_segs[1] = (int64_t)s_pos.size();
    }
  (void)hub_pos_all;
  if (hpos.empty()) return GLV_OK;
  if (need_tab > hub_cap_ || (parallel && !hub_tables_clean_)) {
    TRY(grow_hub(need_tab));
    if (parallel) {
      CK(cudaMemsetAsync(hub_keys_, 0xff, hub_cap_ * sizeof(int32_t), s_));
      CK(cudaMemsetAsync(hub_vals_, 0, hub_cap_ * sizeof(double), s_));
      hub_tables_clean_ = true;
    }
  }
  // per-hub values, aligned with hpos, scattered to their member slots
  int32_t *d_pos;
  int64_t *d_vals;
  const int64_t nh = (int64_t)hpos.size();
  TRY(alloc(&d_pos, nh));
  TRY(upload(s_, d_pos, hpos));
  TRY(alloc(&d_vals, 4 * nh));
  TRY(upload(s_, d_vals, tab_off));
  LAUNCH(k_scatter_i64, grid_for(nh, 256, nsm_ * 4), 256, 0, s_, nh, d_pos, d_vals, hub_off_);
  if (parallel) {
    if (need_occ > hub_occ_cap_) {
      dfree(hub_occ_);
      hub_occ_cap_ = need_occ;
      TRY(alloc(&hub_occ_, hub_occ_cap_));
    }
    if (c_pos.size() > chunk_cap_) {
      dfree(chunk_pos_); dfree(chunk_beg_); dfree(chunk_end_);
      chunk_cap_ = c_pos.size();
      TRY(alloc(&chunk_pos_, chunk_cap_)); TRY(alloc(&chunk_beg_, chunk_cap_));
      TRY(alloc(&chunk_end_, chunk_cap_));
    }
    if (s_pos.size() > seg_cap_) {
      dfree(seg_pos_); dfree(seg_beg_); dfree(seg_end_); dfree(part_g_); dfree(part_c_);
      seg_cap_ = s_pos.size();
      TRY(alloc(&seg_pos_, seg_cap_)); TRY(alloc(&seg_beg_, seg_cap_));
      TRY(alloc(&seg_end_, seg_cap_)); TRY(alloc(&part_g_, seg_cap_)); TRY(alloc(&part_c_, seg_cap_));
    }
    TRY(upload(s_, chunk_pos_, c_pos)); TRY(upload(s_, chunk_beg_, c_beg));
    TRY(upload(s_, chunk_end_, c_end)); TRY(upload(s_, seg_pos_, s_pos));
    TRY(upload(s_, seg_beg_, s_beg)); TRY(upload(s_, seg_end_, s_end));
    std::vector<int64_t> packed;
    packed.reserve(3 * nh);
    packed.insert(packed.end(), occ_off.begin(), occ_off.end());
    packed.insert(packed.end(), seg_b.begin(), seg_b.end());
    packed.insert(packed.end(), seg_e.begin(), seg_e.end());
    TRY(upload(s_, d_vals + nh, packed));
    LAUNCH(k_scatter_i64, grid_for(nh, 256, nsm_ * 4), 256, 0, s_, nh, d_pos, d_vals + nh,
           hub_occ_off_);
    LAUNCH(k_scatter_i64, grid_for(nh, 256, nsm_ * 4), 256, 0, s_, nh, d_pos, d_vals + 2 * nh,
           hub_seg_beg_);
    LAUNCH(k_scatter_i64, grid_for(nh, 256, nsm_ * 4), 256, 0, s_, nh, d_pos, d_vals + 3 * nh,
           hub_seg_end_);
    LAUNCH(k_hub_chunk_counts, grid_for(nh, 256, nsm_ * 4), 256, 0, s_, nh, d_pos, members_, L.ptr,
           hub_seg_beg_, hub_seg_end_, hub_chunk_, hub_left_, hub_segs_left_);
  }
  CK(cudaStreamSynchronize(s_));
  dfree(d_pos);
  dfree(d_vals);
  return GLV_OK;
}

// Iterated greedy passes over the colouring in color_ (recolor.cuh): classes
// in reverse order, each recoloured first-fit against the classes already
// done.  Stops after `passes` or when a pass removes no colour.
int Engine::recolor(const Level &L, int *ncolors, int passes) {
  if (ordered() || L.nv == 0 || passes <= 0) return GLV_OK;
  int32_t *key, *newc, *maxc;
  TRY(alloc(&key, L.nv)); TRY(alloc(&newc, L.nv)); TRY(alloc(&maxc, 1));
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_recolor_pass, kRecolorThreads, 0));
  if (per_sm < 1) return fail(GLV_ERR_CUDA, "recolouring kernel does not fit on an SM");
  const int grid = per_sm * nsm_;
  for (int k = 0; k < passes && *ncolors > 1; ++k) {
    LAUNCH(k_reverse_class_key, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, color_,
           (int32_t)*ncolors, key);
    std::vector<ClassSched> sched;
    TRY(build_schedule(L, key, *ncolors, nullptr, 1, &sched));
    std::vector<StepDesc> steps;
    for (auto &cs : sched)
      for (auto &st : cs.steps) {
        StepDesc d{};
        for (int b = 0; b <= NBINS; ++b) d.seg[b] = st.seg[b];
        d.hub_chunk[0] = st.hub_chunk[0];
        d.hub_chunk[1] = st.hub_chunk[1];
        steps.push_back(d);
      }
    StepDesc *d_steps;
    int64_t *d_ctr;
    TRY(alloc(&d_steps, steps.size()));
    TRY(alloc(&d_ctr, steps.size()));
    TRY(upload(s_, d_steps, steps));
    CK(cudaMemsetAsync(d_ctr, 0, steps.size() * sizeof(int64_t), s_));
    CK(cudaMemsetAsync(newc, 0xff, L.nv * sizeof(int32_t), s_));
    RecolorArgs r{L.ptr, L.tail, members_, newc, d_steps, (int)steps.size(), d_ctr,
                  chunk_pos_, chunk_beg_, chunk_end_, hub_off_, hub_keys_, hub_left_, hub_chunk_};
    void *args[] = {&r};
    CK(cudaLaunchCooperativeKernel((void *)k_recolor_pass, grid, kRecolorThreads, args, 0, s_));
    ++launches_;
    CK(cudaMemsetAsync(maxc, 0xff, sizeof(int32_t), s_));
    LAUNCH(k_max_color, grid_for(L.nv, 256, nsm_ * 8), 256, 0, s_, L.nv, newc, maxc);
    int32_t hm = -1;
    CK(cudaMemcpyAsync(&hm, maxc, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaMemcpyAsync(color_, newc, L.nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, s_));
    CK(cudaStreamSynchronize(s_));
    dfree(d_steps);
    dfree(d_ctr);
    const bool gained = hm + 1 < *ncolors;
    *ncolors = hm + 1;
    if (!gained) break;
  }
  dfree(key); dfree(newc); dfree(maxc);
  return GLV_OK;
}

// ------------------------------------------------------------------- sweeps
constexpr int kWarpCap = 256;   // table_cap(127)
constexpr int kBlockCap = 8192; // table_cap(4095)

int Engine::launch_sweep(const Level &L, const Step &st, SweepArgs a, bool ordered_acc,
                         Probes *pr) {
  const int cap = nsm_ * 16;
  for (int b = 0; b < NBINS; ++b) {
    const int64_t lo = st.seg[b], hi = st.seg[b + 1];
    const int64_t n = hi - lo;
    if (n <= 0) continue;
    int pidx = -1;
    if (pr) TRY(pr->begin(b, 2, s_, &pidx));
    switch (b) {
      case BIN_G4:
        LAUNCH(k_sweep_small<4>, grid_for(n * 4, 256, cap), 256, 0, s_, a, lo, hi);
        break;
      case BIN_G8:
        LAUNCH(k_sweep_small<8>, grid_for(n * 8, 256, cap), 256, 0, s_, a, lo, hi);
        break;
      case BIN_G16:
        LAUNCH(k_sweep_small<16>, grid_for(n * 16, 256, cap), 256, 0, s_, a, lo, hi);
        break;
      case BIN_G32:
        LAUNCH(k_sweep_small<32>, grid_for(n * 32, 256, cap), 256, 0, s_, a, lo, hi);
        break;
      case BIN_WARP: {
        const size_t smem = 8 * kWarpCap * (sizeof(double) + sizeof(int32_t));
        LAUNCH(k_sweep_warp<kWarpCap>, grid_for(n * 32, 256, cap), 256, smem, s_, a, lo, hi);
        break;
      }
      case BIN_T128:
      case BIN_T256:
      case BIN_BLOCK: {
        const size_t smem = (size_t)kBlockCap * (sizeof(double) + sizeof(int32_t));
        LAUNCH(k_sweep_block, (int)std::min<int64_t>(n, nsm_ * 2), 256, smem, s_, a, lo, hi, 0,
               ordered_acc ? 1 : 0);
        break;
      }
      case BIN_HUB:
        if (ordered_acc) {
          LAUNCH(k_sweep_block, (int)std::min<int64_t>(n, nsm_), 512, 0, s_, a, lo, hi, 1, 1);
        } else {
          const HubWork hw = hub_work();
          const int64_t nc = st.hub_chunk[1] - st.hub_chunk[0];
          const int64_t ns = st.hub_segs[1] - st.hub_segs[0];
          LAUNCH(k_hub_accum, (int)std::min<int64_t>(nc, nsm_ * 4), 512,
                 kHubStageSmem, s_, a, hw, st.hub_chunk[0],
                 st.hub_chunk[1]);
          LAUNCH(k_hub_scan, (int)std::min<int64_t>(ns, nsm_ * 8), 256, 0, s_, a, hw,
                 st.hub_segs[0], st.hub_segs[1]);
          LAUNCH(k_hub_final, grid_for(n * 32, 256, nsm_ * 4), 256, 0, s_, a, hw, lo, hi);
        }
        break;
    }
    if (pr) TRY(pr->end(pidx, s_));
  }
  return GLV_OK;
}

int Engine::launch_apply(const ClassSched &cs, bool ordered_upd) {
  const int64_t n = cs.end - cs.begin;
  if (!ordered_upd) {
    LAUNCH(k_apply_deltas, grid_for(n, 256, nsm_ * 16), 256, 0, s_, cs.begin, cs.end, move_old_,
           move_new_, dDeg, dSize, cDeg, cSize);
    return GLV_OK;
  }
  const uint64_t sentinel = (uint64_t)(uint32_t)nv0_ << 32;
  const int end_bit = 32 + bits_for(nv0_);
  LAUNCH(k_delta_records, grid_for(n, 256, nsm_ * 16), 256, 0, s_, cs.begin, cs.end, members_,
         move_old_, move_new_, vDeg, sentinel, dkeys_, drecs_);
  size_t tb = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, dkeys_, dkeys2_, drecs_, drecs2_, 2 * n, 0,
                                     end_bit, s_));
  if (tb > temp_bytes_) return fail(GLV_ERR_CUDA, "sort scratch not reserved before capture");
  CK(cub::DeviceRadixSort::SortPairs(temp_, tb, dkeys_, dkeys2_, drecs_, drecs2_, 2 * n, 0,
                                     end_bit, s_));
  LAUNCH(k_fold_deltas, grid_for(2 * n, 256, nsm_ * 16), 256, 0, s_, 2 * n, dkeys2_, drecs2_,
         sentinel, cDeg, cSize);
  return GLV_OK;
}

int Engine::launch_modularity(const Level &L, const int32_t *Cm, const double *ownw) {
  // one partial pair per block (part_e_ holds at least kConstParts)
  const int nparts = (int)std::max<int64_t>(1, std::min<int64_t>(merge_tiles(L.nv, L.nnz),
                                                                  kConstParts));
  LAUNCH(k_modularity_merge, nparts, 256, 0, s_, L.nv, L.nnz, L.ptr, L.tail, L.w, Cm, ownw, cDeg,
         split_row_, part_e_, part_a_);
  LAUNCH(k_modularity_final, 1, 256, 0, s_, nparts, part_e_, part_a_, cst, mod_out_);
  CK(cudaMemcpyAsync(h_mod_, mod_out_, 3 * sizeof(double), cudaMemcpyDeviceToHost, s_));
  return GLV_OK;
}

// Captures `body` into a CUDA graph (launch count recorded), returns the exec.
template <class F>
static int capture(cudaStream_t s, long *launches, F body, cudaGraphExec_t *exec, long *nodes) {
  cudaGraph_t g;
  const long before = *launches;
  CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  int r = body();
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (r != GLV_OK) {
    if (e == cudaSuccess) cudaGraphDestroy(g);
    return r;
  }
  CK(e);
  *nodes = *launches - before;
  *launches = before;
  cudaError_t ie = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  CK(ie);
  return GLV_OK;
}

int Engine::coloring_phase(const Level &L, int ncolors, bool stale, double lower, double thresh,
                           double *mod, int *itr) {
  const bool debug = getenv("GRAPPOLO_B200_DEBUG") != nullptr;
  double td = now_s();
  TRY(phase_init(L, false));
  int32_t *d_sub = nullptr;
  int nsub = 1;
  if (stale) {
    if (bt_) TRY(sublevels_batch(L, *bt_, &d_sub, &nsub));
    else TRY(sublevels(L, ncolors, &d_sub, &nsub));
  }
  if (debug) { cudaStreamSynchronize(s_); fprintf(stderr, "grappolo_b200: phase init %.4f s\n", now_s() - td); td = now_s(); }
  std::vector<ClassSched> sched;
  auto make_sched = [&](std::vector<ClassSched> *out) -> int {
    sweep_rows_ = persistent();
    int rc = build_schedule(L, color_, ncolors, d_sub, nsub, out);
    relaxed_ = false;
    if (rc == GLV_OK && nsub == 1 && core_color_ < ncolors) {  // core batches
      relaxed_ = true;
      for (ClassSched &cs : *out) cs.relaxed = cs.color >= core_color_;
    } else if (rc == GLV_OK && nsub == 1 && persistent()) {
      rc = group_classes(L, ncolors, out);
    }
    sweep_rows_ = false;
    return rc;
  };
  TRY(make_sched(&sched));
  if (debug) { cudaStreamSynchronize(s_); fprintf(stderr, "grappolo_b200: schedule %.4f s\n", now_s() - td); }
  dfree(d_sub);
  const bool ord = ordered();
  if (ord) {
    if (!dkeys_) {
      TRY(alloc(&dkeys_, 2 * nv0_)); TRY(alloc(&dkeys2_, 2 * nv0_));
      TRY(alloc(&drecs_, 2 * nv0_)); TRY(alloc(&drecs2_, 2 * nv0_));
    }
    size_t tb = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, dkeys_, dkeys2_, drecs_, drecs2_,
                                       2 * std::max<int64_t>(max_class_, 1), 0, 64, s_));
    TRY(temp(tb));
  }
  SweepArgs a{};
  a.ptr = L.ptr; a.tail = L.tail; a.w = L.w; a.C = C; a.target = nullptr; a.own_w = nullptr;
  a.vDeg = vDeg; a.cDeg = cDeg; a.cSize = cSize; a.members = members_;
  a.move_old = move_old_; a.move_new = move_new_; a.dDeg = dDeg; a.dSize = dSize;
  a.atomic_deltas = ord ? 0 : 1;
  a.hub_keys = hub_keys_; a.hub_vals = hub_vals_; a.hub_off = hub_off_;
  CK(cudaMemcpyAsync(&a.constant, cst, sizeof(double), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  a.defer_c = (relaxed_ && persistent()) ? 1 : 0;
  if (persistent() && phase_index_ == 0 && !bt_) {
    TRY(autotune(L, ncolors, &sched, make_sched, a, lower, thresh));
    a.hub_keys = hub_keys_; a.hub_vals = hub_vals_; a.hub_off = hub_off_;
  }
  if (first_cluster_ < 0) first_cluster_ = persistent() ? cluster_ : 0;
  if (debug)
    fprintf(stderr, "grappolo_b200: colour phase: persistent %d ordered %d cluster %d rows %zu\n",
            persistent() ? 1 : 0, ordered() ? 1 : 0, cluster_, hub_pos_h_.size());
  if (persistent()) return run_persistent(L, sched, a, false, lower, thresh, mod, itr);
  cudaGraphExec_t exec = nullptr;
  long nodes = 0;
  Probes pr;
  pr.level = g_profile.load();
  TRY(capture(s_, &launches_, [&]() -> int {
        for (auto &cs : sched) {
          int k;
          TRY(pr.begin(-1, 1, s_, &k));
          for (auto &st : cs.steps) TRY(launch_sweep(L, st, a, ord, &pr));
          TRY(pr.end(k, s_));
          int q;
          TRY(pr.begin(kSlotApply, 2, s_, &q));
          TRY(launch_apply(cs, ord));
          TRY(pr.end(q, s_));
        }
        int q;
        TRY(pr.begin(kSlotModularity, 2, s_, &q));
        TRY(launch_modularity(L, C, nullptr));
        return pr.end(q, s_);
      }, &exec, &nodes));
  double prev = lower;
  int n = 0;
  int rc = GLV_OK;
  while (true) {
    ++n;
    const double t0 = now_s();
    cudaError_t e = cudaGraphLaunch(exec, s_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s_);
    t_sweep += now_s() - t0;
    if (e != cudaSuccess) { g_err = cudaGetErrorString(e); rc = GLV_ERR_CUDA; break; }
    launches_ += nodes;
    edges_swept += (double)L.nnz;
    account(pr, L);
    const double q = h_mod_[0];
    if (q - prev < thresh) break;
    prev = q;
  }
  cudaGraphExecDestroy(exec);
  *mod = prev;
  *itr = n;
  return rc;
}

__global__ void k_rotate(int64_t n, int32_t *past, int32_t *curr, const int32_t *tgt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    past[i] = curr[i];
    curr[i] = tgt[i];
  }
}

// ------------------------------------------------------------- autotuner
// Speed-only knobs of the persistent sweep, picked per graph: the degree above
// which a row is a hub (global table, chunks over many blocks) instead of a
// block row (8192-slot shared table), and the entries per hub chunk.  Neither
// changes a decision: every candidate folds the same per-community sums
// (exactly, on integral weights) and takes the same arg-max.  On the first
// colour phase of a level with at least GRAPPOLO_B200_AUTOTUNE_MIN entries
// (default 2^24; GRAPPOLO_B200_AUTOTUNE=0 switches it off) each candidate runs
// one sweep iteration of the actual level from the phase's start state, which
// is restored after every trial; the fastest (device time of the launch)
// wins and is cached for the process under the graph's signature (vertex and
// entry counts and the row-degree histogram in powers of two), so repeated
// runs on the same graph pay once.
struct TuneChoice {
  int block_max;
  int hub_chunk;
  int cluster;
  double seconds;
};
static std::mutex g_tune_mu;
static std::map<std::string, TuneChoice> g_tune_cache;

__global__ void k_degree_log_hist(int64_t nv, const int64_t *ptr, unsigned long long *hist) {
  __shared__ unsigned int sh[64];
  for (int k = threadIdx.x; k < 64; k += blockDim.x) sh[k] = 0;
  __syncthreads();
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t d = (uint64_t)(ptr[v + 1] - ptr[v]);
    atomicAdd(&sh[d ? 64 - __clzll((long long)d) : 0], 1u);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < 64; k += blockDim.x)
    if (sh[k]) atomicAdd(&hist[k], (unsigned long long)sh[k]);
}

int Engine::autotune(const Level &L, int ncolors, std::vector<ClassSched> *sched,
                     const std::function<int(std::vector<ClassSched> *)> &make_sched,
                     SweepArgs a, double lower, double thresh) {
  const char *on = getenv("GRAPPOLO_B200_AUTOTUNE");
  if (on && on[0] == '0') return GLV_OK;
  const char *mn = getenv("GRAPPOLO_B200_AUTOTUNE_MIN");
  if (L.nnz < (mn ? atoll(mn) : (int64_t(1) << 24))) return GLV_OK;
  (void)ncolors;
  // signature
  unsigned long long *d_hist;
  TRY(alloc(&d_hist, 64));
  CK(cudaMemsetAsync(d_hist, 0, 64 * sizeof(unsigned long long), s_));
  LAUNCH(k_degree_log_hist, grid_for(L.nv, 256, nsm_ * 4), 256, 0, s_, L.nv, L.ptr, d_hist);
  unsigned long long hist[64];
  CK(cudaMemcpyAsync(hist, d_hist, sizeof(hist), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  dfree(d_hist);
  std::string sig = std::to_string(L.nv) + ":" + std::to_string(L.nnz) + ":" +
                    std::to_string(mode_);
  for (int k = 0; k < 64; ++k)
    if (hist[k]) sig += ":" + std::to_string(k) + "=" + std::to_string(hist[k]);
  const bool debug = getenv("GRAPPOLO_B200_DEBUG") != nullptr;
  const BinLimits lim0 = lim_;
  const int chunk0 = hub_chunk_;
  const int cluster0 = cluster_;
  auto apply = [&](int block_max, int chunk, int cl) -> int {
    if (block_max == lim_.block_max && chunk == hub_chunk_ && cl == cluster_) return GLV_OK;
    lim_.block_max = block_max;
    hub_chunk_ = chunk;
    cluster_ = cl;
    return make_sched(sched);
  };
  bool hit = false;
  TuneChoice cached{};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(sig);
    if (it != g_tune_cache.end()) {
      hit = true;
      cached = it->second;
    }
  }
  if (hit) {
    tune_cached_ = true;
    tune_choice_[0] = cached.block_max;
    tune_choice_[1] = cached.hub_chunk;
    return apply(cached.block_max, cached.hub_chunk, cached.cluster);
  }
  // the phase's start state, restored after every trial
  int32_t *C0, *S0;
  double *D0;
  TRY(alloc(&C0, L.nv)); TRY(alloc(&S0, L.nv)); TRY(alloc(&D0, L.nv));
  CK(cudaMemcpyAsync(C0, C, L.nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, s_));
  CK(cudaMemcpyAsync(S0, cSize, L.nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, s_));
  CK(cudaMemcpyAsync(D0, cDeg, L.nv * sizeof(double), cudaMemcpyDeviceToDevice, s_));
  // statistics the trials must not touch
  const double s_t = t_sweep, s_e = edges_swept, s_k = sweep_kernel_s, s_b = sweep_bytes;
  const long s_l = launches_, s_s = sweep_steps, s_g = gated_iterations_;
  // Candidates: hub thresholds 4095 and 2047 with every hub on global tables
  // in 2048-entry chunks, 1024-entry chunks, and the hub rows that fit on
  // 2-block clusters (the larger hubs keep their chunks).
  std::vector<TuneChoice> cands;
  const int bms[3] = {lim0.block_max, 2047, 1023};
  for (int bi = 0; bi < 3; ++bi) {
    if (bms[bi] > lim0.block_max || (bi > 0 && bms[bi] == lim0.block_max)) continue;
    if (bi < 2) cands.push_back(TuneChoice{bms[bi], kHubChunk, 0, INFINITY});
    if (bi == 0) cands.push_back(TuneChoice{bms[bi], kHubChunk / 2, 0, INFINITY});
    if (bi == 0 && cluster_grid(2) > 0) cands.push_back(TuneChoice{bms[bi], kHubChunk, 2, INFINITY});
  }
  TuneChoice best{lim0.block_max, chunk0, cluster0, INFINITY};
  int rc = GLV_OK;
  for (const TuneChoice &cand : cands) {
    {
      rc = apply(cand.block_max, cand.hub_chunk, cand.cluster);
      if (rc != GLV_OK) break;
      SweepArgs ta = a;
      ta.hub_keys = hub_keys_; ta.hub_vals = hub_vals_; ta.hub_off = hub_off_;
      max_iters_ = 1;
      double q = 0;
      int it = 0;
      rc = run_persistent(L, *sched, ta, false, lower, thresh, &q, &it);
      max_iters_ = 0;
      if (rc != GLV_OK) break;
      if (debug)
        fprintf(stderr, "grappolo_b200: autotune block_max %d chunk %d cluster %d: %.3f ms\n",
                cand.block_max, cand.hub_chunk, cand.cluster, last_launch_s_ * 1e3);
      if (last_launch_s_ < best.seconds)
        best = TuneChoice{cand.block_max, cand.hub_chunk, cand.cluster, last_launch_s_};
      cudaMemcpyAsync(C, C0, L.nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, s_);
      cudaMemcpyAsync(cSize, S0, L.nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, s_);
      cudaMemcpyAsync(cDeg, D0, L.nv * sizeof(double), cudaMemcpyDeviceToDevice, s_);
    }
  }
  CK(cudaStreamSynchronize(s_));
  dfree(C0); dfree(S0); dfree(D0);
  t_sweep = s_t; edges_swept = s_e; sweep_kernel_s = s_k; sweep_bytes = s_b;
  launches_ = s_l; sweep_steps = s_s; gated_iterations_ = s_g;
  if (rc != GLV_OK) return rc;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[sig] = best;
  }
  tune_cached_ = false;
  tune_choice_[0] = best.block_max;
  tune_choice_[1] = best.hub_chunk;
  return apply(best.block_max, best.hub_chunk, best.cluster);
}

int Engine::basic_phase(const Level &L, double lower, double thresh, double *mod, int *itr) {
  TRY(phase_init(L, true));
  std::vector<ClassSched> sched;
  sweep_rows_ = persistent();
  const int rc_sched = build_schedule(L, nullptr, 1, nullptr, 1, &sched);
  sweep_rows_ = false;
  TRY(rc_sched);
  const bool ord = ordered();
  if (ord) {
    if (!dkeys_) {
      TRY(alloc(&dkeys_, 2 * nv0_)); TRY(alloc(&dkeys2_, 2 * nv0_));
      TRY(alloc(&drecs_, 2 * nv0_)); TRY(alloc(&drecs2_, 2 * nv0_));
    }
    size_t tb = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, dkeys_, dkeys2_, drecs_, drecs2_,
                                       2 * std::max<int64_t>(max_class_, 1), 0, 64, s_));
    TRY(temp(tb));
  }
  SweepArgs a{};
  a.ptr = L.ptr; a.tail = L.tail; a.w = L.w; a.C = C; a.target = Ctgt; a.own_w = own_w;
  a.vDeg = vDeg; a.cDeg = cDeg; a.cSize = cSize; a.members = members_;
  a.move_old = move_old_; a.move_new = move_new_; a.dDeg = dDeg; a.dSize = dSize;
  a.atomic_deltas = ord ? 0 : 1;
  a.hub_keys = hub_keys_; a.hub_vals = hub_vals_; a.hub_off = hub_off_;
  CK(cudaMemcpyAsync(&a.constant, cst, sizeof(double), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  if (persistent()) {
    TRY(run_persistent(L, sched, a, true, lower, thresh, mod, itr));
    // C = pastCommAss (parallelLouvainMethod.cpp:304-307)
    CK(cudaMemcpyAsync(C, Cpast, L.nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, s_));
    CK(cudaStreamSynchronize(s_));
    return GLV_OK;
  }
  cudaGraphExec_t exec = nullptr;
  long nodes = 0;
  // Q is taken on the state before the moves (parallelLouvainMethod.cpp:244-255);
  // the totals update is applied in the same graph and only matters if the
  // loop continues.
  Probes pr;
  pr.level = g_profile.load();
  TRY(capture(s_, &launches_, [&]() -> int {
        int k;
        TRY(pr.begin(-1, 1, s_, &k));
        for (auto &cs : sched) {
          for (auto &st : cs.steps) TRY(launch_sweep(L, st, a, ord, &pr));
        }
        TRY(pr.end(k, s_));
        TRY(launch_modularity(L, C, own_w));
        for (auto &cs : sched) TRY(launch_apply(cs, ord));
        return GLV_OK;
      }, &exec, &nodes));
  double prev = -1.0;
  int n = 0;
  int rc = GLV_OK;
  while (true) {
    ++n;
    const double t0 = now_s();
    cudaError_t e = cudaGraphLaunch(exec, s_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s_);
    t_sweep += now_s() - t0;
    if (e != cudaSuccess) { g_err = cudaGetErrorString(e); rc = GLV_ERR_CUDA; break; }
    launches_ += nodes;
    edges_swept += (double)L.nnz;
    account(pr, L);
    const double q = h_mod_[0];
    if (q - prev < thresh) break;
    prev = q;
    if (prev < lower) prev = lower;
    LAUNCH(k_rotate, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, Cpast, C, Ctgt);
  }
  cudaGraphExecDestroy(exec);
  // C = pastCommAss (parallelLouvainMethod.cpp:304-307)
  CK(cudaMemcpyAsync(C, Cpast, L.nv * sizeof(int32_t), cudaMemcpyDeviceToDevice, s_));
  CK(cudaStreamSynchronize(s_));
  *mod = prev;
  *itr = n;
  return rc;
}

// Decisions for a vertex list against the state already in C/cDeg/cSize/vDeg
// and cst[0]; targets land in Ctgt[v].
int Engine::decide(const Level &L, const int32_t *verts, int64_t nverts) {
  const int64_t nkeys = NBINS;
  if (nkeys + 1 > hist_cap_) {
    dfree(hist_);
    hist_cap_ = (int)(nkeys + 1);
    TRY(alloc(&hist_, hist_cap_));
  }
  // schedule over the given list: key = bin only
  std::vector<int32_t> hv(nverts);
  std::vector<int64_t> hp(L.nv + 1);
  CK(cudaMemcpyAsync(hv.data(), verts, nverts * sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(hp.data(), L.ptr, (L.nv + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  std::vector<std::vector<int32_t>> byb(NBINS);
  for (int32_t v : hv) byb[degree_bin(hp[v + 1] - hp[v], lim_)].push_back(v);
  std::vector<int32_t> mem;
  ClassSched cs;
  Step st;
  for (int b = 0; b < NBINS; ++b) {
    st.seg[b] = (int64_t)mem.size();
    mem.insert(mem.end(), byb[b].begin(), byb[b].end());
  }
  st.seg[NBINS] = (int64_t)mem.size();
  cs.begin = 0; cs.end = (int64_t)mem.size();
  cs.steps.push_back(st);
  CK(cudaMemcpyAsync(members_, mem.data(), mem.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                     s_));
  CK(cudaStreamSynchronize(s_));
  std::vector<ClassSched> sched{cs};
  TRY(hub_offsets(L, sched));
  SweepArgs a{};
  a.ptr = L.ptr; a.tail = L.tail; a.w = L.w; a.C = C; a.target = Ctgt; a.own_w = own_w;
  a.vDeg = vDeg; a.cDeg = cDeg; a.cSize = cSize; a.members = members_;
  a.move_old = move_old_; a.move_new = move_new_; a.dDeg = dDeg; a.dSize = dSize;
  a.atomic_deltas = 0;
  a.hub_keys = hub_keys_; a.hub_vals = hub_vals_; a.hub_off = hub_off_;
  CK(cudaMemcpyAsync(&a.constant, cst, sizeof(double), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  TRY(launch_sweep(L, st, a, true, nullptr));
  CK(cudaStreamSynchronize(s_));
  return GLV_OK;
}

__global__ void k_trace_append(int64_t nv, const int64_t *ptr, const float *feat,
                               const int32_t *last_move, int32_t iter, uint32_t keep_below,
                               uint32_t salt, float *tx, float *ty, unsigned long long *tn,
                               int64_t cap) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    if (ptr[v + 1] == ptr[v]) continue;
    if (mix32((uint32_t)v ^ salt) > keep_below) continue;
    const unsigned long long k = atomicAdd(tn, 1ull);
    if ((int64_t)k >= cap) continue;
    for (int i = 0; i < kGateIn; ++i) tx[k * kGateIn + i] = feat[(size_t)v * kGateIn + i];
    ty[k] = (last_move[v] == iter) ? 1.0f : 0.0f;
  }
}

// The gate's per-vertex state lives for one phase's sweeps: sized for the
// phase's level and released after its last sweep, so the coarsening that
// follows (the run's memory peak on large graphs) has that memory back.
int Engine::gate_init(int64_t nv, bool tracing) {
  if (rec_own_) return GLV_OK;
  const size_t n = (size_t)nv + 1;
  TRY(alloc(&rec_own_, n)); TRY(alloc(&rec_gain_, n)); TRY(alloc(&last_move_, n));
  TRY(alloc(&skip_, n)); TRY(alloc(&gate_p_, kGateParams));
  if (tracing) TRY(alloc(&feat_, n * kGateIn));  // feature rows only for trace capture
  TRY(alloc(&evald_, 1));
  if (learned()) {
    std::lock_guard<std::mutex> lock(g_gate_mu);
    if ((int)g_gate_params.size() != kGateParams)
      return fail(GLV_ERR_ARG, "learned mode needs gate parameters (glv_gate_set)");
    CK(cudaMemcpyAsync(gate_p_, g_gate_params.data(), kGateParams * sizeof(float),
                       cudaMemcpyHostToDevice, s_));
    CK(cudaStreamSynchronize(s_));
  }
  return GLV_OK;
}

// Device memory an allocation could still get: free on the device, unused in
// the pool, and the blocks in this device's cache (a failed allocation hands
// them back to the pool).
int64_t Engine::avail_bytes() {
  size_t fr = 0, tot = 0;
  if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  uint64_t rc = 0, uc = 0;
  if (pool_) {
    cudaMemPoolGetAttribute(pool_, cudaMemPoolAttrReservedMemCurrent, &rc);
    cudaMemPoolGetAttribute(pool_, cudaMemPoolAttrUsedMemCurrent, &uc);
  }
  size_t cached = 0;
  {
    BlockCache &bc = g_cache[dev_];
    std::lock_guard<std::mutex> lock(bc.mu);
    for (const auto &kv : bc.free) cached += kv.first * kv.second.size();
  }
  return (int64_t)fr + (int64_t)(rc > uc ? rc - uc : 0) + (int64_t)cached;
}

void Engine::gate_release() {
  dfree(rec_own_); dfree(rec_gain_); dfree(last_move_); dfree(skip_); dfree(feat_);
  dfree(gate_p_); dfree(evald_);
}

__global__ void k_scatter_i32(int64_t n, const int32_t *pos, const int32_t *val, int32_t *out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    out[pos[k]] = val[k];
}

// Blocks of the persistent sweep kernel that a cooperative launch with
// clusters of cl blocks keeps resident at once (whole clusters only); 0 when
// none fits.
int Engine::cluster_grid(int cl) {
  if (cl < 1 || cl > kClusterMax) return 0;
  if (cluster_grid_[cl] > 0) return cluster_grid_[cl];
  if (cl == 1) {  // every block is a cluster of its own
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_iteration<true>,
                                                      kPersistThreads, kPersistSmem) !=
        cudaSuccess) {
      cudaGetLastError();
      return 0;
    }
    cluster_grid_[1] = per_sm * nsm_;
    return cluster_grid_[1];
  }
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cl;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(cl * nsm_));
  cfg.blockDim = dim3(kPersistThreads);
  cfg.dynamicSmemBytes = kPersistSmem;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  int nclusters = 0;
  if (cudaOccupancyMaxActiveClusters(&nclusters, (const void *)k_sweep_iteration<true>, &cfg) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  cluster_grid_[cl] = nclusters * cl;
  return cluster_grid_[cl];
}

// One cooperative launch per iteration (persist.cuh).  Colour phases: C is
// updated in place and Q is taken after the sweep; Jacobi phases: targets go
// to Ctgt, Q is taken on the state before the moves, and the loop rotates
// past <- curr <- target after an accepted iteration.
int Engine::run_persistent(const Level &L, const std::vector<ClassSched> &sched, SweepArgs a,
                           bool jacobi, double lower, double thresh, double *mod, int *itr) {
  std::vector<StepDesc> steps;
  std::vector<int64_t> cls_b, cls_e;
  for (auto &cs : sched) {
    cls_b.push_back(cs.begin);
    cls_e.push_back(cs.end);
    for (size_t k = 0; k < cs.steps.size(); ++k) {
      const Step &st = cs.steps[k];
      StepDesc d{};
      d.cls = (int64_t)cls_b.size() - 1;
      for (int b = 0; b <= NBINS; ++b) d.seg[b] = st.seg[b];
      d.hub_chunk[0] = st.hub_chunk[0]; d.hub_chunk[1] = st.hub_chunk[1];
      d.hub_segs[0] = st.hub_segs[0]; d.hub_segs[1] = st.hub_segs[1];
      const bool last = (k + 1 == cs.steps.size());
      d.apply[0] = last ? cs.begin : 0;
      d.apply[1] = last ? cs.end : 0;
      steps.push_back(d);
    }
  }
  // Hub rows as cluster tasks: one per (row, community partition), in the
  // step's hub order; their chunk and segment lists are not used.
  const int cl = (cluster_ > 0 && !hub_pos_h_.empty()) ? cluster_ : 0;
  if (cl > 0) {
    std::vector<int32_t> t_pos, t_part, t_np, p_pos, p_np;
    size_t hk = 0;
    for (auto &d : steps) {
      d.ctask[0] = d.ctask[1] = (int64_t)t_pos.size();
      while (hk < hub_pos_h_.size() && hub_pos_h_[hk] < d.seg[BIN_HUB]) ++hk;
      for (; hk < hub_pos_h_.size() && hub_pos_h_[hk] < d.seg[BIN_HUB + 1]; ++hk) {
        const int32_t pos = hub_pos_h_[hk];
        uint32_t np, cap;
        cluster_row_shape(hub_deg_h_[hk], cl, &np, &cap);
        for (uint32_t q = 0; q < np; ++q) {
          t_pos.push_back((int32_t)pos);
          t_part.push_back((int32_t)q);
          t_np.push_back((int32_t)np);
        }
        if (np > 1) { p_pos.push_back((int32_t)pos); p_np.push_back((int32_t)np); }
      }
      d.ctask[1] = (int64_t)t_pos.size();
    }
    if (t_pos.size() > ct_cap_) {  // task lists and the partitioned rows' partials
      dfree(ct_pos_); dfree(ct_part_); dfree(ct_nparts_); dfree(ct_g_); dfree(ct_c_); dfree(ct_g_); dfree(ct_c_);
      ct_cap_ = t_pos.size();
      TRY(alloc(&ct_pos_, ct_cap_)); TRY(alloc(&ct_part_, ct_cap_)); TRY(alloc(&ct_nparts_, ct_cap_));
      TRY(alloc(&ct_g_, ct_cap_)); TRY(alloc(&ct_c_, ct_cap_));
    }
    TRY(upload(s_, ct_pos_, t_pos)); TRY(upload(s_, ct_part_, t_part));
    TRY(upload(s_, ct_nparts_, t_np));
    if (!p_pos.empty()) {  // partitions still to finish, per partitioned row
      int32_t *d_pp;
      TRY(alloc(&d_pp, 2 * p_pos.size()));
      TRY(upload(s_, d_pp, p_pos));
      CK(cudaMemcpyAsync(d_pp + p_pos.size(), p_np.data(), p_np.size() * sizeof(int32_t),
                         cudaMemcpyHostToDevice, s_));
      LAUNCH(k_scatter_i32, grid_for((int64_t)p_pos.size(), 256, nsm_ * 4), 256, 0, s_,
             (int64_t)p_pos.size(), d_pp, d_pp + p_pos.size(), hub_segs_left_);
      CK(cudaStreamSynchronize(s_));
      dfree(d_pp);
    }
  }
  StepDesc *d_steps = nullptr;
  int64_t *d_ctr = nullptr;
  TRY(alloc(&d_steps, steps.size()));
  TRY(alloc(&d_ctr, 3 * steps.size()));  // block, team and cluster queues of every step
  TRY(upload(s_, d_steps, steps));
  int64_t *d_cls_b = nullptr;
  int32_t *d_kept = nullptr;
  const int nclass = (int)cls_b.size();
  const int64_t nmem = cls_e.empty() ? 0 : cls_e.back();
  Batch *bt = bt_;
  if ((!jacobi && learned()) || bt) {
    TRY(alloc(&d_cls_b, nclass)); TRY(alloc(&d_kept, nclass));
    TRY(upload(s_, d_cls_b, cls_b));
  }
  if (bt) {
    if (!skip_) TRY(alloc(&skip_, nv0_ + 1));
    a.gid = bt->gid;
    a.gcst = bt->gcst;
  }
  IterArgs p{};
  p.a = a;
  p.h = hub_work();
  p.steps = d_steps;
  p.nsteps = (int)steps.size();
  p.jacobi = jacobi ? 1 : 0;
  p.nv = L.nv;
  p.C_mod = C;
  p.own_w_mod = jacobi ? own_w : nullptr;
  p.part_e = part_e_;
  p.part_a = part_a_;
  p.cst = cst;
  p.mod_out = mod_out_;
  p.cDeg = cDeg;
  p.cSize = cSize;
  p.task_ctr = d_ctr;
  p.nnz = L.nnz;
  p.split_row = split_row_;
  // Fast mode on non-integral weights (no exact result to keep): after the
  // first sweep of a phase, e_xx is carried from the moves instead of a pass
  // over every entry.  GRAPPOLO_B200_FULL_MODULARITY=1 keeps the full pass;
  // GRAPPOLO_B200_CHECK_MODULARITY=1 runs both and fails when they differ.
  const char *fm = getenv("GRAPPOLO_B200_FULL_MODULARITY");
  const bool check_exx = getenv("GRAPPOLO_B200_CHECK_MODULARITY") != nullptr;
  bool carry_exx = !jacobi && !bt && !ordered() && !integral && !(fm && fm[0] == '1') &&
                   L.nnz > 0;
  // A step that runs several classes (a core batch) moves neighbours together,
  // and the carried change of each move assumes its neighbours stay put: the
  // entries whose two ends share such a step correct the carried sum.  When
  // they are too many to list, the phase takes the full pass instead.
  int32_t *step_of = nullptr, *pos_of = nullptr, *pair_u = nullptr, *pair_t = nullptr;
  double *pair_w = nullptr;
  int64_t npairs = 0;
  if (carry_exx && relaxed_) {
    std::vector<uint8_t> rel(sched.size());
    for (size_t k = 0; k < sched.size(); ++k) rel[k] = sched[k].relaxed ? 1 : 0;
    uint8_t *d_rel;
    int64_t *d_cb;
    unsigned long long *d_cnt;
    const int64_t cap = std::max<int64_t>(int64_t(1) << 20, L.nnz / 16);
    TRY(alloc(&step_of, L.nv)); TRY(alloc(&pos_of, L.nv));
    TRY(alloc(&d_rel, sched.size())); TRY(alloc(&d_cb, sched.size())); TRY(alloc(&d_cnt, 1));
    TRY(alloc(&pair_u, cap)); TRY(alloc(&pair_t, cap)); TRY(alloc(&pair_w, cap));
    TRY(upload(s_, d_rel, rel));
    TRY(upload(s_, d_cb, cls_b));
    CK(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), s_));
    LAUNCH(k_member_steps, grid_for(nmem, 256, nsm_ * 16), 256, 0, s_, nmem, members_,
           (int)sched.size(), d_cb, step_of, pos_of);
    LAUNCH(k_step_pairs, std::max(1, (int)std::min<int64_t>(merge_tiles(L.nv, L.nnz), nsm_ * 8)),
           256, 0, s_, L.nv, L.nnz, L.ptr, L.tail, L.w, step_of, d_rel, pos_of, split_row_, cap,
           pair_u, pair_t, pair_w, d_cnt);
    unsigned long long hc = 0;
    CK(cudaMemcpyAsync(&hc, d_cnt, sizeof(hc), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    dfree(d_rel); dfree(d_cb); dfree(d_cnt); dfree(step_of); dfree(pos_of);
    if ((int64_t)hc <= cap) {
      npairs = (int64_t)hc;
    } else {
      carry_exx = false;
      dfree(pair_u); dfree(pair_t); dfree(pair_w);
    }
    if (getenv("GRAPPOLO_B200_DEBUG"))
      fprintf(stderr, "grappolo_b200: %llu same-step entries (cap %ld)%s\n", hc, (long)cap,
              carry_exx ? "" : ": full modularity passes");
  }
  p.pair_u = pair_u;
  p.pair_t = pair_t;
  p.pair_w = pair_w;
  p.npairs = npairs;

  if (bt) {
    p.gid = bt->gid;
    p.gacc = bt->gacc;
  }
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_iteration<false>, kPersistThreads,
                                                   kPersistSmem));
  if (per_sm < 1) return fail(GLV_ERR_CUDA, "persistent sweep kernel does not fit on an SM");
  const int grid = cl > 0 ? cluster_grid(cl) : per_sm * nsm_;
  if (grid < 1) return fail(GLV_ERR_CUDA, "no cluster of the persistent sweep kernel fits");
  double *exx_buf = nullptr;
  if (carry_exx) {
    TRY(alloc(&exx_buf, (size_t)grid + 1));  // carried e_xx, then one slot per block
    p.a.exx_delta = exx_buf + 1;
    p.exx_state = exx_buf;
  }
  void *args[] = {&p};
  const bool debug = getenv("GRAPPOLO_B200_DEBUG") != nullptr;
  uint64_t *d_trace = nullptr;
  std::vector<uint64_t> h_trace;
  if (debug) {
    TRY(alloc(&d_trace, 8 * steps.size() + 2));
    CK(cudaMemsetAsync(d_trace, 0, (8 * steps.size() + 2) * sizeof(uint64_t), s_));
    h_trace.resize(8 * steps.size() + 2);
    p.trace = d_trace;
  }
  const int level = g_profile.load();
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (level > 0 || max_iters_ > 0) {
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
  }
  double prev = jacobi ? -1.0 : lower;
  int n = 0;
  int rc = GLV_OK;
  // learned gate / trace capture (colour phases only)
  const bool tracing = !jacobi && g_trace.on && !bt;
  const bool gating = !jacobi && learned() && !bt;
  std::vector<double> bprev;
  if (bt) {
    bprev.assign(bt->G, 0.0);
    for (int g = 0; g < bt->G; ++g) {
      bt->h_act[g] = bt->in_phase[g];
      bprev[g] = jacobi ? -1.0 : bt->lower[g];
      bt->mod[g] = bprev[g];
      bt->itr[g] = 0;
    }
    CK(cudaMemcpyAsync(bt->act, bt->h_act.data(), bt->G, cudaMemcpyHostToDevice, s_));
  }
  if (gating || tracing) {
    TRY(gate_init(L.nv, tracing));
    CK(cudaMemsetAsync(last_move_, 0, L.nv * sizeof(int32_t), s_));
    CK(cudaMemsetAsync(rec_own_, 0, L.nv * sizeof(double), s_));
    CK(cudaMemsetAsync(rec_gain_, 0, L.nv * sizeof(float), s_));
    p.a.rec_own = rec_own_;
    p.a.rec_gain = rec_gain_;
    p.a.last_move = last_move_;
  }
  bool force_full = true;  // the first sweep of a phase is always a full one
  // Gated sweeps only in the phase's tail: once a full sweep gains less than
  // GRAPPOLO_B200_GATE_TAIL (default 16) times the threshold.  Early sweeps
  // move many vertices, and a gate that misses some of them costs iterations.
  double gate_tail = 16.0;
  if (const char *e = getenv("GRAPPOLO_B200_GATE_TAIL")) gate_tail = atof(e);
  double last_full_gain = INFINITY;
  float tau = 0.5f;
  {
    std::lock_guard<std::mutex> lock(g_gate_mu);
    tau = g_gate_tau;
  }
  while (true) {
    ++n;
    const double t0 = now_s();
    p.a.iter = n;
    bool gated_now = false;
    if (gating || tracing) {
      gated_now = gating && !force_full && n >= 2 &&
                  (gate_tail <= 0.0 || last_full_gain < gate_tail * thresh);
      const GateFeatSrc fsrc{L.ptr, vDeg, rec_own_, rec_gain_, last_move_, n, phase_index_};
      if (n >= 2 && tracing)
        LAUNCH(k_gate_features, grid_for(L.nv, 256, nsm_ * 8), 256, 0, s_, L.nv, fsrc, feat_);
      p.a.skip = nullptr;
      if (gated_now) {
        // the features are computed inside the inference kernel unless a
        // trace capture has just written them
        CK(cudaMemsetAsync(evald_, 0, sizeof(unsigned long long), s_));
        LAUNCH(k_gate_infer, std::max(1, (int)std::min<int64_t>((L.nv + 127) / 128, nsm_ * 8)), 256, 0,
               s_, L.nv, tracing ? (const float *)feat_ : nullptr, fsrc, gate_p_, tau, L.ptr,
               (float *)nullptr, skip_, evald_);
        CK(cudaMemsetAsync(d_kept, 0, nclass * sizeof(int32_t), s_));
        LAUNCH(k_class_kept, grid_for(nmem, 256, nsm_ * 8), 256, 0, s_, nclass, d_cls_b, nmem,
               members_, skip_, d_kept);
        p.a.skip = skip_;
      }
      p.class_kept = gated_now ? d_kept : nullptr;
    }
    double batch_edges = 0;
    if (bt) {
      // graphs that have converged (or sit out this phase) are skipped whole
      LAUNCH(k_graph_skip, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, bt->gid, bt->act,
             skip_);
      CK(cudaMemsetAsync(d_kept, 0, nclass * sizeof(int32_t), s_));
      LAUNCH(k_class_kept, grid_for(nmem, 256, nsm_ * 8), 256, 0, s_, nclass, d_cls_b, nmem,
             members_, skip_, d_kept);
      CK(cudaMemsetAsync(bt->gacc, 0, 2 * bt->G * sizeof(double), s_));
      p.a.skip = skip_;
      p.class_kept = d_kept;
      for (int g = 0; g < bt->G; ++g)
        if (bt->h_act[g]) batch_edges += (double)bt->gnnz[g];
    }
    p.exx_mode = (carry_exx && n >= 2) ? (check_exx ? 2 : 1) : 0;
    cudaError_t e = cudaMemsetAsync(d_ctr, 0, 3 * steps.size() * sizeof(int64_t), s_);
    p.h.epoch = ++epoch_;
    if (e0) cudaEventRecord(e0, s_);
    if (e == cudaSuccess && cl > 0) {
      cudaLaunchAttribute at[2];
      at[0].id = cudaLaunchAttributeCooperative;
      at[0].val.cooperative = 1;
      at[1].id = cudaLaunchAttributeClusterDimension;
      at[1].val.clusterDim.x = (unsigned)cl;
      at[1].val.clusterDim.y = 1;
      at[1].val.clusterDim.z = 1;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)grid);
      cfg.blockDim = dim3(kPersistThreads);
      cfg.dynamicSmemBytes = kPersistSmem;
      cfg.stream = s_;
      cfg.attrs = at;
      cfg.numAttrs = 2;
      e = cudaLaunchKernelEx(&cfg, k_sweep_iteration<true>, p);
    } else if (e == cudaSuccess) {
      e = cudaLaunchCooperativeKernel((void *)k_sweep_iteration<false>, grid, kPersistThreads, args,
                                      kPersistSmem, s_);
    }
    if (e1) cudaEventRecord(e1, s_);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h_mod_, mod_out_, 5 * sizeof(double), cudaMemcpyDeviceToHost, s_);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s_);
    t_sweep += now_s() - t0;
    if (e != cudaSuccess) { g_err = cudaGetErrorString(e); rc = GLV_ERR_CUDA; break; }
    if (h_mod_[4] != 0.0) {
      rc = fail(GLV_ERR_CUDA, h_mod_[4] == 2.0
                                  ? "sweep: a hub partition's cluster table overflowed"
                                  : "sweep: a hub's table scan gave up waiting for its chunks");
      break;
    }
    if (p.exx_mode == 2) {
      const double carried = h_mod_[1], full = h_mod_[3];
      if (debug)
        fprintf(stderr, "grappolo_b200: e_xx carried %.17g full %.17g (rel %.3g)\n", carried,
                full, fabs(carried - full) / std::max(1.0, fabs(full)));
      if (!(fabs(carried - full) <= 1e-9 * std::max(1.0, fabs(full)))) {
        rc = fail(GLV_ERR_CUDA, "carried e_xx differs from the full pass");
        break;
      }
    }
    ++launches_;
    if (bt) {
      edges_swept += batch_edges;
    } else if (gated_now) {
      unsigned long long ev = 0;
      CK(cudaMemcpy(&ev, evald_, sizeof(ev), cudaMemcpyDeviceToHost));
      edges_swept += (double)ev;
      ++gated_iterations_;
    } else {
      edges_swept += (double)L.nnz;
    }
    if (tracing && n >= 2) {
      const uint32_t keep = (uint32_t)std::min(4294967295.0, g_trace.rate * 4294967296.0);
      LAUNCH(k_trace_append, grid_for(L.nv, 256, nsm_ * 8), 256, 0, s_, L.nv, L.ptr, feat_,
             last_move_, n, keep, (uint32_t)(n * 7919 + phase_index_ * 104729), g_trace.x,
             g_trace.y, g_trace.n, g_trace.cap);
    }
    if (e0) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) sweep_kernel_s += ms * 1e-3;
      last_launch_s_ = ms * 1e-3;
      // sweep: 16 B per entry + 36 B per vertex; modularity: a full pass 16 B
      // per entry + 12 B per vertex, a carried e_xx 8 B per vertex (cDeg)
      sweep_bytes += (p.exx_mode == 1) ? 16.0 * (double)L.nnz + 44.0 * (double)L.nv
                                       : 32.0 * (double)L.nnz + 48.0 * (double)L.nv;
      ++sweep_steps;
    }
    if (debug) {
      CK(cudaMemcpy(h_trace.data(), d_trace, h_trace.size() * sizeof(uint64_t),
                    cudaMemcpyDeviceToHost));
      CK(cudaMemsetAsync(d_trace, 0, h_trace.size() * sizeof(uint64_t), s_));
      // Stage times per step (a zero slot = stage not run); steps holding
      // only hub rows are summed apart.
      const size_t ns = steps.size();
      uint64_t last = h_trace[4 * ns];
      double acc[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
      int cnt[2] = {0, 0};
      std::vector<double> per(ns, 0.0);
      for (size_t k = 0; k < ns; ++k) {
        const StepDesc &d = steps[k];
        const int hub_only = (d.seg[BIN_HUB] == d.seg[0] && d.seg[NBINS] > d.seg[0]) ? 1 : 0;
        if (h_trace[4 * k] == 0) continue;  // skipped step
        uint64_t t = last;
        for (int q = 0; q < 4; ++q) {
          const uint64_t x = h_trace[4 * k + q];
          if (x == 0 || x < t) continue;
          acc[hub_only][q] += (x - t) * 1e-9;
          t = x;
        }
        per[k] = (t - last) * 1e-9;
        ++cnt[hub_only];
        last = t;
      }
      const double tm = h_trace[4 * ns + 1] > last ? (h_trace[4 * ns + 1] - last) * 1e-9 : 0.0;
      if (const char *tf = getenv("GRAPPOLO_B200_TRACE_FILE")) {
        // one line per step: level size, iteration, step, members per degree
        // bin, hub chunks, then the stage times in microseconds
        if (FILE *f = fopen(tf, "a")) {
          uint64_t t = h_trace[4 * ns];
          for (size_t k = 0; k < ns; ++k) {
            const StepDesc &d = steps[k];
            fprintf(f, "%ld %d %zu", (long)L.nv, n, k);
            for (int b = 0; b < NBINS; ++b) fprintf(f, " %ld", (long)(d.seg[b + 1] - d.seg[b]));
            fprintf(f, " %ld", (long)(d.hub_chunk[1] - d.hub_chunk[0] + d.ctask[1] - d.ctask[0]));
            const uint64_t t0 = t;
            for (int q = 0; q < 4; ++q) {
              const uint64_t x = h_trace[4 * k + q];
              if (x == 0 || x < t) { fprintf(f, " 0"); continue; }
              fprintf(f, " %.2f", (x - t) * 1e-3);
              t = x;
            }
            // when the block queue, the team queue, the warp items and the
            // cluster tasks ran dry
            for (int q = 0; q < 4; ++q) {
              const uint64_t x = h_trace[4 * ns + 2 + 4 * k + q];
              fprintf(f, " %.2f", (x > t0) ? (x - t0) * 1e-3 : 0.0);
            }
            fprintf(f, "\n");
          }
          fclose(f);
        }
      }
      std::vector<double> sorted = per;
      std::sort(sorted.begin(), sorted.end());
      fprintf(stderr,
              "grappolo_b200: iter %d nv=%ld steps=%zu | mixed %d: stage1 %.4f scan %.4f final "
              "%.4f apply %.4f | hub-only %d: stage1 %.4f scan %.4f final %.4f apply %.4f | "
              "modularity %.4f | step median %.1f us p90 %.1f us max %.1f us\n",
              n, (long)L.nv, ns, cnt[0], acc[0][0], acc[0][1], acc[0][2], acc[0][3], cnt[1],
              acc[1][0], acc[1][1], acc[1][2], acc[1][3], tm, sorted[ns / 2] * 1e6,
              sorted[ns * 9 / 10] * 1e6, sorted[ns - 1] * 1e6);
    }
    if (bt) {
      // per-graph Q = e*c - a*c*c and the phase loop's test, graph by graph
      CK(cudaMemcpyAsync(bt->h_acc.data(), bt->gacc, 2 * bt->G * sizeof(double),
                         cudaMemcpyDeviceToHost, s_));
      CK(cudaStreamSynchronize(s_));
      bool any = false;
      for (int g = 0; g < bt->G; ++g) {
        if (!bt->h_act[g]) continue;
        const double c = bt->h_gcst[g];
        const double qg = bt->h_acc[2 * g] * c - bt->h_acc[2 * g + 1] * c * c;
        bt->itr[g] = n;
        if (!(qg - bprev[g] >= bt->thresh)) {  // NaN (no edges) ends the graph too
          bt->h_act[g] = 0;
          bt->mod[g] = bprev[g];
          bt->done_s[g] = now_s();
        } else {
          bprev[g] = qg;
          if (jacobi && bprev[g] < bt->lower[g]) bprev[g] = bt->lower[g];
          any = true;
        }
      }
      if (!any) break;
      CK(cudaMemcpyAsync(bt->act, bt->h_act.data(), bt->G, cudaMemcpyHostToDevice, s_));
      if (jacobi)
        LAUNCH(k_rotate_active, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, bt->gid,
               bt->act, Cpast, C, Ctgt);
      continue;
    }
    const double q = h_mod_[0];
    if (debug)
      fprintf(stderr, "grappolo_b200: iter %d gated %d q %.9f gain %.3e edges %.0f time %.5f\n", n,
              (int)gated_now, q, q - prev, edges_swept, now_s() - t0);
    if (max_iters_ > 0 && n >= max_iters_) {
      prev = q;
      break;
    }
    if (!gated_now) last_full_gain = q - prev;
    if (q - prev < thresh) {
      // A phase ends only after a full (ungated) sweep gains less than thresh.
      if (!gated_now) break;
      if (q > prev) prev = q;
      force_full = true;
      continue;
    }
    prev = q;
    force_full = false;
    if (jacobi) {
      if (prev < lower) prev = lower;
      LAUNCH(k_rotate, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, Cpast, C, Ctgt);
    }
  }
  if (gating || tracing) gate_release();
  dfree(d_trace);
  dfree(d_ctr);
  dfree(pair_u); dfree(pair_t); dfree(pair_w);
  dfree(d_cls_b);
  dfree(d_kept);
  dfree(exx_buf);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  dfree(d_steps);
  *mod = prev;
  *itr = n;
  return rc;
}

// --------------------------------------------------------------- renumbering
int Engine::renumber(int32_t *Cm, int64_t n, int64_t *ncl) {
  if (n == 0) { *ncl = 0; return GLV_OK; }
  int32_t *first, *flag, *scan;
  TRY(alloc(&first, n)); TRY(alloc(&flag, n)); TRY(alloc(&scan, n));
  const int g = grid_for(n, 256, nsm_ * 16);
  LAUNCH(k_fill_i32, g, 256, 0, s_, n, first, INT32_MAX);
  LAUNCH(k_first_occurrence, g, 256, 0, s_, n, Cm, first);
  LAUNCH(k_open_flags, g, 256, 0, s_, n, Cm, first, flag);
  size_t tb = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, scan, n, s_));
  TRY(temp(tb));
  CK(cub::DeviceScan::ExclusiveSum(temp_, tb, flag, scan, n, s_));
  LAUNCH(k_apply_renumber, g, 256, 0, s_, n, Cm, first, scan);
  int32_t h[2];
  CK(cudaMemcpyAsync(&h[0], scan + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(&h[1], flag + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  dfree(first); dfree(flag); dfree(scan);
  *ncl = (int64_t)h[0] + h[1];
  return GLV_OK;
}

// ----------------------------------------------------------------- coarsening
__global__ void k_add_counts(int64_t n, const int64_t *a, const int64_t *b, int64_t *out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (i < n) ? a[i] + b[i] : 0;
}

// Chunked coarsening (phase_kernels.cuh): records for one range of row
// communities at a time, at most about `budget` records per chunk, so a level
// of billions of entries needs a fraction of the two-sort path's buffers.
// vf: the vertex-following graph (Utility/vertexFollowing.cpp:91-255) — no
// zero self-loop seeds, every weight cast to long before it is summed.
int Engine::coarsen_chunked(const Level &in, const int32_t *Cm, int64_t ncl, Level *out,
                            int64_t *num_edges, int64_t budget, bool vf) {
  const int nb = bits_for(std::max<int64_t>(ncl - 1, 1));
  int64_t *cnt, *prefix, *rowc;
  TRY(alloc(&cnt, ncl + 1)); TRY(alloc(&prefix, ncl + 1)); TRY(alloc(&rowc, ncl + 1));
  LAUNCH(k_fill_i64, grid_for(ncl, 256, nsm_ * 16), 256, 0, s_, ncl, cnt, (int64_t)(vf ? 0 : 1));
  CK(cudaMemsetAsync(cnt + ncl, 0, sizeof(int64_t), s_));
  LAUNCH(k_comm_entry_counts, grid_for(in.nv, 256, nsm_ * 16), 256, 0, s_, in.nv, in.ptr, Cm,
         cnt);
  size_t tb = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt, prefix, ncl + 1, s_));
  TRY(temp(tb));
  CK(cub::DeviceScan::ExclusiveSum(temp_, tb, cnt, prefix, ncl + 1, s_));
  int64_t total = 0;
  CK(cudaMemcpyAsync(&total, prefix + ncl, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  const int K = (int)std::max<int64_t>(1, (total + budget - 1) / budget);
  int64_t *bounds, *pb;
  TRY(alloc(&bounds, K + 1)); TRY(alloc(&pb, K + 1));
  LAUNCH(k_chunk_bounds, (K + 1 + 255) / 256, 256, 0, s_, ncl, prefix, K, bounds);
  LAUNCH(k_gather_i64, grid_for(K + 1, 256, nsm_), 256, 0, s_, (int64_t)K + 1, bounds, prefix, pb);
  std::vector<int64_t> hb(K + 1), hp(K + 1);
  CK(cudaMemcpyAsync(hb.data(), bounds, (K + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(hp.data(), pb, (K + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  int64_t maxrec = 1;
  for (int k = 0; k < K; ++k) maxrec = std::max(maxrec, hp[k + 1] - hp[k]);
  // record buffers of at most 2 x budget entries; a chunk with more records
  // (one community with a huge row sum) is read in tile slices whose partial
  // sums are gathered in the accumulation buffer and reduced once more
  // (never below one tile's records plus a chunk's seeds: a slice is at
  // least one merge-path tile)
  int64_t maxseeds = 1;
  for (int k = 0; k < K; ++k) maxseeds = std::max(maxseeds, hb[k + 1] - hb[k]);
  const int64_t cap =
      std::min<int64_t>(maxrec, std::max<int64_t>(2 * budget, 2 * kMergeTile + maxseeds));
  uint64_t *k1, *k2, *uk, *ak;
  double *v1, *v2, *uv, *av;
  unsigned long long *counter, *ndiag;
  int64_t *d_np;
  TRY(alloc(&k1, cap)); TRY(alloc(&k2, cap)); TRY(alloc(&uk, cap));
  TRY(alloc(&v1, cap)); TRY(alloc(&v2, cap)); TRY(alloc(&uv, cap));
  TRY(alloc(&counter, 1)); TRY(alloc(&d_np, 1)); TRY(alloc(&ndiag, 1));
  CK(cudaMemsetAsync(ndiag, 0, sizeof(unsigned long long), s_));
  const bool sliced = maxrec > cap;
  ak = nullptr;
  av = nullptr;
  if (sliced) { TRY(alloc(&ak, cap)); TRY(alloc(&av, cap)); }
  CK(cudaMemsetAsync(rowc, 0, (ncl + 1) * sizeof(int64_t), s_));
  // The rows in community order (vertex id within a community), so that a
  // chunk's rows are one run of merge tiles and each chunk reads only them.
  const int64_t ntiles = merge_tiles(in.nv, in.nnz);
  int32_t *perm, *oid;
  uint32_t *ok1, *ok2;
  int64_t *pdeg, *pptr, *split_perm, *ctile;
  TRY(alloc(&ok1, in.nv)); TRY(alloc(&ok2, in.nv)); TRY(alloc(&oid, in.nv)); TRY(alloc(&perm, in.nv));
  TRY(alloc(&pdeg, in.nv + 1)); TRY(alloc(&pptr, in.nv + 1)); TRY(alloc(&split_perm, ntiles + 1));
  TRY(alloc(&ctile, K + 1));
  LAUNCH(k_comm_order_keys, grid_for(in.nv, 256, nsm_ * 16), 256, 0, s_, in.nv, Cm, ok1, oid);
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, ok1, ok2, oid, perm, in.nv, 0, 32, s_));
  TRY(temp(tb));
  CK(cub::DeviceRadixSort::SortPairs(temp_, tb, ok1, ok2, oid, perm, in.nv, 0, 32, s_));
  LAUNCH(k_perm_degrees, grid_for(in.nv, 256, nsm_ * 16), 256, 0, s_, in.nv, perm, in.ptr, pdeg);
  CK(cudaMemsetAsync(pdeg + in.nv, 0, sizeof(int64_t), s_));
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, pdeg, pptr, in.nv + 1, s_));
  TRY(temp(tb));
  CK(cub::DeviceScan::ExclusiveSum(temp_, tb, pdeg, pptr, in.nv + 1, s_));
  LAUNCH(k_merge_splits, grid_for(ntiles + 1, 256, nsm_ * 8), 256, 0, s_, in.nv, in.nnz, pptr,
         ntiles, split_perm);
  LAUNCH(k_chunk_tiles, (K + 1 + 255) / 256, 256, 0, s_, K, bounds, in.nv, ok2, pptr, ctile);
  std::vector<int64_t> hct(K + 1);
  CK(cudaMemcpyAsync(hct.data(), ctile, (K + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  dfree(ok1); dfree(oid); dfree(pdeg); dfree(ctile);
  // the coarse rows go straight to their place: `total` (records of all
  // chunks) bounds the coarse entries, and a copy of the chunks' outputs
  // would double the peak on levels of billions of entries
  Level o;
  o.nv = ncl;
  o.owned = true;
  int64_t at = 0;
  const int grid = std::max(1, (int)std::min<int64_t>(ntiles, nsm_ * 8));
  // sort + reduce n records of (kin, vin) into (kout, vout); returns the pairs
  auto sort_reduce = [&](uint64_t *ka, uint64_t *kb, double *va, double *vb, int64_t n,
                         int end_bit, uint64_t *kout, double *vout, int64_t *np) -> int {
    cub::DoubleBuffer<uint64_t> dk(ka, kb);
    cub::DoubleBuffer<double> dv(va, vb);
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, n, 0, end_bit, s_));
    TRY(temp(tb));
    CK(cub::DeviceRadixSort::SortPairs(temp_, tb, dk, dv, n, 0, end_bit, s_));
    CK(cub::DeviceReduce::ReduceByKey(nullptr, tb, dk.Current(), kout, dv.Current(), vout, d_np,
                                      cuda::std::plus<>{}, n, s_));
    TRY(temp(tb));
    CK(cub::DeviceReduce::ReduceByKey(temp_, tb, dk.Current(), kout, dv.Current(), vout, d_np,
                                      cuda::std::plus<>{}, n, s_));
    CK(cudaMemcpyAsync(np, d_np, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    return GLV_OK;
  };
  // records of tiles [t0, t1) into (k1, v1); returns their count (may pass cap)
  auto records = [&](int64_t a0, int64_t a1, int64_t t0, int64_t t1, int seeds,
                     int64_t *n) -> int {
    CK(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), s_));
    LAUNCH(k_chunk_records, grid, 256, sizeof(PermTileSmem), s_, in.nv, in.nnz, in.ptr,
           in.tail, in.w, Cm, perm, pptr, split_perm, (int32_t)a0, (int32_t)a1, nb, t0, t1,
           vf ? 0 : seeds, vf ? 1 : 0, (unsigned long long)cap, counter, k1, v1);
    unsigned long long hn = 0;
    CK(cudaMemcpyAsync(&hn, counter, sizeof(hn), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    *n = (int64_t)hn;
    return GLV_OK;
  };
  // The coarse rows go straight to their place.  `total` (records of all
  // chunks) bounds the coarse entries.  A level of that bound is allocated
  // unless it is large and the device could not hold it beside a margin for
  // the next phase (a tenth of the device, at least 8 GB); then the chunks
  // run twice, first only to count, so the level gets its exact size (the
  // counting pass repeats every chunk's records and sorts).
  const int64_t bound_bytes = total * (int64_t)(sizeof(int32_t) + sizeof(double));
  // GRAPPOLO_B200_COARSEN_PASSES=1|2 forces one way.
  const char *cp = getenv("GRAPPOLO_B200_COARSEN_PASSES");
  bool two_pass = getenv("GRAPPOLO_B200_COARSEN_EXACT") != nullptr || (cp && atoi(cp) == 2);
  int64_t avail = -1;
  if (!two_pass && !(cp && atoi(cp) == 1) && bound_bytes > (int64_t(16) << 30)) {
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) cudaGetLastError();
    const int64_t margin = std::max<int64_t>(int64_t(8) << 30, (int64_t)tot / 10);
    avail = avail_bytes();
    two_pass = bound_bytes + margin > avail;
  }
  if (debug_)
    fprintf(stderr, "grappolo_b200: chunked coarsening, %d chunks, bound %.2f GB, available "
            "%.2f GB, %s\n", K, bound_bytes * 1e-9, avail * 1e-9,
            two_pass ? "counting pass first" : "one pass");
  for (int pass = two_pass ? 0 : 1; pass < 2; ++pass) {
    const bool counting = pass == 0;
    if (!counting) {
      const int64_t n_out = two_pass ? at : total;
      TRY(alloc(&o.tail, std::max<int64_t>(n_out, 1)));
      TRY(alloc(&o.w, std::max<int64_t>(n_out, 1)));
      at = 0;
    }
    for (int k = 0; k < K; ++k) {
      const int64_t a0 = hb[k], a1 = hb[k + 1];
      if (a1 <= a0) continue;
      const int end_bit = nb + bits_for(std::max<int64_t>(a1 - a0 - 1, 1));
      // the chunk's tile run (one tile past the start of the next chunk's rows)
      const int64_t tk0 = hct[k], tk1 = std::min<int64_t>(ntiles, hct[k + 1] + 1);
      int64_t np = 0;
      if (hp[k + 1] - hp[k] <= cap) {
        int64_t n = 0;
        TRY(records(a0, a1, tk0, tk1, 1, &n));
        TRY(sort_reduce(k1, k2, v1, v2, n, end_bit, uk, uv, &np));
      } else {
        // slices of tiles; a slice whose records overflow is cut in two
        int64_t acc = 0;
        std::vector<std::pair<int64_t, int64_t>> todo;
        const int64_t nsl = 2 * ((hp[k + 1] - hp[k] + cap - 1) / cap);
        for (int64_t q = nsl - 1; q >= 0; --q)
          todo.push_back({tk0 + (tk1 - tk0) * q / nsl, tk0 + (tk1 - tk0) * (q + 1) / nsl});
        bool first = true;
        while (!todo.empty()) {
          const auto sl = todo.back();
          todo.pop_back();
          int64_t n = 0;
          TRY(records(a0, a1, sl.first, sl.second, first ? 1 : 0, &n));
          if (n > cap) {
            if (sl.second - sl.first <= 1)
              return fail(GLV_ERR_OOM, "a coarsening tile exceeds the record buffer");
            const int64_t mid = (sl.first + sl.second) / 2;
            todo.push_back({mid, sl.second});
            todo.push_back({sl.first, mid});
            continue;
          }
          first = false;
          int64_t pn = 0;
          TRY(sort_reduce(k1, k2, v1, v2, n, end_bit, uk, uv, &pn));
          if (acc + pn > cap) {  // fold what has been gathered so far
            int64_t an = 0;
            TRY(sort_reduce(ak, k1, av, v1, acc, end_bit, k2, v2, &an));
            CK(cudaMemcpyAsync(ak, k2, an * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s_));
            CK(cudaMemcpyAsync(av, v2, an * sizeof(double), cudaMemcpyDeviceToDevice, s_));
            acc = an;
            if (acc + pn > cap) return fail(GLV_ERR_OOM, "coarsening partial sums exceed the buffer");
          }
          CK(cudaMemcpyAsync(ak + acc, uk, pn * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s_));
          CK(cudaMemcpyAsync(av + acc, uv, pn * sizeof(double), cudaMemcpyDeviceToDevice, s_));
          acc += pn;
        }
        TRY(sort_reduce(ak, k1, av, v1, acc, end_bit, uk, uv, &np));
      }
      if (!counting) {
        LAUNCH(k_chunk_emit, grid_for(np, 256, nsm_ * 16), 256, 0, s_, np, uk, nb, (int32_t)a0,
               rowc, o.tail + at, ndiag);
        CK(cudaMemcpyAsync(o.w + at, uv, np * sizeof(double), cudaMemcpyDeviceToDevice, s_));
      }
      at += np;
    }
  }
  dfree(ak); dfree(av);
  dfree(k1); dfree(k2); dfree(uk); dfree(v1); dfree(v2); dfree(uv);
  dfree(ok2); dfree(perm); dfree(pptr); dfree(split_perm);
  unsigned long long hdiag = 0;
  CK(cudaMemcpyAsync(&hdiag, ndiag, sizeof(hdiag), cudaMemcpyDeviceToHost, s_));
  dfree(counter); dfree(d_np); dfree(ndiag); dfree(bounds); dfree(pb); dfree(cnt); dfree(prefix);
  TRY(alloc(&o.ptr, ncl + 1));
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, rowc, o.ptr, ncl + 1, s_));
  TRY(temp(tb));
  CK(cub::DeviceScan::ExclusiveSum(temp_, tb, rowc, o.ptr, ncl + 1, s_));
  o.nnz = at;
  dfree(rowc);
  CK(cudaStreamSynchronize(s_));
  *out = o;
  // off-diagonal pairs once, plus the diagonal ones (every cluster has its
  // seed unless vf)
  *num_edges = (o.nnz - (int64_t)hdiag) / 2 + (int64_t)hdiag;
  return GLV_OK;
}

int Engine::coarsen(const Level &in, const int32_t *Cm, int64_t ncl, Level *out,
                    int64_t *num_edges) {
  // Levels whose two-sort records (32 B per entry) would not fit beside the
  // graph go through the chunked path outside verify mode;
  // GRAPPOLO_B200_COARSEN_CHUNK=<records> forces it with that chunk size.
  {
    const char *cc = getenv("GRAPPOLO_B200_COARSEN_CHUNK");
    const int64_t budget = cc ? std::max<int64_t>(atoll(cc), 1) : (int64_t(1) << 27);
    if (!ordered() && ncl > 0 && (cc || ncl + in.nnz > (int64_t(1) << 30)))
      return coarsen_chunked(in, Cm, ncl, out, num_edges, budget);
  }
  // Fast and learned modes (no entry order to keep): a level with few
  // communities folds its entries into a dense ncl x ncl matrix; the others
  // keep the sorts.  GRAPPOLO_B200_COARSEN=sort|hash forces the sorts or the
  // per-community hash tables on every level.
  if (mode_ != GLV_MODE_VERIFY && ncl > 0) {
    const char *cv = getenv("GRAPPOLO_B200_COARSEN");
    const std::string want = cv ? cv : "";
    if (want == "hash") return coarsen_hash(in, Cm, ncl, out, num_edges, false);
    if (want != "sort" && ncl <= kDenseCoarseMax)
      return coarsen_hash(in, Cm, ncl, out, num_edges, true);
  }
  const bool debug = getenv("GRAPPOLO_B200_DEBUG") != nullptr;
  double tdbg = now_s();
  auto mark = [&](const char *what) {
    if (!debug) return;
    cudaStreamSynchronize(s_);
    const double t = now_s();
    fprintf(stderr, "grappolo_b200: coarsen %s %.4f s\n", what, t - tdbg);
    tdbg = t;
  };
  const int nb = bits_for(std::max<int64_t>(ncl - 1, 1));
  const uint64_t sentinel = 1ull << (2 * nb);
  const int end_bit = 2 * nb + 1;
  const int64_t n_all = ncl + in.nnz;
  if (n_all > crec_cap_) {
    dfree(ck1_); dfree(ck2_); dfree(cv1_); dfree(cv2_);
    // sized for level 0 when that is modest, so every level reuses them
    const int64_t lvl0 = nnz0_ + nv0_;
    crec_cap_ = lvl0 <= (int64_t(1) << 30) ? std::max<int64_t>(n_all, lvl0) : n_all;
    TRY(alloc(&ck1_, crec_cap_)); TRY(alloc(&ck2_, crec_cap_));
    TRY(alloc(&cv1_, crec_cap_)); TRY(alloc(&cv2_, crec_cap_));
  }
  uint64_t *k1 = ck1_, *k2 = ck2_;
  double *v1 = cv1_, *v2 = cv2_;
  TRY(merge_splits(in));
  const int rgrid = std::max(1, (int)std::min<int64_t>(merge_tiles(in.nv, in.nnz), nsm_ * 8));
  // records of the pairs that exist, in entry order (two passes over the tiles)
  const int64_t ntiles = merge_tiles(in.nv, in.nnz);
  int64_t *tile_cnt, *tile_off;
  TRY(alloc(&tile_cnt, ntiles + 1)); TRY(alloc(&tile_off, ntiles + 1));
  CK(cudaMemsetAsync(tile_cnt + ntiles, 0, sizeof(int64_t), s_));
  LAUNCH(k_coarse_tile_counts, rgrid, 256, 0, s_, in.nv, in.nnz, in.ptr, in.tail, Cm, nb,
         split_row_, tile_cnt);
  {
    size_t sb = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, sb, tile_cnt, tile_off, ntiles + 1, s_));
    TRY(temp(sb));
    CK(cub::DeviceScan::ExclusiveSum(temp_, sb, tile_cnt, tile_off, ntiles + 1, s_));
  }
  LAUNCH(k_coarse_records_compact, rgrid, 256, 0, s_, in.nv, in.nnz, in.ptr, in.tail, in.w, Cm,
         ncl, nb, split_row_, tile_off, k1, v1);
  int64_t nrec = 0;
  CK(cudaMemcpyAsync(&nrec, tile_off + ntiles, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  dfree(tile_cnt);
  dfree(tile_off);
  const int64_t n = ncl + nrec;
  size_t tb = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k1, k2, v1, v2, n, 0, end_bit, s_));
  TRY(temp(tb));
  mark("records");
  CK(cub::DeviceRadixSort::SortPairs(temp_, tb, k1, k2, v1, v2, n, 0, end_bit, s_));
  mark("sort");
  uint64_t *ukeys;
  double *uvals;
  int64_t np = 0;
  const int g = grid_for(n, 256, nsm_ * 16);
  if (ordered()) {
    // one thread folds each pair's records in (i, j) order
    int32_t *flag;
    int64_t *uidx;
    TRY(alloc(&flag, n)); TRY(alloc(&uidx, n));
    LAUNCH(k_segment_heads, g, 256, 0, s_, n, k2, sentinel, flag);
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, flag, uidx, n, s_));
    TRY(temp(tb));
    CK(cub::DeviceScan::ExclusiveSum(temp_, tb, flag, uidx, n, s_));
    int64_t hu;
    int32_t hf;
    CK(cudaMemcpyAsync(&hu, uidx + n - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaMemcpyAsync(&hf, flag + n - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    np = hu + hf;
    TRY(alloc(&ukeys, np)); TRY(alloc(&uvals, np));
    LAUNCH(k_fold_pairs, g, 256, 0, s_, n, k2, v2, flag, uidx, sentinel, ukeys, uvals);
    dfree(flag); dfree(uidx);
  } else {
    // reduce-by-key over the sorted records (the sentinel run is dropped by
    // counting only keys below it)
    int64_t *d_np;
    ukeys = k1;
    uvals = v1;
    TRY(alloc(&d_np, 1));
    CK(cub::DeviceReduce::ReduceByKey(nullptr, tb, k2, ukeys, v2, uvals, d_np, cuda::std::plus<>{},
                                      n, s_));
    TRY(temp(tb));
    CK(cub::DeviceReduce::ReduceByKey(temp_, tb, k2, ukeys, v2, uvals, d_np, cuda::std::plus<>{},
                                      n, s_));
    CK(cudaMemcpyAsync(&np, d_np, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    dfree(d_np);
    uint64_t last = 0;
    if (np > 0) {
      CK(cudaMemcpyAsync(&last, ukeys + np - 1, sizeof(uint64_t), cudaMemcpyDeviceToHost, s_));
      CK(cudaStreamSynchronize(s_));
      if (last >= sentinel) --np;
    }
  }
  mark("fold");
  int64_t *lower_cnt, *upper_cnt, *ne_off, *rowc, *lower_first, *upper_first;
  TRY(alloc(&lower_cnt, ncl)); TRY(alloc(&upper_cnt, ncl)); TRY(alloc(&ne_off, 1));
  TRY(alloc(&rowc, ncl + 1)); TRY(alloc(&lower_first, ncl)); TRY(alloc(&upper_first, ncl));
  CK(cudaMemsetAsync(lower_cnt, 0, ncl * sizeof(int64_t), s_));
  CK(cudaMemsetAsync(upper_cnt, 0, ncl * sizeof(int64_t), s_));
  CK(cudaMemsetAsync(ne_off, 0, sizeof(int64_t), s_));
  const int gp = grid_for(np, 256, nsm_ * 16);
  LAUNCH(k_row_counts, gp, 256, 0, s_, np, ukeys, nb, lower_cnt, upper_cnt, ne_off);
  LAUNCH(k_add_counts, grid_for(ncl + 1, 256, nsm_ * 16), 256, 0, s_, ncl, lower_cnt, upper_cnt,
         rowc);
  Level o;
  o.nv = ncl;
  o.owned = true;
  TRY(alloc(&o.ptr, ncl + 1));
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, rowc, o.ptr, ncl + 1, s_));
  TRY(temp(tb));
  CK(cub::DeviceScan::ExclusiveSum(temp_, tb, rowc, o.ptr, ncl + 1, s_));
  int64_t hne;
  CK(cudaMemcpyAsync(&o.nnz, o.ptr + ncl, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaMemcpyAsync(&hne, ne_off, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  mark("emit counts");
  TRY(alloc(&o.tail, o.nnz)); TRY(alloc(&o.w, o.nnz));
  LAUNCH(k_run_first, gp, 256, 0, s_, np, ukeys, nb, sentinel, lower_first);
  uint64_t *tk1 = k2, *tk2;
  double *tv1 = v2, *tv2;
  TRY(alloc(&tk2, np)); TRY(alloc(&tv2, np));
  LAUNCH(k_emit_lower, gp, 256, 0, s_, np, ukeys, uvals, nb, o.ptr, lower_first, o.tail, o.w, tk1,
         tv1, sentinel);
  mark("emit lower");
  // stable on the b bits (and the sentinel bit) only: each b's keys already
  // come in ascending a
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, tk1, tk2, tv1, tv2, np, nb, end_bit, s_));
  TRY(temp(tb));
  CK(cub::DeviceRadixSort::SortPairs(temp_, tb, tk1, tk2, tv1, tv2, np, nb, end_bit, s_));
  mark("emit sort");
  LAUNCH(k_run_first, gp, 256, 0, s_, np, tk2, nb, sentinel, upper_first);
  LAUNCH(k_emit_upper, gp, 256, 0, s_, np, tk2, tv2, nb, o.ptr, lower_cnt, upper_first, o.tail,
         o.w, sentinel);
  CK(cudaStreamSynchronize(s_));
  mark("emit");
  dfree(tk2); dfree(tv2);
  if (ukeys != k1) { dfree(ukeys); dfree(uvals); }
  dfree(lower_cnt); dfree(upper_cnt); dfree(ne_off); dfree(rowc); dfree(lower_first);
  dfree(upper_first);
  *out = o;
  *num_edges = hne + ncl;
  return GLV_OK;
}

// The next level without sorts (coarsen_hash.cuh): per-community hash
// tables, or with `dense` an ncl x ncl matrix of sums (ncl <= kDenseCoarseMax).
int Engine::coarsen_hash(const Level &in, const int32_t *Cm, int64_t ncl, Level *out,
                         int64_t *num_edges, bool dense) {
  const bool debug = getenv("GRAPPOLO_B200_DEBUG") != nullptr;
  double tdbg = now_s();
  auto mark = [&](const char *what) {
    if (!debug) return;
    cudaStreamSynchronize(s_);
    const double t = now_s();
    fprintf(stderr, "grappolo_b200: coarsen %s %.4f s\n", what, t - tdbg);
    tdbg = t;
  };
  const int64_t nv = in.nv;
  const int g_nv = grid_for(nv, 256, nsm_ * 16), g_cl = grid_for(ncl + 1, 256, nsm_ * 16);
  // 1. members in community order and their entry offsets
  uint32_t *mk1, *mk2;
  int32_t *mv1, *mv2;
  int64_t *mdeg, *mptr, *d_nmem;
  TRY(alloc(&mk1, nv)); TRY(alloc(&mk2, nv)); TRY(alloc(&mv1, nv)); TRY(alloc(&mv2, nv));
  TRY(alloc(&mdeg, nv + 1)); TRY(alloc(&mptr, nv + 1)); TRY(alloc(&d_nmem, 1));
  CK(cudaMemsetAsync(d_nmem, 0, sizeof(int64_t), s_));
  CK(cudaMemsetAsync(mdeg + nv, 0, sizeof(int64_t), s_));
  LAUNCH(k_hc_member_keys, g_nv, 256, 0, s_, nv, Cm, in.ptr, ncl, mk1, mv1);
  size_t tb = 0;
  const int kbits = bits_for(ncl);
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, mk1, mk2, mv1, mv2, nv, 0, kbits, s_));
  TRY(temp(tb));
  CK(cub::DeviceRadixSort::SortPairs(temp_, tb, mk1, mk2, mv1, mv2, nv, 0, kbits, s_));
  LAUNCH(k_hc_member_degrees, g_nv, 256, 0, s_, nv, mk2, mv2, in.ptr, ncl, mdeg, d_nmem);
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, mdeg, mptr, nv + 1, s_));
  TRY(temp(tb));
  CK(cub::DeviceScan::ExclusiveSum(temp_, tb, mdeg, mptr, nv + 1, s_));
  int64_t nmem = 0;
  CK(cudaMemcpyAsync(&nmem, d_nmem, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  int64_t E = 0;
  CK(cudaMemcpyAsync(&E, mptr + nmem, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  dfree(mk1); dfree(mv1); dfree(mdeg);
  // 2. community entry ranges; big-community tables or the dense matrix
  int64_t *cE0, *cE1, *capA, *gtoff, *nch, *nchoff, *cnt;
  uint8_t *has_self;
  int32_t *err;
  TRY(alloc(&cE0, ncl + 1)); TRY(alloc(&cE1, ncl + 1)); TRY(alloc(&capA, ncl + 1));
  TRY(alloc(&gtoff, ncl + 1)); TRY(alloc(&nch, ncl + 1)); TRY(alloc(&nchoff, ncl + 1));
  TRY(alloc(&cnt, ncl + 1)); TRY(alloc(&has_self, ncl + 1)); TRY(alloc(&err, 1));
  CK(cudaMemsetAsync(cE0, 0, (ncl + 1) * sizeof(int64_t), s_));
  CK(cudaMemsetAsync(cE1, 0, (ncl + 1) * sizeof(int64_t), s_));
  CK(cudaMemsetAsync(cnt, 0, (ncl + 1) * sizeof(int64_t), s_));
  CK(cudaMemsetAsync(has_self, 0, (ncl + 1) * sizeof(uint8_t), s_));
  CK(cudaMemsetAsync(err, 0, sizeof(int32_t), s_));
  CK(cudaMemsetAsync(capA + ncl, 0, sizeof(int64_t), s_));
  CK(cudaMemsetAsync(nch + ncl, 0, sizeof(int64_t), s_));
  if (nmem > 0)
    LAUNCH(k_hc_community_ranges, grid_for(nmem, 256, nsm_ * 16), 256, 0, s_, nmem, mk2, mptr, cE0,
           cE1);
  int64_t G = 0, nchunks = 0;
  if (!dense) {
    LAUNCH(k_hc_big_caps, g_cl, 256, 0, s_, ncl, cE0, cE1, capA, nch);
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, capA, gtoff, ncl + 1, s_));
    TRY(temp(tb));
    CK(cub::DeviceScan::ExclusiveSum(temp_, tb, capA, gtoff, ncl + 1, s_));
    CK(cub::DeviceScan::ExclusiveSum(temp_, tb, nch, nchoff, ncl + 1, s_));
    CK(cudaMemcpyAsync(&G, gtoff + ncl, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaMemcpyAsync(&nchunks, nchoff + ncl, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  }
  CK(cudaStreamSynchronize(s_));
  int32_t *gkeys = nullptr, *chunk_comm = nullptr, *out_b = nullptr;
  double *gvals = nullptr, *dmat = nullptr, *out_w = nullptr;
  uint32_t *dbits = nullptr;
  if (dense) {
    const int64_t cells = ncl * ncl;
    TRY(alloc(&dmat, cells)); TRY(alloc(&dbits, (cells + 31) / 32));
    CK(cudaMemsetAsync(dmat, 0, cells * sizeof(double), s_));
    CK(cudaMemsetAsync(dbits, 0, ((cells + 31) / 32) * sizeof(uint32_t), s_));
  } else {
    TRY(alloc(&out_b, std::max<int64_t>(E, 1))); TRY(alloc(&out_w, std::max<int64_t>(E, 1)));
    if (G > 0) {
      TRY(alloc(&gkeys, G)); TRY(alloc(&gvals, G)); TRY(alloc(&chunk_comm, nchunks));
      CK(cudaMemsetAsync(gkeys, 0xff, G * sizeof(int32_t), s_));
      CK(cudaMemsetAsync(gvals, 0, G * sizeof(double), s_));
      LAUNCH(k_hc_chunk_list, g_cl, 256, 0, s_, ncl, nchoff, chunk_comm);
    }
  }
  dfree(capA); dfree(nch);
  mark("hash members");
  // 3. tasks: one window of kHashWindow entries' small communities each, then
  // the big communities' chunks
  if (E > 0) {
    const int64_t nwin = (E + kHashWindow - 1) / kHashWindow;
    int64_t *nbch, *nbch_off;
    TRY(alloc(&nbch, ncl + 1)); TRY(alloc(&nbch_off, ncl + 1));
    CK(cudaMemsetAsync(nbch + ncl, 0, sizeof(int64_t), s_));
    unsigned long long *wE0, *wE1;
    TRY(alloc(&wE0, nwin)); TRY(alloc(&wE1, nwin));
    CK(cudaMemsetAsync(wE0, 0xff, nwin * sizeof(unsigned long long), s_));
    CK(cudaMemsetAsync(wE1, 0, nwin * sizeof(unsigned long long), s_));
    LAUNCH(k_hc_windows, g_cl, 256, 0, s_, ncl, cE0, cE1, wE0, wE1, nbch);
    CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, nbch, nbch_off, ncl + 1, s_));
    TRY(temp(tb));
    CK(cub::DeviceScan::ExclusiveSum(temp_, tb, nbch, nbch_off, ncl + 1, s_));
    int64_t nbig = 0;
    CK(cudaMemcpyAsync(&nbig, nbch_off + ncl, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
    CK(cudaStreamSynchronize(s_));
    const int64_t ntask = nwin + nbig;
    unsigned long long *tE0, *tE1;
    int64_t *mlo, *mhi;
    TRY(alloc(&tE0, ntask)); TRY(alloc(&tE1, ntask)); TRY(alloc(&mlo, ntask)); TRY(alloc(&mhi, ntask));
    CK(cudaMemcpyAsync(tE0, wE0, nwin * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s_));
    CK(cudaMemcpyAsync(tE1, wE1, nwin * sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s_));
    dfree(wE0); dfree(wE1);
    if (nbig > 0)
      LAUNCH(k_hc_big_tasks, g_cl, 256, 0, s_, ncl, nwin, cE0, cE1, nbch_off, tE0, tE1);
    LAUNCH(k_hc_tile_members, grid_for(ntask, 256, nsm_ * 16), 256, 0, s_, ntask, tE0, tE1, mptr,
           nmem, mlo, mhi);
    HashTileArgs ha{ntask, nwin, nmem, ncl, mptr, tE0, tE1, mlo, mhi, mk2, mv2, in.ptr, in.tail,
                    in.w, Cm, cE0, gtoff, gkeys, gvals, out_b, out_w, cnt, has_self, err, dmat,
                    dbits};
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hc_tiles, kHashThreads,
                                                     sizeof(HashTileSmem)));
    if (per_sm < 1) return fail(GLV_ERR_CUDA, "coarsening task kernel does not fit on an SM");
    const int grid = (int)std::min<int64_t>(ntask, (int64_t)per_sm * nsm_);
    LAUNCH(k_hc_tiles, grid, kHashThreads, sizeof(HashTileSmem), s_, ha);
    dfree(nbch); dfree(nbch_off); dfree(tE0); dfree(tE1); dfree(mlo); dfree(mhi);
    mark("hash tasks");
    if (nchunks > 0)
      LAUNCH(k_hc_big_emit, (int)std::min<int64_t>(nchunks, nsm_ * 8), 256, 0, s_, nchunks,
             chunk_comm, nchoff, gtoff, gkeys, gvals, cE0, out_b, out_w, cnt, has_self);
    mark("hash big");
  }
  int32_t herr = 0;
  CK(cudaMemcpyAsync(&herr, err, sizeof(int32_t), cudaMemcpyDeviceToHost, s_));
  // 4. rows
  int64_t *rowc;
  TRY(alloc(&rowc, ncl + 1));
  const int g_rows = grid_for(ncl * 32, 256, nsm_ * 16);
  if (dense) LAUNCH(k_hc_dense_counts, g_rows, 256, 0, s_, ncl, dbits, rowc);
  else LAUNCH(k_hc_row_lengths, g_cl, 256, 0, s_, ncl, cnt, has_self, rowc);
  Level o;
  o.nv = ncl;
  o.owned = true;
  TRY(alloc(&o.ptr, ncl + 1));
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb, rowc, o.ptr, ncl + 1, s_));
  TRY(temp(tb));
  CK(cub::DeviceScan::ExclusiveSum(temp_, tb, rowc, o.ptr, ncl + 1, s_));
  CK(cudaMemcpyAsync(&o.nnz, o.ptr + ncl, sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
  CK(cudaStreamSynchronize(s_));
  if (herr) return fail(GLV_ERR_CUDA, "coarsening: a community's table filled up");
  TRY(alloc(&o.tail, o.nnz)); TRY(alloc(&o.w, o.nnz));
  if (dense) {
    LAUNCH(k_hc_dense_emit, g_rows, 256, 0, s_, ncl, dbits, dmat, o.ptr, o.tail, o.w);
  } else {
    const int64_t nct = (o.nnz + kCopyTile - 1) / kCopyTile;
    int64_t *alo, *ahi;
    TRY(alloc(&alo, nct)); TRY(alloc(&ahi, nct));
    LAUNCH(k_hc_copy_rows, grid_for(nct, 256, nsm_ * 16), 256, 0, s_, nct, ncl, o.ptr, alo, ahi);
    LAUNCH(k_hc_compact, (int)std::max<int64_t>(1, std::min<int64_t>(nct, nsm_ * 8)), 256, 0, s_,
           ncl, o.ptr, alo, ahi, cE0, has_self, out_b, out_w, o.tail, o.w);
    dfree(alo); dfree(ahi);
  }
  CK(cudaStreamSynchronize(s_));
  mark("hash rows");
  dfree(mk2); dfree(mv2); dfree(mptr); dfree(d_nmem); dfree(cE0); dfree(cE1); dfree(gtoff);
  dfree(nchoff); dfree(cnt); dfree(has_self); dfree(err); dfree(rowc);
  if (out_b) { dfree(out_b); dfree(out_w); }
  if (gkeys) { dfree(gkeys); dfree(gvals); dfree(chunk_comm); }
  if (dmat) { dfree(dmat); dfree(dbits); }
  *out = o;
  *num_edges = (o.nnz - ncl) / 2 + ncl;  // one (a, a) entry per row, the rest in mirrored pairs
  return GLV_OK;
}

__global__ void k_comm_degrees(int64_t nv, const int32_t *Cm, const double *vDeg, double *cDeg) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int32_t c = Cm[i];
    if (c >= 0) atomicAdd(&cDeg[c], vDeg[i]);
  }
}

// Q of an arbitrary assignment Cm (ids < L.nv, -1 = none) over L.
int Engine::modularity_of(const Level &L, const int32_t *Cm, double *q) {
  TRY(phase_init(L, false));
  CK(cudaMemsetAsync(cDeg, 0, L.nv * sizeof(double), s_));
  LAUNCH(k_comm_degrees, grid_for(L.nv, 256, nsm_ * 16), 256, 0, s_, L.nv, Cm, vDeg, cDeg);
  TRY(launch_modularity(L, Cm, nullptr));
  CK(cudaStreamSynchronize(s_));
  *q = h_mod_[0];
  return GLV_OK;
}

void Engine::free_level(Level &L) {
  if (L.owned) {
    dfree(L.ptr);
    dfree(L.tail);
    dfree(L.w);
  }
  L = Level{};
}

// ------------------------------------------------------------ multiphase
int Engine::run_multiphase(const Level &L0, int32_t *d_C_orig, bool coloring,
                           long min_graph_size, double threshold, double c_threshold,
                           glv_run_stats *st) {
  Level L = L0;
  L.owned = false;
  int ncolors = 0;
  bool recolored = false;
  double tcol = 0;
  if (coloring) {
    TRY(color(L, &ncolors, &tcol, true));
    t_color += tcol;
    recolored = true;
  }
  double prev = -1, curr = -1;
  long phase = 1;
  bool non_color = !coloring;
  int tot_itr = 0;
  int64_t ncl = 0;
  int nrec = 0;
  const long itr_cap = coloring ? 10000 : 100000;
  while (true) {
    prev = curr;
    int itr = 0;
    const bool used_color = !non_color;
    const double ts0 = t_sweep, es0 = edges_swept;
    phase_index_ = (int)phase - 1;
    if (!non_color) {
      // a multi-hash colouring leaves an improper class: sublevels as for stale ones
      TRY(coloring_phase(L, ncolors, !recolored || color_algo_ == 3, curr, c_threshold, &curr,
                         &itr));
    } else {
      TRY(basic_phase(L, curr, threshold, &curr, &itr));
    }
    tot_itr += itr;
    const double tc0 = now_s();
    TRY(renumber(C, L.nv, &ncl));
    LAUNCH(k_compose, grid_for(L0.nv, 256, nsm_ * 16), 256, 0, s_, L0.nv, d_C_orig, C,
           phase == 1 ? 1 : 0);
    CK(cudaStreamSynchronize(s_));
    double tcoarse = now_s() - tc0;
    const glv_phase_stats rec0{L.nv, L.nnz, used_color ? 1 : 0,
                               used_color ? (recolored ? 1 : 0) : 0, used_color ? ncolors : 0,
                               itr, curr, (long)ncl, t_sweep - ts0, 0.0, 0.0,
                               edges_swept - es0};
    glv_phase_stats rec = rec0;
    if (used_color && nrec == 0) rec.time_color = tcol;
    bool stop = (phase > 200) || (tot_itr > itr_cap);
    if (!stop) {
      if ((curr - prev) > threshold) {
        const double tb0 = now_s();
        Level nl;
        int64_t ne = 0;
        TRY(coarsen(L, C, ncl, &nl, &ne));
        free_level(L);
        L = nl;
        tcoarse += now_s() - tb0;
        ++phase;
        recolored = false;
        if (coloring && L.nv > min_graph_size && !non_color) {
          TRY(color(L, &ncolors, &tcol, true));
          t_color += tcol;
          recolored = true;
        }
      } else {
        if (coloring && !non_color) non_color = true;
        else stop = true;
      }
    }
    t_coarsen += tcoarse;
    rec.time_coarsen = tcoarse;
    if (st && nrec < GLV_MAX_PHASES) st->phase[nrec] = rec;
    ++nrec;
    if (stop) break;
  }
  free_level(L);
  if (st) {
    st->phases = (int)phase;
    st->total_iterations = tot_itr;
    st->final_clusters = (long)ncl;
    st->final_modularity = prev;
    st->nphase = std::min(nrec, GLV_MAX_PHASES);
    st->time_clustering = t_sweep;
    st->time_coloring = t_color;
    st->time_building = t_coarsen;
    st->edges_swept = edges_swept;
    st->sweep_kernel_time = sweep_kernel_s;
    st->sweep_bytes = sweep_bytes;
    st->sweep_steps = sweep_steps;
    for (int k = 0; k < kSlots; ++k) st->kernel_time[k] = slot_s[k];
    st->tuned_block_max = tune_choice_[0];
    st->tuned_hub_chunk = tune_choice_[1];
    st->tuned_from_cache = tune_cached_ ? 1 : 0;
    st->hub_cluster = first_cluster_ < 0 ? 0 : first_cluster_;
  }
  return GLV_OK;
}

#include "batch.cuh"

}  // namespace glv

// =========================================================================
// C ABI (include/grappolo_b200.h)
// =========================================================================
namespace glv {

__global__ void k_split_aos(int64_t n, const glv_edge *aos, int32_t *tail, double *w) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    tail[i] = (int32_t)aos[i].tail;
    w[i] = aos[i].weight;
  }
}

__global__ void k_narrow(int64_t n, const int64_t *in, int32_t *out, int32_t *bad, int64_t hi) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t x = in[i];
    if (x < -1 || x >= hi) atomicOr(bad, 1);
    out[i] = (int32_t)x;
  }
}

__global__ void k_widen(int64_t n, const int32_t *in, int64_t *out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}

__global__ void k_fill_aos(int64_t nv, const int64_t *ptr, const int32_t *tail, const double *w,
                           glv_edge *aos) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x)
    for (int64_t j = ptr[v]; j < ptr[v + 1]; ++j) aos[j] = glv_edge{(long)v, (long)tail[j], w[j]};
}

// A call's device context: stream, engine and the uploaded level-0 graph.
struct Call {
  cudaStream_t s = nullptr;
  Engine *eng = nullptr;
  Level L0;
  long launches = 0;
  double t_transfer = 0;
  ~Call() {
    if (getenv("GRAPPOLO_B200_DEBUG")) {
      cudaMemPool_t p = engine_pool();
      uint64_t rc = 0, rh = 0, uc = 0, uh = 0;
      if (p) {
        cudaMemPoolGetAttribute(p, cudaMemPoolAttrReservedMemCurrent, &rc);
        cudaMemPoolGetAttribute(p, cudaMemPoolAttrReservedMemHigh, &rh);
        cudaMemPoolGetAttribute(p, cudaMemPoolAttrUsedMemCurrent, &uc);
        cudaMemPoolGetAttribute(p, cudaMemPoolAttrUsedMemHigh, &uh);
      }
      fprintf(stderr, "grappolo_b200: pool reserved %.3f GB (high %.3f) used %.3f GB (high %.3f)\n",
              rc * 1e-9, rh * 1e-9, uc * 1e-9, uh * 1e-9);
    }
    if (eng) {
      eng->free_level(L0);
      launches += eng->launches_;
      g_launches += eng->launches_;
      delete eng;
      if (s) end_call_block_cache(current_device(), s);
    }
    if (s) cudaStreamSynchronize(s);  // the stream is the device's, kept for the next call
  }
};

// The dynamic shared-memory limits of the kernels that take more than 48 KB
// are a per-device setting: they are raised once for each device, with that
// device current, the first time an entry point runs on it.
static int set_kernel_attributes() {
  const struct { const void *fn; int bytes; } want[] = {
      {(const void *)k_sweep_block, kBlockCap * (int)(sizeof(double) + sizeof(int32_t))},
      {(const void *)k_sweep_iteration<false>, (int)kPersistSmem},
      {(const void *)k_sweep_iteration<true>, (int)kPersistSmem},
      {(const void *)k_hub_accum, kHubStageSmem},
      {(const void *)k_chunk_records, (int)sizeof(PermTileSmem)},
      {(const void *)k_hc_tiles, (int)sizeof(HashTileSmem)},
      {(const void *)k_row_sums_tiles, (int)sizeof(RowSumSmem)},
  };
  for (const auto &k : want) {
    const cudaError_t e =
        cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, k.bytes);
    if (e != cudaSuccess)
      return fail(GLV_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  }
  // clusters of 16 blocks are beyond the portable size of 8
  const cudaError_t e = cudaFuncSetAttribute((const void *)k_sweep_iteration<true>,
                                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess)
    return fail(GLV_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(e));
  return GLV_OK;
}

static int device_ready() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return fail(GLV_ERR_NO_DEVICE, "no CUDA device");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(GLV_ERR_ARG, "device ordinal out of range");
  static std::mutex mu;
  static bool attrs[kMaxDevices] = {};
  std::lock_guard<std::mutex> lock(mu);
  if (!attrs[dev]) {
    TRY(set_kernel_attributes());
    attrs[dev] = true;
  }
  return GLV_OK;
}

static int check_ptr(long nv, const long *ptr) {
  if (nv < 0) return fail(GLV_ERR_ARG, "numVertices < 0");
  if (nv >= (1L << 31) - 1) return fail(GLV_ERR_TOO_LARGE, "numVertices >= 2^31");
  if (!ptr) return fail(GLV_ERR_ARG, "edgeListPtrs is NULL");
  if (ptr[0] != 0) return fail(GLV_ERR_ARG, "edgeListPtrs[0] != 0");
  for (long i = 0; i < nv; ++i)
    if (ptr[i + 1] < ptr[i]) return fail(GLV_ERR_ARG, "edgeListPtrs not non-decreasing");
  return GLV_OK;
}

// Uploads a host CSR (either AoS `edges` or SoA `tail64`/`w`) as level 0.
static int open_call(Call &c, int mode, long nv, const long *ptr, const glv_edge *edges,
                     const long *tail64, const double *w) {
  TRY(device_ready());
  TRY(check_ptr(nv, ptr));
  if (mode < GLV_MODE_VERIFY || mode > GLV_MODE_LEARNED) return fail(GLV_ERR_ARG, "bad mode");
  const int64_t nnz = ptr[nv];
  if (nnz > 0 && !edges && !(tail64 && w)) return fail(GLV_ERR_ARG, "edge arrays are NULL");
  CK(engine_stream(&c.s));
  c.eng = new Engine(c.s, mode);
  TRY(c.eng->init(nv, nnz));
  const double t0 = now_s();
  Level &L = c.L0;
  L.nv = nv;
  L.nnz = nnz;
  L.owned = true;
  // through the engine's allocator: its block cache serves repeated calls
  TRY(c.eng->alloc(&L.ptr, nv + 1));
  TRY(c.eng->alloc(&L.tail, std::max<int64_t>(nnz, 1)));
  TRY(c.eng->alloc(&L.w, std::max<int64_t>(nnz, 1)));
  CK(cudaMemcpyAsync(L.ptr, ptr, (nv + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, c.s));
  // Edges move in chunks through one device staging buffer.
  const int64_t chunk = std::min<int64_t>(std::max<int64_t>(nnz, 1), 1 << 24);
  int nsm = 148;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
  if (edges) {
    glv_edge *stage;
    TRY(c.eng->alloc(&stage, chunk));
    for (int64_t b = 0; b < nnz; b += chunk) {
      const int64_t n = std::min(chunk, nnz - b);
      CK(cudaMemcpyAsync(stage, edges + b, n * sizeof(glv_edge), cudaMemcpyHostToDevice, c.s));
      k_split_aos<<<grid_for(n, 256, nsm * 8), 256, 0, c.s>>>(n, stage, L.tail + b, L.w + b);
      ++c.launches;
      CK(cudaGetLastError());
    }
    c.eng->dfree(stage);
  } else if (nnz > 0) {
    int64_t *stage;
    int32_t *bad;
    TRY(c.eng->alloc(&stage, chunk));
    TRY(c.eng->alloc(&bad, 1));
    CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), c.s));
    for (int64_t b = 0; b < nnz; b += chunk) {
      const int64_t n = std::min(chunk, nnz - b);
      CK(cudaMemcpyAsync(stage, tail64 + b, n * sizeof(int64_t), cudaMemcpyHostToDevice, c.s));
      k_narrow<<<grid_for(n, 256, nsm * 8), 256, 0, c.s>>>(n, stage, L.tail + b, bad, nv);
      ++c.launches;
      CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(L.w, w, nnz * sizeof(double), cudaMemcpyHostToDevice, c.s));
    c.eng->dfree(stage);
    c.eng->dfree(bad);
  }
  CK(cudaStreamSynchronize(c.s));
  c.t_transfer += now_s() - t0;
  return c.eng->upload_check(L);
}

// int32 device ids -> caller's int64 host array.
static int download_ids(Call &c, const int32_t *d, int64_t n, long *host) {
  if (n == 0) return GLV_OK;
  const double t0 = now_s();
  int64_t *tmp;
  CK(cudaMallocFromPoolAsync((void **)&tmp, n * sizeof(int64_t), engine_pool(), c.s));
  k_widen<<<grid_for(n, 256, 148 * 8), 256, 0, c.s>>>(n, d, tmp);
  ++c.launches;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, tmp, n * sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
  CK(cudaFreeAsync(tmp, c.s));
  CK(cudaStreamSynchronize(c.s));
  c.t_transfer += now_s() - t0;
  return GLV_OK;
}

static int upload_ids(Call &c, const long *host, int64_t n, int32_t *d, int64_t hi) {
  if (n == 0) return GLV_OK;
  int64_t *tmp;
  int32_t *bad;
  CK(cudaMallocFromPoolAsync((void **)&tmp, n * sizeof(int64_t), engine_pool(), c.s));
  CK(cudaMallocFromPoolAsync((void **)&bad, sizeof(int32_t), engine_pool(), c.s));
  CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), c.s));
  CK(cudaMemcpyAsync(tmp, host, n * sizeof(int64_t), cudaMemcpyHostToDevice, c.s));
  k_narrow<<<grid_for(n, 256, 148 * 8), 256, 0, c.s>>>(n, tmp, d, bad, hi);
  ++c.launches;
  CK(cudaGetLastError());
  int32_t hb = 0;
  CK(cudaMemcpyAsync(&hb, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, c.s));
  CK(cudaFreeAsync(tmp, c.s));
  CK(cudaFreeAsync(bad, c.s));
  CK(cudaStreamSynchronize(c.s));
  if (hb) return fail(GLV_ERR_ARG, "id out of range");
  return GLV_OK;
}

static int run_host(int mode, long nv, const long *ptr, const glv_edge *edges, const long *tail64,
                    const double *w, long *C_orig, bool coloring, long min_graph_size,
                    double threshold, double c_threshold, glv_run_stats *st,
                    int color_algo = 1, int num_colors = 16) {
  const double t0 = now_s();
  if (!C_orig && nv > 0) return fail(GLV_ERR_ARG, "C_orig is NULL");
  if (st) memset(st, 0, sizeof(*st));
  Call c;
  TRY(open_call(c, mode, nv, ptr, edges, tail64, w));
  c.eng->color_algo_ = color_algo;
  // runMultiPhaseColoring's parameters (Coloring/runMultiPhaseColoring.cpp:77-86)
  c.eng->mhash_nhash_ = 2;
  c.eng->mhash_itrs_ = std::max(1, num_colors / 4);
  int32_t *dC;
  CK(cudaMallocFromPoolAsync((void **)&dC, std::max<long>(nv, 1) * sizeof(int32_t), engine_pool(), c.s));
  TRY(c.eng->run_multiphase(c.L0, dC, coloring, min_graph_size, threshold, c_threshold, st));
  TRY(download_ids(c, dC, nv, C_orig));
  CK(cudaFreeAsync(dC, c.s));
  if (st) {
    st->time_transfer = c.t_transfer;
    st->kernel_launches = c.launches + c.eng->launches_;
    st->time_total = now_s() - t0;
  }
  return GLV_OK;
}

}  // namespace glv

using namespace glv;

extern "C" {

const char *glv_version(void) { return "grappolo_b200 0.1 (sm_100a)"; }
const char *glv_last_error(void) { return g_err.c_str(); }
long glv_kernel_launch_count(void) { return g_launches.load(); }
void glv_release_cached_memory(void) {
  int cur = 0;
  cudaGetDevice(&cur);
  for (int d = 0; d < 128; ++d) {
    if (!g_stream[d]) continue;
    cudaSetDevice(d);
    flush_block_cache(d, g_stream[d]);
    cudaStreamSynchronize(g_stream[d]);
  }
  cudaSetDevice(cur);
  std::lock_guard<std::mutex> lock(g_pool_mu);
  for (auto &p : g_pool)
    if (p) cudaMemPoolTrimTo(p, 0);
}
void glv_set_profiling(int on) { g_profile = on < 0 ? 0 : (on > 2 ? 2 : on); }

int glv_run_multiphase_coloring(const glv_graph *G, long *C_orig, int coloring, int numColors,
                                int replaceMap, long minGraphSize, double threshold,
                                double C_threshold, int mode, glv_run_stats *stats) {
  if (!G) return fail(GLV_ERR_ARG, "G is NULL");
  if (coloring < 1 || coloring > 3) return fail(GLV_ERR_ARG, "coloring must be 1, 2 or 3");
  if (coloring == 3 && 4L * std::max(1, numColors / 4) + 1 >= kMaxColors)
    return fail(GLV_ERR_COLORS, "numColors reaches the colour cap");
  if (replaceMap != 0) return fail(GLV_ERR_UNSUPPORTED, "replaceMap = 1 is not implemented");
  return run_host(mode, G->numVertices, G->edgeListPtrs, G->edgeList, nullptr, nullptr, C_orig,
                  true, minGraphSize, threshold, C_threshold, stats, coloring, numColors);
}

int glv_run_multiphase_basic(const glv_graph *G, long *C_orig, int basicOpt, long minGraphSize,
                             double threshold, double C_threshold, int mode,
                             glv_run_stats *stats) {
  if (!G) return fail(GLV_ERR_ARG, "G is NULL");
  if (basicOpt != 0) return fail(GLV_ERR_UNSUPPORTED, "basicOpt = 1 is not implemented");
  return run_host(mode, G->numVertices, G->edgeListPtrs, G->edgeList, nullptr, nullptr, C_orig,
                  false, minGraphSize, threshold, C_threshold, stats);
}

int glv_run_multiphase_coloring_csr(long nv, const long *ptr, const long *tail,
                                    const double *weight, long *C_orig, long minGraphSize,
                                    double threshold, double C_threshold, int mode,
                                    glv_run_stats *stats) {
  return run_host(mode, nv, ptr, nullptr, tail, weight, C_orig, true, minGraphSize, threshold,
                  C_threshold, stats);
}

int glv_run_multiphase_basic_csr(long nv, const long *ptr, const long *tail, const double *weight,
                                 long *C_orig, double threshold, int mode, glv_run_stats *stats) {
  return run_host(mode, nv, ptr, nullptr, tail, weight, C_orig, false, 0, threshold, 0.0, stats);
}

int glv_dev_run_multiphase(long nv, const long *d_ptr, const int *d_tail, const double *d_weight,
                           int *d_C_orig, int coloring, long minGraphSize, double threshold,
                           double C_threshold, int mode, void *stream, glv_run_stats *stats) {
  const double t0 = now_s();
  TRY(device_ready());
  if (nv < 0) return fail(GLV_ERR_ARG, "nv < 0");
  if (nv >= (1L << 31) - 1) return fail(GLV_ERR_TOO_LARGE, "nv >= 2^31");
  if (mode < GLV_MODE_VERIFY || mode > GLV_MODE_LEARNED) return fail(GLV_ERR_ARG, "bad mode");
  if (stats) memset(stats, 0, sizeof(*stats));
  Call c;
  CK(engine_stream(&c.s));
  if (stream) {
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, (cudaStream_t)stream));
    CK(cudaStreamWaitEvent(c.s, ev, 0));
    cudaEventDestroy(ev);
  } else {
    CK(cudaStreamSynchronize(0));
  }
  int64_t nnz = 0;
  if (nv > 0) {
    CK(cudaMemcpyAsync(&nnz, d_ptr + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
  }
  c.eng = new Engine(c.s, mode);
  TRY(c.eng->init(nv, nnz));
  c.L0.nv = nv;
  c.L0.nnz = nnz;
  c.L0.ptr = (int64_t *)d_ptr;
  c.L0.tail = (int32_t *)d_tail;
  c.L0.w = (double *)d_weight;
  c.L0.owned = false;
  TRY(c.eng->upload_check(c.L0));
  TRY(c.eng->run_multiphase(c.L0, d_C_orig, coloring != 0, minGraphSize, threshold, C_threshold,
                            stats));
  CK(cudaStreamSynchronize(c.s));
  if (stats) {
    stats->kernel_launches = c.launches + c.eng->launches_;
    stats->time_total = now_s() - t0;
  }
  return GLV_OK;
}

// Batches: graph g owns vertices [vertex_offsets[g], vertex_offsets[g+1]) of
// one CSR whose tails are global vertex ids inside the row's own graph.
static int check_offsets(int G, const long *voff, long nv) {
  if (G < 1) return fail(GLV_ERR_ARG, "num_graphs < 1");
  if (!voff) return fail(GLV_ERR_ARG, "vertex_offsets is NULL");
  if (voff[0] != 0 || voff[G] != nv) return fail(GLV_ERR_ARG, "vertex_offsets must span [0, nv]");
  for (int g = 0; g < G; ++g)
    if (voff[g + 1] <= voff[g]) return fail(GLV_ERR_ARG, "every graph needs a vertex");
  return GLV_OK;
}

static int run_batch(Call &c, int G, const long *voff, int32_t *dC, bool coloring,
                     long min_graph_size, double threshold, double C_threshold,
                     glv_batch_stats *st) {
  const int64_t nv = c.L0.nv;
  std::vector<int64_t> off(voff, voff + G + 1);
  // every tail inside its row's graph
  int32_t *gid, *bad;
  int64_t *d_off;
  CK(cudaMallocFromPoolAsync((void **)&gid, nv * sizeof(int32_t), engine_pool(), c.s));
  CK(cudaMallocFromPoolAsync((void **)&bad, sizeof(int32_t), engine_pool(), c.s));
  CK(cudaMallocFromPoolAsync((void **)&d_off, (G + 1) * sizeof(int64_t), engine_pool(), c.s));
  CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), c.s));
  CK(cudaMemcpyAsync(d_off, off.data(), (G + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, c.s));
  k_fill_gid<<<std::max(1, std::min(G, 148 * 16)), 256, 0, c.s>>>(G, d_off, gid);
  k_check_batch_tails<<<grid_for(nv, 256, 148 * 16), 256, 0, c.s>>>(nv, c.L0.ptr, c.L0.tail, gid,
                                                                      d_off, bad);
  c.launches += 2;
  CK(cudaGetLastError());
  int32_t hb = 0;
  CK(cudaMemcpyAsync(&hb, bad, sizeof(int32_t), cudaMemcpyDeviceToHost, c.s));
  CK(cudaFreeAsync(gid, c.s));
  CK(cudaFreeAsync(bad, c.s));
  CK(cudaFreeAsync(d_off, c.s));
  CK(cudaStreamSynchronize(c.s));
  if (hb) return fail(GLV_ERR_ARG, "an edge joins two graphs of the batch");
  std::vector<double> fm(G), ds(G);
  std::vector<int> ph(G), it(G);
  std::vector<long> cl(G);
  BatchResult r{fm.data(), ph.data(), it.data(), cl.data(), ds.data(), 0};
  TRY(c.eng->run_multiphase_batch(c.L0, off, dC, coloring, min_graph_size, threshold,
                                  C_threshold, &r));
  if (st) {
    for (int g = 0; g < G; ++g) {
      if (st->final_modularity) st->final_modularity[g] = fm[g];
      if (st->phases) st->phases[g] = ph[g];
      if (st->iterations) st->iterations[g] = it[g];
      if (st->clusters) st->clusters[g] = cl[g];
      if (st->done_seconds) st->done_seconds[g] = ds[g];
    }
    st->rounds = r.rounds;
    st->time_clustering = c.eng->t_sweep;
    st->time_coloring = c.eng->t_color;
    st->time_building = c.eng->t_coarsen;
    st->edges_swept = c.eng->edges_swept;
  }
  return GLV_OK;
}

static void clear_batch_stats(glv_batch_stats *st) {
  if (!st) return;
  st->rounds = 0;
  st->time_total = st->time_clustering = st->time_coloring = st->time_building = 0;
  st->time_transfer = st->edges_swept = 0;
  st->kernel_launches = 0;
}

int glv_run_batch_csr(int num_graphs, const long *vertex_offsets, const long *ptr,
                      const long *tail, const double *weight, long *C_out, int coloring,
                      long minGraphSize, double threshold, double C_threshold, int mode,
                      glv_batch_stats *stats) {
  const double t0 = now_s();
  clear_batch_stats(stats);
  if (!vertex_offsets || num_graphs < 1) return fail(GLV_ERR_ARG, "no graphs");
  const long nv = vertex_offsets[num_graphs];
  TRY(check_offsets(num_graphs, vertex_offsets, nv));
  if (!C_out) return fail(GLV_ERR_ARG, "C_out is NULL");
  if (mode < GLV_MODE_VERIFY || mode > GLV_MODE_FAST) return fail(GLV_ERR_ARG, "bad mode");
  Call c;
  TRY(open_call(c, mode, nv, ptr, nullptr, tail, weight));
  int32_t *dC;
  CK(cudaMallocFromPoolAsync((void **)&dC, nv * sizeof(int32_t), engine_pool(), c.s));
  TRY(run_batch(c, num_graphs, vertex_offsets, dC, coloring != 0, minGraphSize, threshold,
                C_threshold, stats));
  TRY(download_ids(c, dC, nv, C_out));
  CK(cudaFreeAsync(dC, c.s));
  if (stats) {
    stats->time_transfer = c.t_transfer;
    stats->kernel_launches = c.launches + c.eng->launches_;
    stats->time_total = now_s() - t0;
  }
  return GLV_OK;
}

int glv_dev_run_batch(int num_graphs, const long *vertex_offsets, const long *d_ptr,
                      const int *d_tail, const double *d_weight, int *d_C, int coloring,
                      long minGraphSize, double threshold, double C_threshold, int mode,
                      void *stream, glv_batch_stats *stats) {
  const double t0 = now_s();
  clear_batch_stats(stats);
  TRY(device_ready());
  if (!vertex_offsets || num_graphs < 1) return fail(GLV_ERR_ARG, "no graphs");
  const long nv = vertex_offsets[num_graphs];
  TRY(check_offsets(num_graphs, vertex_offsets, nv));
  if (nv >= (1L << 31) - 1) return fail(GLV_ERR_TOO_LARGE, "nv >= 2^31");
  if (mode < GLV_MODE_VERIFY || mode > GLV_MODE_FAST) return fail(GLV_ERR_ARG, "bad mode");
  Call c;
  CK(engine_stream(&c.s));
  if (stream) {
    cudaEvent_t ev;
    CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventRecord(ev, (cudaStream_t)stream));
    CK(cudaStreamWaitEvent(c.s, ev, 0));
    cudaEventDestroy(ev);
  } else {
    CK(cudaStreamSynchronize(0));
  }
  int64_t nnz = 0;
  CK(cudaMemcpyAsync(&nnz, d_ptr + nv, sizeof(int64_t), cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  c.eng = new Engine(c.s, mode);
  TRY(c.eng->init(nv, nnz));
  c.L0.nv = nv;
  c.L0.nnz = nnz;
  c.L0.ptr = (int64_t *)d_ptr;
  c.L0.tail = (int32_t *)d_tail;
  c.L0.w = (double *)d_weight;
  c.L0.owned = false;
  TRY(c.eng->upload_check(c.L0));
  TRY(run_batch(c, num_graphs, vertex_offsets, d_C, coloring != 0, minGraphSize, threshold,
                C_threshold, stats));
  CK(cudaStreamSynchronize(c.s));
  if (stats) {
    stats->kernel_launches = c.launches + c.eng->launches_;
    stats->time_total = now_s() - t0;
  }
  return GLV_OK;
}

int glv_louvain_coloring_phase(const glv_graph *G, long *C, const int *color, int numColor,
                               double Lower, double thresh, int mode, double *mod, int *numItr,
                               double *totTime) {
  const double t0 = now_s();
  if (!G || !C || (!color && G->numVertices > 0)) return fail(GLV_ERR_ARG, "NULL argument");
  if (numColor < 1 || numColor > kMaxColors) return fail(GLV_ERR_ARG, "numColor out of range");
  Call c;
  TRY(open_call(c, mode, G->numVertices, G->edgeListPtrs, G->edgeList, nullptr, nullptr));
  const long nv = G->numVertices;
  for (long i = 0; i < nv; ++i)
    if (color[i] < 0 || color[i] >= numColor) return fail(GLV_ERR_ARG, "colour out of range");
  CK(cudaMemcpyAsync(c.eng->color_, color, nv * sizeof(int32_t), cudaMemcpyHostToDevice, c.s));
  CK(cudaStreamSynchronize(c.s));
  double q = 0;
  int itr = 0;
  TRY(c.eng->coloring_phase(c.L0, numColor, true, Lower, thresh, &q, &itr));
  TRY(download_ids(c, c.eng->C, nv, C));
  if (mod) *mod = q;
  if (numItr) *numItr = itr;
  if (totTime) *totTime = now_s() - t0;
  return GLV_OK;
}

int glv_louvain_basic_phase(const glv_graph *G, long *C, double Lower, double thresh, int mode,
                            double *mod, int *numItr, double *totTime) {
  const double t0 = now_s();
  if (!G || !C) return fail(GLV_ERR_ARG, "NULL argument");
  Call c;
  TRY(open_call(c, mode, G->numVertices, G->edgeListPtrs, G->edgeList, nullptr, nullptr));
  double q = 0;
  int itr = 0;
  TRY(c.eng->basic_phase(c.L0, Lower, thresh, &q, &itr));
  TRY(download_ids(c, c.eng->C, G->numVertices, C));
  if (mod) *mod = q;
  if (numItr) *numItr = itr;
  if (totTime) *totTime = now_s() - t0;
  return GLV_OK;
}

int glv_distance_one_coloring(const glv_graph *G, int *vtxColor, int mode, int *maxColor,
                              double *totTime) {
  if (!G || (!vtxColor && G->numVertices > 0)) return fail(GLV_ERR_ARG, "NULL argument");
  Call c;
  TRY(open_call(c, mode, G->numVertices, G->edgeListPtrs, G->edgeList, nullptr, nullptr));
  int nc = 0;
  double secs = 0;
  if (G->numVertices > 0) TRY(c.eng->color(c.L0, &nc, &secs));
  CK(cudaMemcpyAsync(vtxColor, c.eng->color_, G->numVertices * sizeof(int32_t),
                     cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  if (maxColor) *maxColor = nc - 1;
  if (totTime) *totTime = secs;
  return GLV_OK;
}

int glv_color_multihash(const glv_graph *G, int *vtxColor, int nHash, int nItrs,
                        int *maxColor, double *totTime) {
  if (!G || (!vtxColor && G->numVertices > 0)) return fail(GLV_ERR_ARG, "NULL argument");
  if (nHash < 1 || nItrs < 1) return fail(GLV_ERR_ARG, "nHash and nItrs must be positive");
  if ((long)2 * nHash * nItrs + 1 >= kMaxColors)
    return fail(GLV_ERR_COLORS, "2 * nHash * nItrs reaches the colour cap");
  Call c;
  TRY(open_call(c, GLV_MODE_VERIFY, G->numVertices, G->edgeListPtrs, G->edgeList, nullptr,
                nullptr));
  c.eng->color_algo_ = 3;
  c.eng->mhash_nhash_ = nHash;
  c.eng->mhash_itrs_ = nItrs;
  int nc = 0;
  double secs = 0;
  TRY(c.eng->color(c.L0, &nc, &secs));
  CK(cudaMemcpyAsync(vtxColor, c.eng->color_, G->numVertices * sizeof(int32_t),
                     cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  if (maxColor) *maxColor = nc - 1;
  if (totTime) *totTime = secs;
  return GLV_OK;
}

int glv_vbase_redistribution(const glv_graph *G, int *vtxColor, int ncolors, int type,
                             long *moves) {
  if (!G || (!vtxColor && G->numVertices > 0)) return fail(GLV_ERR_ARG, "NULL argument");
  if (type != 0 && type != 1) return fail(GLV_ERR_ARG, "type must be 0 or 1");
  if (ncolors <= 0 && G->numVertices > 0) return fail(GLV_ERR_ARG, "ncolors must be positive");
  if (ncolors > kMaxColors) return fail(GLV_ERR_COLORS, "more colours than the 4096 cap");
  for (long v = 0; v < G->numVertices; ++v)
    if (vtxColor[v] < 0 || vtxColor[v] >= ncolors)
      return fail(GLV_ERR_ARG, "a colour outside [0, ncolors)");
  Call c;
  TRY(open_call(c, GLV_MODE_VERIFY, G->numVertices, G->edgeListPtrs, G->edgeList, nullptr,
                nullptr));
  const long nv = G->numVertices;
  if (nv > 0) {
    CK(cudaMemcpyAsync(c.eng->color_, vtxColor, nv * sizeof(int32_t), cudaMemcpyHostToDevice,
                       c.s));
    TRY(c.eng->vbase(c.L0, ncolors, type, moves));
    CK(cudaMemcpyAsync(vtxColor, c.eng->color_, nv * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       c.s));
    CK(cudaStreamSynchronize(c.s));
  } else if (moves) {
    *moves = 0;
  }
  return GLV_OK;
}

int glv_renumber_clusters(long *C, long size, long *numClusters) {
  if (size < 0 || (!C && size > 0)) return fail(GLV_ERR_ARG, "bad arguments");
  if (size >= (1L << 31) - 1) return fail(GLV_ERR_TOO_LARGE, "size >= 2^31");
  TRY(device_ready());
  Call c;
  CK(engine_stream(&c.s));
  c.eng = new Engine(c.s, GLV_MODE_VERIFY);
  TRY(c.eng->init(size, 0));
  TRY(upload_ids(c, C, size, c.eng->C, size));
  int64_t ncl = 0;
  TRY(c.eng->renumber(c.eng->C, size, &ncl));
  TRY(download_ids(c, c.eng->C, size, C));
  if (numClusters) *numClusters = (long)ncl;
  return GLV_OK;
}

int glv_build_next_level(const glv_graph *Gin, glv_graph *Gout, const long *C,
                         long numUniqueClusters, int mode, double *totTime) {
  const double t0 = now_s();
  if (!Gin || !Gout || (!C && Gin->numVertices > 0)) return fail(GLV_ERR_ARG, "NULL argument");
  if (numUniqueClusters < 1 || numUniqueClusters > Gin->numVertices)
    return fail(GLV_ERR_ARG, "numUniqueClusters out of range");
  Call c;
  TRY(open_call(c, mode, Gin->numVertices, Gin->edgeListPtrs, Gin->edgeList, nullptr, nullptr));
  TRY(upload_ids(c, C, Gin->numVertices, c.eng->C, numUniqueClusters));
  Level out;
  int64_t ne = 0;
  TRY(c.eng->coarsen(c.L0, c.eng->C, numUniqueClusters, &out, &ne));
  long *hp = (long *)malloc((numUniqueClusters + 1) * sizeof(long));
  glv_edge *he = (glv_edge *)malloc(std::max<int64_t>(out.nnz, 1) * sizeof(glv_edge));
  if (!hp || !he) {
    free(hp); free(he);
    c.eng->free_level(out);
    return fail(GLV_ERR_OOM, "host allocation failed");
  }
  glv_edge *daos;
  CK(cudaMallocFromPoolAsync((void **)&daos, std::max<int64_t>(out.nnz, 1) * sizeof(glv_edge), engine_pool(), c.s));
  k_fill_aos<<<grid_for(out.nv, 256, 148 * 8), 256, 0, c.s>>>(out.nv, out.ptr, out.tail, out.w,
                                                              daos);
  ++c.launches;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(hp, out.ptr, (numUniqueClusters + 1) * sizeof(long), cudaMemcpyDeviceToHost,
                     c.s));
  CK(cudaMemcpyAsync(he, daos, out.nnz * sizeof(glv_edge), cudaMemcpyDeviceToHost, c.s));
  CK(cudaFreeAsync(daos, c.s));
  CK(cudaStreamSynchronize(c.s));
  c.eng->free_level(out);
  Gout->numVertices = numUniqueClusters;
  Gout->sVertices = numUniqueClusters;
  Gout->numEdges = ne;
  Gout->edgeListPtrs = hp;
  Gout->edgeList = he;
  if (totTime) *totTime = now_s() - t0;
  return GLV_OK;
}

int glv_vertex_following(const glv_graph *G, long *C, long *numVtxToFix) {
  if (!G || (!C && G->numVertices > 0)) return fail(GLV_ERR_ARG, "NULL argument");
  Call c;
  TRY(open_call(c, GLV_MODE_VERIFY, G->numVertices, G->edgeListPtrs, G->edgeList, nullptr,
                nullptr));
  unsigned long long *num;
  CK(cudaMallocFromPoolAsync((void **)&num, sizeof(*num), engine_pool(), c.s));
  CK(cudaMemsetAsync(num, 0, sizeof(*num), c.s));
  if (c.L0.nv > 0) {
    k_vertex_following<<<grid_for(c.L0.nv, 256, 148 * 16), 256, 0, c.s>>>(
        c.L0.nv, c.L0.ptr, c.L0.tail, c.eng->C, num);
    ++c.launches;
    CK(cudaGetLastError());
  }
  unsigned long long h = 0;
  CK(cudaMemcpyAsync(&h, num, sizeof(h), cudaMemcpyDeviceToHost, c.s));
  CK(cudaFreeAsync(num, c.s));
  TRY(download_ids(c, c.eng->C, c.L0.nv, C));
  if (numVtxToFix) *numVtxToFix = (long)h;
  return GLV_OK;
}

int glv_build_new_graph_vf(const glv_graph *Gin, glv_graph *Gout, const long *C,
                           long numUniqueClusters, double *totTime) {
  const double t0 = now_s();
  if (!Gin || !Gout || (!C && Gin->numVertices > 0)) return fail(GLV_ERR_ARG, "NULL argument");
  if (numUniqueClusters < 1 || numUniqueClusters > Gin->numVertices)
    return fail(GLV_ERR_ARG, "numUniqueClusters out of range");
  Call c;
  TRY(open_call(c, GLV_MODE_VERIFY, Gin->numVertices, Gin->edgeListPtrs, Gin->edgeList, nullptr,
                nullptr));
  TRY(upload_ids(c, C, Gin->numVertices, c.eng->C, numUniqueClusters));
  Level out;
  int64_t ne = 0;
  TRY(c.eng->coarsen_chunked(c.L0, c.eng->C, numUniqueClusters, &out, &ne, int64_t(1) << 27,
                             true));
  long *hp = (long *)malloc((numUniqueClusters + 1) * sizeof(long));
  glv_edge *he = (glv_edge *)malloc(std::max<int64_t>(out.nnz, 1) * sizeof(glv_edge));
  if (!hp || !he) {
    free(hp); free(he);
    c.eng->free_level(out);
    return fail(GLV_ERR_OOM, "host allocation failed");
  }
  glv_edge *daos;
  CK(cudaMallocFromPoolAsync((void **)&daos, std::max<int64_t>(out.nnz, 1) * sizeof(glv_edge),
                             engine_pool(), c.s));
  k_fill_aos<<<grid_for(out.nv, 256, 148 * 8), 256, 0, c.s>>>(out.nv, out.ptr, out.tail, out.w,
                                                              daos);
  ++c.launches;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(hp, out.ptr, (numUniqueClusters + 1) * sizeof(long), cudaMemcpyDeviceToHost,
                     c.s));
  CK(cudaMemcpyAsync(he, daos, out.nnz * sizeof(glv_edge), cudaMemcpyDeviceToHost, c.s));
  CK(cudaFreeAsync(daos, c.s));
  CK(cudaStreamSynchronize(c.s));
  c.eng->free_level(out);
  Gout->numVertices = numUniqueClusters;
  Gout->sVertices = numUniqueClusters;
  Gout->numEdges = ne;
  Gout->edgeListPtrs = hp;
  Gout->edgeList = he;
  if (totTime) *totTime = now_s() - t0;
  return GLV_OK;
}

int glv_modularity(const glv_graph *G, const long *C, double *mod) {
  if (!G || !mod || (!C && G->numVertices > 0)) return fail(GLV_ERR_ARG, "NULL argument");
  Call c;
  TRY(open_call(c, GLV_MODE_VERIFY, G->numVertices, G->edgeListPtrs, G->edgeList, nullptr,
                nullptr));
  TRY(upload_ids(c, C, G->numVertices, c.eng->Ctgt, G->numVertices));
  return c.eng->modularity_of(c.L0, c.eng->Ctgt, mod);
}

int glv_decide_batch(long nv, const long *ptr, const long *tail, const double *weight,
                     const long *C, const double *vDeg, const double *cDeg, const long *cSize,
                     double constant, long nverts, const long *verts, long *targets) {
  if (nverts < 0 || (nverts > 0 && (!verts || !targets))) return fail(GLV_ERR_ARG, "bad list");
  for (long k = 0; k < nverts; ++k)
    if (verts[k] < 0 || verts[k] >= nv) return fail(GLV_ERR_ARG, "vertex id out of range");
  if (!C || !vDeg || !cDeg || !cSize) return fail(GLV_ERR_ARG, "NULL state array");
  Call c;
  TRY(open_call(c, GLV_MODE_VERIFY, nv, ptr, nullptr, tail, weight));
  Engine &e = *c.eng;
  TRY(upload_ids(c, C, nv, e.C, nv));
  std::vector<int32_t> cs(nv);
  for (long i = 0; i < nv; ++i) cs[i] = (int32_t)cSize[i];
  CK(cudaMemcpyAsync(e.vDeg, vDeg, nv * sizeof(double), cudaMemcpyHostToDevice, c.s));
  CK(cudaMemcpyAsync(e.cDeg, cDeg, nv * sizeof(double), cudaMemcpyHostToDevice, c.s));
  CK(cudaMemcpyAsync(e.cSize, cs.data(), nv * sizeof(int32_t), cudaMemcpyHostToDevice, c.s));
  double cst2[2] = {constant, 0.0};
  CK(cudaMemcpyAsync(e.cst, cst2, sizeof(cst2), cudaMemcpyHostToDevice, c.s));
  int32_t *dv;
  CK(cudaMallocFromPoolAsync((void **)&dv, std::max<long>(nverts, 1) * sizeof(int32_t), engine_pool(), c.s));
  TRY(upload_ids(c, verts, nverts, dv, nv));
  CK(cudaStreamSynchronize(c.s));
  TRY(e.decide(c.L0, dv, nverts));
  std::vector<int32_t> tg(nv);
  CK(cudaMemcpyAsync(tg.data(), e.Ctgt, nv * sizeof(int32_t), cudaMemcpyDeviceToHost, c.s));
  CK(cudaFreeAsync(dv, c.s));
  CK(cudaStreamSynchronize(c.s));
  for (long k = 0; k < nverts; ++k) targets[k] = tg[verts[k]];
  return GLV_OK;
}

}  // extern "C"

// =========================================================================
// Edge lists to CSR, binary graph files
// =========================================================================
#include "csr_build.cuh"
#include "compare.cuh"

// =========================================================================
// Modularity without allocation (glv_dev_modularity_static)
// =========================================================================
#include <mutex>

namespace glv {

// Largest vertex count the static scratch covers: one partial pair per 256
// vertices, 65,536 pairs -> 16,777,216 vertices, 1 MiB of device memory that
// every GPU which loads this library keeps until the process exits.
constexpr int64_t kStaticModParts = 65536;
constexpr int64_t kStaticModMaxVertices = kStaticModParts * kModVB;

// Block partials of e_xx (first half) and a2_x (second half).  Shared by every
// call on a device: concurrent calls on that device race on it.
static __device__ __align__(256) double g_mod_scratch[2 * kStaticModParts];

static std::mutex g_mod_scratch_mu;
static double *g_mod_scratch_addr[kMaxDevices];  // device address of g_mod_scratch, per device

// The fold of k_modularity_final with the constant passed by value, so the
// call needs no device copy of it.
__global__ void __launch_bounds__(256) k_modularity_final_value(int nparts, const double *part_e,
                                                                const double *part_a,
                                                                double constant, double *out) {
  __shared__ double sh[8];
  double e = 0.0, a = 0.0;
  const int per = (nparts + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per, en = min(nparts, b + per);
  for (int i = b; i < en; ++i) { e = __dadd_rn(e, part_e[i]); a = __dadd_rn(a, part_a[i]); }
  e = block_sum<256>(e, sh);
  a = block_sum<256>(a, sh);
  if (threadIdx.x == 0) {
    out[0] = __dsub_rn(__dmul_rn(e, constant), __dmul_rn(__dmul_rn(a, constant), constant));
    out[1] = e;
    out[2] = a;
  }
}

}  // namespace glv

extern "C" int glv_dev_modularity_static(long nv, const long *d_ptr, const int *d_tail,
                                         const double *d_weight, const int *d_C,
                                         const double *d_cDeg, double constant, double *d_out,
                                         void *stream) {
  using namespace glv;
  if (nv < 1) return fail(GLV_ERR_ARG, "glv_dev_modularity_static: numVertices < 1");
  if (nv > kStaticModMaxVertices)
    return fail(GLV_ERR_LIMIT,
                "glv_dev_modularity_static: numVertices exceeds 16,777,216, the size its "
                "static scratch covers; use the allocating entry points");
  if (!d_ptr || !d_tail || !d_weight || !d_C || !d_cDeg || !d_out)
    return fail(GLV_ERR_ARG, "glv_dev_modularity_static: NULL pointer");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(GLV_ERR_NO_DEVICE, "glv_dev_modularity_static: no CUDA device");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(GLV_ERR_ARG, "glv_dev_modularity_static: device id");
  double *scratch = nullptr;
  {
    // First call on a device: look up the array's device address with that
    // device current.  The address is kept for the life of the process; it
    // belongs to the device's primary context, so a caller that resets the
    // device (cudaDeviceReset) must not call this entry again afterwards.
    std::lock_guard<std::mutex> lock(g_mod_scratch_mu);
    if (!g_mod_scratch_addr[dev]) {
      void *p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_mod_scratch);
      if (e != cudaSuccess || !p) {
        g_err = std::string("glv_dev_modularity_static: cudaGetSymbolAddress: ") +
                cudaGetErrorString(e);
        return GLV_ERR_CUDA;
      }
      g_mod_scratch_addr[dev] = static_cast<double *>(p);
    }
    scratch = g_mod_scratch_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int nparts = (int)((nv + kModVB - 1) / kModVB);
  double *part_e = scratch, *part_a = scratch + kStaticModParts;
  // Every partial read below is written first by this call's k_modularity_part,
  // so nothing in the scratch needs clearing.
  k_modularity_part<<<nparts, 256, 0, s>>>(nv, (const int64_t *)d_ptr, d_tail, d_weight, d_C,
                                           nullptr, d_cDeg, part_e, part_a);
  k_modularity_final_value<<<1, 256, 0, s>>>(nparts, part_e, part_a, constant, d_out);
  g_launches += 2;
  CK(cudaGetLastError());
  return GLV_OK;
}

// =========================================================================
// Learned gate and trace capture (C ABI)
// =========================================================================
namespace glv {

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

static int upload_floats(const float *h, size_t n, DevBuf &d) {
  CK(cudaMalloc(&d.p, std::max<size_t>(n, 1) * sizeof(float)));
  if (n) CK(cudaMemcpy(d.p, h, n * sizeof(float), cudaMemcpyHostToDevice));
  return GLV_OK;
}

// Forward/backward and gradient reduction for rows [0, n) of x/y/w (device),
// parameters `dp` (device, FP32); gradients into dg (zeroed here).
static int gate_grad_device(cudaStream_t s, int64_t n, const float *x, const float *y,
                            const float *w, const float *dp, float *dg, float *work,
                            double *dloss) {
  float *h1 = work, *h2 = h1 + n * kGateHid, *dz1 = h2 + n * kGateHid, *dz2 = dz1 + n * kGateHid,
        *dz3 = dz2 + n * kGateHid;
  CK(cudaMemsetAsync(dg, 0, kGateParams * sizeof(float), s));
  CK(cudaMemsetAsync(dloss, 0, sizeof(double), s));
  const int gb = (int)std::max<int64_t>(1, std::min<int64_t>((n + 127) / 128, 148 * 8));
  k_gate_fwd_bwd<<<gb, 128, 0, s>>>(n, x, y, w, dp, h1, h2, dz1, dz2, dz3, dloss);
  const int ga = (int)std::max<int64_t>(1, std::min<int64_t>((n + 1023) / 1024, 148 * 4));
  k_outer_accum<<<ga, 256, 0, s>>>(n, kGateHid, kGateIn, dz1, kGateHid, x, kGateIn, dg + kGateW1);
  k_outer_accum<<<ga, 256, 0, s>>>(n, kGateHid, 1, dz1, kGateHid, nullptr, 1, dg + kGateB1);
  k_outer_accum<<<ga, 256, 0, s>>>(n, kGateHid, kGateHid, dz2, kGateHid, h1, kGateHid, dg + kGateW2);
  k_outer_accum<<<ga, 256, 0, s>>>(n, kGateHid, 1, dz2, kGateHid, nullptr, 1, dg + kGateB2);
  k_outer_accum<<<ga, 256, 0, s>>>(n, 1, kGateHid, dz3, 1, h2, kGateHid, dg + kGateW3);
  k_outer_accum<<<ga, 256, 0, s>>>(n, 1, 1, dz3, 1, nullptr, 1, dg + kGateB3);
  g_launches += 7;
  CK(cudaGetLastError());
  return GLV_OK;
}

}  // namespace glv

extern "C" {

int glv_gate_set(const float *params, float tau) {
  if (!params) return fail(GLV_ERR_ARG, "params is NULL");
  if (!(tau >= 0.0f && tau <= 1.0f)) return fail(GLV_ERR_ARG, "tau must be in [0, 1]");
  std::lock_guard<std::mutex> lock(g_gate_mu);
  g_gate_params.assign(params, params + kGateParams);
  g_gate_tau = tau;
  return GLV_OK;
}

int glv_gate_infer(long n, const float *d_feat, float *d_prob, void *stream) {
  TRY(device_ready());
  if (n < 0 || (n > 0 && (!d_feat || !d_prob))) return fail(GLV_ERR_ARG, "bad arguments");
  std::vector<float> hp;
  {
    std::lock_guard<std::mutex> lock(g_gate_mu);
    if ((int)g_gate_params.size() != kGateParams) return fail(GLV_ERR_ARG, "no gate parameters");
    hp = g_gate_params;
  }
  DevBuf dp;
  TRY(upload_floats(hp.data(), hp.size(), dp));
  cudaStream_t s = (cudaStream_t)stream;
  if (n > 0) {
    k_gate_infer<<<(int)std::max<long>(1, std::min<long>((n + 127) / 128, 148 * 8)), 256, 0, s>>>(
        n, d_feat, GateFeatSrc{}, (const float *)dp.p, 0.5f, nullptr, d_prob, nullptr, nullptr);
    ++g_launches;
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(s));
  return GLV_OK;
}

int glv_gate_grad(long n, const float *x, const float *y, const float *w, const float *params,
                  float *grad, double *loss) {
  TRY(device_ready());
  if (n < 1 || !x || !y || !w || !params || !grad) return fail(GLV_ERR_ARG, "bad arguments");
  DevBuf dx, dy, dw, dp, dg, work, dl;
  TRY(upload_floats(x, (size_t)n * kGateIn, dx));
  TRY(upload_floats(y, n, dy));
  TRY(upload_floats(w, n, dw));
  TRY(upload_floats(params, kGateParams, dp));
  CK(cudaMalloc(&dg.p, kGateParams * sizeof(float)));
  CK(cudaMalloc(&work.p, (size_t)n * (4 * kGateHid + 1) * sizeof(float)));
  CK(cudaMalloc(&dl.p, sizeof(double)));
  TRY(gate_grad_device(0, n, (float *)dx.p, (float *)dy.p, (float *)dw.p, (float *)dp.p,
                       (float *)dg.p, (float *)work.p, (double *)dl.p));
  CK(cudaMemcpy(grad, dg.p, kGateParams * sizeof(float), cudaMemcpyDeviceToHost));
  double l = 0;
  CK(cudaMemcpy(&l, dl.p, sizeof(double), cudaMemcpyDeviceToHost));
  if (loss) *loss = l / (double)n;
  return GLV_OK;
}

int glv_gate_train(long n, const float *x, const float *y, const float *w, int epochs,
                   long batch, float lr, unsigned seed, float *params, double *loss) {
  TRY(device_ready());
  if (n < 1 || batch < 1 || epochs < 1 || !x || !y || !w || !params)
    return fail(GLV_ERR_ARG, "bad arguments");
  // shuffle rows once on the host (seeded), then walk mini-batches per epoch
  std::vector<long> order(n);
  for (long i = 0; i < n; ++i) order[i] = i;
  uint32_t st = seed * 2654435761u + 12345u;
  for (long i = n - 1; i > 0; --i) {
    st = mix32(st + (uint32_t)i);
    std::swap(order[i], order[st % (uint32_t)(i + 1)]);
  }
  std::vector<float> hx((size_t)n * kGateIn), hy(n), hw(n);
  for (long i = 0; i < n; ++i) {
    for (int k = 0; k < kGateIn; ++k) hx[i * kGateIn + k] = x[order[i] * kGateIn + k];
    hy[i] = y[order[i]];
    hw[i] = w[order[i]];
  }
  const long bs = std::min(batch, n);
  DevBuf dx, dy, dw, dp, dg, dm, dv, work, dl;
  TRY(upload_floats(hx.data(), hx.size(), dx));
  TRY(upload_floats(hy.data(), n, dy));
  TRY(upload_floats(hw.data(), n, dw));
  TRY(upload_floats(params, kGateParams, dp));
  CK(cudaMalloc(&dg.p, kGateParams * sizeof(float)));
  CK(cudaMalloc(&dm.p, kGateParams * sizeof(float)));
  CK(cudaMalloc(&dv.p, kGateParams * sizeof(float)));
  CK(cudaMemset(dm.p, 0, kGateParams * sizeof(float)));
  CK(cudaMemset(dv.p, 0, kGateParams * sizeof(float)));
  CK(cudaMalloc(&work.p, (size_t)bs * (4 * kGateHid + 1) * sizeof(float)));
  CK(cudaMalloc(&dl.p, sizeof(double)));
  const float b1 = 0.9f, b2 = 0.999f;
  long t = 0;
  double epoch_loss = 0;
  for (int e = 0; e < epochs; ++e) {
    epoch_loss = 0;
    for (long b = 0; b < n; b += bs) {
      const long m = std::min(bs, n - b);
      TRY(gate_grad_device(0, m, (float *)dx.p + b * kGateIn, (float *)dy.p + b,
                           (float *)dw.p + b, (float *)dp.p, (float *)dg.p, (float *)work.p,
                           (double *)dl.p));
      ++t;
      const float c1 = 1.0f - std::pow(b1, (float)t), c2 = 1.0f - std::pow(b2, (float)t);
      k_adam<<<(kGateParams + 255) / 256, 256>>>(kGateParams, (float *)dp.p, (float *)dg.p,
                                                  (float *)dm.p, (float *)dv.p, lr, b1, b2, 1e-8f,
                                                  c1, c2);
      ++g_launches;
      CK(cudaGetLastError());
      double l = 0;
      CK(cudaMemcpy(&l, dl.p, sizeof(double), cudaMemcpyDeviceToHost));
      epoch_loss += l;
    }
    epoch_loss /= (double)n;
  }
  CK(cudaMemcpy(params, dp.p, kGateParams * sizeof(float), cudaMemcpyDeviceToHost));
  if (loss) *loss = epoch_loss;
  return GLV_OK;
}

int glv_trace_begin(long capacity, double rate) {
  TRY(device_ready());
  if (capacity < 1 || !(rate > 0.0 && rate <= 1.0)) return fail(GLV_ERR_ARG, "bad arguments");
  glv_trace_end();
  CK(cudaGetDevice(&g_trace.device));
  CK(cudaMalloc((void **)&g_trace.x, (size_t)capacity * kGateIn * sizeof(float)));
  CK(cudaMalloc((void **)&g_trace.y, (size_t)capacity * sizeof(float)));
  CK(cudaMalloc((void **)&g_trace.n, sizeof(unsigned long long)));
  CK(cudaMemset(g_trace.n, 0, sizeof(unsigned long long)));
  g_trace.cap = capacity;
  g_trace.rate = rate;
  g_trace.on = true;
  return GLV_OK;
}

long glv_trace_fetch(float *x, float *y, long cap) {
  if (!g_trace.on) return 0;
  unsigned long long n = 0;
  if (cudaMemcpy(&n, g_trace.n, sizeof(n), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  const long held = (long)std::min<unsigned long long>(n, (unsigned long long)g_trace.cap);
  const long k = std::min(held, cap);
  if (k > 0 && x && y) {
    if (cudaMemcpy(x, g_trace.x, (size_t)k * kGateIn * sizeof(float), cudaMemcpyDeviceToHost) !=
            cudaSuccess ||
        cudaMemcpy(y, g_trace.y, (size_t)k * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
      return -1;
  }
  return held;
}

int glv_trace_end(void) {
  if (g_trace.x) cudaFree(g_trace.x);
  if (g_trace.y) cudaFree(g_trace.y);
  if (g_trace.n) cudaFree(g_trace.n);
  g_trace = TraceSink{};
  return GLV_OK;
}

}  // extern "C"
