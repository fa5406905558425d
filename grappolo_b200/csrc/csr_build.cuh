// Edge lists to CSR on the device, and Grappolo's binary graph files.
//
// The reference builds its graphs on the host: removeEdges drops self-loops
// and repeated (head, tail) pairs (Utility/utilityFunctions.cpp:416-460), the
// loaders (e.g. InputsOutput/loadPajekFormat.cpp:94-150) and
// SortEdgesUndirected (utilityFunctions.cpp:463-498) store every edge in the
// rows of both its ends in list order, and SortNodeEdgesByIndex
// (:501-531) sorts each row by tail.  Here each of those is a handful of
// grid-stride kernels around CUB radix sorts and scans, with the exact output
// order of the reference's one-thread code:
//
//  * kept edges: a stable sort of (head, tail) keys marks the first of each
//    run; removeEdges' compaction fills the dropped slots below NGE, in
//    ascending order, with the kept edges above NGE from the top down, which
//    two scans and two scatters reproduce;
//  * rows: entry 2k + d (kept edge k, d = 0 head side, 1 tail side) is
//    stable-sorted by row, which is the loaders' fill order;
//  * sorted rows: the reference's bottom-up merge takes the right run on equal
//    tails, so equal tails end in descending position; a stable sort by
//    (row, tail) of the entries listed in reverse gives exactly that.
//
// Included into engine.cu after the C ABI helpers (Call, fail, CK, TRY).

namespace glv {

constexpr int kIdBits = 31;
constexpr uint64_t kIdMask = (1ull << kIdBits) - 1;

// Bits that hold every id below nv: sort keys (row, col) take 2 * id_bits(nv)
// bits, so the radix sorts make only the passes the graph needs.
static int id_bits(int64_t nv) {
  int b = 1;
  while (b < kIdBits && (int64_t(1) << b) < nv) ++b;
  return b;
}

// Edge arrays as the kernels read them: AoS glv_edge (stride 3 words) or
// separate int64 heads / tails and double weights (stride 1).  A null weight
// array reads as 1.0.
struct EdgeView {
  const int64_t *head, *tail;
  const double *w;
  int64_t stride;
  __device__ __forceinline__ int64_t h(int64_t i) const { return head[i * stride]; }
  __device__ __forceinline__ int64_t t(int64_t i) const { return tail[i * stride]; }
  __device__ __forceinline__ double wt(int64_t i) const { return w ? w[i * stride] : 1.0; }
};

static EdgeView aos_view(const glv_edge *e) {
  static_assert(sizeof(glv_edge) == 24, "glv_edge is three 8-byte words");
  const int64_t *base = reinterpret_cast<const int64_t *>(e);
  return EdgeView{base, base + 1, reinterpret_cast<const double *>(base + 2), 3};
}

__global__ void k_edge_pair_keys(int64_t ne, EdgeView ev, int64_t nv, int bits, uint64_t *keys,
                                 int64_t *idx, int32_t *bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t h = ev.h(i), t = ev.t(i);
    if (h < 0 || h >= nv || t < 0 || t >= nv) {
      atomicOr(bad, 1);
      h = t = 0;
    }
    keys[i] = ((uint64_t)h << bits) | (uint64_t)t;
    idx[i] = i;
  }
}

// After the stable sort: the first edge of each (head, tail) run is kept
// unless it is a self-loop.
__global__ void k_mark_kept(int64_t ne, int bits, const uint64_t *skeys, const int64_t *sidx,
                            uint8_t *kept, unsigned long long *count) {
  unsigned int mine = 0;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < ne;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = skeys[s];
    const bool first = s == 0 || skeys[s - 1] != k;
    const bool loop = (k >> bits) == (k & ((1ull << bits) - 1));
    const bool g = first && !loop;
    kept[sidx[s]] = g ? 1 : 0;
    mine += g ? 1u : 0u;
  }
  mine = __reduce_add_sync(FULL, mine);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(count, (unsigned long long)mine);
}

// Scan input of the compaction: below NGE the dropped slots, from NGE on the
// kept edges.
__global__ void k_slot_flags(int64_t ne, int64_t nge, const uint8_t *kept, int64_t *f) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne;
       i += (int64_t)gridDim.x * blockDim.x)
    f[i] = (i < nge) ? (kept[i] ? 0 : 1) : (kept[i] ? 1 : 0);
}

__global__ void k_order_low(int64_t nge, const uint8_t *kept, const int64_t *scan, int64_t *order,
                            int64_t *holes) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nge;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (kept[i]) order[i] = i;
    else holes[scan[i]] = i;
  }
}

// Kept edge i >= NGE is the r-th from the top (r = nholes - 1 - its rank
// above NGE) and fills the r-th hole.
__global__ void k_order_high(int64_t ne, int64_t nge, int64_t nholes, const uint8_t *kept,
                             const int64_t *scan, const int64_t *holes, int64_t *order) {
  for (int64_t i = nge + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ne;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (!kept[i]) continue;
    const int64_t r = nholes - 1 - (scan[i] - nholes);
    order[holes[r]] = i;
  }
}

__device__ __forceinline__ void entry_of(int64_t e, const int64_t *order, const EdgeView &ev,
                                         int64_t *src, int64_t *row, int64_t *col) {
  const int64_t k = e >> 1;
  const int64_t i = order ? order[k] : k;
  const int64_t h = ev.h(i), t = ev.t(i);
  *src = i;
  *row = (e & 1) ? t : h;
  *col = (e & 1) ? h : t;
}

// Sort records of the 2 * nk directed entries, one per entry e = 2k + d.
// sorted_rows: listed in reverse, key (row, col), sorted on all 2 * bits;
// otherwise in order, key (col above row), sorted on the row bits only, so
// the column rides along in the key's upper bits.  The weight is the sort
// value: the sorted records are the CSR, with nothing left to gather.
__global__ void k_entry_keys(int64_t m, bool sorted_rows, int bits, int64_t nv,
                             const int64_t *order, EdgeView ev, uint64_t *keys, double *vals,
                             int32_t *bad) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < m;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t e = sorted_rows ? m - 1 - q : q;
    int64_t src, row, col;
    entry_of(e, order, ev, &src, &row, &col);
    if (row < 0 || row >= nv || col < 0 || col >= nv) {
      atomicOr(bad, 1);
      row = col = 0;
    }
    keys[q] = sorted_rows ? (((uint64_t)row << bits) | (uint64_t)col)
                          : (((uint64_t)col << bits) | (uint64_t)row);
    vals[q] = ev.wt(src);
  }
}

__device__ __forceinline__ int64_t key_row(uint64_t k, bool sorted_rows, int bits) {
  return sorted_rows ? (int64_t)(k >> bits) : (int64_t)(k & ((1ull << bits) - 1));
}

__device__ __forceinline__ int64_t key_col(uint64_t k, bool sorted_rows, int bits) {
  return sorted_rows ? (int64_t)(k & ((1ull << bits) - 1)) : (int64_t)(k >> bits);
}

// Row offsets from the sorted records: position s opens every row after the
// previous record's row up to its own (s = m closes the rest).
__global__ void k_row_bounds(int64_t m, int64_t nv, bool sorted_rows, int bits,
                             const uint64_t *skeys, int64_t *ptr) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s <= m;
       s += (int64_t)gridDim.x * blockDim.x) {
    const int64_t here = s < m ? key_row(skeys[s], sorted_rows, bits) : nv;
    const int64_t prev = s > 0 ? key_row(skeys[s - 1], sorted_rows, bits) : -1;
    for (int64_t r = prev + 1; r <= here; ++r) ptr[r] = s;
  }
}

__global__ void k_emit_entries(int64_t m, bool sorted_rows, int bits, const uint64_t *skeys,
                               const double *svals, int32_t *otail, double *ow, glv_edge *oaos) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < m;
       s += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = skeys[s];
    const int64_t col = key_col(k, sorted_rows, bits);
    const double w = svals[s];
    if (otail) otail[s] = (int32_t)col;
    if (ow) ow[s] = w;
    if (oaos) oaos[s] = glv_edge{(long)key_row(k, sorted_rows, bits), (long)col, w};
  }
}

__global__ void k_gather_edges(int64_t n, const int64_t *order, const glv_edge *in, glv_edge *out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (int64_t)gridDim.x * blockDim.x)
    out[k] = in[order[k]];
}

// Row id of every entry of a CSR (one warp per row).
__global__ void k_row_ids(int64_t nv, const int64_t *ptr, int64_t *rowid) {
  const int lane = threadIdx.x & 31;
  for (int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < nv;
       v += ((int64_t)gridDim.x * blockDim.x) >> 5)
    for (int64_t j = ptr[v] + lane; j < ptr[v + 1]; j += 32) rowid[j] = v;
}

// SortNodeEdgesByIndex keys: positions listed in reverse, keyed (row, tail).
__global__ void k_row_sort_keys(int64_t nnz, const int64_t *rowid, const glv_edge *e,
                                uint64_t *keys, int64_t *vals, int32_t *bad) {
  // the row above the tail's 31 bits: tails of a given CSR are not bounded by
  // its row count
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nnz;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = nnz - 1 - q;
    int64_t t = e[p].tail;
    if (t < 0 || t > (int64_t)kIdMask) {
      atomicOr(bad, 1);
      t = 0;
    }
    keys[q] = ((uint64_t)rowid[p] << kIdBits) | (uint64_t)t;
    vals[q] = p;
  }
}

// Binary files: ids of each entry checked against NV while splitting.
__global__ void k_split_checked(int64_t n, const glv_edge *aos, int64_t nv, int32_t *tail,
                                double *w, int32_t *bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = aos[i].tail;
    if (t < 0 || t >= nv) atomicOr(bad, 1);
    tail[i] = (int32_t)t;
    w[i] = aos[i].weight;
  }
}

// Pool allocations released (stream-ordered) when the owner goes out of scope.
struct DevScratch {
  cudaStream_t s;
  std::vector<void *> held;
  explicit DevScratch(cudaStream_t st) : s(st) {}
  ~DevScratch() {
    for (void *p : held) cudaFreeAsync(p, s);
  }
  template <class T>
  int get(T **p, int64_t n) {
    cudaError_t e = cudaMallocFromPoolAsync((void **)p, std::max<int64_t>(n, 1) * sizeof(T),
                                            engine_pool(), s);
    if (e == cudaErrorMemoryAllocation) {
      // hand the pool's unused blocks back and retry once
      cudaGetLastError();
      cudaStreamSynchronize(s);
      cudaMemPoolTrimTo(engine_pool(), 0);
      e = cudaMallocFromPoolAsync((void **)p, std::max<int64_t>(n, 1) * sizeof(T), engine_pool(), s);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      return fail(GLV_ERR_OOM, "device allocation failed while building a CSR");
    }
    held.push_back(*p);
    return GLV_OK;
  }
};

static int csr_grid(int64_t n) { return grid_for(n, 256, 148 * 16); }

// removeEdges on the device: *order[k] = index of the edge that ends in slot
// k < *nge.
static int kept_order(cudaStream_t s, int64_t nv, int64_t ne, EdgeView ev, DevScratch &d,
                      int64_t **order, int64_t *nge, long *launches) {
  uint64_t *k1, *k2;
  int64_t *v1, *v2, *scan, *flags, *holes;
  uint8_t *kept;
  int32_t *bad;
  unsigned long long *cnt;
  TRY(d.get(&k1, ne));
  TRY(d.get(&k2, ne));
  TRY(d.get(&v1, ne));
  TRY(d.get(&v2, ne));
  TRY(d.get(&kept, ne));
  TRY(d.get(&bad, 1));
  TRY(d.get(&cnt, 1));
  CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
  CK(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
  const int bits = id_bits(nv);
  k_edge_pair_keys<<<csr_grid(ne), 256, 0, s>>>(ne, ev, nv, bits, k1, v1, bad);
  ++*launches;
  CK(cudaGetLastError());
  size_t tb = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k1, k2, v1, v2, ne, 0, 2 * bits, s));
  void *temp;
  TRY(d.get((char **)&temp, (int64_t)tb));
  CK(cub::DeviceRadixSort::SortPairs(temp, tb, k1, k2, v1, v2, ne, 0, 2 * bits, s));
  k_mark_kept<<<csr_grid(ne), 256, 0, s>>>(ne, bits, k2, v2, kept, cnt);
  ++*launches;
  CK(cudaGetLastError());
  int32_t hbad = 0;
  unsigned long long hcnt = 0;
  CK(cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&hcnt, cnt, sizeof(hcnt), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (hbad) return fail(GLV_ERR_ARG, "an edge end is outside [0, NV)");
  *nge = (int64_t)hcnt;
  // keys and sort values are free again: reuse them for the compaction
  flags = reinterpret_cast<int64_t *>(k1);
  scan = reinterpret_cast<int64_t *>(k2);
  holes = v1;
  *order = v2;
  k_slot_flags<<<csr_grid(ne), 256, 0, s>>>(ne, *nge, kept, flags);
  ++*launches;
  CK(cudaGetLastError());
  size_t tb2 = 0;
  CK(cub::DeviceScan::ExclusiveSum(nullptr, tb2, flags, scan, ne, s));
  if (tb2 > tb) TRY(d.get((char **)&temp, (int64_t)tb2));
  CK(cub::DeviceScan::ExclusiveSum(temp, tb2, flags, scan, ne, s));
  int64_t nholes = 0;
  if (*nge < ne) {
    CK(cudaMemcpyAsync(&nholes, scan + *nge, sizeof(nholes), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  }
  if (*nge > 0) {
    k_order_low<<<csr_grid(*nge), 256, 0, s>>>(*nge, kept, scan, *order, holes);
    ++*launches;
    CK(cudaGetLastError());
  }
  if (nholes > 0) {
    k_order_high<<<csr_grid(ne - *nge), 256, 0, s>>>(ne, *nge, nholes, kept, scan, holes, *order);
    ++*launches;
    CK(cudaGetLastError());
  }
  return GLV_OK;
}

// The 2 * nk directed entries of the kept edges in row order (sorted_rows:
// rows sorted by tail, equal tails latest first), written as a CSR: d_ptr[nv
// + 1] and any of otail / ow (SoA) and oaos (glv_edge records).  Ids outside
// [0, nv) are GLV_ERR_ARG.
static int row_entries(cudaStream_t s, int64_t nv, int64_t nk, const int64_t *order, EdgeView ev,
                       bool sorted_rows, DevScratch &d, int64_t *d_ptr, int32_t *otail, double *ow,
                       glv_edge *oaos, long *launches) {
  const int64_t m = 2 * nk;
  const int ib = id_bits(nv);
  uint64_t *k1, *k2;
  double *v1, *v2;
  int32_t *bad;
  TRY(d.get(&k1, m));
  TRY(d.get(&k2, m));
  TRY(d.get(&v1, m));
  TRY(d.get(&v2, m));
  TRY(d.get(&bad, 1));
  CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
  if (m > 0) {
    k_entry_keys<<<csr_grid(m), 256, 0, s>>>(m, sorted_rows, ib, nv, order, ev, k1, v1, bad);
    ++*launches;
    CK(cudaGetLastError());
    const int bits = sorted_rows ? 2 * ib : ib;
    size_t tb = 0;
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k1, k2, v1, v2, m, 0, bits, s));
    void *temp;
    TRY(d.get((char **)&temp, (int64_t)tb));
    CK(cub::DeviceRadixSort::SortPairs(temp, tb, k1, k2, v1, v2, m, 0, bits, s));
  }
  k_row_bounds<<<csr_grid(m + 1), 256, 0, s>>>(m, nv, sorted_rows, ib, k2, d_ptr);
  ++*launches;
  CK(cudaGetLastError());
  if (m > 0) {
    k_emit_entries<<<csr_grid(m), 256, 0, s>>>(m, sorted_rows, ib, k2, v2, otail, ow, oaos);
    ++*launches;
    CK(cudaGetLastError());
  }
  int32_t hb = 0;
  CK(cudaMemcpyAsync(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (hb) return fail(GLV_ERR_ARG, "an edge end is outside [0, NV)");
  return GLV_OK;
}

// Device-to-host copy of a large result into ordinary (pageable, possibly
// never touched) host memory, such as the malloc'd arrays the reference's API
// returns.  A plain cudaMemcpy into such memory runs at the speed of one
// thread faulting pages in; here the data moves by DMA into two pinned
// staging buffers while a team of host threads copies the previous chunk out
// (and takes the page faults in parallel).
static bool page_locked(const void *p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

static void parallel_memcpy(char *dst, const char *src, int64_t n) {
  const int nthreads = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<std::thread> team;
  const int64_t part = (n + nthreads - 1) / nthreads;
  for (int t = 0; t < nthreads; ++t) {
    const int64_t a = t * part, b = std::min(n, a + part);
    if (a >= b) break;
    team.emplace_back([=] { memcpy(dst + a, src + a, b - a); });
  }
  for (auto &th : team) th.join();
}

static int d2h_large(cudaStream_t s, void *host, const void *dev, int64_t bytes) {
  if (bytes <= 0) return GLV_OK;
  if (bytes < (int64_t(64) << 20) || page_locked(host)) {
    CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return GLV_OK;
  }
  const int64_t chunk = int64_t(128) << 20;
  char *stage[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  struct Guard {
    char **st;
    cudaEvent_t *ev;
    ~Guard() {
      for (int k = 0; k < 2; ++k) {
        if (ev[k]) {
          cudaEventSynchronize(ev[k]);
          cudaEventDestroy(ev[k]);
        }
        if (st[k]) cudaFreeHost(st[k]);
      }
    }
  } guard{stage, ev};
  for (int k = 0; k < 2; ++k) {
    CK(cudaHostAlloc((void **)&stage[k], chunk, cudaHostAllocDefault));
    CK(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
  }
  auto copy_out = [](const char *src, char *dst, int64_t n) { parallel_memcpy(dst, src, n); };
  const char *d = static_cast<const char *>(dev);
  char *h = static_cast<char *>(host);
  int64_t prev_off = -1, prev_n = 0;
  int k = 0;
  for (int64_t off = 0; off < bytes; off += chunk, k ^= 1) {
    const int64_t n = std::min(chunk, bytes - off);
    CK(cudaMemcpyAsync(stage[k], d + off, n, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(ev[k], s));
    if (prev_off >= 0) {  // the previous chunk's DMA is done: copy it out meanwhile
      CK(cudaEventSynchronize(ev[k ^ 1]));
      copy_out(stage[k ^ 1], h + prev_off, prev_n);
    }
    prev_off = off;
    prev_n = n;
    // stage[k ^ 1] is free again for the next chunk's DMA
  }
  CK(cudaEventSynchronize(ev[k ^ 1]));
  copy_out(stage[k ^ 1], h + prev_off, prev_n);
  return GLV_OK;
}

// Host-to-device counterpart of d2h_large for pageable sources: host threads
// copy chunk i + 1 into a pinned staging buffer while chunk i moves by DMA.
static int h2d_large(cudaStream_t s, void *dev, const void *host, int64_t bytes) {
  if (bytes <= 0) return GLV_OK;
  if (bytes < (int64_t(64) << 20) || page_locked(host)) {
    CK(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s));
    return GLV_OK;
  }
  const int64_t chunk = int64_t(128) << 20;
  char *stage[2] = {nullptr, nullptr};
  cudaEvent_t ev[2] = {nullptr, nullptr};
  struct Guard {
    char **st;
    cudaEvent_t *ev;
    ~Guard() {
      for (int k = 0; k < 2; ++k) {
        if (ev[k]) {
          cudaEventSynchronize(ev[k]);
          cudaEventDestroy(ev[k]);
        }
        if (st[k]) cudaFreeHost(st[k]);
      }
    }
  } guard{stage, ev};
  for (int k = 0; k < 2; ++k) {
    CK(cudaHostAlloc((void **)&stage[k], chunk, cudaHostAllocDefault));
    CK(cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming));
  }
  const char *h = static_cast<const char *>(host);
  char *d = static_cast<char *>(dev);
  int k = 0;
  for (int64_t off = 0; off < bytes; off += chunk, k ^= 1) {
    const int64_t n = std::min(chunk, bytes - off);
    CK(cudaEventSynchronize(ev[k]));  // this buffer's previous DMA has finished
    parallel_memcpy(stage[k], h + off, n);
    CK(cudaMemcpyAsync(d + off, stage[k], n, cudaMemcpyHostToDevice, s));
    CK(cudaEventRecord(ev[k], s));
  }
  return GLV_OK;  // the guard waits for both buffers' last DMA
}

static int upload_edges(cudaStream_t s, const glv_edge *host, int64_t n, DevScratch &d,
                        glv_edge **dev) {
  TRY(d.get(dev, n));
  return h2d_large(s, *dev, host, n * (int64_t)sizeof(glv_edge));
}

static int open_stream(Call &c) {
  TRY(device_ready());
  if (!engine_pool()) return fail(GLV_ERR_CUDA, "could not create the device memory pool");
  CK(engine_stream(&c.s));
  return GLV_OK;
}

static FILE *open_binary(const char *path, const char *how) {
  return path ? fopen(path, how) : nullptr;
}

// Header of a binary graph file (InputsOutput/loadBinary.cpp:26-30).
static int read_binary_header(FILE *f, long *nv, long *ne, long *weighted) {
  long h[3];
  if (fread(h, sizeof(long), 3, f) != 3) return fail(GLV_ERR_IO, "short binary header");
  if (h[0] < 0 || h[1] < 0) return fail(GLV_ERR_IO, "negative sizes in the binary header");
  *nv = h[0];
  *ne = h[1];
  *weighted = h[2];
  return GLV_OK;
}

}  // namespace glv

extern "C" {

int glv_remove_edges(long NV, long NE, glv_edge *edgeList, long *numGoodEdges) {
  if (NV < 0 || NE < 0 || (!edgeList && NE > 0)) return fail(GLV_ERR_ARG, "bad arguments");
  if (NV > (long)kIdMask) return fail(GLV_ERR_TOO_LARGE, "NV >= 2^31");
  Call c;
  TRY(open_stream(c));
  DevScratch d(c.s);
  glv_edge *din, *dout;
  TRY(upload_edges(c.s, edgeList, NE, d, &din));
  int64_t *order = nullptr, nge = 0;
  if (NE > 0) TRY(kept_order(c.s, NV, NE, aos_view(din), d, &order, &nge, &c.launches));
  if (nge > 0) {
    TRY(d.get(&dout, nge));
    k_gather_edges<<<csr_grid(nge), 256, 0, c.s>>>(nge, order, din, dout);
    ++c.launches;
    CK(cudaGetLastError());
    TRY(d2h_large(c.s, edgeList, dout, nge * (int64_t)sizeof(glv_edge)));
  }
  CK(cudaStreamSynchronize(c.s));
  g_launches += c.launches;
  if (numGoodEdges) *numGoodEdges = (long)nge;
  return GLV_OK;
}

int glv_sort_edges_undirected(long NV, long NE, const glv_edge *list1, glv_edge *list2,
                              long *ptrs) {
  if (NV < 0 || NE < 0 || !ptrs || (NE > 0 && (!list1 || !list2)))
    return fail(GLV_ERR_ARG, "bad arguments");
  if (NV > (long)kIdMask) return fail(GLV_ERR_TOO_LARGE, "NV >= 2^31");
  Call c;
  TRY(open_stream(c));
  DevScratch d(c.s);
  glv_edge *din, *dout;
  int64_t *dptr;
  TRY(upload_edges(c.s, list1, NE, d, &din));
  TRY(d.get(&dptr, NV + 1));
  TRY(d.get(&dout, 2 * NE));
  TRY(row_entries(c.s, NV, NE, nullptr, aos_view(din), false, d, dptr, nullptr, nullptr, dout,
                  &c.launches));
  TRY(d2h_large(c.s, list2, dout, 2 * NE * (int64_t)sizeof(glv_edge)));
  CK(cudaMemcpyAsync(ptrs, dptr, (NV + 1) * sizeof(long), cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  ptrs[NV + 1] = 2 * NE;  // the reference's shifted histogram leaves 2*NE here
  g_launches += c.launches;
  return GLV_OK;
}

int glv_sort_node_edges_by_index(long NV, glv_edge *list1, glv_edge *list2, const long *ptrs) {
  (void)list2;
  TRY(check_ptr(NV, ptrs));
  const int64_t nnz = ptrs[NV];
  if (nnz > 0 && !list1) return fail(GLV_ERR_ARG, "list1 is NULL");
  Call c;
  TRY(open_stream(c));
  DevScratch d(c.s);
  glv_edge *din, *dout;
  int64_t *dptr, *rowid, *v1, *v2;
  uint64_t *k1, *k2;
  int32_t *bad;
  TRY(upload_edges(c.s, list1, nnz, d, &din));
  TRY(d.get(&dptr, NV + 1));
  TRY(d.get(&rowid, nnz));
  TRY(d.get(&k1, nnz));
  TRY(d.get(&k2, nnz));
  TRY(d.get(&v1, nnz));
  TRY(d.get(&v2, nnz));
  TRY(d.get(&bad, 1));
  TRY(d.get(&dout, nnz));
  CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), c.s));
  CK(cudaMemcpyAsync(dptr, ptrs, (NV + 1) * sizeof(long), cudaMemcpyHostToDevice, c.s));
  if (nnz > 0) {
    k_row_ids<<<grid_for(NV * 32, 256, 148 * 16), 256, 0, c.s>>>(NV, dptr, rowid);
    k_row_sort_keys<<<csr_grid(nnz), 256, 0, c.s>>>(nnz, rowid, din, k1, v1, bad);
    c.launches += 2;
    CK(cudaGetLastError());
    size_t tb = 0;
    const int bits = kIdBits + id_bits(NV);
    CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, k1, k2, v1, v2, nnz, 0, bits, c.s));
    void *temp;
    TRY(d.get((char **)&temp, (int64_t)tb));
    CK(cub::DeviceRadixSort::SortPairs(temp, tb, k1, k2, v1, v2, nnz, 0, bits, c.s));
    k_gather_edges<<<csr_grid(nnz), 256, 0, c.s>>>(nnz, v2, din, dout);
    ++c.launches;
    CK(cudaGetLastError());
    int32_t hb = 0;
    CK(cudaMemcpyAsync(&hb, bad, sizeof(hb), cudaMemcpyDeviceToHost, c.s));
    CK(cudaStreamSynchronize(c.s));
    if (hb) return fail(GLV_ERR_ARG, "a tail is outside [0, 2^31)");
    TRY(d2h_large(c.s, list1, dout, nnz * (int64_t)sizeof(glv_edge)));
  }
  CK(cudaStreamSynchronize(c.s));
  g_launches += c.launches;
  return GLV_OK;
}

int glv_build_csr(long NV, long NE, const glv_edge *edges, int flags, glv_graph *Gout) {
  if (NV < 0 || NE < 0 || !Gout || (!edges && NE > 0)) return fail(GLV_ERR_ARG, "bad arguments");
  if (NV > (long)kIdMask) return fail(GLV_ERR_TOO_LARGE, "NV >= 2^31");
  if (flags & ~(GLV_CSR_REMOVE_EDGES | GLV_CSR_SORT_ROWS)) return fail(GLV_ERR_ARG, "bad flags");
  Call c;
  TRY(open_stream(c));
  DevScratch d(c.s);
  glv_edge *din, *dout;
  int64_t *dptr, *order = nullptr, nk = NE;
  TRY(upload_edges(c.s, edges, NE, d, &din));
  TRY(d.get(&dptr, NV + 1));
  if (NE > 0 && (flags & GLV_CSR_REMOVE_EDGES))
    TRY(kept_order(c.s, NV, NE, aos_view(din), d, &order, &nk, &c.launches));
  const int64_t m = 2 * nk;
  TRY(d.get(&dout, m));
  TRY(row_entries(c.s, NV, nk, order, aos_view(din), (flags & GLV_CSR_SORT_ROWS) != 0, d, dptr,
                  nullptr, nullptr, dout, &c.launches));
  long *hp = (long *)malloc((NV + 1) * sizeof(long));
  glv_edge *he = (glv_edge *)malloc(std::max<int64_t>(m, 1) * sizeof(glv_edge));
  if (!hp || !he) {
    free(hp);
    free(he);
    return fail(GLV_ERR_OOM, "host allocation failed");
  }
  int rc = d2h_large(c.s, hp, dptr, (NV + 1) * sizeof(long));
  if (rc == GLV_OK) rc = d2h_large(c.s, he, dout, m * (int64_t)sizeof(glv_edge));
  if (rc != GLV_OK) {
    free(hp);
    free(he);
    return rc;
  }
  g_launches += c.launches;
  Gout->numVertices = NV;
  Gout->sVertices = NV;
  Gout->numEdges = nk;
  Gout->edgeListPtrs = hp;
  Gout->edgeList = he;
  return GLV_OK;
}

int glv_dev_build_csr(long NV, long NE, const long *d_head, const long *d_tail,
                      const double *d_weight, int flags, long *d_ptr, int *d_tail_out,
                      double *d_weight_out, long *nnz, void *stream) {
  if (NV < 0 || NE < 0 || !d_ptr || (NE > 0 && (!d_head || !d_tail || !d_tail_out || !d_weight_out)))
    return fail(GLV_ERR_ARG, "bad arguments");
  if (NV > (long)kIdMask) return fail(GLV_ERR_TOO_LARGE, "NV >= 2^31");
  if (flags & ~(GLV_CSR_REMOVE_EDGES | GLV_CSR_SORT_ROWS)) return fail(GLV_ERR_ARG, "bad flags");
  TRY(device_ready());
  if (!engine_pool()) return fail(GLV_ERR_CUDA, "could not create the device memory pool");
  cudaStream_t s = (cudaStream_t)stream;
  long launches = 0;
  int64_t *order = nullptr, nk = NE;
  const EdgeView ev{reinterpret_cast<const int64_t *>(d_head),
                    reinterpret_cast<const int64_t *>(d_tail), d_weight, 1};
  {
    DevScratch d(s);
    if (NE > 0 && (flags & GLV_CSR_REMOVE_EDGES))
      TRY(kept_order(s, NV, NE, ev, d, &order, &nk, &launches));
    TRY(row_entries(s, NV, nk, order, ev, (flags & GLV_CSR_SORT_ROWS) != 0, d,
                    reinterpret_cast<int64_t *>(d_ptr), d_tail_out, d_weight_out, nullptr,
                    &launches));
  }
  CK(cudaStreamSynchronize(s));
  g_launches += launches;
  if (nnz) *nnz = 2 * nk;
  return GLV_OK;
}

int glv_binary_header(const char *path, long *numVertices, long *numEdges, long *weighted) {
  FILE *f = open_binary(path, "rb");
  if (!f) return fail(GLV_ERR_IO, "cannot open the binary file");
  long nv, ne, wt;
  const int rc = read_binary_header(f, &nv, &ne, &wt);
  fclose(f);
  TRY(rc);
  if (numVertices) *numVertices = nv;
  if (numEdges) *numEdges = ne;
  if (weighted) *weighted = wt;
  return GLV_OK;
}

int glv_load_binary(const char *path, glv_graph *G) {
  if (!G) return fail(GLV_ERR_ARG, "G is NULL");
  FILE *f = open_binary(path, "rb");
  if (!f) return fail(GLV_ERR_IO, "cannot open the binary file");
  long nv, ne, wt;
  int rc = read_binary_header(f, &nv, &ne, &wt);
  if (rc != GLV_OK) {
    fclose(f);
    return rc;
  }
  long *p = (long *)malloc((nv + 1) * sizeof(long));
  glv_edge *e = (glv_edge *)malloc(std::max<long>(2 * ne, 1) * sizeof(glv_edge));
  if (!p || !e) {
    fclose(f);
    free(p);
    free(e);
    return fail(GLV_ERR_OOM, "host allocation failed");
  }
  const bool ok = fread(p, sizeof(long), nv + 1, f) == (size_t)(nv + 1) &&
                  fread(e, sizeof(glv_edge), 2 * ne, f) == (size_t)(2 * ne);
  fclose(f);
  if (!ok) {
    free(p);
    free(e);
    return fail(GLV_ERR_IO, "binary file shorter than its header says");
  }
  G->numVertices = nv;
  G->sVertices = nv;
  G->numEdges = ne;
  G->edgeListPtrs = p;
  G->edgeList = e;
  return GLV_OK;
}

int glv_write_binary(const glv_graph *G, const char *path, long weighted) {
  if (!G || G->numVertices < 0 || !G->edgeListPtrs) return fail(GLV_ERR_ARG, "bad graph");
  FILE *f = open_binary(path, "wb");
  if (!f) return fail(GLV_ERR_IO, "cannot create the binary file");
  const long h[3] = {G->numVertices, G->numEdges, weighted};
  const long n2 = 2 * G->numEdges;  // the reference writes 2 * numEdges entries
  bool ok = fwrite(h, sizeof(long), 3, f) == 3 &&
            fwrite(G->edgeListPtrs, sizeof(long), G->numVertices + 1, f) ==
                (size_t)(G->numVertices + 1) &&
            (n2 == 0 || fwrite(G->edgeList, sizeof(glv_edge), n2, f) == (size_t)n2);
  ok = (fclose(f) == 0) && ok;
  return ok ? GLV_OK : fail(GLV_ERR_IO, "write to the binary file failed");
}

int glv_dev_load_binary(const char *path, long numVertices, long nnz, long *d_ptr, int *d_tail,
                        double *d_weight, void *stream) {
  if (numVertices < 0 || nnz < 0 || !d_ptr || (nnz > 0 && (!d_tail || !d_weight)))
    return fail(GLV_ERR_ARG, "bad arguments");
  if (numVertices > (long)kIdMask) return fail(GLV_ERR_TOO_LARGE, "numVertices >= 2^31");
  TRY(device_ready());
  if (!engine_pool()) return fail(GLV_ERR_CUDA, "could not create the device memory pool");
  FILE *f = open_binary(path, "rb");
  if (!f) return fail(GLV_ERR_IO, "cannot open the binary file");
  struct Closer {
    FILE *f;
    ~Closer() { fclose(f); }
  } closer{f};
  long nv, ne, wt;
  TRY(read_binary_header(f, &nv, &ne, &wt));
  if (nv != numVertices || 2 * ne != nnz)
    return fail(GLV_ERR_ARG, "numVertices / nnz differ from the file's header");
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<long> ptr(nv + 1);
  if (fread(ptr.data(), sizeof(long), nv + 1, f) != (size_t)(nv + 1))
    return fail(GLV_ERR_IO, "binary file shorter than its header says");
  if (ptr[0] != 0 || ptr[nv] != nnz) return fail(GLV_ERR_IO, "row offsets do not span 2*NE");
  for (long v = 0; v < nv; ++v)
    if (ptr[v + 1] < ptr[v]) return fail(GLV_ERR_IO, "row offsets decrease");
  CK(cudaMemcpyAsync(d_ptr, ptr.data(), (nv + 1) * sizeof(long), cudaMemcpyHostToDevice, s));
  // Entries stream through two pinned buffers: the file read of one chunk
  // overlaps the copy and split of the previous one.
  const int64_t chunk = std::min<int64_t>(std::max<int64_t>(nnz, 1), int64_t(1) << 22);
  glv_edge *pin[2] = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
  struct PinGuard {
    glv_edge **p;
    cudaEvent_t *ev;
    ~PinGuard() {
      for (int k = 0; k < 2; ++k) {
        if (ev[k]) {
          cudaEventSynchronize(ev[k]);
          cudaEventDestroy(ev[k]);
        }
        if (p[k]) cudaFreeHost(p[k]);
      }
    }
  } guard{pin, done};
  for (int k = 0; k < 2; ++k) {
    CK(cudaHostAlloc((void **)&pin[k], chunk * sizeof(glv_edge), cudaHostAllocDefault));
    CK(cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming));
  }
  long launches = 0;
  int32_t hbad = 0;
  {
    DevScratch d(s);
    glv_edge *stage[2];
    int32_t *bad;
    TRY(d.get(&stage[0], chunk));
    TRY(d.get(&stage[1], chunk));
    TRY(d.get(&bad, 1));
    CK(cudaMemsetAsync(bad, 0, sizeof(int32_t), s));
    int k = 0;
    for (int64_t b = 0; b < nnz; b += chunk, k ^= 1) {
      const int64_t n = std::min(chunk, nnz - b);
      CK(cudaEventSynchronize(done[k]));  // the buffer's previous copy has finished
      if (fread(pin[k], sizeof(glv_edge), n, f) != (size_t)n)
        return fail(GLV_ERR_IO, "binary file shorter than its header says");
      CK(cudaMemcpyAsync(stage[k], pin[k], n * sizeof(glv_edge), cudaMemcpyHostToDevice, s));
      CK(cudaEventRecord(done[k], s));
      k_split_checked<<<csr_grid(n), 256, 0, s>>>(n, stage[k], nv, d_tail + b, d_weight + b, bad);
      ++launches;
      CK(cudaGetLastError());
    }
    CK(cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  }
  g_launches += launches;
  if (hbad) return fail(GLV_ERR_IO, "a tail in the binary file is outside [0, NV)");
  return GLV_OK;
}

}  // extern "C"
