// Comparing two community assignments (Utility/utilityClusterComparisonMetrics.cpp).
//
// computeCommunityComparisons (:50-307) counts, over every pair of vertices
// in one community of C1 (the truth), those in one community of C2 too
// (SameSame, true positives) or not (SameDiff, false negatives), and over
// every pair in one community of C2, those split by C1 (DiffSame, false
// positives) -- by enumerating the pairs, quadratic in community size.  The
// same integers come from the contingency table of (C1, C2) labels:
//
//   SameSame = sum over label pairs (a, b) of C(n_ab, 2)
//   SameDiff = sum over a of C(n_a, 2) - SameSame
//   DiffSame = sum over b of C(n_b, 2) - SameSame
//
// Here: one kernel relabels as the reference does (-1 entries, 0- or 1-based
// ids) and histograms both sides; a radix sort of the (a, b) keys and a
// run-length encode give the n_ab.  The Gini coefficient of each side's
// community sizes (computeGiniCoefficient, :310-330) sorts the sizes and takes
// sum (i + 1) * size_i in exact 64-bit integers (the reference's FP64 running
// sum is exact, and so equal, while it stays below 2^53).
//
// Included into engine.cu after csr_build.cuh (DevScratch, staged copies).

namespace glv {

// Max, zero and -1 presence, and ids below -1, of one label array.  When
// `minus_one_as` >= 0 a -1 counts as that value (C2's rule, :92-93).
__global__ void k_label_stats(int64_t n, const int64_t *C, int64_t minus_one_as,
                              long long *mx, int32_t *flags) {
  long long m = LLONG_MIN;
  int f = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t c = C[i];
    if (c == -1) {
      f |= 2;
      if (minus_one_as < 0) continue;
      c = minus_one_as;
    } else if (c < -1) {
      f |= 4;
      continue;
    }
    if (c == 0) f |= 1;
    m = c > m ? c : m;
  }
  for (int off = 16; off; off >>= 1) {
    m = max(m, (long long)__shfl_xor_sync(FULL, m, off));
    f |= __shfl_xor_sync(FULL, f, off);
  }
  if ((threadIdx.x & 31) == 0) {
    if (m != LLONG_MIN) atomicMax(mx, m);
    if (f) atomicOr(flags, f);
  }
}

// Relabel in place as the reference does (C1: -1 -> fill1, C2: -1 -> fill2),
// map ids to community indices (minus one for 1-based ids), histogram them and
// form the contingency keys (a above b).
__global__ void k_label_pairs(int64_t n, int64_t *C1, int64_t *C2, int64_t fill1, int64_t fill2,
                              int64_t base1, int64_t base2, int bits2,
                              unsigned long long *hist1, unsigned long long *hist2,
                              uint64_t *keys) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int64_t a = C1[i], b = C2[i];
    if (a == -1) C1[i] = a = fill1;
    if (b == -1) C2[i] = b = fill2;
    a -= base1;
    b -= base2;
    atomicAdd(&hist1[a], 1ull);
    atomicAdd(&hist2[b], 1ull);
    keys[i] = ((uint64_t)a << bits2) | (uint64_t)b;
  }
}

// sum of C(n_k, 2) over counts n_k (32- or 64-bit counts).
template <class T>
__global__ void k_pair_sum(int64_t m, const T *counts, unsigned long long *out) {
  unsigned long long acc = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long c = (unsigned long long)counts[i];
    acc += c * (c - (c > 0 ? 1 : 0)) / 2;
  }
  for (int off = 16; off; off >>= 1) acc += __shfl_xor_sync(FULL, acc, off);
  if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

// out[0] += sum over the ascending sizes of (i + 1) * size_i, out[1] += the
// sum of the sizes.
__global__ void k_gini_sums(int64_t m, const unsigned long long *sorted, unsigned long long *out) {
  unsigned long long num = 0, den = 0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    num += (unsigned long long)(i + 1) * sorted[i];
    den += sorted[i];
  }
  for (int off = 16; off; off >>= 1) {
    num += __shfl_xor_sync(FULL, num, off);
    den += __shfl_xor_sync(FULL, den, off);
  }
  if ((threadIdx.x & 31) == 0) {
    if (num) atomicAdd(out, num);
    if (den) atomicAdd(out + 1, den);
  }
}

// computeGiniCoefficient's closing expression (:323), on the exact sums.
static double gini_from(unsigned long long num, unsigned long long den, int numColors) {
  const double numFunc = (double)num, denFunc = (double)den;
  return ((2 * numFunc) / (numColors * denFunc)) - ((double)(numColors + 1) / (double)numColors);
}

// Sizes sorted ascending (into *sorted) and the Gini sums of them
// (sums[0] numerator, sums[1] total); sizes take at most `bits` bits.
static int gini_sums(cudaStream_t s, const unsigned long long *sizes, int64_t m, int bits,
                     DevScratch &d, unsigned long long **sorted, unsigned long long sums[2],
                     long *launches) {
  unsigned long long *acc;
  TRY(d.get(sorted, m));
  TRY(d.get(&acc, 2));
  CK(cudaMemsetAsync(acc, 0, 2 * sizeof(*acc), s));
  size_t tb = 0;
  CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, sizes, *sorted, m, 0, bits, s));
  void *temp;
  TRY(d.get((char **)&temp, (int64_t)tb));
  CK(cub::DeviceRadixSort::SortKeys(temp, tb, sizes, *sorted, m, 0, bits, s));
  k_gini_sums<<<csr_grid(m), 256, 0, s>>>(m, *sorted, acc);
  ++*launches;
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(sums, acc, 2 * sizeof(*acc), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return GLV_OK;
}

// The comparison on device-resident label arrays (int64, relabelled in place).
static int compare_device(cudaStream_t s, int64_t n, int64_t *dC1, int64_t *dC2, DevScratch &d,
                          glv_comparison *out, long *launches) {
  long long *mx;
  int32_t *fl;
  TRY(d.get(&mx, 2));
  TRY(d.get(&fl, 2));
  const long long lo[2] = {LLONG_MIN, LLONG_MIN};
  CK(cudaMemcpyAsync(mx, lo, sizeof(lo), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(fl, 0, 2 * sizeof(int32_t), s));
  k_label_stats<<<csr_grid(n), 256, 0, s>>>(n, dC1, -1, mx, fl);
  k_label_stats<<<csr_grid(n), 256, 0, s>>>(n, dC2, n + 1, mx + 1, fl + 1);
  *launches += 2;
  CK(cudaGetLastError());
  long long hmx[2];
  int32_t hfl[2];
  CK(cudaMemcpyAsync(hmx, mx, sizeof(hmx), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(hfl, fl, sizeof(hfl), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if ((hfl[0] | hfl[1]) & 4) return fail(GLV_ERR_ARG, "a community id below -1");
  // C1 (:63-87): nC1 = largest id, plus one when 0 is an id; -1 entries
  // become nC1, which then grows by one
  const bool z1 = hfl[0] & 1, z2 = hfl[1] & 1;
  int64_t nC1 = (hmx[0] == LLONG_MIN ? -1 : hmx[0]) + (z1 ? 1 : 0);
  const int64_t fill1 = nC1;
  if (hfl[0] & 2) ++nC1;
  // C2 (:89-113): -1 entries become N2 + 1 before the count
  const int64_t nC2 = (int64_t)hmx[1] + (z2 ? 1 : 0);
  if (nC1 <= 0 || nC2 <= 0) return fail(GLV_ERR_ARG, "no community ids in C1 or C2");
  const int64_t base1 = z1 ? 0 : 1, base2 = z2 ? 0 : 1;
  if (nC1 > (int64_t)kIdMask + 1 || nC2 > (int64_t)kIdMask + 1)
    return fail(GLV_ERR_TOO_LARGE, "community ids >= 2^31");
  const int bits1 = id_bits(nC1), bits2 = id_bits(nC2);
  unsigned long long *h1, *h2, *acc;
  uint64_t *k1, *k2, *uniq;
  int64_t *counts, *nruns;
  TRY(d.get(&h1, nC1));
  TRY(d.get(&h2, nC2));
  TRY(d.get(&acc, 3));
  TRY(d.get(&k1, n));
  TRY(d.get(&k2, n));
  TRY(d.get(&uniq, n));
  TRY(d.get(&counts, n));
  TRY(d.get(&nruns, 1));
  CK(cudaMemsetAsync(h1, 0, nC1 * sizeof(*h1), s));
  CK(cudaMemsetAsync(h2, 0, nC2 * sizeof(*h2), s));
  CK(cudaMemsetAsync(acc, 0, 3 * sizeof(*acc), s));
  k_label_pairs<<<csr_grid(n), 256, 0, s>>>(n, dC1, dC2, fill1, n + 1, base1, base2, bits2, h1,
                                            h2, k1);
  ++*launches;
  CK(cudaGetLastError());
  size_t tb = 0, tb2 = 0;
  CK(cub::DeviceRadixSort::SortKeys(nullptr, tb, k1, k2, n, 0, bits1 + bits2, s));
  CK(cub::DeviceRunLengthEncode::Encode(nullptr, tb2, k2, uniq, counts, nruns, n, s));
  void *temp;
  TRY(d.get((char **)&temp, (int64_t)std::max(tb, tb2)));
  CK(cub::DeviceRadixSort::SortKeys(temp, tb, k1, k2, n, 0, bits1 + bits2, s));
  CK(cub::DeviceRunLengthEncode::Encode(temp, tb2, k2, uniq, counts, nruns, n, s));
  int64_t hr = 0;
  CK(cudaMemcpyAsync(&hr, nruns, sizeof(hr), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  k_pair_sum<<<csr_grid(hr), 256, 0, s>>>(hr, counts, acc);
  k_pair_sum<<<csr_grid(nC1), 256, 0, s>>>(nC1, h1, acc + 1);
  k_pair_sum<<<csr_grid(nC2), 256, 0, s>>>(nC2, h2, acc + 2);
  *launches += 3;
  CK(cudaGetLastError());
  unsigned long long pairs[3];
  CK(cudaMemcpyAsync(pairs, acc, sizeof(pairs), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  unsigned long long g1[2], g2[2], *srt;
  // community sizes are at most n: sort only the bits that can be set
  const int size_bits = id_bits(n + 1);
  TRY(gini_sums(s, h1, nC1, size_bits, d, &srt, g1, launches));
  TRY(gini_sums(s, h2, nC2, size_bits, d, &srt, g2, launches));
  const long SameSame = (long)pairs[0];
  const long SameDiff = (long)(pairs[1] - pairs[0]);
  const long DiffSame = (long)(pairs[2] - pairs[0]);
  // :258-263, :265-266
  const double precision = (double)SameSame / (double)(SameSame + DiffSame);
  const double recall = (double)SameSame / (double)(SameSame + SameDiff);
  out->n1 = n;
  out->n2 = n;
  out->num_communities1 = nC1;
  out->num_communities2 = nC2;
  out->same_same = SameSame;
  out->same_diff = SameDiff;
  out->diff_same = DiffSame;
  out->precision = precision;
  out->recall = recall;
  out->f_score = 2 * ((precision * recall) / (precision + recall));
  out->gini1 = gini_from(g1[0], g1[1], (int)nC1);
  out->gini2 = gini_from(g2[0], g2[1], (int)nC2);
  return GLV_OK;
}

}  // namespace glv

extern "C" {

int glv_compare_communities(long *C1, long N1, long *C2, long N2, glv_comparison *out) {
  if (!out || N1 <= 0 || N2 <= 0 || !C1 || !C2) return fail(GLV_ERR_ARG, "bad arguments");
  if (N1 != N2) return fail(GLV_ERR_ARG, "C1 and C2 label different numbers of vertices");
  if (N1 >= (1L << 31) - 2) return fail(GLV_ERR_TOO_LARGE, "N >= 2^31");
  Call c;
  TRY(open_stream(c));
  DevScratch d(c.s);
  int64_t *d1, *d2;
  TRY(d.get(&d1, N1));
  TRY(d.get(&d2, N1));
  TRY(h2d_large(c.s, d1, C1, N1 * (int64_t)sizeof(long)));
  TRY(h2d_large(c.s, d2, C2, N1 * (int64_t)sizeof(long)));
  TRY(compare_device(c.s, N1, d1, d2, d, out, &c.launches));
  TRY(d2h_large(c.s, C1, d1, N1 * (int64_t)sizeof(long)));
  TRY(d2h_large(c.s, C2, d2, N1 * (int64_t)sizeof(long)));
  g_launches += c.launches;
  return GLV_OK;
}

int glv_dev_compare_communities(long n, long *d_C1, long *d_C2, glv_comparison *out,
                                void *stream) {
  if (!out || n <= 0 || !d_C1 || !d_C2) return fail(GLV_ERR_ARG, "bad arguments");
  if (n >= (1L << 31) - 2) return fail(GLV_ERR_TOO_LARGE, "n >= 2^31");
  TRY(device_ready());
  if (!engine_pool()) return fail(GLV_ERR_CUDA, "could not create the device memory pool");
  cudaStream_t s = (cudaStream_t)stream;
  long launches = 0;
  {
    DevScratch d(s);
    TRY(compare_device(s, n, reinterpret_cast<int64_t *>(d_C1), reinterpret_cast<int64_t *>(d_C2),
                       d, out, &launches));
  }
  CK(cudaStreamSynchronize(s));
  g_launches += launches;
  return GLV_OK;
}

int glv_gini_coefficient(long *colorSize, int numColors, double *gini) {
  if (!gini || numColors <= 0 || !colorSize) return fail(GLV_ERR_ARG, "bad arguments");
  Call c;
  TRY(open_stream(c));
  DevScratch d(c.s);
  unsigned long long *dh, *sorted, sums[2];
  TRY(d.get(&dh, numColors));
  CK(cudaMemcpyAsync(dh, colorSize, numColors * sizeof(long), cudaMemcpyHostToDevice, c.s));
  // sizes are counts; a negative one would sort as a huge unsigned value
  long long *mn;
  int32_t *fl;
  TRY(d.get(&mn, 1));
  TRY(d.get(&fl, 1));
  const long long lo = LLONG_MIN;
  CK(cudaMemcpyAsync(mn, &lo, sizeof(lo), cudaMemcpyHostToDevice, c.s));
  CK(cudaMemsetAsync(fl, 0, sizeof(int32_t), c.s));
  k_label_stats<<<csr_grid(numColors), 256, 0, c.s>>>(numColors, (const int64_t *)dh, -1, mn, fl);
  ++c.launches;
  CK(cudaGetLastError());
  int32_t hf = 0;
  CK(cudaMemcpyAsync(&hf, fl, sizeof(hf), cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  if (hf & 6) return fail(GLV_ERR_ARG, "a negative size");
  TRY(gini_sums(c.s, dh, numColors, 64, d, &sorted, sums, &c.launches));
  // the reference sorts colorSize in place
  CK(cudaMemcpyAsync(colorSize, sorted, numColors * sizeof(long), cudaMemcpyDeviceToHost, c.s));
  CK(cudaStreamSynchronize(c.s));
  *gini = gini_from(sums[0], sums[1], numColors);
  g_launches += c.launches;
  return GLV_OK;
}

}  // extern "C"
