// Learned move gate: a 6 -> 64 -> 64 -> 1 MLP that predicts, from what the
// previous sweep saw of a vertex, whether the next sweep will move it.  A
// gated sweep evaluates only the vertices the MLP keeps (p >= tau); the
// others stay where they are.  Weights are BF16 with FP32 accumulation; the
// 64x64 layer runs on the tensor cores (mma.sync m16n8k16 bf16 -> f32).
//
// Features of vertex v at iteration t of a phase (all from iteration t-1):
//   f0 = log1p(row length) / 8           f1 = log1p(weighted degree) / 8
//   f2 = Counter[own] / weighted degree  (fraction of weight into its community)
//   f3 = best positive gain / weighted degree
//   f4 = log1p(sweeps since its last move) / 4
//   f5 = phase index / 8
// Parameter layout (kGateParams floats): W1[64][6], b1[64], W2[64][64] (row =
// output), b2[64], W3[64], b3.
#pragma once

#include <cuda_bf16.h>

#include "glv_common.cuh"

namespace glv {

constexpr int kGateIn = 6, kGateHid = 64;
constexpr int kGateW1 = 0, kGateB1 = kGateW1 + kGateHid * kGateIn, kGateW2 = kGateB1 + kGateHid,
              kGateB2 = kGateW2 + kGateHid * kGateHid, kGateW3 = kGateB2 + kGateHid,
              kGateB3 = kGateW3 + kGateHid, kGateParams = kGateB3 + 1;  // 4673

__device__ __forceinline__ float bf16r(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// What the features of a vertex are computed from (the sweep's state after
// iteration iter - 1 of phase `phase`).
struct GateFeatSrc {
  const int64_t *ptr;
  const double *vDeg;
  const double *rec_own;
  const float *rec_gain;
  const int32_t *last_move;
  int32_t iter, phase;
};

__device__ __forceinline__ void gate_features(int64_t v, const GateFeatSrc &s, float f[kGateIn]) {
  const double deg = (double)(s.ptr[v + 1] - s.ptr[v]);
  const double wd = s.vDeg[v];
  const double inv = wd > 0.0 ? 1.0 / wd : 0.0;
  f[0] = (float)(log1p(deg) * 0.125);
  f[1] = (float)(log1p(wd) * 0.125);
  f[2] = (float)(s.rec_own[v] * inv);
  f[3] = (float)((double)s.rec_gain[v] * inv);
  f[4] = (float)(log1p((double)(s.iter - s.last_move[v])) * 0.25);
  f[5] = (float)s.phase * 0.125f;
}

// The feature rows, for trace capture (the gated sweeps compute them inside
// k_gate_infer instead).
__global__ void k_gate_features(int64_t nv, GateFeatSrc src, float *feat) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nv;
       v += (int64_t)gridDim.x * blockDim.x) {
    float f[kGateIn];
    gate_features(v, src, f);
#pragma unroll
    for (int i = 0; i < kGateIn; ++i) feat[(size_t)v * kGateIn + i] = f[i];
  }
}

// Inference: one warp per 16 vertices.  Layer 1 on the CUDA cores into a
// per-warp BF16 tile, layer 2 with mma.sync (8 column tiles x 4 k-steps),
// layer 3 as a 4-lane reduction.  The features come from `feat` (rows of
// kGateIn floats) or, when feat is NULL, from `src`: lane r computes those of
// the tile's row r and the warp reads them by shuffles.  prob may be NULL;
// skip[v] = (p < tau); *evaluated += row lengths of the kept vertices.
__global__ void __launch_bounds__(256) k_gate_infer(int64_t nv, const float *feat,
                                                    GateFeatSrc src, const float *params,
                                                    float tau, const int64_t *ptr, float *prob,
                                                    uint8_t *skip,
                                                    unsigned long long *evaluated) {
  __shared__ float s_w1[kGateHid * kGateIn], s_b1[kGateHid], s_b2[kGateHid], s_w3[kGateHid];
  __shared__ __align__(16) __nv_bfloat16 s_w2[kGateHid * kGateHid];
  __shared__ __align__(16) __nv_bfloat16 s_h1[8][16 * kGateHid];
  __shared__ float s_b3;
  for (int i = threadIdx.x; i < kGateHid * kGateIn; i += blockDim.x) s_w1[i] = bf16r(params[kGateW1 + i]);
  for (int i = threadIdx.x; i < kGateHid; i += blockDim.x) {
    s_b1[i] = params[kGateB1 + i];
    s_b2[i] = params[kGateB2 + i];
    s_w3[i] = bf16r(params[kGateW3 + i]);
  }
  for (int i = threadIdx.x; i < kGateHid * kGateHid; i += blockDim.x)
    s_w2[i] = __float2bfloat16_rn(params[kGateW2 + i]);
  if (threadIdx.x == 0) s_b3 = params[kGateB3];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  __nv_bfloat16 *h1 = s_h1[warp];
  const int64_t ntile = (nv + 15) / 16;
  unsigned long long local_eval = 0;
  for (int64_t tile = (int64_t)blockIdx.x * 8 + warp; tile < ntile; tile += (int64_t)gridDim.x * 8) {
    const int64_t v0 = tile * 16;
    float mine[kGateIn] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // row `lane`'s features
    if (!feat && lane < 16 && v0 + lane < nv) gate_features(v0 + lane, src, mine);
    // layer 1: lane handles hidden units lane and lane+32 for the 16 rows
    for (int r = 0; r < 16; ++r) {
      const int64_t v = v0 + r;
      float x[kGateIn];
#pragma unroll
      for (int i = 0; i < kGateIn; ++i)
        x[i] = feat ? ((v < nv) ? feat[(size_t)v * kGateIn + i] : 0.0f)
                    : __shfl_sync(FULL, mine[i], r);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const int j = lane + 32 * q;
        float z = s_b1[j];
#pragma unroll
        for (int i = 0; i < kGateIn; ++i) z = fmaf(s_w1[j * kGateIn + i], x[i], z);
        h1[r * kGateHid + j] = __float2bfloat16_rn(fmaxf(z, 0.0f));
      }
    }
    __syncwarp();
    // layer 2 on the tensor cores, bias + ReLU + layer 3 folded into the epilogue
    float z3_lo = 0.0f, z3_hi = 0.0f;  // rows g and g+8, this lane's columns
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
      float d0 = 0.f, d1 = 0.f, d2 = 0.f, d3 = 0.f;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const int k0 = kk * 16 + 2 * t;
        const uint32_t a0 = *reinterpret_cast<const uint32_t *>(&h1[g * kGateHid + k0]);
        const uint32_t a1 = *reinterpret_cast<const uint32_t *>(&h1[(g + 8) * kGateHid + k0]);
        const uint32_t a2 = *reinterpret_cast<const uint32_t *>(&h1[g * kGateHid + k0 + 8]);
        const uint32_t a3 = *reinterpret_cast<const uint32_t *>(&h1[(g + 8) * kGateHid + k0 + 8]);
        const int n = nt * 8 + g;
        const uint32_t b0 = *reinterpret_cast<const uint32_t *>(&s_w2[n * kGateHid + k0]);
        const uint32_t b1 = *reinterpret_cast<const uint32_t *>(&s_w2[n * kGateHid + k0 + 8]);
        asm volatile(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
            "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
            : "+f"(d0), "+f"(d1), "+f"(d2), "+f"(d3)
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
      }
      const int c0 = nt * 8 + 2 * t;
      z3_lo = fmaf(s_w3[c0], fmaxf(d0 + s_b2[c0], 0.f), z3_lo);
      z3_lo = fmaf(s_w3[c0 + 1], fmaxf(d1 + s_b2[c0 + 1], 0.f), z3_lo);
      z3_hi = fmaf(s_w3[c0], fmaxf(d2 + s_b2[c0], 0.f), z3_hi);
      z3_hi = fmaf(s_w3[c0 + 1], fmaxf(d3 + s_b2[c0 + 1], 0.f), z3_hi);
    }
    z3_lo += __shfl_xor_sync(FULL, z3_lo, 1);
    z3_lo += __shfl_xor_sync(FULL, z3_lo, 2);
    z3_hi += __shfl_xor_sync(FULL, z3_hi, 1);
    z3_hi += __shfl_xor_sync(FULL, z3_hi, 2);
    if (t == 0) {
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        const int64_t v = v0 + g + 8 * half;
        if (v >= nv) continue;
        const float p = 1.0f / (1.0f + __expf(-((half ? z3_hi : z3_lo) + s_b3)));
        if (prob) prob[v] = p;
        if (skip) {
          const bool keep = p >= tau;
          skip[v] = keep ? 0 : 1;
          if (keep && evaluated) local_eval += (unsigned long long)(ptr[v + 1] - ptr[v]);
        }
      }
    }
    __syncwarp();
  }
  if (evaluated && local_eval) atomicAdd(evaluated, local_eval);
}

// ---------------------------------------------------------------------------
// Training (CUDA cores, FP32 math on BF16-rounded weights so the forward pass
// is the one inference runs).  Loss: mean over the batch of the weighted
// binary cross-entropy  w * (-(y log p + (1-y) log(1-p))).
// Activations of a batch are stored, then the weight gradients are reduced
// over the batch by a split-K outer-product kernel.

// Forward + backward through the activations, one thread per sample.
__global__ void __launch_bounds__(128) k_gate_fwd_bwd(int64_t n, const float *x, const float *y,
                                                      const float *wt, const float *params,
                                                      float *h1_out, float *h2_out,
                                                      float *dz1_out, float *dz2_out,
                                                      float *dz3_out, double *loss) {
  __shared__ float s_w1[kGateHid * kGateIn], s_b1[kGateHid], s_w2[kGateHid * kGateHid];
  __shared__ float s_b2[kGateHid], s_w3[kGateHid];
  __shared__ float s_b3;
  for (int i = threadIdx.x; i < kGateHid * kGateIn; i += blockDim.x) s_w1[i] = bf16r(params[kGateW1 + i]);
  for (int i = threadIdx.x; i < kGateHid * kGateHid; i += blockDim.x) s_w2[i] = bf16r(params[kGateW2 + i]);
  for (int i = threadIdx.x; i < kGateHid; i += blockDim.x) {
    s_b1[i] = params[kGateB1 + i];
    s_b2[i] = params[kGateB2 + i];
    s_w3[i] = bf16r(params[kGateW3 + i]);
  }
  if (threadIdx.x == 0) s_b3 = params[kGateB3];
  __syncthreads();
  double lsum = 0.0;
  for (int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; b < n;
       b += (int64_t)gridDim.x * blockDim.x) {
    float xi[kGateIn];
    for (int i = 0; i < kGateIn; ++i) xi[i] = x[b * kGateIn + i];
    float *h1 = h1_out + b * kGateHid;
    float *h2 = h2_out + b * kGateHid;
    for (int j = 0; j < kGateHid; ++j) {
      float z = s_b1[j];
      for (int i = 0; i < kGateIn; ++i) z = fmaf(s_w1[j * kGateIn + i], xi[i], z);
      h1[j] = bf16r(fmaxf(z, 0.f));  // the tensor-core layer reads BF16
    }
    float z3 = s_b3;
    for (int j = 0; j < kGateHid; ++j) {
      float z = 0.f;
      for (int k = 0; k < kGateHid; ++k) z = fmaf(s_w2[j * kGateHid + k], h1[k], z);
      const float hv = fmaxf(z + s_b2[j], 0.f);
      h2[j] = hv;
      z3 = fmaf(s_w3[j], hv, z3);
    }
    const float p = 1.0f / (1.0f + expf(-z3));
    const float yy = y[b], ww = wt[b];
    const float pc = fminf(fmaxf(p, 1e-7f), 1.0f - 1e-7f);
    lsum += (double)(ww * -(yy * logf(pc) + (1.f - yy) * logf(1.f - pc)));
    const float dz3 = ww * (p - yy) / (float)n;
    dz3_out[b] = dz3;
    float *dz2 = dz2_out + b * kGateHid;
    for (int j = 0; j < kGateHid; ++j) dz2[j] = (h2[j] > 0.f) ? dz3 * s_w3[j] : 0.f;
    float *dz1 = dz1_out + b * kGateHid;
    for (int k = 0; k < kGateHid; ++k) {
      float s = 0.f;
      for (int j = 0; j < kGateHid; ++j) s = fmaf(s_w2[j * kGateHid + k], dz2[j], s);
      dz1[k] = (h1[k] > 0.f) ? s : 0.f;
    }
  }
  atomicAdd(loss, lsum);
}

// out[m][n] += sum_b A[b][m] * B[b][n] for m < M (<= 64), n < N (<= 64); rows
// of A and B have lda / ldb floats.  B == NULL means a column of ones (bias
// gradients).  Each block reduces a chunk of the batch in shared memory tiles
// and adds its partial sums once.
__global__ void __launch_bounds__(256) k_outer_accum(int64_t nb, int M, int N, const float *A,
                                                     int lda, const float *B, int ldb,
                                                     float *out) {
  __shared__ float sA[64][64], sB[64][64];
  float acc[16];
  for (int q = 0; q < 16; ++q) acc[q] = 0.f;
  const int nout = M * N;
  const int64_t per = (nb + gridDim.x - 1) / gridDim.x;
  const int64_t b0 = (int64_t)blockIdx.x * per, b1 = min(nb, b0 + per);
  for (int64_t base = b0; base < b1; base += 64) {
    const int rows = (int)((b1 - base) < 64 ? (b1 - base) : 64);
    for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) {
      const int r = i / 64, c = i % 64;
      sA[r][c] = (r < rows && c < M) ? A[(base + r) * lda + c] : 0.f;
      sB[r][c] = (r < rows && c < N) ? (B ? B[(base + r) * ldb + c] : 1.f) : 0.f;
    }
    __syncthreads();
    for (int q = 0; q < 16; ++q) {
      const int o = threadIdx.x + q * 256;
      if (o >= nout) break;
      const int m = o / N, nn = o % N;
      float s = 0.f;
      for (int r = 0; r < rows; ++r) s = fmaf(sA[r][m], sB[r][nn], s);
      acc[q] += s;
    }
    __syncthreads();
  }
  for (int q = 0; q < 16; ++q) {
    const int o = threadIdx.x + q * 256;
    if (o >= nout) break;
    if (acc[q] != 0.f) atomicAdd(&out[o], acc[q]);
  }
}

// Adam on the FP32 master parameters.
__global__ void k_adam(int n, float *p, const float *g, float *m, float *v, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace glv
