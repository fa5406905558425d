// Shared device/host helpers for the B200 Louvain engine.
#pragma once

#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "grappolo_b200.h"

namespace glv {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kMaxColors = 4096;  // Coloring/coloringUtils.h MaxDegree

// Degree bins of the local-moving sweep.  A vertex's bin is fixed by its row
// length; each bin has its own work decomposition.
enum Bin : int {
  BIN_G4 = 0,      // degree 0..4      : 4 lanes per vertex, registers only
  BIN_G8 = 1,      // 5..8             : 8 lanes per vertex
  BIN_G16 = 2,     // 9..16            : 16 lanes per vertex
  BIN_G32 = 3,     // 17..32           : one warp per vertex
  BIN_WARP = 4,    // 33..127          : one warp, shared-memory table (<= 256 slots)
  BIN_T128 = 5,    // 128..511         : 128-thread team, shared table (<= 1024 slots)
  BIN_T256 = 6,    // 512..1023        : 256-thread team, shared table (<= 2048 slots)
  BIN_BLOCK = 7,   // 1024..block_max  : 512-thread block, shared table (<= 8192 slots)
  BIN_HUB = 8,     // > block_max      : whole grid per row, global-memory table
  NBINS = 9
};

struct BinLimits {
  int warp_max;   // upper degree of BIN_WARP
  int block_max;  // upper degree of BIN_BLOCK
};

__host__ __device__ inline int degree_bin(int64_t deg, BinLimits lim) {
  if (deg <= 4) return BIN_G4;
  if (deg <= 8) return BIN_G8;
  if (deg <= 16) return BIN_G16;
  if (deg <= 32) return BIN_G32;
  if (deg <= lim.warp_max) return BIN_WARP;
  if (deg > lim.block_max) return BIN_HUB;
  if (deg <= 511) return BIN_T128;
  if (deg <= 1023) return BIN_T256;
  return BIN_BLOCK;
}

// Smallest degree whose bin is `bin` (bins above BIN_G4).
__host__ __device__ inline int64_t first_degree_of_bin(int bin, BinLimits lim) {
  switch (bin) {
    case BIN_G8: return 5;
    case BIN_G16: return 9;
    case BIN_G32: return 17;
    case BIN_WARP: return 33;
    case BIN_T128: return (int64_t)lim.warp_max + 1;
    case BIN_T256: return 512;
    case BIN_BLOCK: return 1024;
    case BIN_HUB: return (int64_t)lim.block_max + 1;
    default: return 0;
  }
}

__host__ __device__ inline uint32_t next_pow2(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

// Hash-table capacity for a row of `deg` entries: distinct keys <= deg + 1.
__host__ __device__ inline uint32_t table_cap(int64_t deg) {
  return next_pow2((uint32_t)(2 * (deg + 1)));
}

// Table slot of a community id.  The product's high bits are folded into the
// low ones: the low bits of key * odd depend only on the key's low bits, and
// vertex ids of R-MAT-like graphs share long runs of zero bits, which would
// pile them into a few slots.
__device__ __forceinline__ uint32_t hash_slot(int32_t key, uint32_t mask) {
  const uint32_t h = (uint32_t)key * 0x9E3779B1u;
  return (h ^ (h >> 15)) & mask;
}

// 32-bit integer mixer (Wang/Jenkins style) used for colouring priorities.
__host__ __device__ inline uint32_t mix32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352dU;
  x ^= x >> 15; x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

// FP64 gain exactly as Utility/utilityClusteringFunctions.cpp:243 evaluates
// it, 2*(eiy - eix) - 2*degree*(ay - ax)*constant, left to right, every
// operation rounded on its own (no FMA contraction).
__device__ __forceinline__ double louvain_gain(double eiy, double eix, double degree, double ay,
                                               double ax, double constant) {
  double t1 = __dmul_rn(2.0, __dsub_rn(eiy, eix));
  double t2 = __dmul_rn(__dmul_rn(__dmul_rn(2.0, degree), __dsub_rn(ay, ax)), constant);
  return __dsub_rn(t1, t2);
}

// (gain, id) arg-max with the reference's tie rule: larger gain wins, equal
// gain goes to the lower community id.  Empty candidates carry gain <= 0 and
// id INT32_MAX and never beat the "stay" default.
__device__ __forceinline__ bool better(double g1, int c1, double g0, int c0) {
  return (g1 > g0) || (g1 == g0 && c1 < c0);
}

}  // namespace glv

#define GLV_CUDA_TRY(expr)                                                        \
  do {                                                                            \
    cudaError_t err_ = (expr);                                                    \
    if (err_ != cudaSuccess) {                                                    \
      fprintf(stderr, "grappolo_b200: CUDA error %s at %s:%d: %s\n",              \
              cudaGetErrorName(err_), __FILE__, __LINE__, cudaGetErrorString(err_)); \
      return err_ == cudaErrorMemoryAllocation ? GLV_ERR_OOM : GLV_ERR_CUDA;     \
    }                                                                             \
  } while (0)
