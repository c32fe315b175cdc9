// common.cuh -- shared device helpers of libstormgpu (sm_100a).
#pragma once

#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "../../include/stormgpu.h"

namespace sg {

constexpr int kMinScore = STORMGPU_MIN_SCORE;
constexpr int kPadBytes = 1024;          // zero (codes) / 0x55 (mask) bytes around sequences
constexpr int kMaxSeeds = STORMGPU_MAX_SEEDS;
constexpr int kMaxSpan = STORMGPU_MAX_SPAN;
constexpr int kMaxPositions = 256;

// One spaced seed as the kernels see it: the offsets of its '#' symbols (seed.c:203-213).
struct SeedDev {
  int weight;
  int span;
  int n_care;
  int8_t care[kMaxSpan];      // offsets of '#', in pattern order
  int n_positions;            // 0: every read position
  int16_t positions[kMaxPositions];
};

struct SeedSet {
  int n;
  SeedDev s[kMaxSeeds];
};

// 2-bit code n of a packed sequence (codes.h:122-130); n may be negative inside padding.
__host__ __device__ __forceinline__ int code_at(const uint8_t* p, int64_t n) {
  return (p[n >> 2] >> ((n & 3) << 1)) & 3;
}

__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace sg

#define SG_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      sg_set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_));    \
      return STORMGPU_ECUDA;                                                               \
    }                                                                                      \
  } while (0)

void sg_set_error(const char* fmt, ...);
