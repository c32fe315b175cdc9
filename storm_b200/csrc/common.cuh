// common.cuh -- shared device helpers of libstormgpu (sm_100a).
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <tuple>
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

// Blocks of `threads` threads of kernel k that fit on the current device at once (the grid of
// a persistent launch), at least one; queried once per (kernel, device, threads, smem).
inline int64_t resident_grid_of(const void* k, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, int, size_t>, int64_t> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_tuple(k, dev, threads, smem);
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int sms = 0, per = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, threads, smem);
  const int64_t g = (int64_t)(per > 0 ? per : 1) * (sms > 0 ? sms : 1);
  cache[key] = g;
  return g;
}
// Allows kernel k up to `bytes` of dynamic shared memory on the current device (the attribute
// is per device: set once for each device a process launches on).
inline void set_smem_attribute_once(const void* k, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, bool> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  bool& d = done[std::make_pair(k, dev)];
  if (!d) {
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    d = true;
  }
}

template <class K>
inline int64_t resident_grid(K* k, int threads, size_t smem = 0) {
  return resident_grid_of(reinterpret_cast<const void*>(k), threads, smem);
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
