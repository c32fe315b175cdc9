// scan.cuh -- device-wide exclusive prefix sum (reduce / scan / down-sweep, recursive on the
// block totals).  Used to turn per-read and per-key counts into offsets.
#pragma once

#include "common.cuh"

namespace sg {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

template <typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* smem_warp, T* total) {
  // smem_warp: >= 32 entries
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) smem_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    T w = lane < nw ? smem_warp[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    if (lane < nw) smem_warp[lane] = w;
  }
  __syncthreads();
  T before = warp ? smem_warp[warp - 1] : T(0);
  if (total) *total = smem_warp[(blockDim.x >> 5) - 1];
  T r = before + x - v;
  __syncthreads();
  return r;
}

template <typename Tin, typename Tout>
__global__ void scan_reduce_kernel(const Tin* __restrict__ in, int64_t n, Tout* __restrict__ sums) {
  __shared__ Tout sw[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile;
  Tout acc = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + (int64_t)k * kScanThreads + threadIdx.x;
    if (i < n) acc += (Tout)in[i];
  }
  Tout tot;
  block_excl_scan<Tout>(acc, sw, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// Exclusive scan of one tile per block; block b adds offs[b] (if offs != nullptr).
template <typename Tin, typename Tout>
__global__ void scan_tile_kernel(const Tin* __restrict__ in, int64_t n, Tout* __restrict__ out,
                                 const Tout* __restrict__ offs, Tout* __restrict__ total_out) {
  __shared__ Tout sw[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  Tout v[kScanItems];
  Tout acc = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + k;
    v[k] = (i < n) ? (Tout)in[i] : Tout(0);
    acc += v[k];
  }
  Tout tot;
  Tout run = block_excl_scan<Tout>(acc, sw, &tot);
  if (offs) run += offs[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int64_t i = base + k;
    if (i < n) out[i] = run;
    run += v[k];
  }
  if (total_out && threadIdx.x == blockDim.x - 1 && blockIdx.x == gridDim.x - 1) *total_out = run;
}

// out[i] = sum(in[0..i)); *total (device pointer, may be null) = sum(in[0..n)).
// `tmp` must hold scan_tmp_elems(n) elements of Tout.
inline int64_t scan_tmp_elems(int64_t n) {
  int64_t t = 0;
  while (n > kScanTile) {
    n = (n + kScanTile - 1) / kScanTile;
    t += n + 1;
  }
  return t + 1;
}

// kernel launches of one exclusive_scan of n elements
inline int scan_launches(int64_t n) {
  return n <= 0 ? 0 : n <= kScanTile ? 1 : 2 + scan_launches((n + kScanTile - 1) / kScanTile);
}

template <typename Tin, typename Tout>
void exclusive_scan(const Tin* in, Tout* out, int64_t n, Tout* total, Tout* tmp, cudaStream_t st) {
  if (n <= 0) {
    if (total) cudaMemsetAsync(total, 0, sizeof(Tout), st);
    return;
  }
  if (n <= kScanTile) {
    scan_tile_kernel<Tin, Tout><<<1, kScanThreads, 0, st>>>(in, n, out, nullptr, total);
    return;
  }
  int64_t nb = (n + kScanTile - 1) / kScanTile;
  Tout* sums = tmp;
  Tout* rest = tmp + nb + 1;
  scan_reduce_kernel<Tin, Tout><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, sums);
  exclusive_scan<Tout, Tout>(sums, sums, nb, total, rest, st);
  scan_tile_kernel<Tin, Tout><<<(unsigned)nb, kScanThreads, 0, st>>>(in, n, out, sums, nullptr);
}

}  // namespace sg
