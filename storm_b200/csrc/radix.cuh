// radix.cuh -- stable LSD radix sort of (32-bit key, 32-bit value) pairs, 8-bit digits.
//
// Per pass: (1) per-tile digit histograms, stored digit-major so that (2) one exclusive scan
// gives every (digit, tile) its output offset, then (3) each tile re-reads its items and
// scatters them, ranking equal digits in input order with __match_any_sync inside a warp and
// per-(warp, digit) offsets across the warps of the tile, through shared memory so that the
// writes of one digit are contiguous.  Stability is what the
// seed index needs: positions are generated in increasing order and must stay so per key.
#pragma once

#include "scan.cuh"

namespace sg {

constexpr int kRadixBits = 8;
constexpr int kRadixBins = 1 << kRadixBits;
constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;

static __global__ void radix_hist_kernel(const uint32_t* __restrict__ keys, int64_t n, int shift,
                                  uint32_t* __restrict__ hist, int ntiles) {
  __shared__ uint32_t h[kRadixBins];
  for (int i = threadIdx.x; i < kRadixBins; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kSortTile;
  for (int r = 0; r < kSortRounds; ++r) {
    int64_t i = base + (int64_t)r * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & (kRadixBins - 1)], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < kRadixBins; d += blockDim.x)
    hist[(int64_t)d * ntiles + blockIdx.x] = h[d];
}

// Each warp owns a contiguous eighth of the tile: 16 rounds of 32 items, held in registers.
// The warps count their digits apart (per-warp counters in shared memory); one block-wide pass
// turns the counts into tile-local offsets (digit-major, warps in order within a digit); the
// warps place their items there in input order, so that the tile sits in shared memory sorted
// by digit, and the block writes it out in that order: each digit's items of the tile go to
// consecutive addresses (whole sectors), not one item per sector.
static __global__ void __launch_bounds__(kSortThreads, 3) radix_scatter_kernel(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, int64_t n, int shift,
    const uint32_t* __restrict__ offs, int ntiles, uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out) {
  constexpr int NW = kSortThreads / 32;
  constexpr int PER_WARP = kSortTile / NW;  // = 32 * kSortRounds
  static_assert(kSortThreads == kRadixBins, "one thread per digit in the offset pass");
  __shared__ uint32_t wc[NW][kRadixBins];
  __shared__ uint32_t lstart[kRadixBins], gbase[kRadixBins], wtot[NW];
  __shared__ uint32_t sk[kSortTile], sv[kSortTile];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int64_t tile0 = (int64_t)blockIdx.x * kSortTile;
  const int64_t base = tile0 + (int64_t)warp * PER_WARP + lane;
  uint32_t k[kSortRounds], v[kSortRounds];
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {
    const int64_t i = base + 32 * r;
    k[r] = i < n ? keys_in[i] : 0u;
    v[r] = i < n ? vals_in[i] : 0u;
  }
  for (int d = lane; d < kRadixBins; d += 32) wc[warp][d] = 0;
  __syncwarp();
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {  // the warp's digit counts
    const bool valid = base + 32 * r < n;
    const int d = valid ? (int)((k[r] >> shift) & (kRadixBins - 1)) : kRadixBins;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    if (valid && __popc(peers & lt) == 0) wc[warp][d] += (uint32_t)__popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {  // thread d: the tile's count of digit d -> its tile-local start (block scan), per-warp offsets
    const int d = threadIdx.x;
    uint32_t c = 0;
#pragma unroll
    for (int w = 0; w < NW; ++w) c += wc[w][d];
    uint32_t x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += t;
    }
    if (lane == 31) wtot[warp] = x;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += wtot[w];
    uint32_t o = before + x - c;
    lstart[d] = o;
    gbase[d] = offs[(int64_t)d * ntiles + blockIdx.x];
#pragma unroll
    for (int w = 0; w < NW; ++w) {
      const uint32_t cw = wc[w][d];
      wc[w][d] = o;
      o += cw;
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kSortRounds; ++r) {  // into shared memory, sorted by digit, stable
    const bool valid = base + 32 * r < n;
    const int d = valid ? (int)((k[r] >> shift) & (kRadixBins - 1)) : kRadixBins;
    const unsigned peers = __match_any_sync(0xffffffffu, d);
    const int rank = __popc(peers & lt);
    uint32_t at = 0;
    if (valid) at = wc[warp][d];
    __syncwarp();
    if (valid) {
      sk[at + rank] = k[r];
      sv[at + rank] = v[r];
      if (rank == 0) wc[warp][d] = at + (uint32_t)__popc(peers);
    }
    __syncwarp();
  }
  __syncthreads();
  const int tn = (int)(n - tile0 < kSortTile ? n - tile0 : kSortTile);
  for (int j = threadIdx.x; j < tn; j += kSortThreads) {  // out in digit order
    const uint32_t key = sk[j];
    const int d = (int)((key >> shift) & (kRadixBins - 1));
    const uint32_t dst = gbase[d] + (uint32_t)j - lstart[d];
    keys_out[dst] = key;
    vals_out[dst] = sv[j];
  }
}

inline int64_t radix_tmp_bytes(int64_t n) {
  int64_t ntiles = (n + kSortTile - 1) / kSortTile;
  int64_t h = ntiles * kRadixBins;
  return (2 * h + scan_tmp_elems(h) + 16) * (int64_t)sizeof(uint32_t);
}

// Sort n pairs by the low `bits` bits of the keys.  Result in (k0, v0) if the number of passes
// is even, else in (k1, v1); returns 0 or 1 accordingly.  n < 2^32.
inline int radix_sort_pairs(uint32_t* k0, uint32_t* v0, uint32_t* k1, uint32_t* v1, int64_t n,
                            int bits, void* tmp, cudaStream_t st) {
  if (n <= 0) return 0;
  const int ntiles = (int)((n + kSortTile - 1) / kSortTile);
  const int64_t h = (int64_t)ntiles * kRadixBins;
  uint32_t* hist = (uint32_t*)tmp;
  uint32_t* offs = hist + h;
  uint32_t* stmp = offs + h;
  int cur = 0;
  for (int shift = 0; shift < bits; shift += kRadixBits) {
    uint32_t *ki = cur ? k1 : k0, *vi = cur ? v1 : v0, *ko = cur ? k0 : k1, *vo = cur ? v0 : v1;
    radix_hist_kernel<<<ntiles, kSortThreads, 0, st>>>(ki, n, shift, hist, ntiles);
    exclusive_scan<uint32_t, uint32_t>(hist, offs, h, (uint32_t*)nullptr, stmp, st);
    radix_scatter_kernel<<<ntiles, kSortThreads, 0, st>>>(ki, vi, n, shift, offs, ntiles, ko, vo);
    cur ^= 1;
  }
  return cur;
}

}  // namespace sg
