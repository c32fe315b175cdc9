// sw_filter.cu -- the banded SW filter on packed 16-bit pairs (DPX), one candidate diagonal
// per thread over a flat candidate list, and the order-preserving compaction of the
// candidates that pass.
//
// Semantics: those of alignment_avx2__align_{hexa,octa,quad,pair} (alignment_simd.c:2613-3404)
// for one hit of W cells, as restated in filter_ref.cuh (sw_filter_one).  Here the W cells of
// one anti-diagonal step live in W/2 registers, two signed 16-bit cells each (filter_core.cuh):
//   * the per-cell score is one prmt whose selector is the difference of a read byte and a
//     genome byte (no compare, no branch);
//   * I = max(P, P of the neighbour cell, 0) with P = max(I[l-1] - ext, M[l-1] - open), and
//     M = max(M[l-2] + score, I) in one __viaddmax_s16x2; cells carry a bias of 256 so that the
//     gap subtractions are plain 32-bit adds;
//   * in the split layout used for reads of at least W codes (cells j and j + W/2 share a
//     register) the neighbour cell is in the neighbouring register, and the code streams move
//     by renaming registers; reads shorter than W use the adjacent-pair layout, which decodes
//     the packed 2-bit streams directly.
// The upper u8 saturation of the reference (adds at 255) is not reproduced: the threshold is
// at most 254, so the first cell that would saturate already has a value above it and the
// hit passes in both; cells are masked before they propagate, so an unmasked run and a
// saturating one agree on pass/fail.  Values stay below 2^15 when L * match < 32000 (checked
// by the host, which otherwise uses the plain 32-bit kernel).
#include "map_kernels.cuh"
#include "sw_filter.cuh"
#include "filter_ref.cuh"
#include "filter_core.cuh"

namespace sg {

// Candidates per thread: a block of 256 threads takes a tile of 256 * rows contiguous
// candidates (rows of 256: kFilterTile, or FilterJob.rows with a cursor).  Tiles go out in
// list order -- from a work cursor to a persistent grid (a block takes the next tile when all
// its warps are done with the last: uneven tiles balance), or by block index to a grid of one
// tile per block -- so the warps resident at any time work on neighbouring candidates: in a batch whose reads are grouped by length, an SM runs
// warps of one read length.  A grid-stride loop over a grid larger than the resident set makes
// every resident block walk the whole list instead, which mixes all lengths on every SM; on a
// 35-150 bp batch that ran the same instructions 1.48x slower, stalled on instruction fetch.
// The tile goes to the whole block, not warp by warp, for the same reason: the warps of a
// block start every tile together and stay close in the long unrolled band code (warps taking
// tiles one by one drift apart in it, which measured 5-15 % slower).
constexpr int kFilterTile = 8;  // rows of a tile unless FilterJob.rows says otherwise

// The block's tiles in list order: by block index, or with a cursor taken from it one at a
// time (all threads of the block make the same calls).  Taking the next tile ahead, to hide
// the atomic's round trip, measured no faster.
struct FilterTiles {
  unsigned long long* cursor;
  int64_t T;  // candidates per tile
  __device__ __forceinline__ int64_t first() { return cursor ? after() : (int64_t)blockIdx.x * T; }
  __device__ __forceinline__ int64_t after() {
    __shared__ unsigned long long s_tile;
    if (!cursor) return INT64_MAX;
    __syncthreads();  // every thread has read the previous tile
    if (threadIdx.x == 0) s_tile = atomicAdd(cursor, 1ull);
    __syncthreads();
    return (int64_t)s_tile * T;
  }
};

// one block's filter counters (cells, candidates, band cells) into the stats: three global
// atomics per block.  `counters` is uniform over the block.
__device__ __forceinline__ void add_filter_counters(unsigned long long* counters, unsigned long long cells,
                                                    unsigned long long cands, unsigned long long band) {
  __shared__ unsigned long long s[3];
  if (threadIdx.x == 0) { s[0] = 0; s[1] = 0; s[2] = 0; }
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) {
    cells += __shfl_xor_sync(0xffffffffu, cells, o);
    cands += __shfl_xor_sync(0xffffffffu, cands, o);
    band += __shfl_xor_sync(0xffffffffu, band, o);
  }
  if ((threadIdx.x & 31) == 0 && cands) {
    atomicAdd(&s[0], cells);
    atomicAdd(&s[1], cands);
    atomicAdd(&s[2], band);
  }
  __syncthreads();
  if (threadIdx.x == 0 && s[1]) {
    atomicAdd(&counters[2], s[0]);
    atomicAdd(&counters[5], s[1]);
    atomicAdd(&counters[6], s[2]);
  }
}

// Calls body(t) for the block's candidates t < n: with a cursor (CURSOR) tiles of `rows` rows
// taken from it one after the other, else the one tile blockIdx.x of kFilterTile rows.  One
// call site of body per instantiation (it is the long unrolled band code).  The one-tile form
// has no barrier and a constant row count, which keeps the W = 8 kernel within 64 registers
// without spilling; run through the cursor loop it measured 3 % slower.
template <bool CURSOR, class Body>
__device__ __forceinline__ void for_filter_tiles(const FilterJob& job, int64_t n, int rows, Body body) {
  if constexpr (CURSOR) {
    FilterTiles tiles{job.cursor, 256 * (int64_t)rows};
    for (int64_t base = tiles.first(); base < n; base = tiles.after())
      for (int i = 0; i < rows; ++i) {
        const int64_t t = base + i * 256 + threadIdx.x;
        if (t >= n) break;
        body(t);
      }
  } else {
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x * kFilterTile + threadIdx.x;
    for (int i = 0; i < kFilterTile; ++i) {
      const int64_t t = t0 + (int64_t)i * blockDim.x;
      if (t >= n) break;
      body(t);
    }
  }
}

// SHORT: the batch has reads shorter than W (band longer than the read), which take the
// stream-decoding variant; without them the kernel holds only the split-layout core and
// fits in 64 registers for W <= 8.  CURSOR: job.cursor is set (persistent grid).
template <int W, bool SHORT, bool CURSOR>
__global__ void __launch_bounds__(256, (W <= 8 ? 4 : 2)) filter_flat_dpx_kernel(FilterJob job) {
  const uint32_t T = (uint32_t)(job.fm & 0xff) | ((uint32_t)((256 - job.fx) & 0xff) << 8) |
                     ((uint32_t)((256 - job.fx) & 0xff) << 16) | ((uint32_t)((256 - job.fx) & 0xff) << 24);
  const uint32_t NFO = (uint32_t)(uint16_t)(-job.fo) * 0x10001u;
  uint32_t TLO, THI, NFE, CFO;  // NFE: -ext in both halves (both layouts)
  filter_split_consts(job.fm, job.fx, job.fo, job.fe, TLO, THI, NFE, CFO);
  unsigned long long cells = 0, cands = 0, band = 0;
  const int64_t n = job.n_dev ? (int64_t)*job.n_dev : job.n;
  for_filter_tiles<CURSOR>(job, n, job.rows > 0 ? job.rows : kFilterTile, [&](int64_t t) {
    const int r = job.fr[t];
    const int d = job.fd[t];
    const int L = job.lengths[r];
    const int64_t pos = (int64_t)d - job.Is;
    int mx;
    if (!SHORT || L >= W)
      mx = filter_split<W>(job.gexp, pos, job.rexp + (int64_t)r * job.rstride, L, TLO, THI, NFE, CFO);
    else
      mx = filter_dpx<W>(job.genome, pos, job.codes + (int64_t)r * job.cstride, job.cstride, L, T, NFE, NFO);
    job.flag[t] = mx > job.fthr ? 1 : 0;
    cells += (unsigned long long)(2 * W) * (unsigned long long)(L + W - 1);
    band += (unsigned long long)L * (2 * job.Is + 1);
    cands++;
  });
  if (job.counters) add_filter_counters(job.counters, cells, cands, band);
}

__global__ void expand_genome_kernel(const uint8_t* __restrict__ codes, int64_t n_codes, uint8_t* __restrict__ gexp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_codes; i += (int64_t)gridDim.x * blockDim.x)
    gexp[i] = (uint8_t)(code_at(codes, i) * 0x11);
}

void launch_expand_genome(const uint8_t* codes, int64_t n_codes, uint8_t* gexp, cudaStream_t st) {
  if (n_codes <= 0) return;
  int64_t blocks = (n_codes + 255) / 256;
  if (blocks > 148 * 64) blocks = 148 * 64;
  expand_genome_kernel<<<(unsigned)blocks, 256, 0, st>>>(codes, n_codes, gexp);
}

// one warp per read: bytes 0xC4 + c * 0x11 for the L codes, 0xC4 (code 0) after
__global__ void expand_reads_kernel(ReadsDev rd, uint8_t* __restrict__ rexp, int64_t rstride) {
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t r = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rd.n; r += nwarps) {
    const int L = rd.lengths[r];
    const uint8_t* c = rd.codes + r * rd.cstride;
    uint32_t* o = reinterpret_cast<uint32_t*>(rexp + r * rstride);
    for (int64_t w = lane; w < rstride / 4; w += 32) {
      uint32_t v = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int i = (int)(4 * w + k);
        const uint32_t b = i < L ? 0xC4u + 0x11u * (uint32_t)code_at(c, i) : 0xC4u;
        v |= b << (8 * k);
      }
      o[w] = v;
    }
  }
}

void launch_expand_reads(const ReadsDev& rd, uint8_t* rexp, int64_t rstride, cudaStream_t st) {
  if (rd.n <= 0) return;
  int64_t blocks = (rd.n + 7) / 8;
  if (blocks > 148 * 32) blocks = 148 * 32;
  expand_reads_kernel<<<(unsigned)blocks, 256, 0, st>>>(rd, rexp, rstride);
}

// Plain 32-bit variant (any score values), the restatement in map_kernels.cu.
template <bool CURSOR>
__global__ void filter_flat_scalar_kernel(FilterJob job, ScoreParams sp) {
  unsigned long long cells = 0, cands = 0, band = 0;
  const int64_t n = job.n_dev ? (int64_t)*job.n_dev : job.n;
  for_filter_tiles<CURSOR>(job, n, job.rows > 0 ? job.rows : kFilterTile, [&](int64_t t) {
    const int r = job.fr[t];
    const int L = job.lengths[r];
    job.flag[t] = sw_filter_dispatch_ext(job.W, job.genome, (int64_t)job.fd[t] - job.Is,
                                         job.codes + (int64_t)r * job.cstride, L, sp) ? 1 : 0;
    cells += (unsigned long long)(2 * job.W) * (unsigned long long)(L + job.W - 1);
    band += (unsigned long long)L * (2 * job.Is + 1);
    cands++;
  });
  if (job.counters) add_filter_counters(job.counters, cells, cands, band);
}

bool filter_dpx_ok(const ScoreParams& sp, int max_len) {
  return sp.fm <= 127 && sp.fx <= 128 && (int64_t)max_len * sp.fm < 32000 && sp.fe <= 32000 && sp.fo <= 32000;
}

// job.n: the candidates, or with job.n_dev an upper bound of them.  One tile per block, or with
// job.cursor at most the resident grid.
void launch_filter_flat_job(const FilterJob& job, const ScoreParams& sp, bool dpx, cudaStream_t st) {
  if (job.n <= 0) return;
  const int64_t tile = 256 * (int64_t)(job.cursor && job.rows > 0 ? job.rows : kFilterTile);
  const int64_t blocks = (job.n + tile - 1) / tile;
  auto grid = [&](const void* k) {
    return (unsigned)(job.cursor ? std::min<int64_t>(blocks, resident_grid_of(k, 256, 0)) : blocks);
  };
#define SG_FILTER(K, ...) K<<<grid(reinterpret_cast<const void*>(K)), 256, 0, st>>>(__VA_ARGS__)
#define SG_FILTER_W(S, C)                                                \
  switch (job.W) {                                                       \
  case 2: SG_FILTER((filter_flat_dpx_kernel<2, S, C>), job); break;      \
  case 4: SG_FILTER((filter_flat_dpx_kernel<4, S, C>), job); break;      \
  case 8: SG_FILTER((filter_flat_dpx_kernel<8, S, C>), job); break;      \
  default: SG_FILTER((filter_flat_dpx_kernel<16, S, C>), job); break;    \
  }
  const bool cur = job.cursor != nullptr, shrt = job.min_len < job.W;
  if (!dpx) {
    if (cur) SG_FILTER(filter_flat_scalar_kernel<true>, job, sp);
    else SG_FILTER(filter_flat_scalar_kernel<false>, job, sp);
  } else if (!shrt) {
    if (cur) { SG_FILTER_W(false, true) } else { SG_FILTER_W(false, false) }
  } else {
    if (cur) { SG_FILTER_W(true, true) } else { SG_FILTER_W(true, false) }
  }
#undef SG_FILTER_W
#undef SG_FILTER
}

// ------------------------------------------------------------------ compaction of passing candidates

// pass bytes -> pass bits, one word per 32 candidates (the scan then runs over words); the
// words of [n_dev, ncap) (all of them from n_dev on, when it is given) are zero
__global__ void pack_flags_kernel(int64_t ncap, const unsigned long long* __restrict__ n_dev,
                                  const uint8_t* __restrict__ flag, uint32_t* __restrict__ words) {
  const int64_t nw = (ncap + 31) / 32;
  const int64_t n = n_dev ? min(ncap, (int64_t)*n_dev) : ncap;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    const int64_t t0 = w * 32;
    if (t0 >= n) {
      words[w] = 0;
      continue;
    }
    if (t0 + 32 <= n) {
      const uint4* p = reinterpret_cast<const uint4*>(flag + t0);  // flag is 16-byte aligned, t0 a multiple of 32
      const uint4 q0 = p[0], q1 = p[1];
      const uint32_t v[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
      for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int b = 0; b < 4; ++b) bits |= ((v[k] >> (8 * b)) & 1u) << (4 * k + b);
    } else {
      for (int64_t t = t0; t < n; ++t) bits |= (uint32_t)(flag[t] & 1) << (t - t0);
    }
    words[w] = bits;
  }
}

void launch_pack_flags(int64_t ncap, const unsigned long long* n_dev, const uint8_t* flag, uint32_t* words,
                       cudaStream_t st) {
  if (ncap <= 0) return;
  int64_t blocks = ((ncap + 31) / 32 + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  pack_flags_kernel<<<(unsigned)blocks, 256, 0, st>>>(ncap, n_dev, flag, words);
}

// passing candidates, in order, into (p_read, p_diag): one thread per word of pass bits
// (slots from pcap on are not written)
__global__ void compact_kernel(int64_t nwords, const uint32_t* __restrict__ flag, const int64_t* __restrict__ woff,
                               const int32_t* __restrict__ fr, const int32_t* __restrict__ fd,
                               int32_t* __restrict__ p_read, int32_t* __restrict__ p_diag, int64_t pcap) {
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t m = flag[w];
    if (!m) continue;
    int64_t o = woff[w];
    while (m && o < pcap) {
      const int64_t t = w * 32 + (__ffs(m) - 1);
      p_read[o] = fr[t];
      p_diag[o] = fd[t];
      ++o;
      m &= m - 1;
    }
  }
}

__global__ void slot_bounds_kernel(int64_t npass, const int64_t* __restrict__ npass_dev,
                                   const int32_t* __restrict__ p_read, int32_t* __restrict__ pstart,
                                   int32_t* __restrict__ pcount) {
  if (npass_dev) npass = *npass_dev;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < npass; s += (int64_t)gridDim.x * blockDim.x) {
    const int r = p_read[s];
    if (s == 0 || p_read[s - 1] != r) pstart[r] = (int32_t)s;
  }
}

__global__ void slot_count_kernel(int64_t npass, const int64_t* __restrict__ npass_dev,
                                  const int32_t* __restrict__ p_read, const int32_t* __restrict__ pstart,
                                  int32_t* __restrict__ pcount) {
  if (npass_dev) npass = *npass_dev;
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < npass; s += (int64_t)gridDim.x * blockDim.x) {
    const int r = p_read[s];
    if (s == npass - 1 || p_read[s + 1] != r) pcount[r] = (int32_t)(s - pstart[r] + 1);
  }
}

void launch_compact(int64_t nwords, const uint32_t* flag, const int64_t* woff, const int32_t* fr, const int32_t* fd,
                    int32_t* p_read, int32_t* p_diag, int64_t pcap, cudaStream_t st) {
  if (nwords <= 0) return;
  int64_t blocks = (nwords + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  compact_kernel<<<(unsigned)blocks, 256, 0, st>>>(nwords, flag, woff, fr, fd, p_read, p_diag, pcap);
}

void launch_slot_bounds(int64_t npass, const int64_t* npass_dev, const int32_t* p_read, int32_t* pstart,
                        int32_t* pcount, cudaStream_t st) {
  if (npass <= 0) return;
  int64_t blocks = (npass + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  slot_bounds_kernel<<<(unsigned)blocks, 256, 0, st>>>(npass, npass_dev, p_read, pstart, pcount);
  slot_count_kernel<<<(unsigned)blocks, 256, 0, st>>>(npass, npass_dev, p_read, pstart, pcount);
}

}  // namespace sg
