// gather.cu -- hit gather: for one read-strand, every (seed, read position) key's CSR list
// (index.c:212-241) shifted by the read position, merged into the ascending, de-duplicated
// diagonals that process_read's heap yields (run.c:577-698): a diagonal is kept iff it is
// strictly greater than the previous one in sorted order, the previous of the first being -I
// (run.c:617, :648, :697).
//
// One warp per read: keys computed from the packed read, CSR offsets read from the
// (L2-resident) key table, positions gathered straight into the warp's shared memory, bitonic
// sort there, de-duplication by ballot, and the surviving diagonals appended to the flat
// candidate list (reads contiguous, diagonals ascending within a read).  Every lane looks up
// several (seed, position) keys before any result is used, so that a read costs two memory
// latencies (key table, positions) rather than two per seed.  Up to 32 positions are sorted in
// registers; more are first reduced to distinct values (warp_dedupe), then bucket-sorted
// (bucket_sort_emit).  Reads with more index positions than a warp can hold go to a
// block-per-read kernel (shared memory up to 32768 positions) and, beyond that, to a
// global-memory variant run one read at a time.
#include <type_traits>

#include "gather.cuh"

namespace sg {


// Seed key at read position rp; codes beyond the read's end read as 0 (seed.c:203-213).
__device__ __forceinline__ uint32_t read_key(const SeedDev& s, const uint8_t* rd, int L, int rp) {
  uint32_t key = 0;
  for (int c = 0; c < s.n_care; ++c) {
    const int p = rp + s.care[c];
    key = (key << 2) | (uint32_t)(p < L ? code_at(rd, p) : 0);
  }
  return key;
}

// The same key from a register window: codes rp .. rp + 31 of a read staged in shared memory
// (4-byte aligned, readable for 12 bytes from word rp / 16), codes from L on masked to 0;
// one shift and mask per care position instead of a shared-memory load.  Seeds of span <= 32.
__device__ __forceinline__ uint32_t read_key_window(const SeedDev& s, const uint8_t* rd, int L, int rp) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(rd) + (rp >> 4);
  const uint64_t lo = (uint64_t)w[0] | ((uint64_t)w[1] << 32);
  const int sh = 2 * (rp & 15);
  uint64_t win = sh ? (lo >> sh) | ((uint64_t)w[2] << (64 - sh)) : lo;  // code rp + k at bits 2k
  const int lim = L - rp;
  if (lim < 32) win &= (1ull << (2 * lim)) - 1ull;
  uint32_t key = 0;
  for (int c = 0; c < s.n_care; ++c) key = (key << 2) | (uint32_t)((win >> (2 * s.care[c])) & 3u);
  return key;
}

__device__ __forceinline__ int seed_npos(const SeedDev& s, int L) {
  return s.n_positions ? s.n_positions : (L - s.span + 1 > 0 ? L - s.span + 1 : 0);
}

// (index offset, count, read position) of item t of seed si
__device__ __forceinline__ void seed_item(const SeedSet& gs, const IndexView& ix, int si, int t, const uint8_t* read,
                                          int L, int& a, int& cnt, int& rp) {
  const SeedDev& s = gs.s[si];
  a = 0; cnt = 0; rp = 0;
  if (t >= seed_npos(s, L)) return;
  rp = s.n_positions ? s.positions[t] : t;
  if (rp < 0 || rp >= L) return;
  const uint32_t key = read_key(s, read, L, rp);
  a = __ldg(ix.first[si] + key);
  cnt = __ldg(ix.first[si] + key + 1) - a;
}

// (index offset, count, read position) of position t of seed s, with that seed's key table;
// `read` is staged in shared memory (see read_key_window)
__device__ __forceinline__ void item_lookup(const int32_t* __restrict__ first, const SeedDev& s, int t,
                                            const uint8_t* read, int L, int& a, int& cnt, int& rp) {
  a = 0; cnt = 0; rp = 0;
  if (t >= seed_npos(s, L)) return;
  rp = s.n_positions ? s.positions[t] : t;
  if (rp < 0 || rp >= L) return;
  const uint32_t key = s.span <= 32 ? read_key_window(s, read, L, rp) : read_key(s, read, L, rp);
  a = __ldg(first + key);
  cnt = __ldg(first + key + 1) - a;
}

__device__ __forceinline__ void warp_bitonic(int32_t* s, int P) {
  const int lane = threadIdx.x & 31;
  for (int k = 2; k <= P; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < P; i += 32) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const int32_t a = s[i], b = s[ixj];
          if ((a > b) == ((i & k) == 0)) { s[i] = b; s[ixj] = a; }
        }
      }
      __syncwarp();
    }
}

// sorted s[0..H) -> accepted diagonals appended to the flat list (one warp)
__device__ __forceinline__ void warp_emit(int32_t* s, int H, int I, int r, const GatherOut& go) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  int U = 0;
  for (int t0 = 0; t0 < H; t0 += 32) {
    const int t = t0 + lane;
    const int32_t v = t < H ? s[t] : 0;
    const int32_t prev = t == 0 ? -I : (t < H ? s[t - 1] : 0);
    const bool keep = t < H && v > prev;
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    __syncwarp();
    if (keep) s[U + __popc(m & lt)] = v;  // compaction in place (writes trail reads)
    U += __popc(m);
    __syncwarp();
  }
  unsigned long long base = 0;
  if (lane == 0 && U) base = atomicAdd(&go.counters[7], (unsigned long long)U);
  base = __shfl_sync(0xffffffffu, base, 0);
  if ((int64_t)(base + U) > go.cap) {
    if (lane == 0) atomicExch(&go.counters[8], 1ull);
    return;
  }
  for (int k = lane; k < U; k += 32) {
    go.fr[base + k] = r;
    go.fd[base + k] = s[k];
  }
}

// Bitonic sort of 32*E values held E per lane (value k of lane l is element k*32 + l):
// partners 32 or more apart are in the same lane (register compare-exchange), closer ones are
// exchanged with __shfl_xor_sync.
template <int E>
__device__ __forceinline__ void reg_bitonic(int32_t (&v)[E]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int kk = 2; kk <= 32 * E; kk <<= 1) {
#pragma unroll
    for (int j = kk >> 1; j > 0; j >>= 1) {
      if (j >= 32) {
#pragma unroll
        for (int k = 0; k < E; ++k) {
          const int k2 = k ^ (j >> 5);
          if (k2 > k) {
            const bool up = ((k * 32 + lane) & kk) == 0;
            const int32_t a = v[k], b = v[k2];
            const bool sw = (a > b) == up;
            v[k] = sw ? b : a;
            v[k2] = sw ? a : b;
          }
        }
      } else {
#pragma unroll
        for (int k = 0; k < E; ++k) {
          const int32_t o = __shfl_xor_sync(0xffffffffu, v[k], j);
          const bool up = ((k * 32 + lane) & kk) == 0;
          const bool lower = (lane & j) == 0;
          v[k] = (lower == up) ? min(v[k], o) : max(v[k], o);
        }
      }
    }
  }
}

// accepted diagonals of the sorted register array (first H valid) -> flat list
template <int E>
__device__ __forceinline__ void reg_emit(const int32_t (&v)[E], int H, int I, int r, const GatherOut& go) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  unsigned m[E];
  int U = 0;
#pragma unroll
  for (int k = 0; k < E; ++k) {
    const int32_t up = __shfl_up_sync(0xffffffffu, v[k], 1);
    const int32_t last = __shfl_sync(0xffffffffu, k ? v[k > 0 ? k - 1 : 0] : 0, 31);
    const int32_t prev = lane ? up : (k ? last : -I);
    const bool keep = (k * 32 + lane) < H && v[k] > prev;
    m[k] = __ballot_sync(0xffffffffu, keep);
    U += __popc(m[k]);
  }
  unsigned long long base = 0;
  if (lane == 0 && U) base = atomicAdd(&go.counters[7], (unsigned long long)U);
  base = __shfl_sync(0xffffffffu, base, 0);
  if ((int64_t)(base + U) > go.cap) {
    if (lane == 0) atomicExch(&go.counters[8], 1ull);
    return;
  }
  int off = 0;
#pragma unroll
  for (int k = 0; k < E; ++k) {
    if ((m[k] >> lane) & 1u) {
      const int64_t o = (int64_t)base + off + __popc(m[k] & lt);
      go.fr[o] = r;
      go.fd[o] = v[k];
    }
    off += __popc(m[k]);
  }
}

template <int E>
__device__ __forceinline__ void sort_emit_regs(const int32_t* s, int H, int I, int r, const GatherOut& go) {
  const int lane = threadIdx.x & 31;
  int32_t v[E];
#pragma unroll
  for (int k = 0; k < E; ++k) {
    const int i = k * 32 + lane;
    v[k] = i < H ? s[i] : 0x7fffffff;
  }
  reg_bitonic<E>(v);
  reg_emit<E>(v, H, I, r, go);
}

// Drop repeated values from a[0..H) (one warp), keeping one of each, compacted to the front
// of a (order not kept); tab[0..cap), cap >= H, is the open-addressing set.  The diagonal a read
// truly maps to comes once per (seed, position) that hits it, so this removes the one large
// group of equal values before the sort.  Returns the number of distinct values.
constexpr int32_t kEmptySlot = 0x7fffffff;  // no diagonal (position - read position) reaches it
__device__ __forceinline__ int warp_dedupe(int32_t* a, int H, int32_t* tab, int cap) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (int i = lane; i < cap; i += 32) tab[i] = kEmptySlot;
  __syncwarp();
  int U = 0;
  for (int i0 = 0; i0 < H; i0 += 32) {
    const int i = i0 + lane;
    bool keep = false;
    int32_t v = 0;
    if (i < H) {
      v = a[i];
      uint32_t h = __umulhi((uint32_t)v * 0x9E3779B1u, (uint32_t)cap);
      for (;;) {
        const int32_t old = atomicCAS(&tab[h], kEmptySlot, v);
        if (old == kEmptySlot) { keep = true; break; }
        if (old == v) break;
        h = h + 1 == (uint32_t)cap ? 0u : h + 1;
      }
    }
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    if (keep) a[U + __popc(m & lt)] = v;  // writes trail the reads of this and later chunks
    U += __popc(m);
    __syncwarp();
  }
  return U;
}

// Sort a[0..H) (one warp) into b[0..H) and emit: 32 buckets of equal width over [min, max]
// (so that bucket order is value order), counted with shared atomics,
// scattered to b, then every lane insertion-sorts its own bucket.  A bucket holding more than
// 64 values (clustered diagonals) falls back to the bitonic sort of a, which needs room for
// the next power of two of H from a on (a and b are adjacent).
__device__ __forceinline__ void bucket_sort_emit(int32_t* a, int32_t* b, int32_t* hist, int H, int I, int r,
                                                 const GatherOut& go) {
  const int lane = threadIdx.x & 31;
  int32_t vmin = 0x7fffffff, vmax = (int32_t)0x80000000;
  for (int i = lane; i < H; i += 32) {
    const int32_t v = a[i];
    vmin = min(vmin, v);
    vmax = max(vmax, v);
  }
  vmin = __reduce_min_sync(0xffffffffu, vmin);
  vmax = __reduce_max_sync(0xffffffffu, vmax);
  // bucket = floor(32 * (v - min) / (range + 1)) as a multiply-high: monotone, all 32 buckets used
  const uint32_t range = (uint32_t)vmax - (uint32_t)vmin;
  const uint32_t mul = range < 32u ? 0u : (uint32_t)((32ull << 32) / ((uint64_t)range + 1ull));
  auto bucket = [&](int32_t v) -> int {
    const uint32_t x = (uint32_t)v - (uint32_t)vmin;
    return range < 32u ? (int)x : (int)__umulhi(x, mul);
  };
  hist[lane] = 0;
  __syncwarp();
  for (int i = lane; i < H; i += 32) atomicAdd(&hist[bucket(a[i])], 1);
  __syncwarp();
  const int c = hist[lane];
  const int incl = warp_incl_scan(c);
  const int base = incl - c;
  if (__reduce_max_sync(0xffffffffu, (unsigned)c) > 64u) {
    int P = 1;
    while (P < H) P <<= 1;
    for (int i = H + lane; i < P; i += 32) a[i] = 0x7fffffff;
    __syncwarp();
    warp_bitonic(a, P);
    warp_emit(a, H, I, r, go);
    return;
  }
  __syncwarp();
  hist[lane] = base;
  __syncwarp();
  for (int i = lane; i < H; i += 32) {
    const int32_t v = a[i];
    b[atomicAdd(&hist[bucket(v)], 1)] = v;
  }
  __syncwarp();
  for (int x = 1; x < c; ++x) {
    const int32_t t = b[base + x];
    int y = x - 1;
    while (y >= 0 && b[base + y] > t) {
      b[base + y + 1] = b[base + y];
      --y;
    }
    b[base + y + 1] = t;
  }
  __syncwarp();
  warp_emit(b, H, I, r, go);
}

constexpr int kGWarps = 4;
// Reads per steal (GatherOut.reads_per_steal, 4 by default): the grid is the resident set, and
// every warp takes the next reads_per_steal reads (in the order of rd.order, or of the batch) from a work cursor until none is left, so
// reads with many index positions balance out, and warps append their candidates in close to
// read order: a batch whose reads are grouped by length gives a candidate list grouped by
// length, which the filter needs to keep one read length per SM.
constexpr int kReadBytes = STORMGPU_MAX_READ_LEN / 4 + 16;

constexpr int kItems = 4;  // (seed, position) items per lane and round: 128 key lookups in flight per warp

__global__ void __launch_bounds__(kGWarps * 32, 8) gather_fused_kernel(ReadsDev rd, IndexView ix, int I, GatherOut go,
                                                                   const __grid_constant__ SeedSet gs) {
  extern __shared__ int32_t sm[];  // per warp 2 * cap: gathered positions, then the set / sorted copy
  __shared__ int32_t shist[kGWarps][32];
  __shared__ int32_t soff[kGWarps][kMaxSeeds + 1];  // first item of every seed, for the current read
  __shared__ const int32_t* s_first[kMaxSeeds];
  __shared__ const int32_t* s_map[kMaxSeeds];
  __shared__ __align__(16) uint8_t srd[kGWarps][kReadBytes];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int nseeds = gs.n;
  if (threadIdx.x < nseeds) {
    s_first[threadIdx.x] = ix.first[threadIdx.x];
    s_map[threadIdx.x] = ix.map[threadIdx.x];
  }
  __syncthreads();
  const int cap = go.warp_cap;
  int32_t* s = sm + (size_t)w * 2 * cap;
  int32_t* so = soff[w];
  uint8_t* rs = srd[w];
  unsigned long long lookups = 0, positions = 0;
  for (;;) {
  unsigned long long k0 = 0;
  if (lane == 0) k0 = atomicAdd(go.cursor, (unsigned long long)go.reads_per_steal);
  k0 = __shfl_sync(0xffffffffu, k0, 0);
  if ((int64_t)k0 >= rd.n) break;
  const int64_t kend = (int64_t)k0 + go.reads_per_steal < rd.n ? (int64_t)k0 + go.reads_per_steal : rd.n;
  for (int64_t kr = (int64_t)k0; kr < kend; ++kr) {
    const int64_t r = rd.order ? (int64_t)rd.order[kr] : kr;
    const int L = rd.lengths[r];
    {  // the read's packed codes into shared memory, and the item offsets of the seeds
      const uint8_t* src = rd.codes + r * rd.cstride;
      const int nb = (L + 3) >> 2;
      for (int b = lane; b < nb; b += 32) rs[b] = src[b];
      const int np = lane < nseeds ? seed_npos(gs.s[lane], L) : 0;
      const int incl = warp_incl_scan(np);
      if (lane <= nseeds) so[lane] = incl - np;
      __syncwarp();
    }
    const uint8_t* read = rs;
    const int T = so[nseeds];
    int H = 0;
    // a read with more positions than the warp holds is only counted from there on and goes to
    // the block kernel with its count (its lookups and positions are counted there)
    for (int r0 = 0; r0 < T; r0 += 32 * kItems) {
      // every lane looks up its items (all key-table loads in flight together) ...
      int a[kItems], cnt[kItems], rp[kItems], sid[kItems];
#pragma unroll
      for (int m = 0; m < kItems; ++m) {
        const int it = r0 + m * 32 + lane;
        int si = 0;
        if (it < T)
          while (it >= so[si + 1]) ++si;
        sid[m] = si;
        item_lookup(s_first[si], gs.s[si], it < T ? it - so[si] : 0x40000000, read, L, a[m], cnt[m], rp[m]);
      }
      // ... then one scan places all of them, and the position loads go out together
      int tot = 0;
#pragma unroll
      for (int m = 0; m < kItems; ++m) tot += cnt[m];
      const int incl = warp_incl_scan(tot);
      int dst[kItems];
      dst[0] = H + incl - tot;
#pragma unroll
      for (int m = 1; m < kItems; ++m) dst[m] = dst[m - 1] + cnt[m - 1];
      H += __shfl_sync(0xffffffffu, incl, 31);
      if (H > cap) continue;  // uniform over the warp: counting only
#pragma unroll
      for (int m = 0; m < kItems; ++m) {
        if (cnt[m] <= 8) {
          const int32_t* mp = s_map[sid[m]] + a[m];
          int32_t tv[8];
#pragma unroll
          for (int u = 0; u < 8; ++u) tv[u] = u < cnt[m] ? __ldg(mp + u) : 0;
#pragma unroll
          for (int u = 0; u < 8; ++u)
            if (u < cnt[m] && dst[m] + u < cap) s[dst[m] + u] = tv[u] - rp[m];
        }
      }
#pragma unroll
      for (int m = 0; m < kItems; ++m) {  // long position lists: the whole warp copies each
        unsigned bm = __ballot_sync(0xffffffffu, cnt[m] > 8);
        while (bm) {
          const int j = __ffs(bm) - 1;
          bm &= bm - 1;
          const int aj = __shfl_sync(0xffffffffu, a[m], j), cj = __shfl_sync(0xffffffffu, cnt[m], j);
          const int dj = __shfl_sync(0xffffffffu, dst[m], j), rj = __shfl_sync(0xffffffffu, rp[m], j);
          const int sj = __shfl_sync(0xffffffffu, sid[m], j);
          const int32_t* mp = s_map[sj];
          for (int u = lane; u < cj; u += 32)
            if (dj + u < cap) s[dj + u] = __ldg(mp + aj + u) - rj;
        }
      }
    }
    if (H > cap) {
      if (lane == 0) {
        if (H <= kSmallGatherCap) {
          const int k = atomicAdd(go.big_count + 2, 1);
          go.small_list[k] = (int32_t)r;
          go.small_h[k] = H;
        } else {
          const int k = atomicAdd(go.big_count, 1);
          go.big_list[k] = (int32_t)r;
          go.big_h[k] = H;
        }
      }
      __syncwarp();
      continue;
    }
    positions += (unsigned long long)H;
    lookups += (unsigned long long)T;
    __syncwarp();
    if (H <= 32) {
      sort_emit_regs<1>(s, H, I, (int)r, go);
    } else {
      const int U = warp_dedupe(s, H, s + cap, cap);
      if (U <= 32) sort_emit_regs<1>(s, U, I, (int)r, go);
      else bucket_sort_emit(s, s + cap, shist[w], U, I, (int)r, go);
    }
    __syncwarp();
  }
  }
  if (lane == 0) {  // both counts are the same in every lane of the warp
    atomicAdd(&go.counters[3], lookups);
    atomicAdd(&go.counters[4], positions);
  }
}

// One block per read of the list, for reads with more index positions than a warp holds: the
// positions go to a block-private slice of a global buffer (scratch: 2 * cap words per block,
// its working set small enough to stay in L2), then a bucket sort without comparisons across
// buckets: min / max, buckets of equal power-of-two width over [min, max] (about 8 values each,
// so that bucket order is value order), counted and scattered with shared atomics, then every
// thread insertion-sorts its buckets, dropping repeated values on the way.  The surviving
// diagonals are appended in order; the smallest is dropped when it is not above -I
// (run.c:617, :648).  Reads with more than `cap` positions are appended to (huge_list,
// huge_h) for a second launch with a larger cap.  The grid is persistent: blocks take the next
// read of the list from `cursor` (zeroed), list_count read on the device when given.
constexpr int kBT = 512;              // threads of a block-gather block
constexpr int kMaxBuckets = 4096;
constexpr int kSmallCap = kSmallGatherCap;  // a read with at most this many positions sorts in shared memory

// exclusive scan of a[0..n) in place (n <= kMaxBuckets, every thread of the block); the total
__device__ __forceinline__ int block_excl_scan(int32_t* a, int n, int* wtot) {
  constexpr int per = kMaxBuckets / kBT;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b0 = threadIdx.x * per;
  int loc = 0;
#pragma unroll
  for (int k = 0; k < per; ++k)
    if (b0 + k < n) loc += a[b0 + k];
  const int incl = warp_incl_scan(loc);
  if (lane == 31) wtot[w] = incl;
  __syncthreads();
  int before = 0, tot = 0;
  for (int q = 0; q < kBT / 32; ++q) {
    if (q < w) before += wtot[q];
    tot += wtot[q];
  }
  int run = before + incl - loc;
#pragma unroll
  for (int k = 0; k < per; ++k)
    if (b0 + k < n) {
      const int v = a[b0 + k];
      a[b0 + k] = run;
      run += v;
    }
  __syncthreads();
  return tot;
}

// SMEM: the slices in dynamic shared memory (every read of the list has at most kSmallCap
// positions).  Without it a launch keeps its shared memory small: the L1 cache shares that
// storage, and the global slices of reads with many positions live off it.
template <bool SMEM>
__global__ void __launch_bounds__(kBT) gather_block_kernel(ReadsDev rd, IndexView ix, int I, const int32_t* __restrict__ list,
                                                           const int32_t* __restrict__ list_h,
                                                           const int32_t* __restrict__ list_count, int64_t nlist,
                                                           GatherOut go, int32_t* __restrict__ scratch, int cap,
                                                           unsigned long long* cursor, int32_t* huge_list, int32_t* huge_h,
                                                           int32_t* huge_count, const __grid_constant__ SeedSet gs) {
  __shared__ int32_t cnt[kMaxBuckets];   // per bucket: count, start, then end
  __shared__ int32_t uoff[kMaxBuckets];  // per bucket: distinct values, then their offset
  __shared__ int wtot[kBT / 32];
  __shared__ int s_read, s_H;
  __shared__ int32_t s_min, s_max;
  __shared__ unsigned long long s_base;
  __shared__ __align__(16) uint8_t srd[kReadBytes];
  extern __shared__ int32_t dsm[];  // 2 * kSmallCap: the slices of a read with few positions
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int32_t* const Ag = scratch + (int64_t)blockIdx.x * 2 * cap;  // the block's slices in global memory
  int32_t* const Bg = Ag + cap;
  const int64_t n = list_count ? (int64_t)*list_count : nlist;
  unsigned long long lookups = 0, positions = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      const unsigned long long k = atomicAdd(cursor, 1ull);
      s_read = (int64_t)k < n ? list[k] : -1;
      s_H = (int64_t)k < n ? list_h[k] : 0;
      s_min = 0x7fffffff;
      s_max = (int32_t)0x80000000;
    }
    __syncthreads();
    const int r = s_read;
    if (r < 0) break;
    const int L = rd.lengths[r];
    {
      const uint8_t* src = rd.codes + (int64_t)r * rd.cstride;
      const int nbytes = (L + 3) >> 2;
      for (int b = threadIdx.x; b < kReadBytes; b += kBT) srd[b] = b < nbytes ? src[b] : 0;
    }
    __syncthreads();
    // the read's position count came with it (the warp gather counted it), so a read above
    // `cap` loads none of its positions here
    int T = 0;
    for (int si = 0; si < gs.n; ++si) T += seed_npos(gs.s[si], L);
    const int H = s_H;
    if (H > cap) {
      if (threadIdx.x == 0) {
        const int k = atomicAdd(huge_count, 1);
        huge_list[k] = r;
        huge_h[k] = H;
      }
      __syncthreads();
      continue;
    }
    lookups += (unsigned long long)T;
    positions += (unsigned long long)H;
    if (H == 0) {
      __syncthreads();
      continue;
    }
    __syncthreads();  // every thread has read s_H
    if (threadIdx.x == 0) s_H = 0;
    __syncthreads();
    // the rest of the read, compiled twice: slices in shared memory (a read with few positions)
    // or in the block's global slices, each with plain shared or global memory operations
    auto per_read = [&](auto in_shared) {
      constexpr bool SMALL = decltype(in_shared)::value;
      int32_t* const A = SMALL ? dsm : Ag;
      int32_t* const B = SMALL ? dsm + kSmallCap : Bg;
      // gather: every (seed, read position) item's CSR range, placed by a block scan; the range
      // of the values is taken on the way
      int32_t vmin = 0x7fffffff, vmax = (int32_t)0x80000000;
      auto put = [&](int k, int32_t v) {
        vmin = min(vmin, v);
        vmax = max(vmax, v);
        A[k] = v;
      };
      for (int si = 0; si < gs.n; ++si) {
        const int np = seed_npos(gs.s[si], L);
        const int32_t* first = ix.first[si];
        const int32_t* mp = ix.map[si];
        for (int t0 = 0; t0 < np; t0 += kBT) {
          int a, c, rp;
          item_lookup(first, gs.s[si], t0 + threadIdx.x, srd, L, a, c, rp);
          const int incl = warp_incl_scan(c);
          if (lane == 31) wtot[w] = incl;
          __syncthreads();
          int before = 0, tot = 0;
          for (int q = 0; q < kBT / 32; ++q) {
            if (q < w) before += wtot[q];
            tot += wtot[q];
          }
          const int dst = s_H + before + incl - c;
          if (c <= 8) {
            for (int u = 0; u < c; ++u) put(dst + u, __ldg(mp + a + u) - rp);
          }
          unsigned bm = __ballot_sync(0xffffffffu, c > 8);  // long lists: the warp copies each
          while (bm) {
            const int j = __ffs(bm) - 1;
            bm &= bm - 1;
            const int aj = __shfl_sync(0xffffffffu, a, j), cj = __shfl_sync(0xffffffffu, c, j);
            const int dj = __shfl_sync(0xffffffffu, dst, j), rj = __shfl_sync(0xffffffffu, rp, j);
            for (int u = lane; u < cj; u += 32) put(dj + u, __ldg(mp + aj + u) - rj);
          }
          __syncthreads();
          if (threadIdx.x == 0) s_H += tot;
          __syncthreads();
        }
      }
      // range
      vmin = __reduce_min_sync(0xffffffffu, vmin);
      vmax = __reduce_max_sync(0xffffffffu, vmax);
      if (lane == 0) {
        atomicMin(&s_min, vmin);
        atomicMax(&s_max, vmax);
      }
      __syncthreads();
      vmin = s_min;
      const uint32_t range = (uint32_t)s_max - (uint32_t)vmin;
      int nb = 1;
      while (nb < kMaxBuckets && nb * 8 < H) nb <<= 1;
      int shift = 0;
      while ((range >> shift) >= (uint32_t)nb) ++shift;
      for (int b = threadIdx.x; b < nb; b += kBT) cnt[b] = 0;
      __syncthreads();
      for (int i = threadIdx.x; i < H; i += kBT) atomicAdd(&cnt[((uint32_t)A[i] - (uint32_t)vmin) >> shift], 1);
      __syncthreads();
      block_excl_scan(cnt, nb, wtot);
      for (int i = threadIdx.x; i < H; i += kBT) {
        const int32_t v = A[i];
        B[atomicAdd(&cnt[((uint32_t)v - (uint32_t)vmin) >> shift], 1)] = v;
      }
      __syncthreads();  // cnt[b] is now the end of bucket b
      for (int b = threadIdx.x; b < nb; b += kBT) {
        const int s0 = b ? cnt[b - 1] : 0, e = cnt[b];
        int u = 0;
        for (int x = s0; x < e; ++x) {  // insertion into the sorted distinct prefix B[s0, s0 + u)
          const int32_t t = B[x];
          int y = u - 1;
          while (y >= 0 && B[s0 + y] > t) --y;
          if (y >= 0 && B[s0 + y] == t) continue;
          for (int z = u - 1; z > y; --z) B[s0 + z + 1] = B[s0 + z];
          B[s0 + y + 1] = t;
          ++u;
        }
        uoff[b] = u;
      }
      __syncthreads();
      const int U = block_excl_scan(uoff, nb, wtot);
      for (int b = threadIdx.x; b < nb; b += kBT) {
        const int s0 = b ? cnt[b - 1] : 0, o = uoff[b];
        const int u = (b + 1 < nb ? uoff[b + 1] : U) - o;
        for (int k = 0; k < u; ++k) A[o + k] = B[s0 + k];
      }
      __syncthreads();
      const int drop = A[0] <= -I ? 1 : 0;  // the first diagonal must exceed -I (run.c:617, :648)
      const int Uo = U - drop;
      if (threadIdx.x == 0) s_base = Uo ? atomicAdd(&go.counters[7], (unsigned long long)Uo) : 0ull;
      __syncthreads();
      const unsigned long long base = s_base;
      if ((int64_t)(base + Uo) > go.cap) {
        if (threadIdx.x == 0) atomicExch(&go.counters[8], 1ull);
      } else {
        for (int k = threadIdx.x; k < Uo; k += kBT) {
          go.fr[base + k] = r;
          go.fd[base + k] = A[k + drop];
        }
      }
    };
    if constexpr (SMEM) per_read(std::true_type{});
    else per_read(std::false_type{});
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    atomicAdd(&go.counters[3], lookups);
    atomicAdd(&go.counters[4], positions);
  }
}

void launch_gather_fused(const ReadsDev& rd, const IndexView& ix, int I, const GatherOut& go, const SeedSet& seeds,
                         cudaStream_t st) {
  if (rd.n <= 0) return;
  set_smem_attribute_once(reinterpret_cast<const void*>(gather_fused_kernel), kGWarps * 2 * kMaxWarpCap * 4);
  const size_t smem = (size_t)kGWarps * 2 * go.warp_cap * sizeof(int32_t);
  const int64_t per_block = (int64_t)kGWarps * go.reads_per_steal;
  const int64_t blocks = std::min<int64_t>((rd.n + per_block - 1) / per_block,
                                          resident_grid(gather_fused_kernel, kGWarps * 32, smem));
  gather_fused_kernel<<<(unsigned)blocks, kGWarps * 32, smem, st>>>(rd, ix, I, go, seeds);
}

constexpr size_t kBlockGatherSmem = 2 * kSmallCap * sizeof(int32_t);

int64_t gather_block_grid(bool smem) {
  if (!smem) return resident_grid(gather_block_kernel<false>, kBT, 0);
  set_smem_attribute_once(reinterpret_cast<const void*>(gather_block_kernel<true>), (int)kBlockGatherSmem);
  return resident_grid(gather_block_kernel<true>, kBT, kBlockGatherSmem);
}

void launch_gather_block(const ReadsDev& rd, const IndexView& ix, int I, const int32_t* list, const int32_t* list_h,
                         int64_t nlist, const int32_t* nlist_dev, const GatherOut& go, int32_t* scratch, int cap,
                         int64_t grid, unsigned long long* cursor, int32_t* huge_list, int32_t* huge_h,
                         int32_t* huge_count, bool smem, const SeedSet& seeds, cudaStream_t st) {
  if (nlist <= 0 || grid <= 0) return;
  if (smem) {
    set_smem_attribute_once(reinterpret_cast<const void*>(gather_block_kernel<true>), (int)kBlockGatherSmem);
    gather_block_kernel<true><<<(unsigned)grid, kBT, kBlockGatherSmem, st>>>(
        rd, ix, I, list, list_h, nlist_dev, nlist, go, scratch, cap, cursor, huge_list, huge_h, huge_count, seeds);
  } else {
    gather_block_kernel<false><<<(unsigned)grid, kBT, 0, st>>>(rd, ix, I, list, list_h, nlist_dev, nlist, go, scratch,
                                                               cap, cursor, huge_list, huge_h, huge_count, seeds);
  }
}

}  // namespace sg
