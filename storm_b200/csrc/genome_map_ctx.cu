// genome_map_ctx.cu -- the contextual placement of the mapping without -M and without -G
// (genome_map.c:233-531, the default genome_map mode): the mapped reads in descending order of
// their best score (ties in read order, genome_map.c:233-299), each placed at the candidate of
// the highest score adjusted to the consensus that the reads placed before it built
// (genome_map.c:366-424), whose positions it then updates (genome_map.c:346-356, 433-531).
//
// The order is sequential only where reads touch the same positions.  Here the reads run in
// waves over one table of the best (earliest-ranked) pending read per reference position,
// updated with atomic minima of the rank (the rank is the position in that order, so the
// minimum is the reference's own tie-break): a pending read whose candidate spans all hold its
// own rank has no earlier pending read on any position it reads, so it is placed in this wave,
// and two reads placed in one wave touch no common position.  The earliest pending read is always
// placed, so every wave makes progress.  The per-position state (6-bit consensus counters packed
// four plus one to a word, genome_map.c:37-48) is kept only for the positions some candidate span
// covers: a bitmap of the covered positions and its word counts give each a dense index.
#include <cstring>
#include <vector>

#include "context.cuh"
#include "radix.cuh"
#include "scan.cuh"
#include "sw_filter.cuh"

namespace {

using namespace sg;

constexpr uint32_t kNoRank = 0xffffffffu;
constexpr int32_t kPending = (int32_t)0xfefefefe;  // a rank not placed yet (a byte fill)
constexpr int kCodes = 4;        // BASE_CODE_COUNT / COLOR_CODE_COUNT (codes.h:25-29)
constexpr int kNoCode = kCodes;  // genome_map.c:26

struct CtxMap {
  const stormgpu_hit* hits;
  const uint8_t* tb;
  int64_t tbs;
  const uint32_t* order;        // rank j -> read
  const uint32_t* base;         // global position of each sequence's position 0
  const uint32_t* size;         // each sequence's size (its map has size + 1 positions)
  const uint8_t* const* codes;  // each sequence's packed codes
  const uint32_t* bits;         // covered global positions
  const int64_t* woff;          // covered positions before each word of bits
  uint8_t* created;             // per covered position
  uint32_t* aligned;
  uint32_t* inserted;           // indels per covered position
  uint32_t* minrank;            // earliest pending rank per covered position
  int indels, colour, match, mismatch;
};

__device__ __forceinline__ int64_t cov_index(const CtxMap& M, uint32_t p) {
  const uint32_t w = M.bits[p >> 5];
  return M.woff[p >> 5] + __popc(w & ((1u << (p & 31)) - 1u));
}

// The global span [a, b] of rank k of read r: the positions its traceback can reach (each
// operation advances one position at most; the map of a sequence ends at position size);
// false for an empty slot.
__device__ __forceinline__ bool cand_span(const CtxMap& M, int64_t r, int k, uint32_t* a, uint32_t* b) {
  const stormgpu_hit& h = M.hits[r * 4 + k];
  if (h.ref_start == STORMGPU_UNMAPPED) return false;
  const uint32_t s0 = M.base[h.ref_id] + (uint32_t)h.ref_start;
  const uint32_t last = M.base[h.ref_id] + M.size[h.ref_id];
  *a = s0;
  *b = min(s0 + (uint32_t)max(h.tb_len, 0), last);
  return s0 <= last;
}

// the candidates a read has: ranks below the first empty slot (genome_map.c:436-441)
__device__ __forceinline__ int cand_count(const CtxMap& M, int64_t r) {
  int k = 0;
  while (k < 4 && M.hits[r * 4 + k].ref_start != STORMGPU_UNMAPPED) ++k;
  return k;
}

__device__ __forceinline__ int get6(uint32_t c, int code) { return (int)((c >> (code * 6)) & 0x3F); }
__device__ __forceinline__ uint32_t inc6(uint32_t c, int code) {
  const uint32_t v = (uint32_t)((get6(c, code) + 1) & 0x3F);
  return (c & ~(0x3Fu << (code * 6))) | (v << (code * 6));
}

// GET_PAIR_TYPE (alignment.h:87-94)
__device__ __forceinline__ int pair_type(int code, int colour) {
  if ((code & 0xC) == 0x4) return 0x4;
  if (colour && (code & 0xC) == 0x8) return 0x8;
  if ((code & 0xC) == 0xC) return 0xC;
  return code;
}

__device__ __forceinline__ int tb_op(const uint8_t* t, int i) { return (t[i >> 1] >> ((i & 1) ? 0 : 4)) & 0xF; }

// genome_map__get_direct_consensus_code (genome_map.c:312-337); p in the candidate's span
__device__ int consensus(const CtxMap& M, uint32_t p, int offset, int ref_code) {
  const int64_t i = cov_index(M, p);
  if (!M.created[i] || offset >= M.indels) return ref_code;
  const uint32_t cnt = offset < 0 ? M.aligned[i] : M.inserted[i * M.indels + offset];
  int best = ref_code;
  for (int s = 0; s <= kCodes; ++s)
    if (get6(cnt, s) > get6(cnt, best)) best = s;
  if (get6(cnt, best) == 0) best = kNoCode;
  return best;
}

// genome_map__update_consensus_code (genome_map.c:346-356)
__device__ void update(const CtxMap& M, uint32_t p, int offset, int code) {
  const int64_t i = cov_index(M, p);
  M.created[i] = 1;
  if (offset >= 0) {
    if (offset < M.indels) M.inserted[i * M.indels + offset] = inc6(M.inserted[i * M.indels + offset], code);
  } else {
    M.aligned[i] = inc6(M.aligned[i], code);
  }
}

// genome_map__compute_adjusted_score (genome_map.c:366-424)
__device__ int adjusted_score(const CtxMap& M, int64_t r, int k) {
  const stormgpu_hit& h = M.hits[r * 4 + k];
  const uint8_t* t = M.tb + (r * 4 + k) * M.tbs;
  const uint8_t* codes = M.codes[h.ref_id];
  uint32_t a, b;
  cand_span(M, r, k, &a, &b);
  int score = 0, indel = 0;
  int64_t pos = h.ref_start;
  uint32_t gp = a;
  for (int i = 0; i < h.tb_len; ++i) {
    const int cell = tb_op(t, i);
    if (gp > b) break;  // beyond the map of the sequence (no alignment reaches it)
    switch (pair_type(cell, M.colour)) {
    case 0x3: {
      const int rc = code_at(codes, pos);
      score += rc == consensus(M, gp, -1, rc) ? M.match : M.mismatch;
      ++pos; ++gp;
      indel = 0;
      break;
    }
    case 0x1:
      score += consensus(M, gp, -1, kNoCode) == kNoCode ? M.match : M.mismatch;
      ++pos; ++gp;
      indel = 0;
      break;
    case 0x4:
    case 0x8: {
      const int c = cell & 3;
      score += c == consensus(M, gp, -1, c) ? M.match : M.mismatch;
      ++pos; ++gp;
      indel = 0;
      break;
    }
    case 0xC: {
      const int c = cell & 3;
      score += c == consensus(M, gp, indel, c) ? M.match : M.mismatch;
      ++indel;
      break;
    }
    default:
      break;
    }
  }
  return score;
}

// the consensus update along the placed candidate (genome_map.c:500-531)
__device__ void place_updates(const CtxMap& M, int64_t r, int k) {
  const stormgpu_hit& h = M.hits[r * 4 + k];
  const uint8_t* t = M.tb + (r * 4 + k) * M.tbs;
  const uint8_t* codes = M.codes[h.ref_id];
  uint32_t a, b;
  cand_span(M, r, k, &a, &b);
  M.created[cov_index(M, a)] = 1;  // genome_map__create_position_data at the placed start
  int64_t pos = h.ref_start;
  uint32_t gp = a;
  int insertions = -1;
  for (int i = 0; i < h.tb_len && gp <= b; ++i) {
    const int cell = tb_op(t, i);
    switch (pair_type(cell, M.colour)) {
    case 0xC: insertions++; update(M, gp, insertions, cell & 3); break;
    case 0x3: insertions = -1; update(M, gp, -1, code_at(codes, pos)); break;
    case 0x4: insertions = -1; update(M, gp, -1, cell & 3); break;
    case 0x1: insertions = -1; update(M, gp, -1, kNoCode); break;
    case 0x8: insertions = -1; update(M, gp, -1, cell & 3); break;
    default: break;
    }
    for (int p = insertions + 1; p < M.indels; ++p) update(M, gp, p, kNoCode);
    if (insertions < 0) { ++pos; ++gp; }
  }
}

// -------------------------------------------------------------------------------- kernels

// sort keys of the mapped reads, in read order: descending unsigned best score (the reference
// sorts the unsigned score by 4-bit digits into buckets 15 - digit, genome_map.c:233-299)
__global__ void ctx_keys_kernel(int64_t n, const stormgpu_hit* __restrict__ hits, const uint8_t* __restrict__ mapped,
                                const int64_t* __restrict__ off, uint32_t* __restrict__ keys,
                                uint32_t* __restrict__ vals) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    if (mapped[r]) {
      keys[off[r]] = ~(uint32_t)hits[r * 4].score;
      vals[off[r]] = (uint32_t)r;
    }
}

__global__ void rank_iota_kernel(int64_t nm, uint32_t* __restrict__ out) {
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nm; j += (int64_t)gridDim.x * blockDim.x)
    out[j] = (uint32_t)j;
}

__global__ void mapped_flags_kernel(int64_t n, const uint8_t* __restrict__ mapped, uint8_t* __restrict__ f) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    f[r] = mapped[r] ? 1 : 0;
}

// a warp per read (of `list`, or rank j itself without one): the words of every candidate span
__device__ __forceinline__ int64_t warp_id() { return ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int64_t warp_count() { return ((int64_t)gridDim.x * blockDim.x) >> 5; }

__global__ void ctx_mark_kernel(int64_t nm, CtxMap M, uint32_t* __restrict__ bits) {
  const int lane = threadIdx.x & 31;
  for (int64_t j = warp_id(); j < nm; j += warp_count()) {
    const int64_t r = M.order[j];
    const int nk = cand_count(M, r);
    for (int k = 0; k < nk; ++k) {
      uint32_t a, b;
      if (!cand_span(M, r, k, &a, &b)) continue;
      for (uint32_t w = (a >> 5) + lane; w <= (b >> 5); w += 32) {
        uint32_t m = 0xffffffffu;
        if (w == (a >> 5)) m &= 0xffffffffu << (a & 31);
        if (w == (b >> 5)) m &= 0xffffffffu >> (31 - (b & 31));
        atomicOr(&bits[w], m);
      }
    }
  }
}

// Waves run back to back without the host: wave w takes the list `pending` of counts[cur]
// reads and appends the reads it leaves to the other list, counted in counts[cur ^ 1] (zeroed by
// its first kernel); counts[2] counts the waves that had pending reads.

// every position of every span of the pending reads: the earliest rank
__global__ void ctx_rank_kernel(unsigned long long* __restrict__ counts, int cur, const uint32_t* __restrict__ pending,
                                CtxMap M) {
  const int lane = threadIdx.x & 31;
  const int64_t np = (int64_t)counts[cur];
  if (blockIdx.x == 0 && threadIdx.x == 0) counts[cur ^ 1] = 0;
  for (int64_t q = warp_id(); q < np; q += warp_count()) {
    const uint32_t j = pending[q];
    const int64_t r = M.order[j];
    const int nk = cand_count(M, r);
    for (int k = 0; k < nk; ++k) {
      uint32_t a, b;
      if (!cand_span(M, r, k, &a, &b)) continue;
      for (uint32_t p = a + lane; p <= b; p += 32) atomicMin(&M.minrank[cov_index(M, p)], j);
    }
  }
}

// the pending reads that are earliest on every position they read: placed now
__global__ void ctx_place_kernel(const unsigned long long* __restrict__ counts, int cur,
                                 const uint32_t* __restrict__ pending, CtxMap M, int uniqueness,
                                 int uniqueness_threshold, int32_t* __restrict__ placed) {
  const int lane = threadIdx.x & 31;
  const int64_t np = (int64_t)counts[cur];
  for (int64_t q = warp_id(); q < np; q += warp_count()) {
    const uint32_t j = pending[q];
    const int64_t r = M.order[j];
    const int nk = cand_count(M, r);
    bool mine = true;
    for (int k = 0; k < nk; ++k) {
      uint32_t a, b;
      if (!cand_span(M, r, k, &a, &b)) continue;
      for (uint32_t p = a + lane; p <= b && mine; p += 32) mine = M.minrank[cov_index(M, p)] == j;
    }
    if (!__all_sync(0xffffffffu, mine)) continue;
    if (lane == 0) {
      // genome_map.c:436-470: the best adjusted score (first of equals), the uniqueness test
      int adj[4] = {STORMGPU_MIN_SCORE, STORMGPU_MIN_SCORE, STORMGPU_MIN_SCORE, STORMGPU_MIN_SCORE};
      int best_rank = -1, best = STORMGPU_MIN_SCORE;
      for (int k = 0; k < nk; ++k) {
        adj[k] = adjusted_score(M, r, k);
        if (adj[k] > best) { best = adj[k]; best_rank = k; }
      }
      if (best_rank < 0 || (uniqueness && !(adj[0] - adj[1] > uniqueness_threshold))) {
        placed[j] = -1;
      } else {
        place_updates(M, r, best_rank);
        placed[j] = best_rank;
      }
    }
  }
}

// the spans of this wave's pending reads back to no rank; the reads still pending to `next`
__global__ void ctx_reset_kernel(unsigned long long* __restrict__ counts, int cur, const uint32_t* __restrict__ pending,
                                 CtxMap M, const int32_t* __restrict__ placed, uint32_t* __restrict__ next) {
  const int lane = threadIdx.x & 31;
  const int64_t np = (int64_t)counts[cur];
  unsigned long long* next_count = counts + (cur ^ 1);
  if (blockIdx.x == 0 && threadIdx.x == 0 && np > 0) counts[2]++;
  for (int64_t q = warp_id(); q < np; q += warp_count()) {
    const uint32_t j = pending[q];
    const int64_t r = M.order[j];
    const int nk = cand_count(M, r);
    for (int k = 0; k < nk; ++k) {
      uint32_t a, b;
      if (!cand_span(M, r, k, &a, &b)) continue;
      for (uint32_t p = a + lane; p <= b; p += 32) M.minrank[cov_index(M, p)] = kNoRank;
    }
    if (lane == 0 && placed[j] == kPending) next[atomicAdd(next_count, 1ull)] = j;
  }
}

// output sort keys, in rank order: the placed start (global position) or "not placed"
__global__ void ctx_out_keys_kernel(int64_t nm, CtxMap M, const int32_t* __restrict__ placed,
                                    uint32_t* __restrict__ keys, uint32_t* __restrict__ vals,
                                    unsigned long long* __restrict__ count) {
  unsigned long long cnt = 0;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nm; j += (int64_t)gridDim.x * blockDim.x) {
    const int k = placed[j];
    uint32_t key = kNoRank;
    if (k >= 0) {
      const stormgpu_hit& h = M.hits[(int64_t)M.order[j] * 4 + k];
      key = M.base[h.ref_id] + (uint32_t)h.ref_start;
      ++cnt;
    }
    keys[j] = key;
    vals[j] = (uint32_t)j;
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(count, cnt);
}

__global__ void ctx_out_kernel(int64_t npl, const uint32_t* __restrict__ sorted_j, const uint32_t* __restrict__ order,
                               const int32_t* __restrict__ placed, int32_t* __restrict__ read,
                               int32_t* __restrict__ rank) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < npl; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t j = sorted_j[i];
    read[i] = (int32_t)order[j];
    rank[i] = placed[j];
  }
}

unsigned grid_for(int64_t items, int per_block) {
  const int64_t b = (items + per_block - 1) / per_block;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

}  // namespace

namespace {

// device allocations of one call, freed with it
struct Scratch {
  std::vector<void*> ptrs;
  template <typename T>
  T* get(int64_t n) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(T) * (size_t)std::max<int64_t>(n, 1)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
  }
};

}  // namespace

extern "C" int stormgpu_genome_map_contextual(stormgpu_ctx* c, int32_t uniqueness, int32_t uniqueness_threshold,
                                              int32_t* read, int32_t* rank, int64_t* n_placed) {
  if (!c || !read || !rank || !n_placed) {
    sg_set_error("stormgpu_genome_map_contextual: null argument");
    return STORMGPU_EINVAL;
  }
  if (c->last_n < 0) {
    sg_set_error("stormgpu_genome_map_contextual: no stormgpu_map call yet");
    return STORMGPU_ESTATE;
  }
  SG_CUDA(cudaSetDevice(c->p.device));
  const int64_t n = c->last_n;
  *n_placed = 0;
  if (n == 0) return 0;
  const size_t nref = c->refs.size();
  std::vector<uint32_t> base(nref), size(nref);
  std::vector<const uint8_t*> codes(nref);
  uint64_t acc = 0;
  for (size_t s = 0; s < nref; ++s) {
    base[s] = (uint32_t)acc;
    size[s] = (uint32_t)c->refs[s].n;
    codes[s] = c->refs[s].d_codes;
    acc += (uint64_t)c->refs[s].n + 1;
  }
  if (acc + 64 >= 0xffffffffull || n >= (int64_t)kNoRank) {
    sg_set_error("stormgpu_genome_map_contextual: more than 2^32 - 64 reference positions or reads");
    return STORMGPU_EINVAL;
  }
  cudaStream_t st = c->st;
  Scratch S;
  auto nomem = [&]() {
    sg_set_error("stormgpu_genome_map_contextual: device allocation failed");
    return STORMGPU_ENOMEM;
  };
  // the mapped reads, by descending best score, ties in read order
  uint8_t* flags = S.get<uint8_t>(n);
  int64_t* off = S.get<int64_t>(n + 1);
  int64_t* stmp = S.get<int64_t>(scan_tmp_elems(n) + 8);
  uint32_t* d_base = S.get<uint32_t>((int64_t)nref);
  uint32_t* d_size = S.get<uint32_t>((int64_t)nref);
  const uint8_t** d_codes = S.get<const uint8_t*>((int64_t)nref);
  if (!flags || !off || !stmp || !d_base || !d_size || !d_codes) return nomem();
  SG_CUDA(cudaMemcpyAsync(d_base, base.data(), sizeof(uint32_t) * nref, cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemcpyAsync(d_size, size.data(), sizeof(uint32_t) * nref, cudaMemcpyHostToDevice, st));
  SG_CUDA(cudaMemcpyAsync(d_codes, codes.data(), sizeof(const uint8_t*) * nref, cudaMemcpyHostToDevice, st));
  mapped_flags_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, c->mapped.p, flags);
  exclusive_scan<uint8_t, int64_t>(flags, off, n, off + n, stmp, st);
  int64_t nm = 0;
  SG_CUDA(cudaMemcpyAsync(&nm, off + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  if (nm == 0) return 0;
  uint32_t *k0 = S.get<uint32_t>(nm), *v0 = S.get<uint32_t>(nm), *k1 = S.get<uint32_t>(nm), *v1 = S.get<uint32_t>(nm);
  void* rtmp = S.get<uint8_t>(radix_tmp_bytes(nm));
  if (!k0 || !v0 || !k1 || !v1 || !rtmp) return nomem();
  ctx_keys_kernel<<<grid_for(n, 256), 256, 0, st>>>(n, c->hits.p, c->mapped.p, off, k0, v0);
  const uint32_t* order = radix_sort_pairs(k0, v0, k1, v1, nm, 32, rtmp, st) ? v1 : v0;

  CtxMap M;
  memset(&M, 0, sizeof(M));
  M.hits = c->hits.p; M.tb = c->tb.p; M.tbs = c->last_tbs; M.order = order;
  M.base = d_base; M.size = d_size; M.codes = d_codes;
  M.indels = c->p.allowed_indels; M.colour = c->p.colour; M.match = c->p.match; M.mismatch = c->p.mismatch;
  // the covered positions and their dense index
  const int64_t nwords = (int64_t)(acc >> 5) + 2;
  uint32_t* bits = S.get<uint32_t>(nwords);
  int64_t* woff = S.get<int64_t>(nwords + 1);
  int64_t* wtmp = S.get<int64_t>(scan_tmp_elems(nwords) + 8);
  if (!bits || !woff || !wtmp) return nomem();
  SG_CUDA(cudaMemsetAsync(bits, 0, sizeof(uint32_t) * nwords, st));
  ctx_mark_kernel<<<grid_for(nm * 32, 256), 256, 0, st>>>(nm, M, bits);
  exclusive_scan<PassWord, int64_t>(reinterpret_cast<const PassWord*>(bits), woff, nwords, woff + nwords, wtmp, st);
  int64_t cov = 0;
  SG_CUDA(cudaMemcpyAsync(&cov, woff + nwords, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  M.bits = bits;
  M.woff = woff;
  M.created = S.get<uint8_t>(cov);
  M.aligned = S.get<uint32_t>(cov);
  M.inserted = S.get<uint32_t>(cov * std::max(M.indels, 1));
  M.minrank = S.get<uint32_t>(cov);
  int32_t* placed = S.get<int32_t>(nm);
  uint32_t *pend0 = S.get<uint32_t>(nm), *pend1 = S.get<uint32_t>(nm);
  unsigned long long* cnt = S.get<unsigned long long>(3);
  if (!M.created || !M.aligned || !M.inserted || !M.minrank || !placed || !pend0 || !pend1 || !cnt) return nomem();
  SG_CUDA(cudaMemsetAsync(M.created, 0, (size_t)cov, st));
  SG_CUDA(cudaMemsetAsync(M.aligned, 0, sizeof(uint32_t) * cov, st));
  SG_CUDA(cudaMemsetAsync(M.inserted, 0, sizeof(uint32_t) * cov * std::max(M.indels, 1), st));
  SG_CUDA(cudaMemsetAsync(M.minrank, 0xff, sizeof(uint32_t) * cov, st));
  SG_CUDA(cudaMemsetAsync(placed, 0xfe, sizeof(int32_t) * nm, st));  // kPending in every rank
  rank_iota_kernel<<<grid_for(nm, 256), 256, 0, st>>>(nm, pend0);  // every rank pending
  // waves in groups of kGroup between two reads of the pending count (a wave with none pending
  // costs three near-empty launches)
  constexpr int kGroup = 16;
  const unsigned long long init[3] = {(unsigned long long)nm, 0, 0};
  SG_CUDA(cudaMemcpyAsync(cnt, init, sizeof(init), cudaMemcpyHostToDevice, st));
  const unsigned g = grid_for(nm * 32, 256);
  uint32_t* lists[2] = {pend0, pend1};
  int cur = 0;
  unsigned long long h[3] = {(unsigned long long)nm, 0, 0};
  static_assert(kGroup % 2 == 0, "a group ends on the list it started from");
  for (;;) {
    for (int k = 0; k < kGroup; ++k, cur ^= 1) {
      ctx_rank_kernel<<<g, 256, 0, st>>>(cnt, cur, lists[cur], M);
      ctx_place_kernel<<<g, 256, 0, st>>>(cnt, cur, lists[cur], M, uniqueness, uniqueness_threshold, placed);
      ctx_reset_kernel<<<g, 256, 0, st>>>(cnt, cur, lists[cur], M, placed, lists[cur ^ 1]);
    }
    const unsigned long long before = h[cur];
    SG_CUDA(cudaMemcpyAsync(h, cnt, sizeof(h), cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    SG_CUDA(cudaGetLastError());
    if (h[cur] == 0) break;
    if (h[cur] >= before) {  // cannot happen: the earliest pending rank is always placed
      sg_set_error("stormgpu_genome_map_contextual: %d waves placed no read", kGroup);
      return STORMGPU_ECUDA;
    }
  }
  c->stats.placement_waves = (int64_t)h[2];
  // the placed reads by start position, ties in placement order (genome_map.c:551-796)
  SG_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), st));
  ctx_out_keys_kernel<<<grid_for(nm, 256), 256, 0, st>>>(nm, M, placed, k0, pend0, cnt);
  const uint32_t* sj = radix_sort_pairs(k0, pend0, k1, pend1, nm, 32, rtmp, st) ? pend1 : pend0;
  unsigned long long npl = 0;
  SG_CUDA(cudaMemcpyAsync(&npl, cnt, sizeof(npl), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  if (npl) {
    int32_t* d_read = S.get<int32_t>((int64_t)npl);
    int32_t* d_rank = S.get<int32_t>((int64_t)npl);
    if (!d_read || !d_rank) return nomem();
    ctx_out_kernel<<<grid_for((int64_t)npl, 256), 256, 0, st>>>((int64_t)npl, sj, order, placed, d_read, d_rank);
    SG_CUDA(cudaMemcpyAsync(read, d_read, sizeof(int32_t) * npl, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaMemcpyAsync(rank, d_rank, sizeof(int32_t) * npl, cudaMemcpyDeviceToHost, st));
  }
  SG_CUDA(cudaStreamSynchronize(st));
  SG_CUDA(cudaGetLastError());
  *n_placed = (int64_t)npl;
  return 0;
}
