// stormgpu.cu -- the C ABI of include/stormgpu.h: context, reference upload, index build,
// and the mapping pipeline (per reference sequence, per strand: hit gather -> filter ->
// full alignment -> top-4 replay), plus the unit-level entry points used by the tests.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "index_build.cuh"
#include "map_kernels.cuh"
#include "scan.cuh"
#include "sw_filter.cuh"
#include "gather.cuh"
#include "radix.cuh"
#include "context.cuh"

static thread_local char g_err[1024];
thread_local sg::WorkBudget* sg::g_work_budget = nullptr;

void sg_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

extern "C" const char* stormgpu_version(void) { return "storm-b200 0.1 (sm_100a)"; }
extern "C" const char* stormgpu_last_error(void) { return g_err; }

extern "C" int stormgpu_device_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
  return n > 0 ? 1 : 0;
}

namespace {

using namespace sg;

// seed.c:25-135: ';'-separated patterns of '#'/'1' (care) and '-'/'0' (don't care), each with
// an optional ":p1 p2,p3" list of read positions.
int parse_seeds(const char* list, SeedSet* out) {
  memset(out, 0, sizeof(*out));
  if (!list) return STORMGPU_EINVAL;
  std::string s(list);
  size_t p = 0;
  while (p <= s.size()) {
    size_t e = s.find(';', p);
    if (e == std::string::npos) e = s.size();
    std::string tok = s.substr(p, e - p);
    p = e + 1;
    if (tok.empty()) { if (e == s.size()) break; continue; }
    if (out->n >= kMaxSeeds) return STORMGPU_EINVAL;
    SeedDev& sd = out->s[out->n];
    size_t colon = tok.find(':');
    std::string pat = tok.substr(0, colon);
    if (pat.empty() || (int)pat.size() > kMaxSpan) return STORMGPU_EINVAL;
    sd.span = (int)pat.size();
    for (int i = 0; i < sd.span; ++i) {
      char c = pat[i];
      if (c == '#' || c == '1') sd.care[sd.n_care++] = (int8_t)i;
      else if (c != '-' && c != '0') return STORMGPU_EINVAL;
    }
    sd.weight = sd.n_care;
    if (sd.weight == 0 || sd.weight > 15) return STORMGPU_EINVAL;
    if (colon != std::string::npos && tok.size() - colon > 1) {
      std::string rest = tok.substr(colon + 1);
      int v;
      if (sscanf(rest.c_str(), "%d", &v) == 1) {
        char* save = nullptr;
        std::vector<char> buf(rest.begin(), rest.end());
        buf.push_back(0);
        for (char* t = strtok_r(buf.data(), ", ", &save); t; t = strtok_r(nullptr, ", ", &save)) {
          if (sscanf(t, "%d", &v) != 1 || sd.n_positions >= kMaxPositions) break;
          sd.positions[sd.n_positions++] = (int16_t)v;
        }
      }
    }
    out->n++;
    if (e == s.size()) break;
  }
  return out->n > 0 ? 0 : STORMGPU_EINVAL;
}

}  // namespace

namespace sg {

int filter_width(int is) { return is <= 1 ? 2 : is <= 3 ? 4 : is <= 7 ? 8 : 16; }

ScoreParams make_score_params(const stormgpu_params& p) {
  ScoreParams sp;
  memset(&sp, 0, sizeof(sp));
  sp.colour = p.colour;
  sp.I = p.allowed_indels;
  sp.Is = p.allowed_indels < 15 ? p.allowed_indels : 15;
  sp.W = filter_width(sp.Is);
  sp.fm = std::abs(p.match) & 0xff;
  sp.fx = std::abs(p.mismatch) & 0xff;
  sp.fo = std::abs(p.gap_open) & 0xff;
  sp.fe = std::abs(p.gap_extend) & 0xff;
  unsigned z = (unsigned)p.min_score_filter;
  sp.fthr = z >= 255u ? 254 : (int)z;
  for (int l = 0; l < 4; ++l) {
    sp.pair[0][l] = (int)(((p.match) * (l + 1) + 0.) / 4);     // SCALE_SCORE, alignment.h:30
    sp.pair[1][l] = (int)(((p.mismatch) * (l + 1) + 0.) / 4);
  }
  sp.gap_open = p.gap_open;
  sp.gap_ext = p.gap_extend;
  sp.min_score = p.min_score;
  // packed cells (align_one_nuc): scores and penalties below 256 in magnitude, at most 200
  // indels, a read's largest gain below 48000 (a floored cell stays under MIN_SCORE) and -t
  // minus that gain above the floor's score -2^16
  int maxpair = 0;
  for (int l = 0; l < 4; ++l) maxpair = std::max({maxpair, std::abs(sp.pair[0][l]), std::abs(sp.pair[1][l])});
  sp.packed = !p.colour && p.allowed_indels >= 0 && p.allowed_indels <= 200 && maxpair <= 255 &&
              std::abs(p.gap_open) <= 255 && std::abs(p.gap_extend) <= 255 &&
              (int64_t)STORMGPU_MAX_READ_LEN * maxpair < 48000 &&
              (int64_t)p.min_score - (int64_t)STORMGPU_MAX_READ_LEN * maxpair > -60000;
  sp.one = 1u;
  sp.open1 = (uint32_t)p.gap_open * 8192u + 1u;
  sp.open1_tc = sp.open1 + (1u << 11) - (1u << 12);
  const uint32_t dx = (uint32_t)(p.gap_extend - p.gap_open);
  sp.kt = 4u * dx - (1u << 22);
  sp.kl = 8u * dx - (1u << 22);
  for (int k = 0; k < 32; ++k) sp.pw[k] = 1u << k;
  return sp;
}

}  // namespace sg



extern "C" int stormgpu_open(const stormgpu_params* params, const char* seeds, stormgpu_ctx** out) {
  if (!params || !out) { sg_set_error("null argument"); return STORMGPU_EINVAL; }
  *out = nullptr;
  SeedSet ss;
  if (parse_seeds(seeds, &ss) != 0) { sg_set_error("invalid seed list \"%s\"", seeds ? seeds : "(null)"); return STORMGPU_EINVAL; }
  if (params->allowed_indels < 0 || params->allowed_indels > STORMGPU_MAX_INDELS) { sg_set_error("allowed_indels out of range"); return STORMGPU_EINVAL; }
  if (params->min_score < STORMGPU_MIN_SCORE) { sg_set_error("min_score below MIN_SCORE is not supported"); return STORMGPU_EINVAL; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    sg_set_error("no CUDA device available: the mapping path runs on the GPU only");
    return STORMGPU_ECUDA;
  }
  if (params->device < 0 || params->device >= ndev) { sg_set_error("bad device ordinal"); return STORMGPU_EINVAL; }
  SG_CUDA(cudaSetDevice(params->device));
  {
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, params->device) == cudaSuccess) {
      uint64_t keep = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  }
  stormgpu_ctx* c = new stormgpu_ctx();
  c->p = *params;
  c->seeds = ss;
  memset(&c->stats, 0, sizeof(c->stats));
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    sg_set_error("cudaStreamCreate failed");
    return STORMGPU_ECUDA;
  }
  for (auto& e : c->ev) cudaEventCreate(&e);
  for (auto& e : c->rev) cudaEventCreate(&e);
  if (const char* g = getenv("STORMGPU_GRAPHS")) c->graphs = atoi(g) != 0;
  *out = c;
  return 0;
}

extern "C" int stormgpu_set_graphs(stormgpu_ctx* c, int enable) {
  if (!c) { sg_set_error("null argument"); return STORMGPU_EINVAL; }
  c->graphs = enable != 0;
  return 0;
}

extern "C" void stormgpu_close(stormgpu_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->p.device);
  cudaStreamSynchronize(c->st);
  if (c->owns_refs)
    for (auto& r : c->refs) {
      cudaFree(r.d_codes_alloc);
      cudaFree(r.d_mask_alloc);
      cudaFree(r.d_gexp_alloc);
      for (auto& ix : r.idx) { cudaFree(ix.first); cudaFree(ix.map); }
    }
  c->rcodes.release(); c->rlevels.release(); c->fcodes.release(); c->flevels.release();
  c->first_levels.release(); c->lengths.release(); c->hits.release(); c->tb.release();
  c->mapped.release();
  c->pstart.release(); c->pcount.release(); c->p_read.release(); c->p_diag.release();
  c->big_list.release(); c->big_h.release(); c->small_list.release(); c->small_h.release();
  c->big_count.release(); c->huge_list.release(); c->huge_h.release(); c->gstate.release();
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  for (auto& e : c->gev) cudaEventDestroy(e);
  c->scan_tmp64.release();
  c->a_score.release(); c->a_bound.release(); c->a_tblen.release(); c->big_tmp.release();
  c->a_pos.release(); c->a_tb.release(); c->scratch.release(); c->counters.release();
  c->foff.release(); c->fr.release(); c->fd.release(); c->flag.release(); c->flagw.release();
  c->rexp.release();
  c->gm_k0.release(); c->gm_v0.release(); c->gm_k1.release(); c->gm_v1.release(); c->gm_tmp.release();
  c->gm_base.release();
  c->ord.release(); c->ord_tmp.release();
  c->thr.release(); c->round_slots.release(); c->rounds.release();
  for (auto& e : c->ev) cudaEventDestroy(e);
  for (auto& e : c->rev) cudaEventDestroy(e);
  cudaStreamDestroy(c->st);
  delete c;
}

extern "C" int stormgpu_add_reference(stormgpu_ctx* c, const uint8_t* codes, const uint8_t* mask,
                                      int64_t n_codes, const int32_t* rs, const int32_t* re,
                                      int32_t n_regions) {
  if (!c || !codes || n_codes < 0 || (n_regions > 0 && (!rs || !re))) { sg_set_error("bad reference arguments"); return STORMGPU_EINVAL; }
  if (n_codes >= INT32_MAX) { sg_set_error("reference sequence longer than 2^31 codes"); return STORMGPU_EINVAL; }
  SG_CUDA(cudaSetDevice(c->p.device));
  RefSeq r;
  r.n = n_codes;
  const int64_t nb = (n_codes + 3) / 4;
  const int64_t tot = nb + 2 * kPadBytes + 16;
  SG_CUDA(cudaMalloc(&r.d_codes_alloc, tot));
  SG_CUDA(cudaMalloc(&r.d_mask_alloc, tot));
  r.d_codes = r.d_codes_alloc + kPadBytes;
  r.d_mask = r.d_mask_alloc + kPadBytes;
  SG_CUDA(cudaMemsetAsync(r.d_codes_alloc, 0, tot, c->st));
  SG_CUDA(cudaMemsetAsync(r.d_mask_alloc, 0x55, tot, c->st));
  std::vector<uint8_t> hc(codes, codes + nb);
  if (n_codes & 3) hc[nb - 1] &= (uint8_t)((1u << (2 * (n_codes & 3))) - 1);  // zero past the end
  SG_CUDA(cudaMemcpyAsync(r.d_codes, hc.data(), nb, cudaMemcpyHostToDevice, c->st));
  std::vector<uint8_t> hm(nb, 0);
  if (mask) memcpy(hm.data(), mask, nb);
  for (int64_t k = n_codes; k & 3; ++k) hm[k >> 2] |= (uint8_t)(1u << ((k & 3) << 1));  // masked past the end
  SG_CUDA(cudaMemcpyAsync(r.d_mask, hm.data(), nb, cudaMemcpyHostToDevice, c->st));
  SG_CUDA(cudaMalloc(&r.d_gexp_alloc, n_codes + 2 * kGexpPad + 16));
  SG_CUDA(cudaMemsetAsync(r.d_gexp_alloc, 0, n_codes + 2 * kGexpPad + 16, c->st));
  r.d_gexp = r.d_gexp_alloc + kGexpPad;
  launch_expand_genome(r.d_codes, n_codes, r.d_gexp, c->st);
  r.rs.assign(rs, rs + std::max(n_regions, 0));
  r.re.assign(re, re + std::max(n_regions, 0));
  SG_CUDA(cudaStreamSynchronize(c->st));
  c->refs.push_back(std::move(r));
  c->indexed = false;
  return 0;
}

extern "C" int stormgpu_build_index(stormgpu_ctx* c) {
  if (!c) return STORMGPU_EINVAL;
  SG_CUDA(cudaSetDevice(c->p.device));
  SG_CUDA(cudaEventRecord(c->ev[0], c->st));
  int64_t launches = 0;
  for (auto& r : c->refs) {
    for (auto& ix : r.idx) { cudaFree(ix.first); cudaFree(ix.map); }
    r.idx.assign(c->seeds.n, DevIndex());
    for (int si = 0; si < c->seeds.n; ++si) {
      int rc = build_one_index(r.d_codes, r.n, r.rs.data(), r.re.data(), (int)r.rs.size(), c->seeds.s[si],
                               c->p.stdev_distance, &r.idx[si], c->st, &launches);
      if (rc) return rc;
    }
  }
  SG_CUDA(cudaEventRecord(c->ev[1], c->st));
  SG_CUDA(cudaStreamSynchronize(c->st));
  float ms = 0;
  cudaEventElapsedTime(&ms, c->ev[0], c->ev[1]);
  c->stats.ms_index = ms;
  c->stats.kernels += launches;
  c->indexed = true;
  return 0;
}

// Candidate lists of one strand pass are bounded: a batch that would need more is mapped in
// halves (reads are independent, so the results are the same).
constexpr int64_t kMaxCandidatesPerPass = 1000000000;
constexpr int64_t kMaxPassingPerPass = 100000000;  // their tracebacks are kept until the replay
constexpr int kSplitBatch = 1;

// S += s (everything but the index build time)
static void add_stats(stormgpu_stats& S, const stormgpu_stats& s) {
  S.candidates += s.candidates; S.filter_passed += s.filter_passed; S.aligned += s.aligned;
  S.seed_lookups += s.seed_lookups; S.hit_positions += s.hit_positions; S.filter_cells += s.filter_cells;
  S.align_cells += s.align_cells; S.kernels += s.kernels; S.filter_band_cells += s.filter_band_cells;
  S.ms_gather += s.ms_gather; S.ms_filter += s.ms_filter; S.ms_align += s.ms_align; S.passes += s.passes;
  S.ms_replay += s.ms_replay; S.ms_total += s.ms_total; S.graph_passes += s.graph_passes;
}

// sort keys of the length order: key = read length, value = read index
static __global__ void length_keys_kernel(const int16_t* __restrict__ lengths, int64_t n, uint32_t* __restrict__ keys,
                                          uint32_t* __restrict__ vals) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    keys[i] = (uint32_t)(uint16_t)lengths[i];
    vals[i] = (uint32_t)i;
  }
}

// Work weight of a read: its seed positions, about L - 15 (candidates grow with them).
static inline double read_weight(int L) { return L > 16 ? (double)(L - 15) : 1.0; }

// ------------------------------------------------------------------------------ graph passes
//
// Every strand pass of a call as one CUDA graph: the lists are sized up front (from the densest
// pass of the last call, +25 %), every launch takes its list size from device memory, and a
// one-thread gate after the gather and after the filter writes the size the next stages take,
// or 0 with a status when a list would not fit (or the batch must be cut): the passes from there
// on then do nothing, and the host, reading the status once after the graph, maps the call
// again with the host-synced passes.

constexpr int kGraphRetry = 2;

// words of the graph's device state (c->gstate)
enum : int {
  kGsCand = 0,    // candidates the filter of the current pass takes (0: skipped)
  kGsPass,        // passing candidates the alignment of the current pass takes (0: skipped)
  kGsStatus,      // 1: a list outgrew its capacity, 2: the batch must be cut, 4: too many passing
  kGsLookups,     // sums over the passes of the stage counters
  kGsPositions,
  kGsCandidates,
  kGsCells,
  kGsBand,
  kGsAlignCells,
  kGsPassed,
  kGsMaxCand,     // densest pass
  kGsMaxPass,
  kGsWords = 16
};

static __global__ void gate_gather_kernel(const unsigned long long* __restrict__ counters,
                                          const int32_t* __restrict__ big_count, int64_t cand_cap, int64_t cand_max,
                                          unsigned long long* __restrict__ gs) {
  const unsigned long long u = counters[7];
  unsigned long long s = gs[kGsStatus];
  // candidate list overflow, a read above the slices of the last gather launch, or a full list
  if (counters[8] || big_count[3] > 0 || u > (unsigned long long)cand_cap) s |= 1;
  if (u > (unsigned long long)cand_max) s |= 2;
  gs[kGsStatus] = s;
  gs[kGsCand] = s ? 0 : u;
  gs[kGsLookups] += counters[3];
  gs[kGsPositions] += counters[4];
  if (u > gs[kGsMaxCand]) gs[kGsMaxCand] = u;
}

static __global__ void gate_filter_kernel(const int64_t* __restrict__ total, int64_t pass_cap, int64_t pass_max,
                                          int64_t nreads, unsigned long long* __restrict__ gs) {
  const int64_t p = *total;
  unsigned long long s = gs[kGsStatus];
  if (p > pass_cap) s |= 4;
  if (p > pass_max && nreads > 1) s |= 2;
  gs[kGsStatus] = s;
  gs[kGsPass] = s ? 0 : (unsigned long long)p;
  if (!s) gs[kGsPassed] += (unsigned long long)p;
  if ((unsigned long long)p > gs[kGsMaxPass]) gs[kGsMaxPass] = (unsigned long long)p;
}

static __global__ void pass_sums_kernel(const unsigned long long* __restrict__ counters,
                                        unsigned long long* __restrict__ gs) {
  gs[kGsCandidates] += counters[5];
  gs[kGsCells] += counters[2];
  gs[kGsBand] += counters[6];
  gs[kGsAlignCells] += counters[13];
}

static void set_densities(stormgpu_ctx* c, double cand, double pass) {
  c->dens_cand = cand;
  c->dens_pass = pass;
  c->gdens_cand = std::max(cand, 0.9 * c->gdens_cand);
  c->gdens_pass = std::max(pass, 0.9 * c->gdens_pass);
}

// What the passes of one call share (set up by map_device_once before them).
struct PassSetup {
  ScoreParams sp;
  ReadsDev fwd, rev;
  int64_t n;
  int maxL, minL;
  double wsum;
  int wpr;          // scratch words per row of an alignment
  int64_t tbs;      // traceback bytes per passing candidate
  stormgpu_results* out;
};

// The lists a graph call needs (false: they could not be allocated, and the call runs without a
// graph).
static bool graph_buffers(stormgpu_ctx* c, const PassSetup& P, int64_t* cand_cap, int64_t* pass_cap,
                          int64_t* grid_h) {
  const int64_t n = P.n;
  const int64_t want_cand = (int64_t)(c->gdens_cand * P.wsum * 1.25) + 65536;
  const int64_t want_pass = (int64_t)(c->gdens_pass * P.wsum * 1.25) + 4096;
  const int64_t grid_b = gather_block_grid(false);
  *grid_h = std::max<int64_t>(1, std::min<int64_t>(grid_b, ((int64_t)1 << 25) / c->huge_cap));
  const int rounds = std::max(1, std::min<int>(c->tune.align_rounds, kMaxAlignRounds));
  if (c->fr.grow(want_cand) || c->fd.grow(want_cand) || c->big_count.grow(4) || c->gstate.grow(kGsWords) ||
      c->big_tmp.grow(std::max(grid_b * 2 * (int64_t)kBlockGatherCap, *grid_h * 2 * c->huge_cap)) ||
      c->rexp.grow(n * rexp_stride(P.maxL)))
    return false;
  *cand_cap = std::min(c->fr.cap, c->fd.cap);
  const int64_t nw = (*cand_cap + 31) / 32;
  if (c->flag.grow(nw * 32) || c->flagw.grow(nw) || c->foff.grow(nw + 1) ||
      c->scan_tmp64.grow(scan_tmp_elems(std::max<int64_t>(nw, n)) + 8) || c->p_read.grow(want_pass) ||
      c->p_diag.grow(want_pass) || c->a_score.grow(want_pass) || c->a_bound.grow(want_pass) ||
      c->a_tblen.grow(want_pass) || c->a_pos.grow(want_pass * 4) || c->a_tb.grow(want_pass * P.tbs))
    return false;
  *pass_cap = std::min({c->p_read.cap, c->p_diag.cap, c->a_score.cap, c->a_bound.cap, c->a_tblen.cap,
                        c->a_pos.cap / 4, c->a_tb.cap / P.tbs});
  if (c->scratch.grow(align_workers(*pass_cap, P.sp) * (int64_t)P.maxL * P.wpr)) return false;
  if (rounds > 1 && (c->thr.grow(n) || c->round_slots.grow(*pass_cap) || c->rounds.grow(16))) return false;
  return true;
}

// The launches of every pass on c's stream, each list size read from the device (captured into
// the graph; nothing here waits for the device).  E: the stage events, per_pass per pass.
static int enqueue_graph_passes(stormgpu_ctx* c, const PassSetup& P, int64_t cand_cap, int64_t pass_cap,
                                int64_t grid_h, int per_pass, int64_t& launches) {
  cudaStream_t st = c->st;
  const ScoreParams& sp = P.sp;
  const int64_t n = P.n;
  unsigned long long* gs = c->gstate.p;
  const int64_t nw = (cand_cap + 31) / 32;
  const int rounds = std::max(1, std::min<int>(c->tune.align_rounds, kMaxAlignRounds));
  const int64_t rstride = rexp_stride(P.maxL);
  const int64_t grid_s = gather_block_grid(true), grid_b = gather_block_grid(false);
  auto rec = [&](cudaEvent_t e) { return cudaEventRecordWithFlags(e, st, cudaEventRecordExternal); };
  SG_CUDA(cudaMemsetAsync(gs, 0, sizeof(unsigned long long) * kGsWords, st));
  int pi = 0;
  for (size_t ref_id = 0; ref_id < c->refs.size(); ++ref_id) {
    RefSeq& R = c->refs[ref_id];
    IndexView ix;
    memset(&ix, 0, sizeof(ix));
    for (int si = 0; si < c->seeds.n; ++si) { ix.first[si] = R.idx[si].first; ix.map[si] = R.idx[si].map; }
    for (int strand = 0; strand < 2; ++strand) {
      if (!(c->p.senses & (1 << strand))) continue;
      const ReadsDev& rd = strand ? P.rev : P.fwd;
      cudaEvent_t* E = c->gev.data() + (size_t)pi * per_pass;
      ++pi;
      SG_CUDA(rec(E[0]));
      // hit gather: the warp kernel, then the block kernels over the lists it filled, then the
      // reads above the block kernel's slices (reads above this launch's slices end the graph
      // call: the host-synced passes size their slices to fit)
      SG_CUDA(cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long) * 32, st));
      SG_CUDA(cudaMemsetAsync(c->big_count.p, 0, sizeof(int32_t) * 4, st));
      GatherOut go;
      go.fr = c->fr.p; go.fd = c->fd.p; go.cap = cand_cap; go.counters = c->counters.p;
      go.big_list = c->big_list.p; go.big_h = c->big_h.p; go.small_list = c->small_list.p;
      go.small_h = c->small_h.p; go.big_count = c->big_count.p;
      go.cursor = c->counters.p + 12;
      go.reads_per_steal = c->tune.gather_reads_per_steal;
      go.warp_cap = c->tune.gather_warp_cap;
      launch_gather_fused(rd, ix, sp.I, go, c->seeds, st);
      launch_gather_block(rd, ix, sp.I, c->small_list.p, c->small_h.p, n, c->big_count.p + 2, go, c->big_tmp.p,
                          kBlockGatherCap, grid_s, c->counters.p + 9, c->huge_list.p, c->huge_h.p, c->big_count.p + 1,
                          true, c->seeds, st);
      launch_gather_block(rd, ix, sp.I, c->big_list.p, c->big_h.p, n, c->big_count.p + 0, go, c->big_tmp.p,
                          kBlockGatherCap, grid_b, c->counters.p + 14, c->huge_list.p, c->huge_h.p,
                          c->big_count.p + 1, false, c->seeds, st);
      launch_gather_block(rd, ix, sp.I, c->huge_list.p, c->huge_h.p, n, c->big_count.p + 1, go, c->big_tmp.p,
                          (int)c->huge_cap, grid_h, c->counters.p + 15, c->huge_list.p + n, c->huge_h.p + n,
                          c->big_count.p + 3, false, c->seeds, st);
      gate_gather_kernel<<<1, 1, 0, st>>>(c->counters.p, c->big_count.p, cand_cap, kMaxCandidatesPerPass, gs);
      launches += 5;
      SG_CUDA(rec(E[1]));
      // filter over the gate's candidate count
      FilterJob job;
      memset(&job, 0, sizeof(job));
      if (c->tune.filter_cursor) job.cursor = c->counters.p + 10;
      job.rows = c->tune.filter_rows;
      job.n = cand_cap; job.n_dev = gs + kGsCand;
      job.fr = c->fr.p; job.fd = c->fd.p; job.flag = c->flag.p; job.codes = rd.codes;
      job.cstride = rd.cstride; job.lengths = rd.lengths; job.genome = R.d_codes; job.W = sp.W; job.Is = sp.Is;
      job.fm = sp.fm; job.fx = sp.fx; job.fo = sp.fo; job.fe = sp.fe; job.fthr = sp.fthr;
      job.counters = c->counters.p;
      launch_expand_reads(rd, c->rexp.p, rstride, st);
      job.gexp = R.d_gexp; job.rexp = c->rexp.p; job.rstride = rstride; job.min_len = P.minL;
      launch_filter_flat_job(job, sp, filter_dpx_ok(sp, P.maxL), st);
      launches += 2;
      SG_CUDA(rec(E[2]));
      // passing candidates, in order, over the whole capacity (the words past the count are zero)
      launch_pack_flags(cand_cap, gs + kGsCand, c->flag.p, c->flagw.p, st);
      exclusive_scan<PassWord, int64_t>(reinterpret_cast<const PassWord*>(c->flagw.p), c->foff.p, nw, c->foff.p + nw,
                                        c->scan_tmp64.p, st);
      gate_filter_kernel<<<1, 1, 0, st>>>(c->foff.p + nw, pass_cap, kMaxPassingPerPass, n, gs);
      launches += 2 + scan_launches(nw);
      const int64_t* np = reinterpret_cast<const int64_t*>(gs + kGsPass);
      PassBuffers pb;
      memset(&pb, 0, sizeof(pb));
      pb.pstart = c->pstart.p; pb.pcount = c->pcount.p;
      pb.counters = c->counters.p;
      SG_CUDA(cudaMemsetAsync(c->pcount.p, 0, sizeof(int32_t) * n, st));
      pb.p_read = c->p_read.p; pb.p_diag = c->p_diag.p; pb.p_cap = pass_cap;
      launch_compact(nw, c->flagw.p, c->foff.p, c->fr.p, c->fd.p, c->p_read.p, c->p_diag.p, pass_cap, st);
      launch_slot_bounds(pass_cap, np, c->p_read.p, c->pstart.p, c->pcount.p, st);
      launches += 3;
      pb.a_score = c->a_score.p; pb.a_bound = c->a_bound.p; pb.a_tblen = c->a_tblen.p;
      pb.a_pos = c->a_pos.p; pb.a_tb = c->a_tb.p; pb.tbs = P.tbs;
      pb.cursor = c->counters.p + 11;
      pb.npass_dev = np;
      pb.steal = c->tune.align_steal;
      pb.a_scratch = c->scratch.p;
      pb.cells = c->counters.p + 13;
      if (rounds == 1) {
        launch_align(rd, sp, R.d_codes, R.d_mask, 0, pass_cap, pb, st);
        launches++;
        SG_CUDA(rec(E[3]));
        launch_replay(n, sp, (int)ref_id, strand ? -1 : 1, pb, P.out->hits, P.out->tb, P.out->tb_stride,
                      P.out->mapped, st);
        launches++;
      } else {
        SG_CUDA(cudaMemsetAsync(c->rounds.p, 0, sizeof(int64_t) * 16, st));
        launch_round_lists(pass_cap, np, rounds, c->p_read.p, c->pstart.p, c->rounds.p,
                           reinterpret_cast<unsigned long long*>(c->rounds.p + 8), c->round_slots.p, st);
        launches += 2;
        pb.round_slots = c->round_slots.p;
        pb.round_count = c->rounds.p;
        pb.thr = c->thr.p;
        SG_CUDA(rec(E[5]));
        for (int k = 0; k < rounds; ++k) {
          pb.round = k;
          pb.cursor = c->counters.p + 16 + k;
          launch_align(rd, sp, R.d_codes, R.d_mask, 0, pass_cap, pb, st);
          SG_CUDA(rec(E[6 + 2 * k]));
          launch_replay_round(n, sp, (int)ref_id, strand ? -1 : 1, pb, rounds, P.out->hits, P.out->tb,
                              P.out->tb_stride, P.out->mapped, st);
          SG_CUDA(rec(E[7 + 2 * k]));
          launches += 2;
        }
        SG_CUDA(rec(E[3]));
      }
      pass_sums_kernel<<<1, 1, 0, st>>>(c->counters.p, gs);
      launches++;
      SG_CUDA(rec(E[4]));
    }
  }
  return 0;
}

// Every pass of the call as one graph.  0: done (results in P.out, stats in c->stats);
// kGraphRetry: the results are not usable (a list did not fit, or graphs do not work here) and
// the call must run the host-synced passes; else an error code.
static int map_passes_graph(stormgpu_ctx* c, const PassSetup& P, int64_t launches) {
  cudaStream_t st = c->st;
  int64_t cand_cap = 0, pass_cap = 0, grid_h = 0;
  if (!graph_buffers(c, P, &cand_cap, &pass_cap, &grid_h)) {
    cudaGetLastError();
    c->work.over = false;  // the host-synced passes allocate what they need, no more
    return kGraphRetry;
  }
  const int rounds = std::max(1, std::min<int>(c->tune.align_rounds, kMaxAlignRounds));
  const int per_pass = 5 + (rounds > 1 ? 1 + 2 * rounds : 0);
  int npasses = 0;
  for (size_t r = 0; r < c->refs.size(); ++r)
    for (int strand = 0; strand < 2; ++strand) npasses += (c->p.senses >> strand) & 1;
  while (c->gev.size() < (size_t)npasses * per_pass) {
    cudaEvent_t e;
    SG_CUDA(cudaEventCreate(&e));
    c->gev.push_back(e);
  }
  // capture (nothing runs), then update the last call's executable graph in place when the
  // shape is the same, else instantiate anew
  cudaGraph_t g = nullptr;
  auto broken = [&]() {
    cudaGetLastError();
    if (g) cudaGraphDestroy(g);
    c->graph_broken = true;
    return kGraphRetry;
  };
  if (cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed) != cudaSuccess) return broken();
  const int erc = enqueue_graph_passes(c, P, cand_cap, pass_cap, grid_h, per_pass, launches);
  const cudaError_t ece = cudaStreamEndCapture(st, &g);
  if (erc || ece != cudaSuccess || !g) return broken();
  bool ready = false;
  if (c->gexec) {
    cudaGraphExecUpdateResultInfo info;
    ready = cudaGraphExecUpdate(c->gexec, g, &info) == cudaSuccess;
    if (!ready) {
      cudaGetLastError();
      cudaGraphExecDestroy(c->gexec);
      c->gexec = nullptr;
    }
  }
  if (!ready && cudaGraphInstantiate(&c->gexec, g, 0) != cudaSuccess) {
    c->gexec = nullptr;
    return broken();
  }
  cudaGraphDestroy(g);
  g = nullptr;
  unsigned long long h[kGsWords];
  SG_CUDA(cudaEventRecord(c->ev[6], st));
  SG_CUDA(cudaGraphLaunch(c->gexec, st));
  SG_CUDA(cudaEventRecord(c->ev[7], st));
  SG_CUDA(cudaMemcpyAsync(h, c->gstate.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  SG_CUDA(cudaStreamSynchronize(st));
  SG_CUDA(cudaGetLastError());
  if (h[kGsStatus]) return kGraphRetry;
  stormgpu_stats& S = c->stats;
  S.candidates = (int64_t)h[kGsCandidates];
  S.filter_cells = (int64_t)h[kGsCells];
  S.filter_band_cells = (int64_t)h[kGsBand];
  S.seed_lookups = (int64_t)h[kGsLookups];
  S.hit_positions = (int64_t)h[kGsPositions];
  S.filter_passed = (int64_t)h[kGsPassed];
  S.aligned = (int64_t)h[kGsPassed];
  S.align_cells = (int64_t)h[kGsAlignCells];
  S.passes = npasses;
  S.graph_passes = npasses;
  // stage times from the graph's events (as the host-synced passes split them)
  float tg = 0, tf = 0, ta = 0, tr = 0, tt = 0;
  for (int pi = 0; pi < npasses; ++pi) {
    const cudaEvent_t* E = c->gev.data() + (size_t)pi * per_pass;
    float a = 0, b = 0, d = 0, e = 0;
    cudaEventElapsedTime(&a, E[0], E[1]);
    cudaEventElapsedTime(&b, E[1], E[2]);
    cudaEventElapsedTime(&d, E[2], E[3]);
    cudaEventElapsedTime(&e, E[3], E[4]);
    for (int k = 0; rounds > 1 && k < rounds; ++k) {
      float x = 0;
      cudaEventElapsedTime(&x, E[6 + 2 * k], E[7 + 2 * k]);
      d -= x;
      e += x;
    }
    tg += a; tf += b; ta += d; tr += e;
  }
  cudaEventElapsedTime(&tt, c->ev[6], c->ev[7]);
  cudaGetLastError();
  S.ms_gather = tg; S.ms_filter = tf; S.ms_align = ta; S.ms_replay = tr; S.ms_total = tt;
  S.kernels = launches;
  if (P.wsum > 0) set_densities(c, (double)h[kGsMaxCand] / P.wsum, (double)h[kGsMaxPass] / P.wsum);
  return 0;
}

static int map_device_once(stormgpu_ctx* c, const stormgpu_reads* reads, stormgpu_results* out) {
  if (!c->indexed) { sg_set_error("stormgpu_build_index must be called before mapping"); return STORMGPU_ESTATE; }
  cudaStream_t st = c->st;
  const int64_t n = reads->n;
  const ScoreParams sp = make_score_params(c->p);
  stormgpu_stats& S = c->stats;
  double ms_index = S.ms_index;
  memset(&S, 0, sizeof(S));
  S.ms_index = ms_index;
  int64_t launches = 0;
  int maxL = 0, minL = STORMGPU_MAX_READ_LEN;
  double wsum = 0;  // the batch's work weight (read_weight)
  {
    std::vector<int16_t> hl(n > 0 ? n : 1);
    if (n > 0) SG_CUDA(cudaMemcpyAsync(hl.data(), reads->lengths, sizeof(int16_t) * n, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaStreamSynchronize(st));
    for (int64_t r = 0; r < n; ++r) {
      maxL = std::max<int>(maxL, hl[r]);
      minL = std::min<int>(minL, hl[r]);
      wsum += read_weight(hl[r]);
    }
    if (maxL > STORMGPU_MAX_READ_LEN) { sg_set_error("read longer than %d", STORMGPU_MAX_READ_LEN); return STORMGPU_EINVAL; }
  }
  if (out->tb_stride < (maxL + c->p.allowed_indels + 1) / 2) { sg_set_error("tb_stride too small"); return STORMGPU_EINVAL; }
  launch_init_results(n, out->hits, out->mapped, out->tb, out->tb_stride, st);
  launches++;
  if (n == 0) return 0;
  ReadsDev fwd{n, reads->codes, reads->code_stride, reads->levels, reads->level_stride, reads->lengths, nullptr};
  if (minL != maxL) {
    // reads of several lengths: the gather visits them grouped by length (a stable sort of the
    // read indices by length); a batch in any read order then runs like one sorted by length
    if (c->ord.grow(4 * n) || c->ord_tmp.grow(radix_tmp_bytes(n) / 4 + 16)) return STORMGPU_ENOMEM;
    uint32_t *k0 = c->ord.p, *v0 = k0 + n, *k1 = v0 + n, *v1 = k1 + n;
    length_keys_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 8), 256, 0, st>>>(reads->lengths, n, k0, v0);
    int bits = 1;
    while ((1 << bits) <= maxL) ++bits;
    const int which = radix_sort_pairs(k0, v0, k1, v1, n, bits, c->ord_tmp.p, st);
    fwd.order = reinterpret_cast<const int32_t*>(which ? v1 : v0);
    launches += 1 + 3 * ((bits + kRadixBits - 1) / kRadixBits);
  }
  ReadsDev rev = fwd;
  if (c->p.senses & 2) {
    if (c->rcodes.grow(n * reads->code_stride)) return STORMGPU_ENOMEM;
    if (reads->levels && c->rlevels.grow(n * reads->level_stride)) return STORMGPU_ENOMEM;
    launch_reverse_reads(fwd, c->p.colour ? reads->first_levels : nullptr, c->p.colour, c->rcodes.p,
                         reads->levels ? c->rlevels.p : nullptr, st);
    launches++;
    rev.codes = c->rcodes.p;
    rev.levels = reads->levels ? c->rlevels.p : nullptr;
  }
  if (c->pstart.grow(n) || c->pcount.grow(n) || c->scan_tmp64.grow(scan_tmp_elems(n) + 8) ||
      c->big_list.grow(n) || c->big_h.grow(n) || c->small_list.grow(n) || c->small_h.grow(n) ||
      c->huge_list.grow(2 * n) || c->huge_h.grow(2 * n) || c->big_count.grow(3) ||
      c->counters.grow(32) || c->fr.grow(std::max<int64_t>(n * 64, 1 << 20)) ||
      c->fd.grow(std::max<int64_t>(n * 64, 1 << 20)))
    return STORMGPU_ENOMEM;
  const int BW = 2 * sp.I + 1;
  const int wpr = (2 * BW + 31) / 32 + (sp.colour ? (BW + 31) / 32 : 0);
  const int64_t tbs = ((maxL + sp.I + 1) / 2 + 7) & ~7LL;
  if (c->graphs && !c->graph_broken && c->gdens_cand > 0 && c->huge_cap <= ((int64_t)1 << 22)) {
    const PassSetup P{sp, fwd, rev, n, maxL, minL, wsum, wpr, tbs, out};
    const int g = map_passes_graph(c, P, launches);
    if (g != kGraphRetry) return g;
    // a list outgrew its capacity: the passes again, each sized by the host (the graph's
    // replays may have updated the results of its first passes)
    launch_init_results(n, out->hits, out->mapped, out->tb, out->tb_stride, st);
    launches++;
  }
  float tg = 0, tf = 0, ta = 0, tr = 0;
  int64_t max_cand = 0, max_pass = 0;  // densest strand pass of this call
  SG_CUDA(cudaEventRecord(c->ev[6], st));
  for (size_t ref_id = 0; ref_id < c->refs.size(); ++ref_id) {
    RefSeq& R = c->refs[ref_id];
    IndexView ix;
    memset(&ix, 0, sizeof(ix));
    for (int si = 0; si < c->seeds.n; ++si) { ix.first[si] = R.idx[si].first; ix.map[si] = R.idx[si].map; }
    for (int strand = 0; strand < 2; ++strand) {
      if (!(c->p.senses & (1 << strand))) continue;
      const ReadsDev& rd = strand ? rev : fwd;
      int64_t utot = 0;
      SG_CUDA(cudaEventRecord(c->ev[0], st));
      for (int attempt = 0;; ++attempt) {
        // fused hit gather: sorted, de-duplicated diagonals of every read, appended to the flat
        // candidate list (fr, fd); reads with many index positions go to the block kernel
        SG_CUDA(cudaMemsetAsync(c->counters.p, 0, sizeof(unsigned long long) * 32, st));
        SG_CUDA(cudaMemsetAsync(c->big_count.p, 0, sizeof(int32_t) * 3, st));
        GatherOut go;
        go.fr = c->fr.p; go.fd = c->fd.p; go.cap = c->fr.cap; go.counters = c->counters.p;
        go.big_list = c->big_list.p; go.big_h = c->big_h.p; go.small_list = c->small_list.p;
        go.small_h = c->small_h.p; go.big_count = c->big_count.p;
        go.cursor = c->counters.p + 12;  // zeroed just above
        go.reads_per_steal = c->tune.gather_reads_per_steal;
        go.warp_cap = c->tune.gather_warp_cap;
        launch_gather_fused(rd, ix, sp.I, go, c->seeds, st);
        launches++;
        int32_t nbig[3] = {0, 0, 0};  // handed to the block gather with many positions, above its slice, with few
        SG_CUDA(cudaMemcpyAsync(nbig, c->big_count.p, sizeof(nbig), cudaMemcpyDeviceToHost, st));
        SG_CUDA(cudaStreamSynchronize(st));
        if (nbig[2] > 0) {  // reads with few positions: sorted in shared memory
          const int64_t grid_s = std::min<int64_t>(nbig[2], gather_block_grid(true));
          launch_gather_block(rd, ix, sp.I, c->small_list.p, c->small_h.p, nbig[2], nullptr, go, c->big_tmp.p, kBlockGatherCap,
                              grid_s, c->counters.p + 9, c->huge_list.p, c->huge_h.p, c->big_count.p + 1, true,
                              c->seeds, st);
          launches++;
        }
        if (nbig[0] > 0) {  // reads with many positions: a block each, slices in global memory
          const int64_t grid = std::min<int64_t>(nbig[0], gather_block_grid(false));
          if (c->big_tmp.grow(grid * 2 * (int64_t)kBlockGatherCap)) return STORMGPU_ENOMEM;
          launch_gather_block(rd, ix, sp.I, c->big_list.p, c->big_h.p, nbig[0], nullptr, go, c->big_tmp.p, kBlockGatherCap,
                              grid, c->counters.p + 14, c->huge_list.p, c->huge_h.p, c->big_count.p + 1, false,
                              c->seeds, st);
          launches++;
          SG_CUDA(cudaMemcpyAsync(nbig + 1, c->big_count.p + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
          SG_CUDA(cudaStreamSynchronize(st));
          if (nbig[1] > 0) {  // beyond kBlockGatherCap: the same with a slice of the largest read's size
            std::vector<int32_t> hh(nbig[1]);
            SG_CUDA(cudaMemcpyAsync(hh.data(), c->huge_h.p, sizeof(int32_t) * nbig[1], cudaMemcpyDeviceToHost, st));
            SG_CUDA(cudaStreamSynchronize(st));
            int64_t cap2 = kBlockGatherCap;
            for (int k = 0; k < nbig[1]; ++k) while (cap2 < hh[k]) cap2 <<= 1;
            if (cap2 > (int64_t)1 << 30) { sg_set_error("a read has %lld index positions", (long long)cap2); return STORMGPU_EINVAL; }
            c->huge_cap = std::max<int64_t>(c->huge_cap, cap2);
            // at most 1 GiB of slices
            const int64_t grid2 = std::max<int64_t>(1, std::min<int64_t>({(int64_t)nbig[1], gather_block_grid(false),
                                                                           ((int64_t)1 << 27) / cap2}));
            if (c->big_tmp.grow(grid2 * 2 * cap2)) return STORMGPU_ENOMEM;
            launch_gather_block(rd, ix, sp.I, c->huge_list.p, c->huge_h.p, nbig[1], nullptr, go, c->big_tmp.p, (int)cap2,
                                grid2, c->counters.p + 15, c->huge_list.p + n, c->huge_h.p + n, c->big_count.p + 1,
                                false, c->seeds, st);
            launches++;
          }
        }
        unsigned long long g[9];
        SG_CUDA(cudaMemcpyAsync(g, c->counters.p, sizeof(g), cudaMemcpyDeviceToHost, st));
        SG_CUDA(cudaStreamSynchronize(st));
        utot = (int64_t)g[7];
        max_cand = std::max(max_cand, utot);
        if (utot > kMaxCandidatesPerPass) return kSplitBatch;
        if (!g[8]) break;
        if (attempt > 2) { sg_set_error("internal: candidate list overflow"); return STORMGPU_EINVAL; }
        if (c->fr.grow(utot + utot / 4 + 1024) || c->fd.grow(utot + utot / 4 + 1024)) return STORMGPU_ENOMEM;
      }
      const int64_t nwords = (utot + 31) / 32;
      if (c->flag.grow(std::max<int64_t>(nwords * 32, 1)) || c->flagw.grow(std::max<int64_t>(nwords, 1)) ||
          c->foff.grow(nwords + 1) ||
          c->scan_tmp64.grow(scan_tmp_elems(std::max<int64_t>(nwords, n)) + 8))
        return STORMGPU_ENOMEM;
      SG_CUDA(cudaEventRecord(c->ev[1], st));
      FilterJob job;
      memset(&job, 0, sizeof(job));
      if (c->tune.filter_cursor) job.cursor = c->counters.p + 10;  // zeroed with the counters of the pass
      job.rows = c->tune.filter_rows;
      job.n = utot; job.fr = c->fr.p; job.fd = c->fd.p; job.flag = c->flag.p; job.codes = rd.codes;
      job.cstride = rd.cstride; job.lengths = rd.lengths; job.genome = R.d_codes; job.W = sp.W; job.Is = sp.Is;
      job.fm = sp.fm; job.fx = sp.fx; job.fo = sp.fo; job.fe = sp.fe; job.fthr = sp.fthr;
      job.counters = c->counters.p;
      const int64_t rstride = rexp_stride(maxL);
      if (c->rexp.grow(n * rstride)) return STORMGPU_ENOMEM;
      launch_expand_reads(rd, c->rexp.p, rstride, st);
      job.gexp = R.d_gexp; job.rexp = c->rexp.p; job.rstride = rstride; job.min_len = minL;
      launch_filter_flat_job(job, sp, filter_dpx_ok(sp, maxL), st);
      launches += 2;
      S.passes++;
      SG_CUDA(cudaEventRecord(c->ev[2], st));
      launch_pack_flags(utot, nullptr, c->flag.p, c->flagw.p, st);
      launches += (utot > 0 ? 1 : 0) + scan_launches(nwords);
      exclusive_scan<PassWord, int64_t>(reinterpret_cast<const PassWord*>(c->flagw.p), c->foff.p, nwords,
                                        c->foff.p + nwords, c->scan_tmp64.p, st);
      unsigned long long cnt[8];
      int64_t npass = 0;
      SG_CUDA(cudaMemcpyAsync(&npass, c->foff.p + nwords, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaMemcpyAsync(cnt, c->counters.p, sizeof(cnt), cudaMemcpyDeviceToHost, st));
      SG_CUDA(cudaStreamSynchronize(st));
      if (utot == 0) npass = 0;
      S.candidates += (int64_t)cnt[5];
      S.filter_cells += (int64_t)cnt[2];
      S.filter_band_cells += (int64_t)cnt[6];
      S.seed_lookups += (int64_t)cnt[3];
      S.hit_positions += (int64_t)cnt[4];
      S.filter_passed += npass;
      max_pass = std::max(max_pass, npass);
      if (npass > kMaxPassingPerPass && n > 1) return kSplitBatch;
      PassBuffers pb;
      memset(&pb, 0, sizeof(pb));
      pb.pstart = c->pstart.p; pb.pcount = c->pcount.p;
      pb.counters = c->counters.p;
      SG_CUDA(cudaMemsetAsync(c->pcount.p, 0, sizeof(int32_t) * n, st));
      const int rounds = std::max(1, std::min<int>(c->tune.align_rounds, kMaxAlignRounds));
      if (npass > 0) {
        if (c->p_read.grow(npass) || c->p_diag.grow(npass) || c->a_score.grow(npass) || c->a_bound.grow(npass) ||
            c->a_tblen.grow(npass) || c->a_pos.grow(npass * 4) || c->a_tb.grow(npass * tbs))
          return STORMGPU_ENOMEM;
        pb.p_read = c->p_read.p; pb.p_diag = c->p_diag.p; pb.p_cap = c->p_read.cap;
        launch_compact(nwords, c->flagw.p, c->foff.p, c->fr.p, c->fd.p, c->p_read.p, c->p_diag.p, c->p_read.cap, st);
        launch_slot_bounds(npass, nullptr, c->p_read.p, c->pstart.p, c->pcount.p, st);
        launches += 3;
        pb.a_score = c->a_score.p; pb.a_bound = c->a_bound.p; pb.a_tblen = c->a_tblen.p;
        pb.a_pos = c->a_pos.p; pb.a_tb = c->a_tb.p; pb.tbs = tbs;
        // one persistent launch over all passing candidates; scratch for its threads only
        pb.cursor = c->counters.p + 11;  // zeroed with the counters at the start of the pass
        pb.steal = c->tune.align_steal;
        const int64_t per_slot = (int64_t)maxL * wpr;
        if (c->scratch.grow(align_workers(npass, sp) * per_slot)) return STORMGPU_ENOMEM;
        pb.a_scratch = c->scratch.p;
        pb.cells = c->counters.p + 13;
        if (rounds == 1) {
          launch_align(rd, sp, R.d_codes, R.d_mask, 0, npass, pb, st);
          launches++;
        } else {
          // rounds of increasing rank, each aligned with the thresholds the replay of the rounds
          // before left, then replayed
          if (c->thr.grow(n) || c->round_slots.grow(npass) || c->rounds.grow(16)) return STORMGPU_ENOMEM;
          SG_CUDA(cudaMemsetAsync(c->rounds.p, 0, sizeof(int64_t) * 16, st));
          launch_round_lists(npass, nullptr, rounds, c->p_read.p, c->pstart.p, c->rounds.p,
                             reinterpret_cast<unsigned long long*>(c->rounds.p + 8), c->round_slots.p, st);
          launches += 2;
          pb.round_slots = c->round_slots.p;
          pb.round_count = c->rounds.p;
          pb.thr = c->thr.p;
          SG_CUDA(cudaEventRecord(c->rev[0], st));
          for (int k = 0; k < rounds; ++k) {
            pb.round = k;
            pb.cursor = c->counters.p + 16 + k;  // zeroed with the counters of the pass
            launch_align(rd, sp, R.d_codes, R.d_mask, 0, npass, pb, st);
            SG_CUDA(cudaEventRecord(c->rev[2 * k + 1], st));
            launch_replay_round(n, sp, (int)ref_id, strand ? -1 : 1, pb, rounds, out->hits, out->tb, out->tb_stride,
                                out->mapped, st);
            SG_CUDA(cudaEventRecord(c->rev[2 * k + 2], st));
            launches += 2;
          }
        }
        S.aligned += npass;
      }
      SG_CUDA(cudaEventRecord(c->ev[3], st));
      if (npass > 0 && rounds == 1) {
        launch_replay(n, sp, (int)ref_id, strand ? -1 : 1, pb, out->hits, out->tb, out->tb_stride, out->mapped, st);
        launches++;
      }
      SG_CUDA(cudaEventRecord(c->ev[4], st));
      SG_CUDA(cudaEventSynchronize(c->ev[4]));
      float a, b, d, e;
      cudaEventElapsedTime(&a, c->ev[0], c->ev[1]);
      cudaEventElapsedTime(&b, c->ev[1], c->ev[2]);
      cudaEventElapsedTime(&d, c->ev[2], c->ev[3]);
      cudaEventElapsedTime(&e, c->ev[3], c->ev[4]);
      if (npass > 0 && rounds > 1) {  // the rounds' replays count as replay time
        for (int k = 0; k < rounds; ++k) {
          float x = 0;
          cudaEventElapsedTime(&x, c->rev[2 * k + 1], c->rev[2 * k + 2]);
          d -= x;
          e += x;
        }
      }
      tg += a; tf += b; ta += d; tr += e;
      if (npass > 0) {
        unsigned long long cells = 0;
        SG_CUDA(cudaMemcpyAsync(&cells, c->counters.p + 13, sizeof(cells), cudaMemcpyDeviceToHost, st));
        SG_CUDA(cudaStreamSynchronize(st));
        S.align_cells += (int64_t)cells;
      }
    }
  }
  SG_CUDA(cudaEventRecord(c->ev[7], st));
  SG_CUDA(cudaEventSynchronize(c->ev[7]));
  SG_CUDA(cudaGetLastError());
  float tt = 0;
  cudaEventElapsedTime(&tt, c->ev[6], c->ev[7]);
  S.ms_gather = tg; S.ms_filter = tf; S.ms_align = ta; S.ms_replay = tr; S.ms_total = tt;
  S.kernels = launches;
  if (n > 0 && wsum > 0) set_densities(c, (double)max_cand / wsum, (double)max_pass / wsum);
  return 0;
}

// Maps reads[lo, hi) into the matching part of out.
static int map_range(stormgpu_ctx* c, const stormgpu_reads* reads, stormgpu_results* out, int64_t lo, int64_t hi) {
  stormgpu_reads r = *reads;
  stormgpu_results o = *out;
  r.n = hi - lo;
  r.codes += lo * reads->code_stride;
  if (r.levels) r.levels += lo * reads->level_stride;
  r.lengths += lo;
  if (r.first_levels) r.first_levels += lo;
  o.hits += 4 * lo;
  o.tb += 4 * lo * out->tb_stride;
  o.mapped += lo;
  return sg::map_device_impl(c, &r, &o);
}

// Maps the batch as consecutive pieces [cuts[q], cuts[q + 1]), the stats summed.
static int map_cuts(stormgpu_ctx* c, const stormgpu_reads* reads, stormgpu_results* out,
                    const std::vector<int64_t>& cuts) {
  stormgpu_stats acc;
  memset(&acc, 0, sizeof(acc));
  for (size_t q = 0; q + 1 < cuts.size(); ++q) {
    if (cuts[q + 1] <= cuts[q]) continue;
    if (const int e = map_range(c, reads, out, cuts[q], cuts[q + 1])) return e;
    add_stats(acc, c->stats);
  }
  acc.ms_index = c->stats.ms_index;
  c->stats = acc;
  return 0;
}

// k consecutive pieces of (nearly) equal size
static int map_pieces(stormgpu_ctx* c, const stormgpu_reads* reads, stormgpu_results* out, int64_t k) {
  std::vector<int64_t> cuts;
  for (int64_t q = 0; q <= k; ++q) cuts.push_back(reads->n * q / k);
  return map_cuts(c, reads, out, cuts);
}

int sg::map_device_impl(stormgpu_ctx* c, const stormgpu_reads* reads, stormgpu_results* out) {
  if (reads->n > 1 && (c->dens_cand > 0 || c->dens_pass > 0)) {
    // at the last call's density per unit of work weight the batch would be cut after its
    // gather: cut it now, into pieces of equal weight (a batch's reads need not be mixed: a file
    // of several lengths often lists them one length after the other).  0.8: the pieces still
    // differ in repeat content; one that overflows is cut after its gather.
    const int64_t n = reads->n;
    std::vector<int16_t> hl(n);
    SG_CUDA(cudaMemcpyAsync(hl.data(), reads->lengths, sizeof(int16_t) * n, cudaMemcpyDeviceToHost, c->st));
    SG_CUDA(cudaStreamSynchronize(c->st));
    std::vector<double> cum(n + 1, 0.0);
    for (int64_t r = 0; r < n; ++r) cum[r + 1] = cum[r] + read_weight(hl[r]);
    const double W = cum[n];
    const double need = std::max(c->dens_cand * W / (0.8 * (double)kMaxCandidatesPerPass),
                                 c->dens_pass * W / (0.8 * (double)kMaxPassingPerPass));
    if (need > 1.0) {
      const int64_t k = std::min<int64_t>(n, (int64_t)std::ceil(need));
      std::vector<int64_t> cuts(1, 0);
      for (int64_t q = 1; q < k; ++q) {  // strictly increasing, every piece smaller than the batch
        int64_t cut = std::lower_bound(cum.begin(), cum.end(), W * (double)q / (double)k) - cum.begin();
        cut = std::min<int64_t>(std::max<int64_t>(cut, cuts.back() + 1), n - (k - q));
        cuts.push_back(cut);
      }
      cuts.push_back(n);
      return map_cuts(c, reads, out, cuts);
    }
  }
  WorkBudget* saved = g_work_budget;
  g_work_budget = &c->work;
  c->work.over = false;
  int rc = map_device_once(c, reads, out);
  g_work_budget = saved;
  const int64_t n = reads->n;
  if (rc == STORMGPU_ENOMEM && c->work.over) {
    if (n <= 1) {
      sg_set_error("one read needs more than the working memory limit of %lld bytes", (long long)c->work.limit);
      return STORMGPU_ENOMEM;
    }
    rc = kSplitBatch;
  }
  if (rc != kSplitBatch) return rc;
  if (n <= 1) {
    sg_set_error("one read has more than %lld candidate diagonals", (long long)kMaxCandidatesPerPass);
    return STORMGPU_ENOMEM;
  }
  return map_pieces(c, reads, out, 2);
}

extern "C" int stormgpu_map_device(stormgpu_ctx* c, const stormgpu_reads* reads, stormgpu_results* out,
                                   void* stream) {
  if (!c || !reads || !out) { sg_set_error("null argument"); return STORMGPU_EINVAL; }
  SG_CUDA(cudaSetDevice(c->p.device));
  cudaStream_t user = (cudaStream_t)stream;
  if (user) {
    cudaEvent_t e;
    SG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    SG_CUDA(cudaEventRecord(e, user));
    SG_CUDA(cudaStreamWaitEvent(c->st, e, 0));
    cudaEventDestroy(e);
  }
  int rc = map_device_impl(c, reads, out);
  if (rc == 0 && user) {
    cudaEvent_t e;
    SG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    SG_CUDA(cudaEventRecord(e, c->st));
    SG_CUDA(cudaStreamWaitEvent(user, e, 0));
    cudaEventDestroy(e);
  }
  return rc;
}

extern "C" int stormgpu_sync(stormgpu_ctx* c) {
  if (!c) return STORMGPU_EINVAL;
  SG_CUDA(cudaStreamSynchronize(c->st));
  return 0;
}

extern "C" int stormgpu_map(stormgpu_ctx* c, const stormgpu_reads* reads, stormgpu_results* out) {
  if (!c || !reads || !out || reads->n < 0) { sg_set_error("null argument"); return STORMGPU_EINVAL; }
  SG_CUDA(cudaSetDevice(c->p.device));
  const int64_t n = reads->n;
  cudaStream_t st = c->st;
  if (c->fcodes.grow(std::max<int64_t>(n * reads->code_stride, 1)) || c->lengths.grow(std::max<int64_t>(n, 1)) ||
      c->hits.grow(std::max<int64_t>(n * 4, 1)) || c->tb.grow(std::max<int64_t>(n * 4 * out->tb_stride, 1)) ||
      c->mapped.grow(std::max<int64_t>(n, 1)))
    return STORMGPU_ENOMEM;
  if (reads->levels && c->flevels.grow(std::max<int64_t>(n * reads->level_stride, 1))) return STORMGPU_ENOMEM;
  if (reads->first_levels && c->first_levels.grow(std::max<int64_t>(n, 1))) return STORMGPU_ENOMEM;
  if (n > 0) {
    SG_CUDA(cudaMemcpyAsync(c->fcodes.p, reads->codes, n * reads->code_stride, cudaMemcpyHostToDevice, st));
    SG_CUDA(cudaMemcpyAsync(c->lengths.p, reads->lengths, sizeof(int16_t) * n, cudaMemcpyHostToDevice, st));
    if (reads->levels) SG_CUDA(cudaMemcpyAsync(c->flevels.p, reads->levels, n * reads->level_stride, cudaMemcpyHostToDevice, st));
    if (reads->first_levels) SG_CUDA(cudaMemcpyAsync(c->first_levels.p, reads->first_levels, n, cudaMemcpyHostToDevice, st));
  }
  stormgpu_reads dr = *reads;
  dr.codes = c->fcodes.p;
  dr.levels = reads->levels ? c->flevels.p : nullptr;
  dr.lengths = c->lengths.p;
  dr.first_levels = reads->first_levels ? c->first_levels.p : nullptr;
  stormgpu_results dres;
  dres.hits = c->hits.p;
  dres.tb = c->tb.p;
  dres.tb_stride = out->tb_stride;
  dres.mapped = c->mapped.p;
  int rc = map_device_impl(c, &dr, &dres);
  if (rc) return rc;
  c->last_n = n;
  c->last_tbs = out->tb_stride;
  if (n > 0) {
    SG_CUDA(cudaMemcpyAsync(out->hits, c->hits.p, sizeof(stormgpu_hit) * n * 4, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaMemcpyAsync(out->tb, c->tb.p, n * 4 * out->tb_stride, cudaMemcpyDeviceToHost, st));
    SG_CUDA(cudaMemcpyAsync(out->mapped, c->mapped.p, n, cudaMemcpyDeviceToHost, st));
  }
  SG_CUDA(cudaStreamSynchronize(st));
  return 0;
}

extern "C" int stormgpu_get_stats(stormgpu_ctx* c, stormgpu_stats* out) {
  if (!c || !out) return STORMGPU_EINVAL;
  *out = c->stats;
  return 0;
}

// ------------------------------------------------------------------------------ unit level

namespace {
int upload_padded(const uint8_t* h, int64_t n_codes, int64_t pad_codes, uint8_t fill, uint8_t** alloc,
                  uint8_t** base) {
  (void)pad_codes;
  const int64_t nb = (n_codes + 3) / 4;
  const int64_t tot = nb + 2 * kPadBytes + 16;
  SG_CUDA(cudaMalloc(alloc, tot));
  SG_CUDA(cudaMemset(*alloc, fill, tot));
  *base = *alloc + kPadBytes;
  if (nb) {
    std::vector<uint8_t> v(h, h + nb);
    for (int64_t k = n_codes; k & 3; ++k) {  // codes past the end: 0 (sequence) or 1 (mask)
      v[k >> 2] &= (uint8_t)~(3u << ((k & 3) << 1));
      if (fill) v[k >> 2] |= (uint8_t)(1u << ((k & 3) << 1));
    }
    SG_CUDA(cudaMemcpy(*base, v.data(), nb, cudaMemcpyHostToDevice));
  }
  return 0;
}
}  // namespace

extern "C" int stormgpu_sw_filter(int W, int read_len, uint32_t match, uint32_t mismatch, uint32_t gapopen,
                                  uint32_t gapext, uint32_t threshold, const uint8_t* genome, int64_t n_codes,
                                  int64_t pad, const int32_t* pos, int64_t n, const uint8_t* read, uint8_t* pass) {
  if (!(W == 2 || W == 4 || W == 8 || W == 16) || read_len <= 0 || read_len > STORMGPU_MAX_READ_LEN || n < 0) {
    sg_set_error("bad filter arguments");
    return STORMGPU_EINVAL;
  }
  for (int64_t k = 0; k < n; ++k)
    if (pos[k] < -(4 * (int64_t)kPadBytes - 64) || pos[k] + read_len + 2 * W > n_codes + 4 * (int64_t)kPadBytes - 64) {
      sg_set_error("window %lld outside the padded genome", (long long)pos[k]);
      return STORMGPU_EINVAL;
    }
  ScoreParams sp;
  memset(&sp, 0, sizeof(sp));
  sp.fm = match & 0xff; sp.fx = mismatch & 0xff; sp.fo = gapopen & 0xff; sp.fe = gapext & 0xff;
  sp.fthr = threshold >= 255u ? 254 : (int)threshold;
  sp.W = W;
  uint8_t *ga, *gb, *dr, *dp;
  int32_t* dpos;
  if (upload_padded(genome, n_codes, pad, 0, &ga, &gb)) return STORMGPU_ECUDA;
  const int rb = (read_len + 2 * W + 16) / 4 + 16;
  std::vector<uint8_t> hr(rb, 0);
  memcpy(hr.data(), read, (read_len + 3) / 4);
  SG_CUDA(cudaMalloc(&dr, rb));
  SG_CUDA(cudaMemcpy(dr, hr.data(), rb, cudaMemcpyHostToDevice));
  SG_CUDA(cudaMalloc(&dpos, sizeof(int32_t) * std::max<int64_t>(n, 1)));
  SG_CUDA(cudaMalloc(&dp, std::max<int64_t>(n, 1)));
  if (n) SG_CUDA(cudaMemcpy(dpos, pos, sizeof(int32_t) * n, cudaMemcpyHostToDevice));
  {
    int16_t L16 = (int16_t)read_len;
    int16_t* dl;
    int32_t* dzero;
    SG_CUDA(cudaMalloc(&dl, sizeof(int16_t)));
    SG_CUDA(cudaMemcpy(dl, &L16, sizeof(int16_t), cudaMemcpyHostToDevice));
    SG_CUDA(cudaMalloc(&dzero, sizeof(int32_t) * std::max<int64_t>(n, 1)));
    SG_CUDA(cudaMemset(dzero, 0, sizeof(int32_t) * std::max<int64_t>(n, 1)));
    uint8_t *gx, *rx;
    const int64_t rstride = rexp_stride(read_len);
    SG_CUDA(cudaMalloc(&gx, n_codes + 2 * kGexpPad + 16));
    SG_CUDA(cudaMemset(gx, 0, n_codes + 2 * kGexpPad + 16));
    SG_CUDA(cudaMalloc(&rx, rstride));
    launch_expand_genome(gb, n_codes, gx + kGexpPad, 0);
    ReadsDev one{1, dr, rb, nullptr, 0, dl};
    launch_expand_reads(one, rx, rstride, 0);
    FilterJob job;
    memset(&job, 0, sizeof(job));
    job.n = n; job.fr = dzero; job.fd = dpos; job.flag = dp; job.codes = dr; job.cstride = rb;
    job.lengths = dl; job.genome = gb; job.W = W; job.Is = 0;
    job.gexp = gx + kGexpPad; job.rexp = rx; job.rstride = rstride; job.min_len = read_len;
    job.fm = sp.fm; job.fx = sp.fx; job.fo = sp.fo; job.fe = sp.fe; job.fthr = sp.fthr;
    launch_filter_flat_job(job, sp, filter_dpx_ok(sp, read_len), 0);
    SG_CUDA(cudaGetLastError());
    SG_CUDA(cudaDeviceSynchronize());
    cudaFree(dl);
    cudaFree(dzero);
    cudaFree(gx);
    cudaFree(rx);
  }
  SG_CUDA(cudaGetLastError());
  SG_CUDA(cudaDeviceSynchronize());
  if (n) SG_CUDA(cudaMemcpy(pass, dp, n, cudaMemcpyDeviceToHost));
  cudaFree(ga); cudaFree(dr); cudaFree(dpos); cudaFree(dp);
  return 0;
}

extern "C" int stormgpu_align(const stormgpu_params* params, const uint8_t* read, const uint8_t* levels,
                              int read_len, const uint8_t* genome, const uint8_t* mask, int64_t n_codes,
                              int64_t pad, const int32_t* win, int64_t n, int32_t* score, int32_t* bound,
                              int16_t* best, int32_t* tb_len, uint8_t* tb, int64_t tb_stride) {
  if (!params || read_len <= 0 || read_len > STORMGPU_MAX_READ_LEN || n < 0 ||
      params->allowed_indels < 0 || params->allowed_indels > STORMGPU_MAX_INDELS) {
    sg_set_error("bad align arguments");
    return STORMGPU_EINVAL;
  }
  const int I = params->allowed_indels;
  if (tb_stride < (read_len + I + 1) / 2) { sg_set_error("tb_stride too small"); return STORMGPU_EINVAL; }
  for (int64_t k = 0; k < n; ++k)
    if (win[k] < -(4 * (int64_t)kPadBytes - 64) || win[k] + read_len + 2 * I > n_codes + 4 * (int64_t)kPadBytes - 64) {
      sg_set_error("window outside the padded genome");
      return STORMGPU_EINVAL;
    }
  ScoreParams sp = make_score_params(*params);
  sp.Is = 1 << 28;              // window = diag - I exactly
  sp.min_score = -(1 << 29);    // always trace back
  sp.packed = 0;                // every cell exact: no floor
  uint8_t *ga, *gb, *ma, *mb;
  if (upload_padded(genome, n_codes, pad, 0, &ga, &gb)) return STORMGPU_ECUDA;
  if (upload_padded(mask, n_codes, pad, 0x55, &ma, &mb)) return STORMGPU_ECUDA;
  const int64_t rb = ((read_len + 3) / 4 + 15) & ~7;
  std::vector<uint8_t> hr(rb, 0), hq(rb, 0);
  memcpy(hr.data(), read, (read_len + 3) / 4);
  if (levels) memcpy(hq.data(), levels, (read_len + 3) / 4);
  uint8_t *dr, *dq = nullptr;
  int16_t* dl;
  SG_CUDA(cudaMalloc(&dr, rb));
  SG_CUDA(cudaMemcpy(dr, hr.data(), rb, cudaMemcpyHostToDevice));
  if (levels) {
    SG_CUDA(cudaMalloc(&dq, rb));
    SG_CUDA(cudaMemcpy(dq, hq.data(), rb, cudaMemcpyHostToDevice));
  }
  int16_t L16 = (int16_t)read_len;
  SG_CUDA(cudaMalloc(&dl, sizeof(int16_t)));
  SG_CUDA(cudaMemcpy(dl, &L16, sizeof(int16_t), cudaMemcpyHostToDevice));
  ReadsDev rd{1, dr, rb, dq, rb, dl};
  PassBuffers pb;
  memset(&pb, 0, sizeof(pb));
  const int64_t nn = std::max<int64_t>(n, 1);
  const int BW = 2 * I + 1;
  const int wpr = (2 * BW + 31) / 32 + (params->colour ? (BW + 31) / 32 : 0);
  const int64_t tbs = ((read_len + I + 1) / 2 + 7) & ~7LL;
  std::vector<int32_t> zeros(nn, 0), diag(nn, 0);
  for (int64_t k = 0; k < n; ++k) diag[k] = win[k] + I;
  SG_CUDA(cudaMalloc(&pb.p_read, sizeof(int32_t) * nn));
  SG_CUDA(cudaMalloc(&pb.p_diag, sizeof(int32_t) * nn));
  SG_CUDA(cudaMalloc(&pb.a_score, sizeof(int32_t) * nn));
  SG_CUDA(cudaMalloc(&pb.a_bound, sizeof(int32_t) * nn));
  SG_CUDA(cudaMalloc(&pb.a_tblen, sizeof(int32_t) * nn));
  SG_CUDA(cudaMalloc(&pb.a_pos, sizeof(int16_t) * 4 * nn));
  SG_CUDA(cudaMalloc(&pb.a_tb, tbs * nn));
  SG_CUDA(cudaMalloc(&pb.a_scratch, sizeof(uint32_t) * (size_t)read_len * wpr * nn));
  pb.tbs = tbs;
  SG_CUDA(cudaMemcpy(pb.p_read, zeros.data(), sizeof(int32_t) * nn, cudaMemcpyHostToDevice));
  SG_CUDA(cudaMemcpy(pb.p_diag, diag.data(), sizeof(int32_t) * nn, cudaMemcpyHostToDevice));
  launch_align(rd, sp, gb, mb, 0, n, pb, 0);
  SG_CUDA(cudaGetLastError());
  SG_CUDA(cudaDeviceSynchronize());
  if (n) {
    SG_CUDA(cudaMemcpy(score, pb.a_score, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    SG_CUDA(cudaMemcpy(bound, pb.a_bound, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    SG_CUDA(cudaMemcpy(best, pb.a_pos, sizeof(int16_t) * 4 * n, cudaMemcpyDeviceToHost));
    SG_CUDA(cudaMemcpy(tb_len, pb.a_tblen, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    std::vector<uint8_t> htb(tbs * n);
    SG_CUDA(cudaMemcpy(htb.data(), pb.a_tb, tbs * n, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < n; ++k) {
      memset(tb + k * tb_stride, 0, tb_stride);
      memcpy(tb + k * tb_stride, htb.data() + k * tbs, std::min<int64_t>(tbs, tb_stride));
    }
  }
  cudaFree(ga); cudaFree(ma); cudaFree(dr); if (dq) cudaFree(dq); cudaFree(dl);
  cudaFree(pb.p_read); cudaFree(pb.p_diag); cudaFree(pb.a_score); cudaFree(pb.a_bound);
  cudaFree(pb.a_tblen); cudaFree(pb.a_pos); cudaFree(pb.a_tb); cudaFree(pb.a_scratch);
  return 0;
}

extern "C" int stormgpu_index_one(const char* seed, int32_t stdev_distance, const uint8_t* codes, int64_t n_codes,
                                  int64_t pad, const int32_t* rs, const int32_t* re, int32_t n_regions,
                                  int32_t* first, int32_t* map, int64_t map_capacity, int64_t* map_len) {
  SeedSet ss;
  if (parse_seeds(seed, &ss) != 0 || ss.n < 1) { sg_set_error("invalid seed"); return STORMGPU_EINVAL; }
  uint8_t *ga, *gb;
  if (upload_padded(codes, n_codes, pad, 0, &ga, &gb)) return STORMGPU_ECUDA;
  DevIndex ix;
  int rc = build_one_index(gb, n_codes, rs, re, n_regions, ss.s[0], stdev_distance, &ix, 0, nullptr);
  if (rc) { cudaFree(ga); return rc; }
  SG_CUDA(cudaDeviceSynchronize());
  SG_CUDA(cudaMemcpy(first, ix.first, sizeof(int32_t) * (ix.nkeys + 1), cudaMemcpyDeviceToHost));
  if (ix.n > map_capacity) { sg_set_error("map_capacity too small"); cudaFree(ga); return STORMGPU_EINVAL; }
  if (ix.n) SG_CUDA(cudaMemcpy(map, ix.map, sizeof(int32_t) * ix.n, cudaMemcpyDeviceToHost));
  *map_len = ix.n;
  cudaFree(ix.first);
  if (ix.map) cudaFree(ix.map);
  cudaFree(ga);
  return 0;
}
