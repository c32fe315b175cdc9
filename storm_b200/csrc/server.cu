// server.cu -- the served form of the mapping path (stormgpu_server_* in include/stormgpu.h).
//
// The reference and the index of every step of an -O seed chain stay resident.  Batches of
// reads are submitted from any host thread and admitted, in arrival order, as soon as one of
// the `slots` workers is free and the device memory their reads need fits what the batches in
// flight leave of the server's budget (continuous batching); every worker has its own stream
// and buffers, so admitted batches overlap on the GPU.  A batch runs the whole chain on the
// device: step k maps the reads that no earlier step mapped (the reads for which the reference
// writes nothing but the -O FASTQ, hit_map.c:514-579) with the k-th seed family, in the same
// relative order, exactly as the reference run again on its own -O output would (README:97-101).
// Each read's results are those of the step that mapped it, plus that step's number.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>

#include "context.cuh"
#include "map_kernels.cuh"
#include "scan.cuh"

namespace {

using namespace sg;

__global__ void iota_kernel(int32_t* ids, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    ids[i] = (int32_t)i;
}

// Results of the reads mapped at this step go to their place in the batch; unmapped[i] = 1
// for the others (the next step's reads).
__global__ void chain_scatter_kernel(int64_t m, const int32_t* __restrict__ ids, const stormgpu_hit* __restrict__ hits,
                                     const uint8_t* __restrict__ tb, const uint8_t* __restrict__ mapped, int64_t tbs,
                                     int step, stormgpu_hit* __restrict__ hits_all, uint8_t* __restrict__ tb_all,
                                     uint8_t* __restrict__ mapped_all, uint8_t* __restrict__ step_all,
                                     uint8_t* __restrict__ unmapped) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const bool mp = mapped[i] != 0;
    unmapped[i] = mp ? 0 : 1;
    if (!mp) continue;
    const int64_t o = ids[i];
    for (int k = 0; k < 4; ++k) hits_all[o * 4 + k] = hits[i * 4 + k];
    for (int64_t b = 0; b < 4 * tbs; ++b) tb_all[o * 4 * tbs + b] = tb[i * 4 * tbs + b];
    mapped_all[o] = 1;
    step_all[o] = (uint8_t)step;
  }
}

// Order-preserving compaction of the unmapped reads into the other chain buffer.
__global__ void chain_compact_kernel(int64_t m, const uint8_t* __restrict__ unmapped, const int64_t* __restrict__ off,
                                     const uint8_t* __restrict__ codes, int64_t cstride,
                                     const uint8_t* __restrict__ levels, int64_t lstride,
                                     const int16_t* __restrict__ lengths, const uint8_t* __restrict__ first_levels,
                                     const int32_t* __restrict__ ids, uint8_t* __restrict__ codes2,
                                     uint8_t* __restrict__ levels2, int16_t* __restrict__ lengths2,
                                     uint8_t* __restrict__ first_levels2, int32_t* __restrict__ ids2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    if (!unmapped[i]) continue;
    const int64_t o = off[i];
    for (int64_t b = 0; b < cstride; ++b) codes2[o * cstride + b] = codes[i * cstride + b];
    if (levels)
      for (int64_t b = 0; b < lstride; ++b) levels2[o * lstride + b] = levels[i * lstride + b];
    lengths2[o] = lengths[i];
    if (first_levels) first_levels2[o] = first_levels[i];
    ids2[o] = ids[i];
  }
}

unsigned grid_for(int64_t n) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)(b > 0 ? b : 1);
}

struct Request {
  int64_t ticket = 0;
  stormgpu_reads reads;
  stormgpu_results out;
  uint8_t* step = nullptr;
  int64_t bytes = 0;
  std::chrono::steady_clock::time_point t_submit, t_done;
  int status = 1;  // 1 pending, 0 done, < 0 error
  std::string err;
};

// One worker: a view context (stream + mapping buffers, whose working memory is capped) and a
// pinned host staging area for the batch's copies.
struct Slot {
  stormgpu_ctx* ws = nullptr;
  // candidates and passing candidates per unit of work weight of the densest pass of the last
  // batch, per chain step (each step's seeds have their own): the sizes of a step's graph
  double dens[16][4] = {};
  uint8_t* staging = nullptr;  // pinned host memory
  int64_t staging_cap = 0;
  std::thread th;
  void release() {
    if (staging) cudaFreeHost(staging);
    staging = nullptr;
    staging_cap = 0;
  }
};

// The device memory of one batch's chain, besides the slot's mapping buffers: two copies of its
// reads (the reads of the current step and the compacted unmapped ones), their indices, the
// results of a step and of the batch, and the bookkeeping of the compaction; one stream-ordered
// allocation of exactly this size per batch, returned when the batch ends.
struct ChainLayout {
  int64_t codes[2], levels[2], first_levels[2], lengths[2], ids[2];
  int64_t hits, hits_all, tb, tb_all, mapped, mapped_all, step_all, unmapped, off, scan_tmp;
  int64_t bytes;
};

ChainLayout chain_layout(const stormgpu_reads* r, int64_t tbs) {
  const int64_t n = std::max<int64_t>(r->n, 1);
  ChainLayout L;
  int64_t at = 0;
  auto take = [&](int64_t bytes) {
    const int64_t o = at;
    at += (bytes + 255) & ~255LL;
    return o;
  };
  for (int k = 0; k < 2; ++k) {
    L.codes[k] = take(n * r->code_stride);
    L.levels[k] = take(r->levels ? n * r->level_stride : 0);
    L.first_levels[k] = take(r->first_levels ? n : 0);
    L.lengths[k] = take(n * (int64_t)sizeof(int16_t));
    L.ids[k] = take(n * (int64_t)sizeof(int32_t));
  }
  L.hits = take((n * 4 + 4) * (int64_t)sizeof(stormgpu_hit));
  L.hits_all = take((n * 4 + 4) * (int64_t)sizeof(stormgpu_hit));
  L.tb = take(n * 4 * tbs + 4);
  L.tb_all = take(n * 4 * tbs + 4);
  L.mapped = take(n + 1);
  L.mapped_all = take(n + 1);
  L.step_all = take(n + 1);
  L.unmapped = take(n + 1);
  L.off = take((n + 2) * (int64_t)sizeof(int64_t));
  L.scan_tmp = take((scan_tmp_elems(n + 1) + 8) * (int64_t)sizeof(int64_t));
  L.bytes = at;
  return L;
}

}  // namespace

struct stormgpu_server {
  stormgpu_params p;
  std::vector<stormgpu_ctx*> steps;
  std::vector<Slot*> slots;
  int nslots = 1;
  // budget: device memory for the batches, besides the resident sequences and indexes.  Half
  // of it is the slots' mapping buffers (work_cap each, never exceeded: a pass that would need
  // more maps its reads in halves); the other half, chain_budget, is shared by the chains of the
  // batches in flight, each charged its exact chain size when admitted.
  int64_t budget = 0, work_cap = 0, chain_budget = 0, in_use = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::map<int64_t, Request*> reqs;
  int64_t next_ticket = 1;
  bool built = false, stop = false;
  stormgpu_tuning tune = {768, 4, 8, 32, 0, 4};  // launch parameters of every slot
};

namespace {

int run_chain(stormgpu_server* s, Slot* sl, Request* q, std::string& err) {
  stormgpu_ctx* ws = sl->ws;
  cudaStream_t st = ws->st;
  const stormgpu_reads& R = q->reads;
  const int64_t n = R.n, cs = R.code_stride, ls = R.levels ? R.level_stride : 0, tbs = q->out.tb_stride;
  const bool lv = R.levels != nullptr, fl = R.first_levels != nullptr;
  auto fail = [&](int rc) { err = stormgpu_last_error(); return rc; };
  const ChainLayout lay = chain_layout(&R, tbs);
  uint8_t* blk = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void**>(&blk), (size_t)lay.bytes, st) != cudaSuccess) {
    cudaGetLastError();
    err = "stormgpu_submit: the chain buffers of the batch (" + std::to_string(lay.bytes) + " bytes) could not be allocated";
    return STORMGPU_ENOMEM;
  }
  struct ChainView {
    uint8_t *codes[2], *levels[2], *first_levels[2];
    int16_t* lengths[2];
    int32_t* ids[2];
    stormgpu_hit *hits, *hits_all;
    uint8_t *tb, *tb_all, *mapped, *mapped_all, *step_all, *unmapped;
    int64_t *off, *scan_tmp;
  } cv;
  for (int k = 0; k < 2; ++k) {
    cv.codes[k] = blk + lay.codes[k];
    cv.levels[k] = blk + lay.levels[k];
    cv.first_levels[k] = blk + lay.first_levels[k];
    cv.lengths[k] = reinterpret_cast<int16_t*>(blk + lay.lengths[k]);
    cv.ids[k] = reinterpret_cast<int32_t*>(blk + lay.ids[k]);
  }
  cv.hits = reinterpret_cast<stormgpu_hit*>(blk + lay.hits);
  cv.hits_all = reinterpret_cast<stormgpu_hit*>(blk + lay.hits_all);
  cv.tb = blk + lay.tb;
  cv.tb_all = blk + lay.tb_all;
  cv.mapped = blk + lay.mapped;
  cv.mapped_all = blk + lay.mapped_all;
  cv.step_all = blk + lay.step_all;
  cv.unmapped = blk + lay.unmapped;
  cv.off = reinterpret_cast<int64_t*>(blk + lay.off);
  cv.scan_tmp = reinterpret_cast<int64_t*>(blk + lay.scan_tmp);
  // the chain block goes back to the pool on every way out (stream-ordered, no device sync)
  struct FreeAtEnd {
    uint8_t* p;
    cudaStream_t st;
    ~FreeAtEnd() {
      cudaFreeAsync(p, st);
      cudaStreamSynchronize(st);
    }
  } free_at_end{blk, st};
#define SGS(call)                                                        \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      err = std::string(#call) + ": " + cudaGetErrorString(e_);          \
      return STORMGPU_ECUDA;                                             \
    }                                                                    \
  } while (0)
  // host copies through the slot's pinned staging: the transfers then overlap the other slots'
  // kernels; results come back the same way
  const int64_t in_bytes = n * cs + n * (int64_t)sizeof(int16_t) + (lv ? n * ls : 0) + (fl ? n : 0);
  const int64_t out_bytes = n * 4 * (int64_t)sizeof(stormgpu_hit) + n * 4 * tbs + 2 * n;
  const int64_t stage = std::max(in_bytes, out_bytes) + 64;
  if (sl->staging_cap < stage) {
    if (sl->staging) cudaFreeHost(sl->staging);
    sl->staging = nullptr;
    sl->staging_cap = 0;
    if (cudaMallocHost(reinterpret_cast<void**>(&sl->staging), (size_t)stage) != cudaSuccess) {
      cudaGetLastError();
      err = "stormgpu_submit: pinned host staging of " + std::to_string(stage) + " bytes could not be allocated";
      return STORMGPU_ENOMEM;
    }
    sl->staging_cap = stage;
  }
  if (n > 0) {
    uint8_t* h = sl->staging;
    int64_t o = 0;
    memcpy(h + o, R.codes, (size_t)(n * cs));
    SGS(cudaMemcpyAsync(cv.codes[0], h + o, n * cs, cudaMemcpyHostToDevice, st));
    o += n * cs;
    memcpy(h + o, R.lengths, (size_t)n * sizeof(int16_t));
    SGS(cudaMemcpyAsync(cv.lengths[0], h + o, n * sizeof(int16_t), cudaMemcpyHostToDevice, st));
    o += n * (int64_t)sizeof(int16_t);
    if (lv) {
      memcpy(h + o, R.levels, (size_t)(n * ls));
      SGS(cudaMemcpyAsync(cv.levels[0], h + o, n * ls, cudaMemcpyHostToDevice, st));
      o += n * ls;
    }
    if (fl) {
      memcpy(h + o, R.first_levels, (size_t)n);
      SGS(cudaMemcpyAsync(cv.first_levels[0], h + o, n, cudaMemcpyHostToDevice, st));
    }
  }
  launch_init_results(n, cv.hits_all, cv.mapped_all, cv.tb_all, tbs, st);
  SGS(cudaMemsetAsync(cv.step_all, 0xff, std::max<int64_t>(n, 1), st));
  iota_kernel<<<grid_for(n), 256, 0, st>>>(cv.ids[0], n);
  int cur = 0;
  int64_t m = n;
  const int nsteps = (int)s->steps.size();
  for (int k = 0; k < nsteps && m > 0; ++k) {
    stormgpu_ctx* src = s->steps[k];
    ws->refs = src->refs;
    ws->seeds = src->seeds;
    ws->indexed = true;
    stormgpu_reads r{m, cv.codes[cur], cs, lv ? cv.levels[cur] : nullptr, ls, cv.lengths[cur],
                     fl ? cv.first_levels[cur] : nullptr};
    stormgpu_results o{cv.hits, cv.tb, tbs, cv.mapped};
    const int ks = std::min(k, 15);
    double* dk = sl->dens[ks];
    ws->dens_cand = dk[0]; ws->dens_pass = dk[1]; ws->gdens_cand = dk[2]; ws->gdens_pass = dk[3];
    if (const int rc = map_device_impl(ws, &r, &o)) return fail(rc);
    dk[0] = ws->dens_cand; dk[1] = ws->dens_pass; dk[2] = ws->gdens_cand; dk[3] = ws->gdens_pass;
    chain_scatter_kernel<<<grid_for(m), 256, 0, st>>>(m, cv.ids[cur], cv.hits, cv.tb, cv.mapped, tbs, k,
                                                      cv.hits_all, cv.tb_all, cv.mapped_all,
                                                      cv.step_all, cv.unmapped);
    if (k + 1 == nsteps) break;
    exclusive_scan<uint8_t, int64_t>(cv.unmapped, cv.off, m, cv.off + m, cv.scan_tmp, st);
    const int nx = 1 - cur;
    chain_compact_kernel<<<grid_for(m), 256, 0, st>>>(
        m, cv.unmapped, cv.off, cv.codes[cur], cs, lv ? cv.levels[cur] : nullptr, ls,
        cv.lengths[cur], fl ? cv.first_levels[cur] : nullptr, cv.ids[cur], cv.codes[nx],
        lv ? cv.levels[nx] : nullptr, cv.lengths[nx], fl ? cv.first_levels[nx] : nullptr, cv.ids[nx]);
    int64_t next = 0;
    SGS(cudaMemcpyAsync(&next, cv.off + m, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    SGS(cudaStreamSynchronize(st));
    m = next;
    cur = nx;
  }
  SGS(cudaGetLastError());
  if (n > 0) {
    uint8_t* h = sl->staging;
    const int64_t oh = 0, ot = oh + n * 4 * (int64_t)sizeof(stormgpu_hit), om = ot + n * 4 * tbs, os = om + n;
    SGS(cudaMemcpyAsync(h + oh, cv.hits_all, n * 4 * sizeof(stormgpu_hit), cudaMemcpyDeviceToHost, st));
    SGS(cudaMemcpyAsync(h + ot, cv.tb_all, n * 4 * tbs, cudaMemcpyDeviceToHost, st));
    SGS(cudaMemcpyAsync(h + om, cv.mapped_all, n, cudaMemcpyDeviceToHost, st));
    if (q->step) SGS(cudaMemcpyAsync(h + os, cv.step_all, n, cudaMemcpyDeviceToHost, st));
    SGS(cudaStreamSynchronize(st));
    memcpy(q->out.hits, h + oh, (size_t)n * 4 * sizeof(stormgpu_hit));
    memcpy(q->out.tb, h + ot, (size_t)(n * 4 * tbs));
    memcpy(q->out.mapped, h + om, (size_t)n);
    if (q->step) memcpy(q->step, h + os, (size_t)n);
  }
  SGS(cudaStreamSynchronize(st));
#undef SGS
  return 0;
}

void worker(stormgpu_server* s, Slot* sl) {
  cudaSetDevice(s->p.device);
  for (;;) {
    Request* q = nullptr;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      // arrival order; the first waiting batch goes as soon as its memory fits
      s->cv_work.wait(lk, [&] {
        return s->stop || (!s->queue.empty() && s->in_use + s->queue.front()->bytes <= s->chain_budget);
      });
      if (s->stop) return;
      q = s->queue.front();
      s->queue.pop_front();
      s->in_use += q->bytes;
    }
    std::string err;
    const int rc = run_chain(s, sl, q, err);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->in_use -= q->bytes;
      q->t_done = std::chrono::steady_clock::now();
      q->status = rc;
      q->err = err;
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

}  // namespace

extern "C" int stormgpu_server_open(const stormgpu_params* params, const char* const* chain, int nsteps, int slots,
                                    int64_t budget_bytes, stormgpu_server** out) {
  if (!params || !chain || !out || nsteps <= 0 || nsteps > 255 || slots <= 0 || slots > 64 || budget_bytes <= 0) {
    sg_set_error("stormgpu_server_open: bad arguments");
    return STORMGPU_EINVAL;
  }
  *out = nullptr;
  stormgpu_server* s = new stormgpu_server;
  s->p = *params;
  s->nslots = slots;
  s->budget = budget_bytes;
  s->work_cap = budget_bytes / (2 * slots);
  s->chain_budget = budget_bytes - s->work_cap * slots;
  for (int k = 0; k < nsteps; ++k) {
    stormgpu_ctx* c = nullptr;
    const int rc = stormgpu_open(params, chain[k], &c);
    if (rc) {
      for (auto* x : s->steps) stormgpu_close(x);
      delete s;
      return rc;
    }
    s->steps.push_back(c);
  }
  *out = s;
  return 0;
}

extern "C" int stormgpu_server_add_reference(stormgpu_server* s, const uint8_t* codes, const uint8_t* mask,
                                             int64_t n_codes, const int32_t* region_starts,
                                             const int32_t* region_ends, int32_t n_regions) {
  if (!s || s->built) { sg_set_error("stormgpu_server_add_reference: no server, or already built"); return STORMGPU_ESTATE; }
  return stormgpu_add_reference(s->steps[0], codes, mask, n_codes, region_starts, region_ends, n_regions);
}

extern "C" int stormgpu_server_build(stormgpu_server* s) {
  if (!s || s->built) { sg_set_error("stormgpu_server_build: no server, or already built"); return STORMGPU_ESTATE; }
  SG_CUDA(cudaSetDevice(s->p.device));
  // every step maps the sequences uploaded once (step 0 owns them) with an index of its own
  for (size_t k = 1; k < s->steps.size(); ++k) {
    s->steps[k]->refs.clear();
    for (const RefSeq& r0 : s->steps[0]->refs) {
      RefSeq r = r0;
      r.d_codes_alloc = r.d_mask_alloc = r.d_gexp_alloc = nullptr;
      r.idx.clear();
      s->steps[k]->refs.push_back(r);
    }
  }
  for (auto* c : s->steps)
    if (const int rc = stormgpu_build_index(c)) return rc;
  for (int i = 0; i < s->nslots; ++i) {
    Slot* sl = new Slot;
    stormgpu_ctx* v = new stormgpu_ctx;
    v->owns_refs = false;
    v->p = s->p;
    v->seeds = s->steps[0]->seeds;
    v->tune = s->tune;
    v->work.limit = s->work_cap;
    memset(&v->stats, 0, sizeof(v->stats));
    if (cudaStreamCreateWithFlags(&v->st, cudaStreamNonBlocking) != cudaSuccess) {
      cudaGetLastError();
      delete v;
      delete sl;
      sg_set_error("stormgpu_server_build: stream creation failed");
      return STORMGPU_ECUDA;
    }
    for (auto& e : v->ev) cudaEventCreate(&e);
    for (auto& e : v->rev) cudaEventCreate(&e);
    sl->ws = v;
    s->slots.push_back(sl);
  }
  s->built = true;
  for (auto* sl : s->slots) sl->th = std::thread(worker, s, sl);
  return 0;
}

extern "C" int stormgpu_server_set_tuning(stormgpu_server* s, const stormgpu_tuning* t) {
  if (!s || !t) { sg_set_error("stormgpu_server_set_tuning: null argument"); return STORMGPU_EINVAL; }
  if (s->built) { sg_set_error("stormgpu_server_set_tuning: call it before stormgpu_server_build"); return STORMGPU_ESTATE; }
  if (const int rc = stormgpu_set_tuning(s->steps[0], t)) return rc;  // range check
  s->tune = *t;
  return 0;
}

extern "C" int stormgpu_submit(stormgpu_server* s, const stormgpu_reads* reads, stormgpu_results* out, uint8_t* step,
                               int64_t* ticket) {
  if (!s || !s->built) { sg_set_error("stormgpu_submit: server not built"); return STORMGPU_ESTATE; }
  if (!reads || !out || !ticket || reads->n < 0 || (reads->n > 0 && (!reads->codes || !reads->lengths || !out->hits ||
                                                                     !out->tb || !out->mapped))) {
    sg_set_error("stormgpu_submit: bad arguments");
    return STORMGPU_EINVAL;
  }
  int maxL = 0;
  for (int64_t r = 0; r < reads->n; ++r) maxL = std::max<int>(maxL, reads->lengths[r]);
  if (maxL > STORMGPU_MAX_READ_LEN || out->tb_stride < (maxL + s->p.allowed_indels + 1) / 2) {
    sg_set_error("stormgpu_submit: read longer than %d or tb_stride too small", STORMGPU_MAX_READ_LEN);
    return STORMGPU_EINVAL;
  }
  Request* q = new Request;
  q->reads = *reads;
  q->out = *out;
  q->step = step;
  q->bytes = chain_layout(reads, out->tb_stride).bytes;
  if (q->bytes > s->chain_budget) {
    sg_set_error("stormgpu_submit: the chain buffers of a batch of %lld reads take %lld bytes of device memory, "
                 "more than the %lld the server's budget leaves for batches in flight; split it",
                 (long long)reads->n, (long long)q->bytes, (long long)s->chain_budget);
    delete q;
    return STORMGPU_EINVAL;
  }
  q->t_submit = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    q->ticket = s->next_ticket++;
    s->reqs[q->ticket] = q;
    s->queue.push_back(q);
    *ticket = q->ticket;
  }
  s->cv_work.notify_all();
  return 0;
}

extern "C" int stormgpu_poll(stormgpu_server* s, int64_t ticket, int timeout_ms, double* latency_ms) {
  if (!s) { sg_set_error("stormgpu_poll: no server"); return STORMGPU_EINVAL; }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) { sg_set_error("stormgpu_poll: unknown ticket %lld", (long long)ticket); return STORMGPU_EINVAL; }
  Request* q = it->second;
  if (q->status == 1) {
    if (timeout_ms < 0) s->cv_done.wait(lk, [&] { return q->status != 1; });
    else s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return q->status != 1; });
  }
  if (q->status == 1) return 1;
  const int rc = q->status;
  if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count();
  if (rc) sg_set_error("%s", q->err.c_str());
  s->reqs.erase(it);
  delete q;
  return rc;
}

extern "C" void stormgpu_server_close(stormgpu_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto* sl : s->slots)
    if (sl->th.joinable()) sl->th.join();
  cudaSetDevice(s->p.device);
  for (auto* sl : s->slots) {
    sl->release();
    stormgpu_close(sl->ws);
    delete sl;
  }
  for (size_t k = s->steps.size(); k-- > 0;) stormgpu_close(s->steps[k]);  // step 0 (owner of the sequences) last
  for (auto& kv : s->reqs) delete kv.second;
  delete s;
}
