// context.cuh -- the mapping context behind the C ABI (stormgpu.cu) and the server
// (server.cu): the device copies of the reference sequences and their indexes, and the
// per-batch working buffers.
#pragma once

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "index_build.cuh"

namespace sg {

struct RefSeq {
  int64_t n = 0;
  uint8_t* d_gexp_alloc = nullptr;
  uint8_t* d_gexp = nullptr;     // byte-expanded codes (filter streams)
  uint8_t* d_codes_alloc = nullptr;
  uint8_t* d_mask_alloc = nullptr;
  uint8_t* d_codes = nullptr;
  uint8_t* d_mask = nullptr;
  std::vector<int32_t> rs, re;
  std::vector<DevIndex> idx;
};

// Working memory of one mapping context (its DevBufs grown while it maps), with an optional
// limit: a growth past it fails with STORMGPU_ENOMEM and sets `over`, and the mapping call then
// maps the batch in halves instead (the reads are independent).  Set for the thread that maps
// (g_work_budget) around the context's mapping.
struct WorkBudget {
  int64_t used = 0;   // bytes of the DevBufs grown while it was set
  int64_t limit = 0;  // 0: none
  bool over = false;
};
extern thread_local WorkBudget* g_work_budget;

template <typename T>
struct DevBuf {
  T* p = nullptr;
  int64_t cap = 0;
  int grow(int64_t n) {
    if (n <= cap) return 0;
    WorkBudget* b = g_work_budget;
    int64_t c = std::max<int64_t>(n, cap + cap / 2);
    if (b && b->limit > 0 && b->used + (c - cap) * (int64_t)sizeof(T) > b->limit) {
      c = n;  // the exact size, when the usual headroom does not fit
      if (b->used + (c - cap) * (int64_t)sizeof(T) > b->limit) {
        b->over = true;
        sg_set_error("working memory limit of %lld bytes reached", (long long)b->limit);
        return STORMGPU_ENOMEM;
      }
    }
    if (p) cudaFree(p);
    p = nullptr;
    if (b) b->used -= cap * (int64_t)sizeof(T);
    cap = 0;
    if (cudaMalloc(&p, sizeof(T) * (size_t)std::max<int64_t>(c, 1)) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      sg_set_error("device allocation of %lld bytes failed", (long long)(sizeof(T) * c));
      return STORMGPU_ENOMEM;
    }
    cap = c;
    if (b) b->used += cap * (int64_t)sizeof(T);
    return 0;
  }
  void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};


}  // namespace sg

struct stormgpu_ctx {
  bool owns_refs = true;  // false: a view of another context's sequences and indexes
  stormgpu_params p;
  sg::SeedSet seeds;
  cudaStream_t st = nullptr;
  std::vector<sg::RefSeq> refs;
  bool indexed = false;
  stormgpu_stats stats;
  stormgpu_tuning tune = {768, 4, 8, 32, 0, 4};  // launch parameters of the stages (no effect on results)
  // per-batch read buffers
  sg::DevBuf<uint8_t> rcodes, rlevels, fcodes, flevels, first_levels;
  sg::DevBuf<int16_t> lengths;
  sg::DevBuf<stormgpu_hit> hits;
  sg::DevBuf<uint8_t> tb, mapped;
  // pass buffers
  sg::DevBuf<int32_t> pstart, pcount, p_read, p_diag, big_list, big_h, small_list, small_h, big_count, huge_list,
      huge_h;
  sg::DevBuf<int64_t> scan_tmp64, foff;
  sg::DevBuf<int32_t> fr, fd;
  sg::DevBuf<uint8_t> flag;       // pass byte per candidate
  sg::DevBuf<uint32_t> flagw;     // pass bits, one word per 32 candidates
  sg::DevBuf<uint8_t> rexp;
  sg::DevBuf<int32_t> a_score, a_bound, a_tblen, big_tmp;
  sg::DevBuf<int16_t> a_pos;
  sg::DevBuf<uint8_t> a_tb;
  sg::DevBuf<uint32_t> scratch;
  sg::DevBuf<int32_t> thr, round_slots;  // alignment rounds: per-read threshold, per-round slot lists
  sg::DevBuf<int64_t> rounds;           // [0, 8): slots per round, [8, 16): the lists' fill cursors
  sg::DevBuf<unsigned long long> counters;
  sg::DevBuf<uint32_t> ord, ord_tmp;  // length order of a mixed-length batch: sort keys and values, sort scratch
  cudaEvent_t ev[8];
  cudaEvent_t rev[2 * 6 + 1];  // alignment rounds: before the first, after each round's alignment and replay
  int64_t last_n = -1;  // reads of the last stormgpu_map call (its results stay in hits / mapped)
  int64_t last_tbs = 0;  // its traceback stride
  sg::WorkBudget work;  // working memory of the mapping buffers; work.limit 0 = no limit
  // candidates and passing candidates per read of the densest strand pass of the last mapping
  // call: a batch that would exceed a pass's bounds at that density is cut up front instead of
  // after its gather
  double dens_cand = 0, dens_pass = 0;
  // the same densities for the list sizes of a graph call: the larger of the last call's and
  // 0.9 x the value before it, so that calls of different densities in turn (one read length
  // after another) do not outgrow their lists each time
  double gdens_cand = 0, gdens_pass = 0;
  // CUDA graph of the strand passes: on unless turned off (stormgpu_set_graphs, STORMGPU_GRAPHS=0)
  // or broken (a capture or instantiation that failed turns it off for the context); the
  // executable graph of the last call, updated in place by the next call of the same shape; its
  // stage events; its device state (list sizes, status, sums of the counters)
  bool graphs = true;
  bool graph_broken = false;
  cudaGraphExec_t gexec = nullptr;
  std::vector<cudaEvent_t> gev;
  sg::DevBuf<unsigned long long> gstate;
  // slice size (index positions) of the graph's launch for reads with the most positions: the
  // largest the host-synced passes needed so far
  int64_t huge_cap = 1 << 17;
  // genome_map placement
  sg::DevBuf<uint32_t> gm_k0, gm_v0, gm_k1, gm_v1, gm_tmp, gm_base;
};

namespace sg {

// One batch on c's stream (every pointer in reads / out on the device); synchronous.
int map_device_impl(stormgpu_ctx* c, const stormgpu_reads* reads, stormgpu_results* out);

}  // namespace sg
