// autotune.cu -- the launch parameters of the mapping stages (stormgpu_tuning) and the
// autotuner that picks them by timing.
//
// None of the parameters changes a result: the gather's hit bucket (positions a warp holds in
// shared memory) trades occupancy against reads sent to the block-per-read kernel, its reads
// per steal trade work-cursor atomics against load balance, the filter's tile rows trade
// block barriers against the tail, its persistent grid (tiles from a work cursor) trades
// the cursor's atomics and barriers against the block scheduler's tail, and the alignment's
// run per steal trades atomics against
// balance across candidates that stop early.  The best values depend on the read lengths, the
// band and how repetitive the index is, so they are measured on the caller's own reads: every
// candidate value of one parameter is run on a sample (the others at their best so far), the
// stage it affects is timed with the CUDA events of stormgpu_map, and the fastest stays.
// The reference has no counterpart (it has no GPU).
#include <cstring>
#include <vector>

#include "common.cuh"
#include "context.cuh"
#include "map_kernels.cuh"
#include "gather.cuh"

namespace {

bool tuning_ok(const stormgpu_tuning& t) {
  return t.gather_warp_cap >= 256 && t.gather_warp_cap <= sg::kMaxWarpCap &&
         t.gather_reads_per_steal >= 1 && t.gather_reads_per_steal <= 64 && t.filter_rows >= 1 &&
         t.filter_rows <= 64 && t.align_steal >= 32 && t.align_steal <= 1024 && t.align_steal % 32 == 0 &&
         (t.filter_cursor == 0 || t.filter_cursor == 1) && t.align_rounds >= 1 &&
         t.align_rounds <= sg::kMaxAlignRounds;
}

}  // namespace

extern "C" int stormgpu_get_tuning(stormgpu_ctx* c, stormgpu_tuning* out) {
  if (!c || !out) { sg_set_error("null argument"); return STORMGPU_EINVAL; }
  *out = c->tune;
  return 0;
}

extern "C" int stormgpu_set_tuning(stormgpu_ctx* c, const stormgpu_tuning* t) {
  if (!c || !t) { sg_set_error("null argument"); return STORMGPU_EINVAL; }
  if (!tuning_ok(*t)) {
    sg_set_error("tuning out of range (warp cap %d, reads per steal %d, filter rows %d, align steal %d, "
                 "filter cursor %d)", t->gather_warp_cap, t->gather_reads_per_steal, t->filter_rows, t->align_steal,
                 t->filter_cursor);
    return STORMGPU_EINVAL;
  }
  c->tune = *t;
  return 0;
}

extern "C" int stormgpu_autotune(stormgpu_ctx* c, const stormgpu_reads* reads, int64_t sample,
                                 stormgpu_tuning* out) {
  if (!c || !reads || reads->n < 0) { sg_set_error("null argument"); return STORMGPU_EINVAL; }
  if (!c->indexed) { sg_set_error("stormgpu_build_index must be called before stormgpu_autotune"); return STORMGPU_ESTATE; }
  // the sample: reads spread evenly over the batch (a batch sorted by length keeps its mix),
  // grown until one mapping of it takes kMinSampleMs: on a sample whose stages take a fraction of
  // a millisecond the fixed costs of the launches decide, and the pick can be the worst setting
  // for the batch (the colour workload's 2M reads, on an 8000-read sample: the largest hit bucket,
  // gather 40 ms, where the smallest gives 26 ms)
  constexpr double kMinSampleMs = 50.0;
  stormgpu_reads r;
  std::vector<uint8_t> sc, sl, sf;
  std::vector<int16_t> slen;
  std::vector<stormgpu_hit> hits;
  std::vector<uint8_t> tb, mapped;
  stormgpu_results res;
  auto make_sample = [&](int64_t m) {
    r = *reads;
    if (m > 0 && r.n > m) {
      sc.assign((size_t)(m * r.code_stride), 0);
      sl.assign(r.levels ? (size_t)(m * r.level_stride) : 0, 0);
      sf.assign(r.first_levels ? (size_t)m : 0, 0);
      slen.assign((size_t)m, 0);
      for (int64_t k = 0; k < m; ++k) {
        const int64_t j = k * reads->n / m;
        memcpy(sc.data() + k * r.code_stride, reads->codes + j * r.code_stride, (size_t)r.code_stride);
        if (r.levels) memcpy(sl.data() + k * r.level_stride, reads->levels + j * r.level_stride, (size_t)r.level_stride);
        if (r.first_levels) sf[(size_t)k] = reads->first_levels[j];
        slen[(size_t)k] = reads->lengths[j];
      }
      r.n = m;
      r.codes = sc.data();
      r.levels = r.levels ? sl.data() : nullptr;
      r.first_levels = r.first_levels ? sf.data() : nullptr;
      r.lengths = slen.data();
    }
    int maxL = 0;
    for (int64_t k = 0; k < r.n; ++k) maxL = std::max<int>(maxL, r.lengths[k]);
    const int64_t tbs = ((maxL + c->p.allowed_indels + 1) / 2 + 7) & ~7LL;
    hits.assign((size_t)std::max<int64_t>(r.n * 4, 1), stormgpu_hit{});
    tb.assign((size_t)std::max<int64_t>(r.n * 4 * tbs, 1), 0);
    mapped.assign((size_t)std::max<int64_t>(r.n, 1), 0);
    res = stormgpu_results{hits.data(), tb.data(), tbs, mapped.data()};
  };
  int64_t m = sample > 0 ? sample : reads->n;
  make_sample(m);
  if (r.n == 0) {  // nothing to time: the parameters stay as they are
    if (out) *out = c->tune;
    return 0;
  }
  const stormgpu_stats saved = c->stats;
  for (int grow = 0; grow < 8 && r.n < reads->n; ++grow) {
    for (int k = 0; k < 2; ++k)  // the first run of a larger sample may grow the buffers
      if (const int rc = stormgpu_map(c, &r, &res)) { c->stats = saved; return rc; }
    const double ms = c->stats.ms_total;
    if (ms >= kMinSampleMs) break;
    const double f = ms > 0 ? std::min(16.0, 1.2 * kMinSampleMs / ms) : 16.0;
    m = std::min<int64_t>(reads->n, std::max<int64_t>(m + 1, (int64_t)((double)m * f)));
    make_sample(m);
  }

  // stage time of one setting: best of two runs after a warm-up (which also sizes the buffers)
  auto time_of = [&](const stormgpu_tuning& t, double stormgpu_stats::*stage, double* ms) -> int {
    c->tune = t;
    double best = 1e300;
    for (int k = 0; k < 3; ++k) {
      if (const int rc = stormgpu_map(c, &r, &res)) return rc;
      if (k > 0) best = std::min(best, c->stats.*stage);
    }
    *ms = best;
    return 0;
  };
  // one knob = the candidate settings of one or two fields (the filter's grid form and its tile
  // rows go together: the rows only apply with a cursor)
  struct Knob {
    int32_t stormgpu_tuning::*f1;
    int32_t stormgpu_tuning::*f2;  // may be null
    double stormgpu_stats::*stage;
    std::vector<std::pair<int32_t, int32_t>> values;
  };
  const Knob knobs[] = {
      {&stormgpu_tuning::gather_warp_cap, nullptr, &stormgpu_stats::ms_gather, {{512, 0}, {768, 0}, {1024, 0}, {1536, 0}}},
      {&stormgpu_tuning::gather_reads_per_steal, nullptr, &stormgpu_stats::ms_gather,
       {{1, 0}, {2, 0}, {4, 0}, {8, 0}, {16, 0}}},
      {&stormgpu_tuning::filter_cursor, &stormgpu_tuning::filter_rows, &stormgpu_stats::ms_filter,
       {{0, 8}, {1, 2}, {1, 4}, {1, 8}, {1, 16}}},
      {&stormgpu_tuning::align_steal, nullptr, &stormgpu_stats::ms_align, {{32, 0}, {64, 0}, {128, 0}}},
      // with rounds the replays run between the alignment launches: compare whole passes
      {&stormgpu_tuning::align_rounds, nullptr, &stormgpu_stats::ms_total, {{1, 0}, {3, 0}, {4, 0}, {6, 0}}},
  };
  stormgpu_tuning best = c->tune;
  int rc = 0;
  for (const Knob& kn : knobs) {
    double best_ms = 1e300;
    stormgpu_tuning pick = best;
    for (const auto& v : kn.values) {
      stormgpu_tuning t = best;
      t.*kn.f1 = v.first;
      if (kn.f2) t.*kn.f2 = v.second;
      double ms = 0;
      if ((rc = time_of(t, kn.stage, &ms))) break;
      if (ms < best_ms) { best_ms = ms; pick = t; }
    }
    if (rc) break;
    best = pick;
  }
  c->tune = best;
  c->stats = saved;
  if (rc) return rc;
  if (out) *out = best;
  return 0;
}
