// sw_filter.cuh -- packed 16-bit banded filter over a flat candidate list (sw_filter.cu).
#pragma once

#include "map_kernels.cuh"

namespace sg {

struct FilterJob {
  int64_t n;                    // candidates
  const int32_t* fr;            // read of each candidate
  const int32_t* fd;            // diagonal of each candidate (window start = diag - Is)
  uint8_t* flag;                // out: 1 = passes
  const uint8_t* codes;         // packed reads
  int64_t cstride;
  const int16_t* lengths;
  const uint8_t* genome;
  int W, Is;
  int fm, fx, fo, fe, fthr;
  unsigned long long* counters;  // [2] += filter cells L*(2*Is+1), [5] += candidates
};

bool filter_dpx_ok(const ScoreParams& sp, int max_len);
void launch_filter_flat_job(const FilterJob& job, const ScoreParams& sp, bool dpx, cudaStream_t st);
void launch_flatten(int64_t n, const int64_t* hoff, const int32_t* cand, const int32_t* ucount,
                    const int64_t* uoff, int32_t* fr, int32_t* fd, cudaStream_t st);
void launch_compact(int64_t n, const uint8_t* flag, const int64_t* off, const int32_t* fr, const int32_t* fd,
                    int32_t* p_read, int32_t* p_diag, cudaStream_t st);
void launch_slot_bounds(int64_t npass, const int32_t* p_read, int32_t* pstart, int32_t* pcount, cudaStream_t st);

}  // namespace sg
