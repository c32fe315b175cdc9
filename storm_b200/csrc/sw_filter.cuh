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
  unsigned long long* counters;  // [2] += cell updates W*2*(L+W-1), [5] += candidates, [6] += L*(2*Is+1)
  const uint8_t* gexp;          // byte-expanded genome (code c -> c * 0x11), code 0
  const uint8_t* rexp;          // read streams (bytes 0xC4 + c * 0x11), rstride bytes per read
  int64_t rstride;
  int min_len;                  // shortest read of the batch (reads shorter than W take another path)
  // may be null; else the candidate count is read from here when the kernel starts (the hit
  // gather's cursor), and n is only an upper bound for the grid
  const unsigned long long* n_dev;
  // may be null; else a zeroed work cursor: the grid is the resident set, and every block takes
  // the next tile of 256 * kFilterTile candidates from it, in list order, until none is left
  unsigned long long* cursor;
  int rows;  // with a cursor: rows of 256 candidates in a block's tile (0 = 8); without: 8
};

constexpr int64_t kGexpPad = 4096;   // bytes of padding around a byte-expanded sequence
inline int64_t rexp_stride(int max_len) { return ((int64_t)max_len + 16 + 8 + 15) & ~15LL; }
void launch_expand_genome(const uint8_t* codes, int64_t n_codes, uint8_t* gexp, cudaStream_t st);
void launch_expand_reads(const ReadsDev& rd, uint8_t* rexp, int64_t rstride, cudaStream_t st);

bool filter_dpx_ok(const ScoreParams& sp, int max_len);
void launch_filter_flat_job(const FilterJob& job, const ScoreParams& sp, bool dpx, cudaStream_t st);
// pass bytes of the ncap candidates -> words of 32 pass bits (bit t & 31 of word t >> 5); with
// n_dev (may be null) only the first *n_dev candidates count, the words after them are zero
void launch_pack_flags(int64_t ncap, const unsigned long long* n_dev, const uint8_t* flag, uint32_t* words,
                       cudaStream_t st);
// A word of pass bits, counted as its number of passing candidates when scanned.
struct PassWord {
  uint32_t bits;
  __host__ __device__ explicit operator int64_t() const {
#if defined(__CUDA_ARCH__)
    return __popc(bits);
#else
    return __builtin_popcount(bits);
#endif
  }
};
// passing candidates, in order: word w's set bits go to woff[w], woff[w] + 1, ... (those below
// pcap: the capacity of p_read / p_diag)
void launch_compact(int64_t nwords, const uint32_t* flag, const int64_t* woff, const int32_t* fr, const int32_t* fd,
                    int32_t* p_read, int32_t* p_diag, int64_t pcap, cudaStream_t st);
// pstart / pcount of every read with passing candidates; npass is the slot count, or with
// npass_dev (may be null) an upper bound for the grid and the count is read from there
void launch_slot_bounds(int64_t npass, const int64_t* npass_dev, const int32_t* p_read, int32_t* pstart,
                        int32_t* pcount, cudaStream_t st);

}  // namespace sg
