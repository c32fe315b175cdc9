// filter_ref.cuh -- the banded u8 SW filter on plain 32-bit integers (one cell per
// register), a direct restatement of the reference semantics; used for scoring values that
// do not fit the packed 16-bit kernel, and by the unit-level checks.
#pragma once

#include "map_kernels.cuh"

namespace sg {

// The banded saturating-u8 SW of alignment_avx2__align_* (alignment_simd.c:2613-3404) for one
// hit: W cells; before the loop the genome register holds window codes 0..W-1 (cell k = code
// W-1-k); odd steps shift one more genome code in at cell 0, even steps one more read code in
// at cell W-1; per cell M = subs(adds(M[l-2], match if equal), mismatch if different),
// I = max(subs(max(I[l-1], I[l-1] of the neighbour), ext), subs(max(M[l-1], M[l-1] of the
// neighbour), open)) (neighbour below at odd steps, above at even steps, 0 at the edge),
// M = max(M, I) & mask[l], Max = max(Max, M); pass iff Max > thr.  The mask table of
// alignment_avx2__setlength_* (:2282-2507) is rebuilt incrementally per step.
template <int W>
__device__ __forceinline__ bool sw_filter_one(const uint8_t* __restrict__ genome, int64_t pos,
                                              const uint8_t* read, int L, int fm, int fx, int fo,
                                              int fe, int fthr) {
  constexpr uint32_t FULLC = (W == 16) ? 0xffffffffu : ((1u << (2 * W)) - 1u);
  constexpr uint32_t FULLM = (1u << W) - 1u;
  int M1[W], M2[W], I1[W];
#pragma unroll
  for (int k = 0; k < W; ++k) { M1[k] = 0; M2[k] = 0; I1[k] = 0; }
  uint32_t A = 0, B = 0;
  int64_t g = pos;
#pragma unroll
  for (int d = 0; d < W; ++d) B = ((B << 2) | (uint32_t)code_at(genome, g++)) & FULLC;
  const int prlength = 2 * (L + W - 1);
  uint32_t msk = 1u << (W - 1);
  int Max = 0, r = 0;
  for (int l = 0; l < prlength; ++l) {
    if (l > 0 && !(l & 1)) {
      if (l >= prlength - 2 * (W - 1)) msk = (msk >> 1) & FULLM;
      else if (l <= 2 * (W - 1)) msk = msk | ((msk >> 1) & FULLM);
    }
    const bool odd = l & 1;
    if (odd) B = ((B << 2) | (uint32_t)code_at(genome, g++)) & FULLC;
    else A = (A >> 2) | ((uint32_t)code_at(read, r++) << (2 * (W - 1)));
    const uint32_t x = A ^ B;
    int Mn[W], In[W];
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const bool eq = ((x >> (2 * k)) & 3u) == 0u;
      int m = eq ? min(M2[k] + fm, 255) : max(M2[k] - fx, 0);
      int Is_, Ms_;
      if (odd) { Is_ = k > 0 ? I1[k - 1] : 0; Ms_ = k > 0 ? M1[k - 1] : 0; }
      else { Is_ = k < W - 1 ? I1[k + 1] : 0; Ms_ = k < W - 1 ? M1[k + 1] : 0; }
      const int Im = max(I1[k], Is_), Mm = max(M1[k], Ms_);
      const int iv = max(max(Im - fe, 0), max(Mm - fo, 0));
      m = max(m, iv);
      if (!((msk >> k) & 1u)) m = 0;
      Max = max(Max, m);
      Mn[k] = m;
      In[k] = iv;
    }
#pragma unroll
    for (int k = 0; k < W; ++k) { M2[k] = M1[k]; M1[k] = Mn[k]; I1[k] = In[k]; }
  }
  return Max > fthr;
}

__device__ __forceinline__ bool sw_filter_dispatch(int W, const uint8_t* genome, int64_t pos,
                                                   const uint8_t* read, int L, const ScoreParams& sp) {
  switch (W) {
  case 2: return sw_filter_one<2>(genome, pos, read, L, sp.fm, sp.fx, sp.fo, sp.fe, sp.fthr);
  case 4: return sw_filter_one<4>(genome, pos, read, L, sp.fm, sp.fx, sp.fo, sp.fe, sp.fthr);
  case 8: return sw_filter_one<8>(genome, pos, read, L, sp.fm, sp.fx, sp.fo, sp.fe, sp.fthr);
  default: return sw_filter_one<16>(genome, pos, read, L, sp.fm, sp.fx, sp.fo, sp.fe, sp.fthr);
  }
}


__device__ __forceinline__ bool sw_filter_dispatch_ext(int W, const uint8_t* genome, int64_t pos,
                                                       const uint8_t* read, int L, const ScoreParams& sp) {
  return sw_filter_dispatch(W, genome, pos, read, L, sp);
}

}  // namespace sg
