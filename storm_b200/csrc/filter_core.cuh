// filter_core.cuh -- the per-hit arithmetic of the packed 16-bit banded filter (see
// sw_filter.cu for the layout and the argument that it reproduces the reference's pass/fail).
// Host-and-device so that the exact kernel code can be checked against the oracle on a CPU.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sg {

#define SG_HD __host__ __device__ __forceinline__

SG_HD uint32_t ldg32(const uint32_t* p) {
#if defined(__CUDA_ARCH__)
  return __ldg(p);
#else
  return *p;
#endif
}

// prmt.b32, generic mode: nibble n of s picks byte (s_n & 7) of {b, a}; if (s_n & 8) the
// sign bit of that byte is replicated over the output byte (PTX ISA, prmt).  __byte_perm is
// not used: it documents only the 3 low bits of each nibble.
SG_HD uint32_t prmt(uint32_t a, uint32_t b, uint32_t s) {
#if defined(__CUDA_ARCH__)
  uint32_t d;
  asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(s));
  return d;
#else
  const uint64_t src = ((uint64_t)b << 32) | a;
  uint32_t d = 0;
  for (int n = 0; n < 4; ++n) {
    const uint32_t sel = (s >> (4 * n)) & 0xF;
    uint32_t byte = (uint32_t)(src >> (8 * (sel & 7))) & 0xFF;
    if (sel & 8) byte = (byte & 0x80) ? 0xFF : 0x00;
    d |= byte << (8 * n);
  }
  return d;
#endif
}

// per-register 0xFFFF/0 masks of cells (2j, 2j+1) from the W-bit cell mask
SG_HD uint32_t mask_word(uint32_t m, int j) {
  return (((m >> (2 * j)) & 1u) ? 0x0000FFFFu : 0u) | (((m >> (2 * j + 1)) & 1u) ? 0xFFFF0000u : 0u);
}

template <int W, bool ODD, bool MASKED>
SG_HD void fstep(uint32_t (&A)[W / 2], uint32_t (&B)[W / 2], uint32_t (&M1)[W / 2],
                                      uint32_t (&M2)[W / 2], uint32_t (&I1)[W / 2], uint32_t& Max,
                                      uint32_t nb, uint32_t T, uint32_t NFE, uint32_t NFO, uint32_t m) {
  constexpr int NR = W / 2;
  if (ODD) {  // genome register: every cell takes the code of the cell below, cell 0 the new one
#pragma unroll
    for (int j = NR - 1; j > 0; --j) B[j] = prmt(B[j - 1], B[j], 0x0041);
    B[0] = prmt(nb, B[0], 0x0040);
  } else {    // read register: every cell takes the code of the cell above, cell W-1 the new one
#pragma unroll
    for (int j = 0; j < NR - 1; ++j) A[j] = prmt(A[j], A[j + 1], 0x0041);
    A[NR - 1] = prmt(A[NR - 1], nb, 0x0041);
  }
  uint32_t P[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) P[j] = __viaddmax_s16x2(I1[j], NFE, __viaddmax_s16x2(M1[j], NFO, 0x80008000u));
  uint32_t Mn[NR], In[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    const uint32_t nbr = ODD ? prmt(j > 0 ? P[j - 1] : 0u, P[j], 0x5432)
                             : prmt(P[j], j < NR - 1 ? P[j + 1] : 0u, 0x5432);
    In[j] = __vimax_s16x2_relu(P[j], nbr);
    const uint32_t sc = prmt(T, 0u, (A[j] ^ B[j]) | 0x8080u);
    uint32_t mv = __viaddmax_s16x2_relu(M2[j], sc, In[j]);
    if (MASKED) mv &= mask_word(m, j);
    Mn[j] = mv;
  }
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    Max = __vimax_s16x2_relu(Max, Mn[j]);
    M2[j] = M1[j];
    M1[j] = Mn[j];
    I1[j] = In[j];
  }
}

// genome code stream starting at code `pos` (may be negative inside the padding): 64-bit
// window refilled with one aligned 32-bit word every 16 codes, uniformly across lanes.
struct GStream {
  const uint32_t* w;
  uint64_t win;
  int sh;       // 32 - 2*sub: bit where the next word goes
  int used;     // codes consumed since the last refill
  SG_HD void init(const uint8_t* genome, int64_t pos) {
    const int64_t wi = pos >> 4;
    const int sub = (int)(pos & 15);
    w = reinterpret_cast<const uint32_t*>(genome) + wi;
    const uint64_t lo = ldg32(w), hi = ldg32(w + 1);
    win = ((hi << 32) | lo) >> (2 * sub);
    sh = 32 - 2 * sub;
    used = 0;
    w += 2;
  }
  SG_HD uint32_t next_byte() {
    const uint32_t c = (uint32_t)win & 3u;
    win >>= 2;
    if (++used == 16) {
      win |= (uint64_t)ldg32(w) << sh;
      ++w;
      used = 0;
    }
    return c * 0x11u;
  }
};

struct RStream {
  const uint32_t* w;
  const uint32_t* end;
  uint32_t cur;
  int used;
  SG_HD void init(const uint8_t* read, int64_t stride_bytes) {
    w = reinterpret_cast<const uint32_t*>(read);
    end = w + (stride_bytes >> 2);
    cur = w < end ? ldg32(w) : 0u;
    ++w;
    used = 0;
  }
  SG_HD uint32_t next_byte() {
    const uint32_t c = cur & 3u;
    cur >>= 2;
    if (++used == 16) {
      cur = w < end ? ldg32(w) : 0u;
      ++w;
      used = 0;
    }
    return c * 0x11u;
  }
};

template <int W>
SG_HD uint32_t mask_update(uint32_t m, int l, int prlength) {
  constexpr uint32_t FULL = (1u << W) - 1u;
  if (!(l & 1)) {
    if (l >= prlength - 2 * (W - 1)) m = (m >> 1) & FULL;
    else if (l <= 2 * (W - 1)) m = m | ((m >> 1) & FULL);
  }
  return m;
}

// One hit.  Returns max over all cells of M (before comparing with the threshold).
template <int W>
SG_HD int filter_dpx(const uint8_t* __restrict__ genome, int64_t pos, const uint8_t* read,
                                          int64_t rstride, int L, uint32_t T, uint32_t NFE, uint32_t NFO) {
  constexpr int NR = W / 2;
  uint32_t A[NR], B[NR], M1[NR], M2[NR], I1[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) { A[j] = 0; B[j] = 0; M1[j] = 0; M2[j] = 0; I1[j] = 0; }
  uint32_t Max = 0;
  GStream gs;
  gs.init(genome, pos);
  RStream rs;
  rs.init(read, rstride);
#pragma unroll
  for (int d = 0; d < W; ++d) {  // B = window codes 0..W-1, cell k = code W-1-k
    const uint32_t nb = gs.next_byte();
#pragma unroll
    for (int j = NR - 1; j > 0; --j) B[j] = prmt(B[j - 1], B[j], 0x0041);
    B[0] = prmt(nb, B[0], 0x0040);
  }
  const int prlength = 2 * (L + W - 1);
  uint32_t m = 1u << (W - 1);
  if (L >= W) {
    int l = 0;
    for (; l < 2 * (W - 1); l += 2) {  // prologue: cells above the read are masked
      if (l > 0) m = mask_update<W>(m, l, prlength);
      fstep<W, false, true>(A, B, M1, M2, I1, Max, rs.next_byte(), T, NFE, NFO, m);
      fstep<W, true, true>(A, B, M1, M2, I1, Max, gs.next_byte(), T, NFE, NFO, m);
    }
    for (; l < 2 * L; l += 2) {        // body: full band
      fstep<W, false, false>(A, B, M1, M2, I1, Max, rs.next_byte(), T, NFE, NFO, 0u);
      fstep<W, true, false>(A, B, M1, M2, I1, Max, gs.next_byte(), T, NFE, NFO, 0u);
    }
    m = (1u << W) - 1u;
    for (; l < prlength; l += 2) {     // epilogue: cells below the read are masked
      m = mask_update<W>(m, l, prlength);
      fstep<W, false, true>(A, B, M1, M2, I1, Max, rs.next_byte(), T, NFE, NFO, m);
      fstep<W, true, true>(A, B, M1, M2, I1, Max, gs.next_byte(), T, NFE, NFO, m);
    }
  } else {
    for (int l = 0; l < prlength; l += 2) {
      if (l > 0) m = mask_update<W>(m, l, prlength);
      fstep<W, false, true>(A, B, M1, M2, I1, Max, rs.next_byte(), T, NFE, NFO, m);
      fstep<W, true, true>(A, B, M1, M2, I1, Max, gs.next_byte(), T, NFE, NFO, m);
    }
  }
  const int lo = (int)(int16_t)(Max & 0xffffu), hi = (int)(int16_t)(Max >> 16);
  return lo > hi ? lo : hi;
}

// ------------------------------------------------------------------------------------------
// Version with biased cells and byte-expanded streams (used when L >= W).
//
// Every M and I value is stored with a bias of FB (256) in each 16-bit half, so that the gap
// penalties are subtracted with a plain 32-bit add (no borrow between halves: every half is
// >= FB >= open, extend) on the FMA pipe, and "max(., 0)" becomes "max(., FB)".  The genome is
// read from a byte-expanded copy (code c -> c * 0x11) and the read from a per-read stream of
// bytes 0xC4 + c * 0x11, so that for a cell the byte difference (read byte - genome byte) is
// (4 + c - g) | (12 + c - g) << 4: a prmt selector (no borrow between bytes) that picks the
// match score when c == g (byte 4 of {lo, hi}) and the mismatch score otherwise, with the
// sign replicated into the high byte.  Codes enter the band registers with constant-selector
// prmts from 4-byte stream words: four read codes and four genome codes per block of 4 step
// pairs.  Pair p of the band covers read positions i = p - W + 1 + k (cell k); blocks whose
// pairs all have 0 <= i < L for every cell run without the mask.
constexpr uint32_t kFB = 256u;
constexpr uint32_t kFBB = kFB * 0x10001u;

template <int W, bool ODD, bool MASKED, int T>
SG_HD void fstep3(uint32_t (&A)[W / 2], uint32_t (&B)[W / 2], uint32_t (&M1)[W / 2], uint32_t (&M2)[W / 2],
                  uint32_t (&I1)[W / 2], uint32_t& Max, uint32_t rcur, uint32_t gcur, uint32_t TLO,
                  uint32_t THI, uint32_t CFE, uint32_t CFO, const uint32_t (&mw)[W / 2]) {
  constexpr int NR = W / 2;
  if (ODD) {
#pragma unroll
    for (int j = NR - 1; j > 0; --j) B[j] = prmt(B[j - 1], B[j], 0x0041);
    B[0] = prmt(gcur, B[0], 0x0040u | (uint32_t)T);
  } else {
#pragma unroll
    for (int j = 0; j < NR - 1; ++j) A[j] = prmt(A[j], A[j + 1], 0x0041);
    A[NR - 1] = prmt(A[NR - 1], rcur, 0x0001u | ((uint32_t)(4 + T) << 4));
  }
  uint32_t P[NR], Mn[NR], In[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) P[j] = __vimax_s16x2_relu(I1[j] - CFE, M1[j] - CFO);  // halves are positive: relu is a no-op
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    const uint32_t nbr = ODD ? prmt(j > 0 ? P[j - 1] : kFBB, P[j], 0x5432)
                             : prmt(P[j], j < NR - 1 ? P[j + 1] : kFBB, 0x5432);
    In[j] = __vimax3_s16x2(P[j], nbr, kFBB);
    const uint32_t sc = prmt(TLO, THI, A[j] - B[j]);
    uint32_t mv = __viaddmax_s16x2(M2[j], sc, In[j]);
    if (MASKED) mv = (mv & mw[j]) | (kFBB & ~mw[j]);
    Mn[j] = mv;
  }
  if (NR == 1) {
    Max = __vimax_s16x2_relu(Max, Mn[0]);
  } else {
#pragma unroll
    for (int j = 0; j + 1 < NR; j += 2) Max = __vimax3_s16x2(Max, Mn[j], Mn[j + 1]);
  }
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    M2[j] = M1[j];
    M1[j] = Mn[j];
    I1[j] = In[j];
  }
}

// mask words of pair p: cell k enabled iff 0 <= p - W + 1 + k <= L - 1
template <int W>
SG_HD void pair_mask(int p, int L, uint32_t (&mw)[W / 2]) {
  const int kmin = (W - 1 - p) > 0 ? (W - 1 - p) : 0;
  const int kmax = (L + W - 2 - p) < (W - 1) ? (L + W - 2 - p) : (W - 1);
  uint32_t m = 0;
  if (kmax >= kmin) m = ((kmax >= 31) ? 0xffffffffu : ((2u << kmax) - 1u)) & ~((1u << kmin) - 1u);
#pragma unroll
  for (int j = 0; j < W / 2; ++j) mw[j] = mask_word(m, j);
}

template <int W, bool MASKED>
SG_HD void fblock3(int p0, int L, uint32_t (&A)[W / 2], uint32_t (&B)[W / 2], uint32_t (&M1)[W / 2],
                   uint32_t (&M2)[W / 2], uint32_t (&I1)[W / 2], uint32_t& Max, uint32_t rcur, uint32_t gcur,
                   uint32_t TLO, uint32_t THI, uint32_t CFE, uint32_t CFO) {
  uint32_t mw[W / 2];
#pragma unroll
  for (int j = 0; j < W / 2; ++j) mw[j] = 0xffffffffu;
  if (MASKED) pair_mask<W>(p0 + 0, L, mw);
  fstep3<W, false, MASKED, 0>(A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO, mw);
  fstep3<W, true, MASKED, 0>(A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO, mw);
  if (MASKED) pair_mask<W>(p0 + 1, L, mw);
  fstep3<W, false, MASKED, 1>(A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO, mw);
  fstep3<W, true, MASKED, 1>(A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO, mw);
  if (MASKED) pair_mask<W>(p0 + 2, L, mw);
  fstep3<W, false, MASKED, 2>(A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO, mw);
  fstep3<W, true, MASKED, 2>(A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO, mw);
  if (MASKED) pair_mask<W>(p0 + 3, L, mw);
  fstep3<W, false, MASKED, 3>(A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO, mw);
  fstep3<W, true, MASKED, 3>(A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO, mw);
}

// gexp: byte-expanded genome (code c -> c * 0x11) at code 0, 4-byte aligned, readable in its
// padding; rexp: read stream bytes 0xC4 + c * 0x11, 4-byte aligned, readable for L + W + 8
// bytes.  Returns the band maximum (unbiased).  Requires L >= W.
template <int W>
SG_HD int filter_v3(const uint8_t* __restrict__ gexp, int64_t pos, const uint8_t* __restrict__ rexp, int L,
                    uint32_t TLO, uint32_t THI, uint32_t CFE, uint32_t CFO) {
  constexpr int NR = W / 2;
  uint32_t A[NR], B[NR], M1[NR], M2[NR], I1[NR];
#pragma unroll
  for (int j = 0; j < NR; ++j) {
    A[j] = 0xC4C4u;  // code 0 in read format
    // window codes 0..W-1, cell k = code W-1-k
    B[j] = (uint32_t)gexp[pos + W - 1 - 2 * j] | ((uint32_t)gexp[pos + W - 2 - 2 * j] << 8);
    M1[j] = kFBB; M2[j] = kFBB; I1[j] = kFBB;
  }
  uint32_t Max = kFBB;
  const int64_t g0 = pos + W;
  const uint32_t* gw = reinterpret_cast<const uint32_t*>(gexp) + (g0 >> 2);
  const uint32_t s = (uint32_t)(g0 & 3);
  const uint32_t fsel = s | ((s + 1) << 4) | ((s + 2) << 8) | ((s + 3) << 12);
  const uint32_t* rw = reinterpret_cast<const uint32_t*>(rexp);
  const int npairs = L + W - 1;
  const int nblocks = (npairs + 3) >> 2;
  uint32_t w0 = ldg32(gw), w1 = ldg32(gw + 1);
  for (int b = 0; b < nblocks; ++b) {
    const uint32_t gcur = prmt(w0, w1, fsel);
    const uint32_t rcur = ldg32(rw + b);
    w0 = w1;
    w1 = ldg32(gw + b + 2);
    const int p0 = 4 * b;
    if (p0 >= W - 1 && p0 + 3 <= L - 1)
      fblock3<W, false>(p0, L, A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO);
    else
      fblock3<W, true>(p0, L, A, B, M1, M2, I1, Max, rcur, gcur, TLO, THI, CFE, CFO);
  }
  const int lo = (int)(int16_t)(Max & 0xffffu), hi = (int)(int16_t)(Max >> 16);
  return (lo > hi ? lo : hi) - (int)kFB;
}

SG_HD void filter_v3_consts(int fm, int fx, int fo, int fe, uint32_t& TLO, uint32_t& THI, uint32_t& CFE,
                            uint32_t& CFO) {
  const uint32_t mis = (uint32_t)((256 - fx) & 0xff);
  TLO = (mis << 8) | (mis << 16) | (mis << 24);
  THI = (uint32_t)(fm & 0xff) | (mis << 8) | (mis << 16) | (mis << 24);
  CFE = (uint32_t)fe * 0x10001u;
  CFO = (uint32_t)fo * 0x10001u;
}

}  // namespace sg
