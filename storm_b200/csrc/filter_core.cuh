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
// prmts from 4-byte stream words: four read codes and four genome codes per 4 step pairs.
// Pair p of the band covers read positions i = p - W + 1 + k (cell k); blocks whose pairs all
// have 0 <= i < L for every cell run without the mask.
//
// Split layout: register j of the band holds cells j (low half) and j + H (high half),
// H = W / 2.  The neighbour of cell k (k - 1 on genome steps, k + 1 on read steps) is then the
// same half of register j - 1 or j + 1, and shifting a code stream by one cell is a renaming
// of the registers: logical register j of the read codes is A[(j + ra) mod H] after ra read
// steps, and of the genome codes B[(j - rb) mod H] after rb genome steps.  Only the seam
// register (where a half crosses over) needs a prmt, for the neighbour values and for the
// entering code.  Blocks of BP = max(4, H) step pairs return the rotation to 0, so every
// index is a constant.
constexpr uint32_t kFB = 256u;
constexpr uint32_t kFBB = kFB * 0x10001u;

// Cells of pair p inside the read (0 <= p - W + 1 + k <= L - 1), for the pairs where that is
// a constant: prologue pairs p < W - 1 (cells k >= W - 1 - p) and epilogue pairs p = L + e,
// e < W - 1 (cells k <= W - 2 - e).  Every pair in between has all W cells inside.
template <int W> __host__ __device__ constexpr uint32_t full_mask() { return (uint32_t)((1ull << W) - 1ull); }
template <int W, int MODE, int K> __host__ __device__ constexpr uint32_t split_pair_mask() {
  return MODE == 0 ? full_mask<W>()
       : MODE == 1 ? full_mask<W>() & ~((1u << (W - 1 - K)) - 1u)
                   : (2u << (W - 2 - K)) - 1u;
}

// One step of a pair whose index is Q mod H: ODD = genome step.  T = byte of the stream words
// holding the entering codes; MB = the pair's cells inside the read (a constant, so that a
// register with both halves outside costs nothing and one with a half outside one LOP3).
template <int W, bool ODD, int T, int Q, uint32_t MB>
SG_HD void fstep_split(uint32_t (&A)[W / 2], uint32_t (&B)[W / 2], uint32_t (&M1)[W / 2], uint32_t (&M2)[W / 2],
                       uint32_t (&I1)[W / 2], uint32_t& Max, uint32_t rcur, uint32_t gcur, uint32_t TLO,
                       uint32_t THI, uint32_t NFE, uint32_t CFO) {
  constexpr int H = W / 2;
  constexpr int RA = (Q + 1) % H;                // read steps done (mod H), this one included
  constexpr int RB = (ODD ? Q + 1 : Q) % H;      // genome steps done (mod H)
  if (ODD) {  // new code into cell 0; old cell H - 1 moves to cell H
    constexpr int idx = (H - 1 - Q % H + H) % H;
    B[idx] = prmt(gcur, B[idx], 0x0040u | (uint32_t)T);
  } else {    // old cell H moves to cell H - 1; new code into cell W - 1
    constexpr int idx = Q % H;
    A[idx] = prmt(A[idx], rcur, 0x0001u | ((uint32_t)(4 + T) << 4));
  }
  uint32_t P[H], Mn[H], In[H];
#pragma unroll
  // P = max(I1 - ext, M1 - open) as one add-max: NFE holds -ext in both halves, and every half
  // stays positive (cells are biased by 256, ext and open are below 256)
  for (int j = 0; j < H; ++j) P[j] = __viaddmax_s16x2(I1[j], NFE, M1[j] - CFO);
#pragma unroll
  for (int j = 0; j < H; ++j) {
    uint32_t nbr;
    if (ODD) nbr = j > 0 ? P[j - 1] : prmt(kFBB, P[H - 1], 0x5410);
    else     nbr = j < H - 1 ? P[j + 1] : prmt(P[0], kFBB, 0x5432);
    In[j] = __vimax3_s16x2(P[j], nbr, kFBB);
    const bool lo = (MB >> j) & 1u, hi = (MB >> (j + H)) & 1u;
    if (!lo && !hi) {
      Mn[j] = kFBB;  // M of cells outside the read is 0; their I still propagates
    } else {
      const uint32_t sc = prmt(TLO, THI, A[(j + RA) % H] - B[(j - RB + H) % H]);
      const uint32_t mv = __viaddmax_s16x2(M2[j], sc, In[j]);
      Mn[j] = (lo && hi) ? mv : lo ? ((mv & 0x0000FFFFu) | (kFBB & 0xFFFF0000u))
                                   : ((mv & 0xFFFF0000u) | (kFBB & 0x0000FFFFu));
    }
  }
  if (H == 1) {
    Max = __vimax_s16x2_relu(Max, Mn[0]);
  } else {
#pragma unroll
    for (int j = 0; j + 1 < H; j += 2) Max = __vimax3_s16x2(Max, Mn[j], Mn[j + 1]);
  }
#pragma unroll
  for (int j = 0; j < H; ++j) {
    M2[j] = M1[j];
    M1[j] = Mn[j];
    I1[j] = In[j];
  }
}

// Pairs K..NP-1 of a group whose pair 0 has index QB mod H; pair k takes byte k % 4 of the
// stream words rc[k / 4], gc[k / 4].  MODE: 0 main (all cells inside), 1 prologue (pair index
// k), 2 epilogue (pair L + k).
template <int W, int MODE, int QB, int K, int NP, int NWD>
SG_HD void run_pairs_split(uint32_t (&A)[W / 2], uint32_t (&B)[W / 2], uint32_t (&M1)[W / 2], uint32_t (&M2)[W / 2],
                           uint32_t (&I1)[W / 2], uint32_t& Max, const uint32_t (&rc)[NWD],
                           const uint32_t (&gc)[NWD], uint32_t TLO, uint32_t THI, uint32_t NFE, uint32_t CFO) {
  if constexpr (K < NP) {
    constexpr uint32_t MB = split_pair_mask<W, MODE, K>();
    fstep_split<W, false, K % 4, QB + K, MB>(A, B, M1, M2, I1, Max, rc[K / 4], gc[K / 4], TLO, THI, NFE, CFO);
    fstep_split<W, true, K % 4, QB + K, MB>(A, B, M1, M2, I1, Max, rc[K / 4], gc[K / 4], TLO, THI, NFE, CFO);
    run_pairs_split<W, MODE, QB, K + 1, NP, NWD>(A, B, M1, M2, I1, Max, rc, gc, TLO, THI, NFE, CFO);
  }
}

// remainder pairs K.. while K < r (r < NP): guarded, constant rotation
template <int W, int QB, int K, int NP, int NWD>
SG_HD void run_rest_split(int r, uint32_t (&A)[W / 2], uint32_t (&B)[W / 2], uint32_t (&M1)[W / 2],
                          uint32_t (&M2)[W / 2], uint32_t (&I1)[W / 2], uint32_t& Max, const uint32_t (&rc)[NWD],
                          const uint32_t (&gc)[NWD], uint32_t TLO, uint32_t THI, uint32_t NFE, uint32_t CFO) {
  if constexpr (K < NP) {
    if (K < r) {
      run_pairs_split<W, 0, QB, K, K + 1, NWD>(A, B, M1, M2, I1, Max, rc, gc, TLO, THI, NFE, CFO);
      run_rest_split<W, QB, K + 1, NP, NWD>(r, A, B, M1, M2, I1, Max, rc, gc, TLO, THI, NFE, CFO);
    }
  }
}

// selector of prmt(w0, w1, .) picking bytes s..s+3 of the 8-byte pair (s < 4)
SG_HD uint32_t funnel_sel(uint32_t s) { return s | ((s + 1) << 4) | ((s + 2) << 8) | ((s + 3) << 12); }

// gexp: byte-expanded genome (code c -> c * 0x11) at code 0, 4-byte aligned, readable in its
// padding; rexp: read stream bytes 0xC4 + c * 0x11, 4-byte aligned, readable for L + 24
// bytes.  Returns the band maximum (unbiased).  Requires L >= W.
//
// Pairs 0..W-2 (prologue) and L..L+W-2 (epilogue) run with their constant cell masks, pairs
// W-1..L-1 (main) unmasked in blocks of BP pairs; the main remainder (fewer than BP pairs)
// keeps constant rotations, and the registers are rotated back to rotation 0 once, before
// the epilogue.
template <int W>
SG_HD int filter_split(const uint8_t* __restrict__ gexp, int64_t pos, const uint8_t* __restrict__ rexp, int L,
                       uint32_t TLO, uint32_t THI, uint32_t NFE, uint32_t CFO) {
  constexpr int H = W / 2;
  constexpr int BP = H > 4 ? H : 4;
  constexpr int NPRO = W - 1;
  constexpr int NWP = (NPRO + 3) / 4;  // stream words of the prologue / epilogue
  constexpr int NWB = BP / 4;          // stream words of a main block
  uint32_t A[H], B[H], M1[H], M2[H], I1[H];
#pragma unroll
  for (int j = 0; j < H; ++j) {
    A[j] = 0xC4C4u;  // code 0 in read format (cells outside the read)
    // window codes 0..W-1, cell k = code W-1-k
    B[j] = (uint32_t)gexp[pos + W - 1 - j] | ((uint32_t)gexp[pos + W - 1 - j - H] << 8);
    M1[j] = kFBB; M2[j] = kFBB; I1[j] = kFBB;
  }
  uint32_t Max = kFBB;
  const uint32_t* gx = reinterpret_cast<const uint32_t*>(gexp);
  const uint32_t* rw = reinterpret_cast<const uint32_t*>(rexp);
  const int64_t g0 = pos + W;  // genome byte entering at pair 0
  {  // prologue: pairs 0..W-2, read bytes 0.., genome bytes g0..
    uint32_t rc[NWP], gc[NWP];
    const uint32_t* gw = gx + (g0 >> 2);
    const uint32_t sel = funnel_sel((uint32_t)(g0 & 3));
    uint32_t wp = ldg32(gw);
#pragma unroll
    for (int k = 0; k < NWP; ++k) {
      rc[k] = ldg32(rw + k);
      const uint32_t wn = ldg32(gw + k + 1);
      gc[k] = prmt(wp, wn, sel);
      wp = wn;
    }
    run_pairs_split<W, 1, 0, 0, NPRO, NWP>(A, B, M1, M2, I1, Max, rc, gc, TLO, THI, NFE, CFO);
  }
  {  // main: pairs W-1..L-1, index W-1 = H-1 mod H at every block start
    const int nmain = L - W + 1;
    const int64_t gb = g0 + W - 1;
    const uint32_t* gw = gx + (gb >> 2);
    const uint32_t gsel = funnel_sel((uint32_t)(gb & 3));
    const uint32_t* rwm = rw + ((W - 1) >> 2);
    constexpr uint32_t rsel = ((W - 1) & 3) | ((((W - 1) & 3) + 1) << 4) | ((((W - 1) & 3) + 2) << 8) |
                              ((((W - 1) & 3) + 3) << 12);
    uint32_t gp = ldg32(gw), rp = ldg32(rwm);
    int pm = 0;
    for (; pm + BP <= nmain; pm += BP) {
      uint32_t rc[NWB], gc[NWB];
      const int q = pm >> 2;
#pragma unroll
      for (int k = 0; k < NWB; ++k) {
        const uint32_t gn = ldg32(gw + q + k + 1), rn = ldg32(rwm + q + k + 1);
        gc[k] = prmt(gp, gn, gsel);
        rc[k] = prmt(rp, rn, rsel);
        gp = gn;
        rp = rn;
      }
      run_pairs_split<W, 0, H - 1, 0, BP, NWB>(A, B, M1, M2, I1, Max, rc, gc, TLO, THI, NFE, CFO);
    }
    const int r = nmain - pm;
    if (r > 0) {
      uint32_t rc[NWB], gc[NWB];
      const int q = pm >> 2;
#pragma unroll
      for (int k = 0; k < NWB; ++k) {
        const uint32_t gn = ldg32(gw + q + k + 1), rn = ldg32(rwm + q + k + 1);
        gc[k] = prmt(gp, gn, gsel);
        rc[k] = prmt(rp, rn, rsel);
        gp = gn;
        rp = rn;
      }
      run_rest_split<W, H - 1, 0, BP, NWB>(r, A, B, M1, M2, I1, Max, rc, gc, TLO, THI, NFE, CFO);
    }
  }
  if (H > 1) {  // back to rotation 0: logical read register j = A[(j + L) mod H], genome B[(j - L) mod H]
    const int s = L & (H - 1);
#pragma unroll
    for (int b = 1; b < H; b <<= 1) {
      const bool on = (s & b) != 0;
      uint32_t ta[H], tb[H];
#pragma unroll
      for (int j = 0; j < H; ++j) {
        ta[j] = A[(j + b) % H];
        tb[j] = B[(j - b + H) % H];
      }
#pragma unroll
      for (int j = 0; j < H; ++j) {
        A[j] = on ? ta[j] : A[j];
        B[j] = on ? tb[j] : B[j];
      }
    }
  }
  {  // epilogue: pairs L..L+W-2; the entering read codes stay in cells outside the read
    uint32_t rc[NWP], gc[NWP];
    const int64_t ge = g0 + L;
    const uint32_t* gw = gx + (ge >> 2);
    const uint32_t sel = funnel_sel((uint32_t)(ge & 3));
    uint32_t wp = ldg32(gw);
#pragma unroll
    for (int k = 0; k < NWP; ++k) {
      rc[k] = 0xC4C4C4C4u;
      const uint32_t wn = ldg32(gw + k + 1);
      gc[k] = prmt(wp, wn, sel);
      wp = wn;
    }
    run_pairs_split<W, 2, 0, 0, NPRO, NWP>(A, B, M1, M2, I1, Max, rc, gc, TLO, THI, NFE, CFO);
  }
  const int lo = (int)(int16_t)(Max & 0xffffu), hi = (int)(int16_t)(Max >> 16);
  return (lo > hi ? lo : hi) - (int)kFB;
}

SG_HD void filter_split_consts(int fm, int fx, int fo, int fe, uint32_t& TLO, uint32_t& THI, uint32_t& NFE,
                            uint32_t& CFO) {
  const uint32_t mis = (uint32_t)((256 - fx) & 0xff);
  TLO = (mis << 8) | (mis << 16) | (mis << 24);
  THI = (uint32_t)(fm & 0xff) | (mis << 8) | (mis << 16) | (mis << 24);
  NFE = (uint32_t)(uint16_t)(-fe) * 0x10001u;
  CFO = (uint32_t)fo * 0x10001u;
}

}  // namespace sg
