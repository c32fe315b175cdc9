// map_kernels.cu -- the kernels of one mapping pass (one reference sequence x one strand).
//
//  (hit gather: gather.cu; banded filter: sw_filter.cu)
//  align                                            banded DP + traceback (alignment.c:488-734)
//  replay                                           per-read top-4 update (run.c:664-691,
//                                                   hit_map.c:50-144)
#include "map_kernels.cuh"

namespace sg {

// ------------------------------------------------------------------------------ reads

__global__ void reverse_reads_kernel(ReadsDev in, const uint8_t* __restrict__ first_levels, int colour,
                                     uint8_t* __restrict__ rcodes, uint8_t* __restrict__ rlevels) {
  int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= in.n) return;
  const int L = in.lengths[r];
  const uint8_t* c = in.codes + r * in.cstride;
  uint8_t* rc = rcodes + r * in.cstride;
  for (int64_t b = 0; b < in.cstride; ++b) rc[b] = 0;
  // read__reverse (reads_data.c:9-35): nucleotide = reverse complement, colour = reverse
  for (int i = 0; i < L; ++i) {
    int v = code_at(c, i);
    if (!colour) v = 3 - v;
    int o = L - 1 - i;
    rc[o >> 2] |= (uint8_t)(v << ((o & 3) << 1));
  }
  if (in.levels) {
    const uint8_t* q = in.levels + r * in.lstride;
    uint8_t* rq = rlevels + r * in.lstride;
    for (int64_t b = 0; b < in.lstride; ++b) rq[b] = 0;
    if (!colour) {
      for (int i = 0; i < L; ++i) rq[i >> 2] |= (uint8_t)(code_at(q, L - 1 - i) << ((i & 3) << 1));
    } else {
      // quality__reverse_compressed, colour (read_quality.c:238-241)
      int fl = first_levels ? first_levels[r] : 3;
      rq[(L - 1) >> 2] |= (uint8_t)((fl & 3) << (((L - 1) & 3) << 1));
      for (int i = 0; i < L - 1; ++i) rq[i >> 2] |= (uint8_t)(code_at(q, L - 2 - i) << ((i & 3) << 1));
    }
  }
}

void launch_reverse_reads(const ReadsDev& in, const uint8_t* first_levels, int colour,
                          uint8_t* rcodes, uint8_t* rlevels, cudaStream_t st) {
  if (in.n <= 0) return;
  reverse_reads_kernel<<<(unsigned)((in.n + 127) / 128), 128, 0, st>>>(in, first_levels, colour, rcodes, rlevels);
}

__global__ void init_results_kernel(int64_t n, stormgpu_hit* __restrict__ hits, uint8_t* __restrict__ mapped) {
  int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * 4) return;
  stormgpu_hit h;
  h.score = kMinScore;
  h.ref_id = h.ref_start = h.ref_end = -1;
  h.read_start = h.read_end = -1;
  h.sense = 0;
  h.tb_len = 0;
  hits[t] = h;
  if ((t & 3) == 0) mapped[t >> 2] = 0;
}

void launch_init_results(int64_t n, stormgpu_hit* hits, uint8_t* mapped, uint8_t* tb, int64_t tbs,
                         cudaStream_t st) {
  if (n <= 0) return;
  init_results_kernel<<<(unsigned)((n * 4 + 255) / 256), 256, 0, st>>>(n, hits, mapped);
  cudaMemsetAsync(tb, 0, (size_t)(n * 4 * tbs), st);  // the 4n traceback rows are contiguous
}

// ------------------------------------------------------------------------------ align

// Cell state packed in 16 bits: from (2) | indels (7) | colour checksum (2) | auto-correct (2)
// | freshness (3).  "from": 3 corner, 2 top, 1 left (alignment.c:13-19).
__device__ __forceinline__ int st_from(int s) { return s & 3; }
__device__ __forceinline__ int st_ind(int s) { return (s >> 2) & 127; }
__device__ __forceinline__ int st_chk(int s) { return (s >> 9) & 3; }
__device__ __forceinline__ int st_ac(int s) { return (s >> 11) & 3; }
__device__ __forceinline__ int st_fr(int s) { return (s >> 13) & 7; }
__device__ __forceinline__ int st_make(int from, int ind, int chk, int ac, int fr) {
  return from | (ind << 2) | (chk << 9) | (ac << 11) | (fr << 13);
}

constexpr int kMaxBand = 2 * STORMGPU_MAX_INDELS + 1;

// alignment.c:326-360 (init), :488-632 (rows 1..L-1, corner > top > left on ties, gaps only
// while indels < I, affine through the predecessor's direction, colour checksum state
// machine :535-603 with the SNP adjustment :465-468), best cell on the last row (:621-630),
// traceback :642-734.  The direction of every cell (2 bits) and, in colour space, whether its
// pair score was made positive by the SNP adjustment (the `score > corner score` test of
// :693) go to the scratch, column-minor: word (row*wpr + k)*ns + sl for scratch column sl of
// ns (the slot's index in a one-per-thread launch, the thread's index in a persistent one).
// Genome and mask codes of the band of one row, 2 bits each in registers, for a constant band
// width: row i + 1 is row i moved by one code, so each row loads one genome and one mask code
// (instead of BW of each).
template <int BWT>
struct BandWindow {
  static_assert(BWT > 0 && BWT <= 64, "band width");
  uint64_t g[2] = {0, 0}, m[2] = {0, 0};
  __device__ __forceinline__ void put(int c, int gc, int mc) {
    g[c >> 5] |= (uint64_t)gc << (2 * (c & 31));
    m[c >> 5] |= (uint64_t)mc << (2 * (c & 31));
  }
  // codes [base, base + BWT)
  __device__ __forceinline__ void load(const uint8_t* genome, const uint8_t* mask, int64_t base) {
#pragma unroll
    for (int c = 0; c < BWT; ++c) put(c, code_at(genome, base + c), code_at(mask, base + c));
  }
  // drop cell 0, the others move down one cell, code `pos` becomes cell BWT - 1
  __device__ __forceinline__ void advance(const uint8_t* genome, const uint8_t* mask, int64_t pos) {
    if (BWT > 32) {
      g[0] = (g[0] >> 2) | (g[1] << 62);
      m[0] = (m[0] >> 2) | (m[1] << 62);
      g[1] >>= 2;
      m[1] >>= 2;
    } else {
      g[0] >>= 2;
      m[0] >>= 2;
    }
    put(BWT - 1, code_at(genome, pos), code_at(mask, pos));
  }
  __device__ __forceinline__ int gcode(int c) const { return (int)((g[c >> 5] >> (2 * (c & 31))) & 3u); }
  __device__ __forceinline__ int mcode(int c) const { return (int)((m[c >> 5] >> (2 * (c & 31))) & 3u); }
};

// BWT > 0: the band width 2I + 1 as a constant, so that the row arrays live in registers;
// BWT = 0: any width up to kMaxBand (arrays in local memory).  CM: 0 nucleotide, 1 colour
// space (the colour state machine compiled in), -1 either (sp.colour); the kernel's CM = 2 runs
// the packed nucleotide form below (align_one_nuc).
// A candidate whose running abort bound falls below the replay's threshold stops at that row:
// -t, or with rounds the running threshold its read had after the rounds before (the replay's
// threshold only rises, so the candidate is aborted whatever comes before it), and neither its
// score nor its traceback is read.
// One slot; its direction bits in scratch column sl of ns.  Returns the rows it computed.
template <int BWT, int CM>
__device__ __forceinline__ int align_one(const ReadsDev& rd, const ScoreParams& sp, const uint8_t* __restrict__ genome,
                                         const uint8_t* __restrict__ mask, int64_t slot, int64_t sl, int64_t ns,
                                         const PassBuffers& pb) {
  constexpr int NB = BWT > 0 ? BWT : kMaxBand;
  const int r = pb.p_read[slot];
  // the first round, and a launch without rounds, stop at -t only: pb.thr holds the read's
  // threshold after the rounds before this one (in the first round, a previous pass's value)
  const int thr = (pb.thr && pb.round > 0) ? max(sp.min_score, pb.thr[r]) : sp.min_score;
  const int d = pb.p_diag[slot];
  const int I = sp.I, BW = BWT > 0 ? BWT : 2 * I + 1, colour = CM >= 0 ? CM : sp.colour;
  const int L = rd.lengths[r];
  const uint8_t* rdc = rd.codes + (int64_t)r * rd.cstride;
  const uint8_t* rdq = rd.levels ? rd.levels + (int64_t)r * rd.lstride : nullptr;
  const int win = max(d - I, -sp.Is);  // run.c:667
  const int wpr_dir = (2 * BW + 31) / 32, wpr = wpr_dir + (colour ? (BW + 31) / 32 : 0);
  uint32_t* scr = pb.a_scratch;
  int sc[NB], stt[NB];
  const int mbest = sp.pair[0][3];
  BandWindow<(BWT > 0 ? BWT : 1)> bwin;
  if (BWT > 0) bwin.load(genome, mask, win);
  // row 0
  {
    const int rc = code_at(rdc, 0), q = rdq ? code_at(rdq, 0) : 3;
    uint32_t wd[(2 * NB + 31) / 32] = {};
#pragma unroll
    for (int c = 0; c < BW; ++c) {
      const int64_t j = (int64_t)win + c;
      const int f = BWT > 0 ? bwin.gcode(c) : code_at(genome, j);
      int chk = 0, score;
      if ((BWT > 0 ? bwin.mcode(c) : code_at(mask, j)) == 0) {
        chk = colour ? (rc ^ f) : 0;
        score = sp.pair[colour ? (chk ? 1 : 0) : (rc != f)][q];
      } else score = kMinScore;
      sc[c] = score;
      stt[c] = st_make(3, 0, chk, chk, (colour && chk) ? q : 0);
      wd[(2 * c) >> 5] |= 3u << ((2 * c) & 31);
    }
    for (int k = 0; k < wpr; ++k) scr[(int64_t)k * ns + sl] = k < wpr_dir ? wd[k] : 0u;
  }
  int best_possible = (colour ? (L - 2) : L) * mbest;
  long long bound = 0x7fffffffLL;
  int rows = L;
  for (int i = 1; i < L; ++i) {
    const int rc = code_at(rdc, i), q = rdq ? code_at(rdq, i) : 3;
    int max_on_line = kMinScore;
    int lsc = kMinScore, lst = st_make(3, I, 0, 0, 0);  // left border
    uint32_t wd[(2 * NB + 31) / 32] = {};
    uint32_t wc[(NB + 31) / 32] = {};
    if (BWT > 0) bwin.advance(genome, mask, (int64_t)win + i + BW - 1);
#pragma unroll
    for (int c = 0; c < BW; ++c) {
      const int64_t j = (int64_t)win + i + c;
      const int f = BWT > 0 ? bwin.gcode(c) : code_at(genome, j);
      // initial values of this cell (alignment__init_matrix)
      int chk0 = 0, ac0 = 0, fr0 = 0, s0;
      if ((BWT > 0 ? bwin.mcode(c) : code_at(mask, j)) == 0) {
        if (colour) { chk0 = ac0 = rc ^ f; fr0 = ac0 ? q : 0; s0 = sp.pair[chk0 ? 1 : 0][q]; }
        else s0 = sp.pair[rc != f][q];
      } else s0 = kMinScore;
      const int csc = sc[c], cst = stt[c];
      const int tsc = c + 1 < BW ? sc[c + 1] : kMinScore;
      const int tst = c + 1 < BW ? stt[c + 1] : st_make(3, I, 0, 0, 0);
      int ms = s0;
      if (colour) {
        const int prev = st_chk(cst), cmp = prev ^ chk0;
        if (prev && (cmp == 0 || cmp == st_ac(cst)) && s0 != kMinScore && s0 < 0) ms = -2 * s0;
      }
      int score = csc + ms, it = 0, tmp;
      if (st_ind(tst) < I && (tmp = tsc + ((st_from(tst) ^ 2) ? sp.gap_open : sp.gap_ext)) > score) { it = 1; score = tmp; }
      if (st_ind(lst) < I && (tmp = lsc + ((st_from(lst) ^ 1) ? sp.gap_open : sp.gap_ext)) > score) { it = 2; score = tmp; }
      int from = 3, ind, chk = chk0, ac = ac0, fr = fr0;
      if (it == 0) {
        ind = st_ind(cst);
        if (colour) {
          const int cchk = st_chk(cst), cac = st_ac(cst), cfr = st_fr(cst);
          chk = chk0 ^ cchk;
          if (cchk != chk) {
            if (cchk == 0) { ac = chk; fr = q; }
            else if (chk == cac) { ac = 0; chk = 0; fr = 0; }
            else if (chk == 0) { if (cfr - 1 > 0) { ac = cac; fr = cfr - 1; } else { ac = 0; fr = 0; } }
            else { if (cfr - 1 > 0) { ac = cac; fr = cfr - 1; } else { ac = chk; fr = q; } }
          } else {
            if (cac != 0) {
              if (cfr - 1 > 0) {
                if (chk == 0) { ac = 0; fr = 0; } else { ac = cac; fr = cfr - 1; }
              }
            } else { chk = 0; ac = 0; fr = 0; }
          }
        }
      } else if (it == 1) {
        from = 2;
        ind = st_ind(tst) + 1;
        if (colour) {
          chk = st_chk(tst) ^ rc;
          if (st_fr(tst) - 1 > 0) { fr = st_fr(tst) - 1; ac = st_ac(cst); }
        }
      } else {
        from = 1;
        ind = st_ind(lst) + 1;
        if (colour) {
          chk = st_chk(lst) ^ f;
          if (st_fr(lst) - 1 > 0) { fr = st_fr(lst) - 1; ac = st_ac(cst); }
        }
      }
      const int nst = st_make(from, ind, chk, ac, fr);
      sc[c] = score;
      stt[c] = nst;
      lsc = score;
      lst = nst;
      if (max_on_line < score) max_on_line = score;
      wd[(2 * c) >> 5] |= (uint32_t)from << ((2 * c) & 31);
      if (colour && it == 0 && ms > 0) wc[c >> 5] |= 1u << (c & 31);
    }
    if ((long long)max_on_line + best_possible < bound) bound = (long long)max_on_line + best_possible;
    best_possible -= mbest;
    for (int k = 0; k < wpr_dir; ++k) scr[((int64_t)i * wpr + k) * ns + sl] = wd[k];
    if (colour)
      for (int k = wpr_dir; k < wpr; ++k) scr[((int64_t)i * wpr + k) * ns + sl] = wc[k - wpr_dir];
    if (bound < thr) {  // aborted at any threshold it can meet
      rows = i + 1;
      break;
    }
  }
  int best = kMinScore, bi = -1, bj = -1;
#pragma unroll
  for (int c = 0; c < BW; ++c)
    if (best < sc[c]) { best = sc[c]; bi = L - 1; bj = L - 1 + c; }
  const int32_t bnd = bound > 0x7fffffffLL ? 0x7fffffff : (int32_t)bound;
  pb.a_score[slot] = best;
  pb.a_bound[slot] = bnd;
  int i0 = bi, j0 = bj, tl = 0;
  uint8_t* tb = pb.a_tb + slot * pb.tbs;
  if (bi >= 0 && bnd >= thr && best > thr) {
    int i = bi, c = bj - bi, colr = 0;
    uint8_t cur = 0;
    while (i >= 0 && i < L && c >= 0 && c < BW) {
      const int j = i + c;
      i0 = i;
      j0 = j;
      const uint32_t wdir = scr[((int64_t)i * wpr + ((2 * c) >> 5)) * ns + sl];
      const int from = (wdir >> ((2 * c) & 31)) & 3;
      const int rc = code_at(rdc, i);
      int op;
      if (from == 2) op = 0xC | rc;
      else if (from == 1) op = 0x1;
      else {
        const int f = code_at(genome, (int64_t)win + j);
        if (rc != f) {
          if (!colour) op = 0x4 | rc;
          else {
            bool adj = false;
            if (i != 0 && j != 0) {
              const uint32_t wcol = scr[((int64_t)i * wpr + wpr_dir + (c >> 5)) * ns + sl];
              adj = (wcol >> (c & 31)) & 1u;
            }
            if (colr || adj) { op = 0x8 | rc; colr ^= rc ^ f; }
            else op = 0x4 | rc;
          }
        } else op = 0x3;
      }
      if (tl & 1) { cur |= (uint8_t)op; tb[tl >> 1] = cur; }
      else { cur = (uint8_t)(op << 4); tb[tl >> 1] = cur; }
      tl++;
      if (from == 2) { i--; c++; }
      else if (from == 1) { c--; }
      else { i--; }
    }
  }
  pb.a_tblen[slot] = tl;
  pb.a_pos[slot * 4 + 0] = (int16_t)bi;
  pb.a_pos[slot * 4 + 1] = (int16_t)bj;
  pb.a_pos[slot * 4 + 2] = (int16_t)i0;
  pb.a_pos[slot * 4 + 3] = (int16_t)j0;
  return rows;
}

// Nucleotide space with a constant band: the DP of align_one with each cell in one register,
//   score << 13 | from << 10 (one-hot: corner 4, top 2, left 1) | guard << 8 | ind',
// ind' = indels + 256 - I in 8 bits, whose carry into the guard bit marks indels == I (no gap
// may leave such a cell).  The largest candidate value is the reference's choice
// (alignment.c:521-532: the higher score, on equal scores corner before top before left) and
// carries its direction and indel count, so a cell is one three-way max.  The gap candidates
// are formed with integer multiply-adds, which issue on the FMA pipe beside the ALU's logic and
// max operations: t + (open << 13 | 1) relabelled as a gap, plus (t & (its from bit | guard))
// times a constant K chosen modulo 2^32 so that the from bit adds (ext - open) << 13 (an
// extension) and the guard about -2^30, which puts a gap the reference does not allow below
// every cell.  Direction bits are moved into the row's words by multiply-adds too.
// Cells are floored at score -2^16 (every 16 rows, and in rows with masked cells): a floored
// cell, and any cell whose value derives from one, stays below -2^16 + L * (largest pair score),
// under the row maximum's start MIN_SCORE and below every cell of a path the replay can keep
// (sp.packed holds only when -t - L * match stays above it); so every score, bound and traceback
// the replay reads is the reference's, and no packed value overflows.
constexpr int kCellShift = 13;
constexpr int kCellFloor = -(1 << 29);
constexpr uint32_t kFromC = 1u << 12, kFromT = 1u << 11, kFromL = 1u << 10, kFromAll = kFromC | kFromT | kFromL;
constexpr uint32_t kGuard = 1u << 8;

__device__ __forceinline__ uint32_t mad_lo(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
__device__ __forceinline__ uint32_t mad_hi(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("mad.hi.u32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// One row of the packed DP: v[] holds the previous row and becomes this one; mis / msk hold a
// bit at 2c for a mismatching / masked cell c (word c >> 4); returns the row maximum.  The
// corner relabelling of v[c + 1] serves both this cell's top candidate and the next cell's
// corner.  Rows without masked cells skip the floor (align_one_nuc floors every cell every 16
// rows: between those a cell falls by at most 16 * 255 << 13, so nothing overflows and a gap
// the reference forbids still lands below every cell); rows with masked cells (MIN_SCORE)
// floor every cell.
template <int BW, bool MASKED>
__device__ __forceinline__ int packed_row(int (&v)[BW], uint32_t (&wd)[(2 * BW + 31) / 32], const uint32_t* mis,
                                          const uint32_t* msk, int SM, int SX, int MINS, const ScoreParams& sp) {
  int mol = MINS, left = 0, pend = MINS;
  uint32_t cv = ((uint32_t)v[0] & ~kFromAll) | kFromC;  // v[c] relabelled as a corner source
#pragma unroll
  for (int c = 0; c < BW; ++c) {
    const uint32_t bit = 1u << (2 * (c & 15));
    int s0 = (mis[c >> 4] & bit) ? SX : SM;
    if (MASKED && (msk[c >> 4] & bit)) s0 = MINS;
    int nv = (int)mad_lo((uint32_t)s0, sp.one, cv);
    if (MASKED) nv = max(nv, kCellFloor);
    int top = 0, lft = 0;
    if (c + 1 < BW) {
      const uint32_t t = (uint32_t)v[c + 1];
      cv = (t & ~kFromAll) | kFromC;
      top = (int)mad_lo(t & (kFromT | kGuard), sp.kt, mad_lo(cv, sp.one, sp.open1_tc));
    }
    if (c > 0) {
      const uint32_t l = (uint32_t)left;
      const uint32_t b = (mad_lo(l, sp.one, sp.open1) & ~kFromAll) | kFromL;
      lft = (int)mad_lo(l & (kFromL | kGuard), sp.kl, b);
    }
    if (c > 0 && c + 1 < BW) nv = __vimax3_s32(nv, top, lft);
    else if (c + 1 < BW) nv = max(nv, top);
    else if (c > 0) nv = max(nv, lft);
    v[c] = nv;
    left = nv;
    if (c & 1) mol = __vimax3_s32(mol, pend, nv);
    else if (c + 1 == BW) mol = max(mol, nv);
    else pend = nv;
    const uint32_t x = (uint32_t)nv & (kFromC | kFromT);  // direction: 2 corner, 1 top, 0 left
    const int p = 2 * (c & 15);
    if (p <= 10) wd[c >> 4] = mad_hi(x, sp.pw[21 + p], wd[c >> 4]);
    else wd[c >> 4] = mad_lo(x, sp.pw[p - 11], wd[c >> 4]);
  }
  return mol;
}

template <int BW>
__device__ __forceinline__ int align_one_nuc(const ReadsDev& rd, const ScoreParams& sp,
                                             const uint8_t* __restrict__ genome, const uint8_t* __restrict__ mask,
                                             int64_t slot, int64_t sl, int64_t ns, const PassBuffers& pb) {
  static_assert(BW <= 48, "three direction words per row at most");
  const int r = pb.p_read[slot];
  const int thr = (pb.thr && pb.round > 0) ? max(sp.min_score, pb.thr[r]) : sp.min_score;
  const int d = pb.p_diag[slot];
  const int I = sp.I;
  const int L = rd.lengths[r];
  const uint8_t* rdc = rd.codes + (int64_t)r * rd.cstride;
  const uint8_t* rdq = rd.levels ? rd.levels + (int64_t)r * rd.lstride : nullptr;
  const int win = max(d - I, -sp.Is);  // run.c:667
  constexpr int wpr = (2 * BW + 31) / 32;
  constexpr int NW64 = (BW + 31) / 32;
  uint32_t* scr = pb.a_scratch;
  const int MINS = kMinScore * (1 << kCellShift);
  int v[BW];
  const int mbest = sp.pair[0][3];
  BandWindow<BW> bwin;
  bwin.load(genome, mask, win);
  {  // row 0: pair scores only (alignment.c:326-360); indels 0
    const int rc = code_at(rdc, 0), q = rdq ? code_at(rdq, 0) : 3;
    const int SM = sp.pair[0][q] * (1 << kCellShift), SX = sp.pair[1][q] * (1 << kCellShift);
    const int init = (int)kFromC | (256 - I);
    uint32_t wd[wpr] = {};
#pragma unroll
    for (int c = 0; c < BW; ++c) {
      v[c] = (bwin.mcode(c) == 0 ? (rc != bwin.gcode(c) ? SX : SM) : MINS) | init;
      wd[(2 * c) >> 5] |= 2u << ((2 * c) & 31);
    }
#pragma unroll
    for (int k = 0; k < wpr; ++k) scr[(int64_t)k * ns + sl] = wd[k];
  }
  int best_possible = L * mbest;
  long long bound = 0x7fffffffLL;
  int rows = L;
  for (int i = 1; i < L; ++i) {
    const int rc = code_at(rdc, i), q = rdq ? code_at(rdq, i) : 3;
    const int SM = sp.pair[0][q] * (1 << kCellShift), SX = sp.pair[1][q] * (1 << kCellShift);
    bwin.advance(genome, mask, (int64_t)win + i + BW - 1);
    uint32_t mis[2 * NW64], msk[2 * NW64];
    bool masked = false;
    const uint64_t rrep = (uint64_t)rc * 0x5555555555555555ull;
#pragma unroll
    for (int k = 0; k < NW64; ++k) {
      const uint64_t x = bwin.g[k] ^ rrep;
      const uint64_t mm = (x | (x >> 1)) & 0x5555555555555555ull;
      const uint64_t mk = (bwin.m[k] | (bwin.m[k] >> 1)) & 0x5555555555555555ull;
      mis[2 * k] = (uint32_t)mm;
      mis[2 * k + 1] = (uint32_t)(mm >> 32);
      msk[2 * k] = (uint32_t)mk;
      msk[2 * k + 1] = (uint32_t)(mk >> 32);
      masked |= mk != 0;
    }
    uint32_t wd[wpr] = {};
    if ((i & 15) == 0) {
#pragma unroll
      for (int c = 0; c < BW; ++c) v[c] = max(v[c], kCellFloor);
    }
    const int mol = masked ? packed_row<BW, true>(v, wd, mis, msk, SM, SX, MINS, sp)
                           : packed_row<BW, false>(v, wd, mis, msk, SM, SX, MINS, sp);
    const long long ml = (long long)(mol >> kCellShift) + best_possible;
    if (ml < bound) bound = ml;
    best_possible -= mbest;
#pragma unroll
    for (int k = 0; k < wpr; ++k) scr[((int64_t)i * wpr + k) * ns + sl] = wd[k];
    if (bound < thr) {
      rows = i + 1;
      break;
    }
  }
  int best = kMinScore, bi = -1, bj = -1;
#pragma unroll
  for (int c = 0; c < BW; ++c) {
    const int s = v[c] >> kCellShift;
    if (best < s) { best = s; bi = L - 1; bj = L - 1 + c; }
  }
  const int32_t bnd = bound > 0x7fffffffLL ? 0x7fffffff : (int32_t)bound;
  pb.a_score[slot] = best;
  pb.a_bound[slot] = bnd;
  int i0 = bi, j0 = bj, tl = 0;
  uint8_t* tb = pb.a_tb + slot * pb.tbs;
  if (bi >= 0 && bnd >= thr && best > thr) {  // alignment.c:642-734
    int i = bi, c = bj - bi;
    uint8_t cur = 0;
    while (i >= 0 && i < L && c >= 0 && c < BW) {
      const int j = i + c;
      i0 = i;
      j0 = j;
      const uint32_t wdir = scr[((int64_t)i * wpr + ((2 * c) >> 5)) * ns + sl];
      const int from = (wdir >> ((2 * c) & 31)) & 3;  // 2 corner, 1 top, 0 left
      const int rc = code_at(rdc, i);
      int op;
      if (from == 1) op = 0xC | rc;
      else if (from == 0) op = 0x1;
      else op = rc != code_at(genome, (int64_t)win + j) ? 0x4 | rc : 0x3;
      if (tl & 1) { cur |= (uint8_t)op; tb[tl >> 1] = cur; }
      else { cur = (uint8_t)(op << 4); tb[tl >> 1] = cur; }
      tl++;
      if (from == 1) { i--; c++; }
      else if (from == 0) { c--; }
      else { i--; }
    }
  }
  pb.a_tblen[slot] = tl;
  pb.a_pos[slot * 4 + 0] = (int16_t)bi;
  pb.a_pos[slot * 4 + 1] = (int16_t)bj;
  pb.a_pos[slot * 4 + 2] = (int16_t)i0;
  pb.a_pos[slot * 4 + 3] = (int16_t)j0;
  return rows;
}

// Slots slot0 .. slot0 + nslots: one per thread (scratch column = slot - slot0), or with
// pb.cursor a persistent grid whose warps take the next 32 slots from the cursor (the slot
// count read from pb.npass_dev when it is given; scratch column = the thread's index in the
// grid, so the scratch holds align_workers() columns).
template <int BWT, int CM>
__global__ void __launch_bounds__(128, CM == 2 ? (BWT > 0 && BWT <= 15 ? 7 : BWT == 31 ? 5 : BWT == 41 ? 4 : 1)
                                              : (BWT > 0 && BWT <= 15 ? 5 : BWT == 31 ? 4 : BWT == 41 ? 3 : 1)) align_kernel(ReadsDev rd, ScoreParams sp, const uint8_t* __restrict__ genome,
                                                    const uint8_t* __restrict__ mask, int64_t slot0, int64_t nslots,
                                                    PassBuffers pb) {
  // one call site of align_one (its band code is large and fully unrolled)
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool steal = pb.cursor != nullptr;
  int64_t n = steal && pb.npass_dev ? *pb.npass_dev : nslots;
  int64_t list0 = 0;  // with rounds: this round's slots are round_slots[list0 .. list0 + n)
  if (pb.round_slots) {
    n = pb.round_count[pb.round];
    for (int k = 0; k < pb.round; ++k) list0 += pb.round_count[k];
  }
  const int64_t ns = steal ? (int64_t)gridDim.x * blockDim.x : nslots;
  const int lane = threadIdx.x & 31;
  const int take = pb.steal >= 32 ? pb.steal & ~31 : 32;
  unsigned long long rows = 0;
  int64_t s = tid, end = steal ? 0 : tid + 1;  // stealing: every lane takes the first run together
  for (;;) {
    if (steal && s >= end) {  // the warp's next run of `take` slots
      unsigned long long b = 0;
      if (lane == 0) b = atomicAdd(pb.cursor, (unsigned long long)take);
      s = (int64_t)__shfl_sync(0xffffffffu, b, 0);
      if (s >= n) break;
      end = s + take;
      s += lane;
    }
    if (s < n) {
      const int64_t slot = pb.round_slots ? (int64_t)pb.round_slots[list0 + s] : slot0 + s;
      if constexpr (CM == 2)
        rows += (unsigned long long)align_one_nuc<BWT>(rd, sp, genome, mask, slot, steal ? tid : s, ns, pb);
      else
        rows += (unsigned long long)align_one<BWT, CM>(rd, sp, genome, mask, slot, steal ? tid : s, ns, pb);
    }
    if (!steal) break;
    s += 32;
  }
  if (pb.cells) {
    for (int o = 16; o > 0; o >>= 1) rows += __shfl_xor_sync(0xffffffffu, rows, o);
    if (lane == 0 && rows) atomicAdd(pb.cells, rows * (unsigned long long)(2 * sp.I + 1));
  }
}

static const void* align_kernel_of(const ScoreParams& sp) {
#define SG_ALIGN(BW) \
  case BW: return sp.colour ? (const void*)align_kernel<BW, 1> \
                  : sp.packed ? (const void*)align_kernel<BW, 2> : (const void*)align_kernel<BW, 0>;
  switch (2 * sp.I + 1) {
    SG_ALIGN(7)
    SG_ALIGN(15)
    SG_ALIGN(31)
    SG_ALIGN(41)
  default: return (const void*)align_kernel<0, -1>;
  }
#undef SG_ALIGN
}

int64_t align_workers(int64_t nslots, const ScoreParams& sp) {
  const int64_t g = resident_grid_of(align_kernel_of(sp), 128, 0) * 128;
  return std::min<int64_t>(g, (nslots + 127) / 128 * 128);
}

void launch_align(const ReadsDev& r, const ScoreParams& sp, const uint8_t* genome,
                  const uint8_t* mask, int64_t slot0, int64_t nslots, PassBuffers& pb,
                  cudaStream_t st) {
  if (nslots <= 0) return;
  const void* k = align_kernel_of(sp);
  const unsigned blocks = (unsigned)(pb.cursor ? align_workers(nslots, sp) / 128 : (nslots + 127) / 128);
  void* args[] = {(void*)&r, (void*)&sp, (void*)&genome, (void*)&mask, (void*)&slot0, (void*)&nslots, (void*)&pb};
  cudaLaunchKernel(k, dim3(blocks), dim3(128), args, 0, st);  // errors surface at the caller's next check
}

// ------------------------------------------------------------------------------ replay

__device__ __forceinline__ int tbget(const uint8_t* t, int i) { return (t[i >> 1] >> ((i & 1) ? 0 : 4)) & 0xF; }

// process_read's acceptance (run.c:664-691) in the reference's order, with the
// threshold starting at -t for every (sequence, strand, read): aborted iff the bound is
// below the running threshold; accepted iff not aborted and score > threshold; then
// hit_map__update (hit_map.c:50-144) and threshold = max(threshold, 4th score).
// With rounds, the ranks [lo, hi) of each read, starting from the threshold the ranks before
// left in pb.thr (the first round starts from -t), which it updates.
__global__ void replay_kernel(int64_t n, ScoreParams sp, int ref_id, int sense, PassBuffers pb, int lo, int hi,
                              stormgpu_hit* __restrict__ hits, uint8_t* __restrict__ tbo, int64_t tbs,
                              uint8_t* __restrict__ mapped) {
  const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int P = pb.pcount[r];
  if (P <= lo) return;
  const int64_t s0 = pb.pstart[r];
  int T = (pb.thr && lo > 0) ? pb.thr[r] : sp.min_score;
  stormgpu_hit* h = hits + r * 4;
  const int kend = P < hi ? P : hi;
  for (int k = lo; k < kend; ++k) {
    const int64_t slot = s0 + k;
    const int score = pb.a_score[slot];
    if (!(pb.a_bound[slot] >= T && score > T)) continue;
    const int win = max(pb.p_diag[slot] - sp.I, -sp.Is);
    const int bi = pb.a_pos[slot * 4 + 0], bj = pb.a_pos[slot * 4 + 1];
    const int i0 = pb.a_pos[slot * 4 + 2], j0 = pb.a_pos[slot * 4 + 3];
    mapped[r] = 1;
    int q;
    bool dup_worse = false;
    for (q = 0; q < 4 && h[q].ref_id != -1; ++q) {
      if (h[q].ref_id == ref_id &&
          ((h[q].ref_start == win + j0 && h[q].read_start == i0) ||
           (h[q].ref_end == win + bj && h[q].read_end == bi))) {
        if (score > h[q].score) break;
        dup_worse = true;
        break;
      }
    }
    if (!dup_worse) {
      if (q == 4) q--;
      int i = q;
      while (i >= 0 && score > h[i].score) i--;
      if (i != 3) {
        for (int j = q; j > i + 1; --j) {
          h[j] = h[j - 1];
          for (int64_t b = 0; b < tbs; ++b) tbo[(r * 4 + j) * tbs + b] = tbo[(r * 4 + j - 1) * tbs + b];
        }
        stormgpu_hit nh;
        nh.score = score;
        nh.ref_id = ref_id;
        nh.ref_start = win + j0;
        nh.ref_end = win + bj;
        nh.read_start = (int16_t)i0;
        nh.read_end = (int16_t)bi;
        nh.sense = sense;
        const int tl = pb.a_tblen[slot];
        nh.tb_len = tl;
        h[i + 1] = nh;
        uint8_t* dst = tbo + (r * 4 + i + 1) * tbs;
        const uint8_t* srcb = pb.a_tb + slot * pb.tbs;
        for (int64_t b = 0; b < tbs; ++b) dst[b] = 0;
        for (int p = 0; p < tl; ++p) {
          int v = tbget(srcb, tl - 1 - p);
          if (p & 1) dst[p >> 1] |= (uint8_t)v;
          else dst[p >> 1] |= (uint8_t)(v << 4);
        }
      }
    }
    if (h[3].score > T) T = h[3].score;
  }
  if (pb.thr) pb.thr[r] = T;
}

void launch_replay(int64_t n, const ScoreParams& sp, int ref_id, int sense, PassBuffers& pb,
                   stormgpu_hit* hits, uint8_t* tb, int64_t tbs, uint8_t* mapped, cudaStream_t st) {
  if (n <= 0) return;
  replay_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n, sp, ref_id, sense, pb, 0, 0x7fffffff, hits, tb, tbs,
                                                             mapped);
}

void launch_replay_round(int64_t n, const ScoreParams& sp, int ref_id, int sense, PassBuffers& pb, int rounds,
                         stormgpu_hit* hits, uint8_t* tb, int64_t tbs, uint8_t* mapped, cudaStream_t st) {
  if (n <= 0) return;
  const int lo = align_round_bound(pb.round, rounds), hi = align_round_bound(pb.round + 1, rounds);
  replay_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n, sp, ref_id, sense, pb, lo, hi, hits, tb, tbs, mapped);
}

// ------------------------------------------------------------------------------ rounds

__device__ __forceinline__ int round_of_rank(int rank, int rounds) {
  int k = 0;
  while (k + 1 < rounds && rank >= align_round_bound(k + 1, rounds)) ++k;
  return k;
}

// per round: slots whose rank falls in it (one atomic per warp and round)
__global__ void round_count_kernel(int64_t npass, const int64_t* __restrict__ npass_dev, int rounds,
                                   const int32_t* __restrict__ p_read, const int32_t* __restrict__ pstart,
                                   int64_t* __restrict__ count) {
  if (npass_dev) npass = *npass_dev;
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < npass; base += stride) {
    const int64_t s = base + lane;
    const int k = s < npass ? round_of_rank((int)(s - pstart[p_read[s]]), rounds) : -1;
    for (int j = 0; j < rounds; ++j) {
      const unsigned m = __ballot_sync(0xffffffffu, k == j);
      if (m && lane == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&count[j]), (unsigned long long)__popc(m));
    }
  }
}

// the lists: a warp's slots of one round go out together, in slot order
__global__ void round_scatter_kernel(int64_t npass, const int64_t* __restrict__ npass_dev, int rounds,
                                     const int32_t* __restrict__ p_read, const int32_t* __restrict__ pstart,
                                     const int64_t* __restrict__ count, unsigned long long* __restrict__ cursors,
                                     int32_t* __restrict__ slots) {
  if (npass_dev) npass = *npass_dev;
  const int lane = threadIdx.x & 31;
  int64_t start[kMaxAlignRounds];
  int64_t acc = 0;
  for (int j = 0; j < kMaxAlignRounds; ++j) {
    start[j] = acc;
    if (j < rounds) acc += count[j];
  }
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < npass; base += stride) {
    const int64_t s = base + lane;
    const int k = s < npass ? round_of_rank((int)(s - pstart[p_read[s]]), rounds) : -1;
    for (int j = 0; j < rounds; ++j) {
      const unsigned m = __ballot_sync(0xffffffffu, k == j);
      if (!m) continue;
      unsigned long long b = 0;
      if (lane == 0) b = atomicAdd(&cursors[j], (unsigned long long)__popc(m));
      b = __shfl_sync(0xffffffffu, b, 0);
      if (k == j) slots[start[j] + (int64_t)b + __popc(m & ((1u << lane) - 1u))] = (int32_t)s;
    }
  }
}

void launch_round_lists(int64_t npass, const int64_t* npass_dev, int rounds, const int32_t* p_read,
                        const int32_t* pstart, int64_t* round_count, unsigned long long* cursors, int32_t* round_slots,
                        cudaStream_t st) {
  if (npass <= 0) return;
  int64_t blocks = (npass + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  round_count_kernel<<<(unsigned)blocks, 256, 0, st>>>(npass, npass_dev, rounds, p_read, pstart, round_count);
  round_scatter_kernel<<<(unsigned)blocks, 256, 0, st>>>(npass, npass_dev, rounds, p_read, pstart, round_count,
                                                         cursors, round_slots);
}

}  // namespace sg
