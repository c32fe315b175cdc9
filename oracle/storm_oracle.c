/*
 * storm_oracle.c -- TEST INFRASTRUCTURE ONLY: single-threaded C restatement of the
 * reference mapper's hot path, the checker of the CUDA path.  See storm_oracle.h.
 * Every function states the reference lines it follows (file:line within laurentnoe/storm).
 */
#include "storm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MINS STORMGPU_MIN_SCORE

/* code n of a packed sequence; n may be negative when the buffer is padded before code 0
 * (codes.h:122-130: byte n>>2, bits 2*(n&3)) */
static inline int code_at(const uint8_t *p, int64_t n) {
  return (p[n >> 2] >> ((n & 3) << 1)) & 3;
}

/* ------------------------------------------------------------------------------ seeds */

/* seed.c:25-88 (seed__create): '#'/'1' care, '-'/'0' don't care, optional ":p1 p2,p3" */
static int parse_one_seed(const char *pat, or_seed *s) {
  memset(s, 0, sizeof(*s));
  const char *colon = strchr(pat, ':');
  int len = colon ? (int)(colon - pat) : (int)strlen(pat);
  if (len <= 0 || len > STORMGPU_MAX_SPAN) return -1;
  for (int i = 0; i < len; ++i) {
    char c = pat[i];
    if (c == '#' || c == '1') { s->care[i] = 1; s->weight++; }
    else if (c == '-' || c == '0') s->care[i] = 0;
    else return -1;
  }
  if (s->weight == 0 || s->weight > 15) return -1;
  s->span = len;
  if (colon && strlen(colon) > 1) {
    int v;
    if (sscanf(colon + 1, "%d", &v) == 1) {
      /* tokens separated by ' ' or ',', parsed until the first non-number (seed.c:78-84) */
      char buf[4096];
      strncpy(buf, colon + 1, sizeof(buf) - 1);
      buf[sizeof(buf) - 1] = 0;
      char *save = NULL;
      for (char *tok = strtok_r(buf, ", ", &save); tok; tok = strtok_r(NULL, ", ", &save)) {
        if (sscanf(tok, "%d", &v) != 1 || s->n_positions >= 256) break;
        s->positions[s->n_positions++] = v;
      }
    }
  }
  return 0;
}

/* seed.c:97-135 (seed__parse_list): ';'-separated, empty tokens skipped */
int or_parse_seeds(const char *list, or_seed *out, int max_seeds) {
  char buf[8192];
  if (!list || !*list) return 0;
  strncpy(buf, list, sizeof(buf) - 1);
  buf[sizeof(buf) - 1] = 0;
  int n = 0;
  char *save = NULL;
  for (char *tok = strtok_r(buf, ";", &save); tok; tok = strtok_r(NULL, ";", &save)) {
    if (n >= max_seeds) return -1;
    if (parse_one_seed(tok, &out[n]) != 0) return -1;
    n++;
  }
  return n;
}

/* seed.c:203-213: key = 2-bit codes at the '#' offsets, first offset most significant */
uint32_t or_seed_key(const or_seed *s, const uint8_t *packed, int64_t pos) {
  uint32_t key = 0;
  for (int i = 0; i < s->span; ++i)
    if (s->care[i]) key = (key << 2) | (uint32_t)code_at(packed, pos + i);
  return key;
}

/* ------------------------------------------------------------------------------ index */

/* index.c:19-195.  Positions are visited in increasing order; a window is skipped while
 * i + span >= start of the next masked region, jumping to end-1 of that region, and the
 * position reached by the jump is indexed without re-checking the loop bound (the `continue`
 * at index.c:534 continues the inner while, not the for).  Keys whose count c satisfies
 * c - avg > l * sd are erased (index.c:117-155, avg and sd as written there).  The CSR is
 * first[k] = number of kept positions with key < k, positions ascending (index.c:161-188). */
int64_t or_index_build(const or_seed *s, int stdev_distance, const uint8_t *codes,
                       int64_t n_codes, const int32_t *rs, const int32_t *re, int nreg,
                       int32_t *first, int32_t *map, int64_t map_capacity) {
  int64_t index_size = (int64_t)1 << (2 * s->weight);
  int64_t map_size = n_codes - s->span + 1;
  for (int64_t k = 0; k <= index_size; ++k) first[k] = 0;
  if (map_size <= 0) return 0;
  int32_t *counts = calloc((size_t)index_size, sizeof(int32_t));
  int64_t *pos_list = malloc(sizeof(int64_t) * (size_t)(map_size + nreg + 1));
  uint32_t *key_list = malloc(sizeof(uint32_t) * (size_t)(map_size + nreg + 1));
  int64_t count = 0;
  if (s->span < n_codes) {
    int r = 0;
    for (int64_t i = 0; i < map_size; ++i) {
      while (r < nreg && i + s->span >= rs[r]) {
        i = re[r] - 1;
        r++;
      }
      uint32_t key = or_seed_key(s, codes, i);
      counts[key]++;
      pos_list[count] = i;
      key_list[count] = key;
      count++;
    }
  }
  uint8_t *erased = calloc((size_t)index_size, 1);
  if (stdev_distance > 0 && count > 0) {
    /* index.c:117-155 computes avg = sum(c^2)/count^2 and sd = sqrt(sum_{c>0}(c-avg)^2/count)
     * in double; here both come from the exact integer moments, in long double, which
     * agrees with the reference except on exact ties of c - avg against l*sd. */
    int64_t s2 = 0, nocc = 0;
    for (int64_t k = 0; k < index_size; ++k)
      if (counts[k] > 0) { s2 += (int64_t)counts[k] * counts[k]; nocc++; }
    long double n = (long double)count;
    long double avg = (long double)s2 / n / n;
    long double var = ((long double)s2 - 2.0L * avg * n + (long double)nocc * avg * avg) / n;
    long double sd = sqrtl(var > 0 ? var : 0);
    for (int64_t k = 0; k < index_size; ++k)
      if (counts[k] && ((long double)counts[k] - avg) > (long double)stdev_distance * sd) erased[k] = 1;
  }
  int64_t acc = 0;
  for (int64_t k = 0; k < index_size; ++k) {
    first[k] = (int32_t)acc;
    if (!erased[k]) acc += counts[k];
  }
  first[index_size] = (int32_t)acc;
  if (acc > map_capacity) { acc = -1; goto out; }
  {
    int64_t *cur = malloc(sizeof(int64_t) * (size_t)index_size);
    for (int64_t k = 0; k < index_size; ++k) cur[k] = first[k];
    for (int64_t t = 0; t < count; ++t) {
      uint32_t k = key_list[t];
      if (!erased[k]) map[cur[k]++] = (int32_t)pos_list[t];
    }
    free(cur);
  }
out:
  free(counts);
  free(pos_list);
  free(key_list);
  free(erased);
  return acc;
}

/* --------------------------------------------------------------------------- candidates */

static int cmp_i32(const void *a, const void *b) {
  int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

/* run.c:577-698: every (seed, read position) contributes its whole CSR list shifted by the
 * read position; the heap pops them in ascending order; a popped diagonal is kept iff it is
 * strictly greater than the previously popped one, the "previous" starting at -I
 * (run.c:617, :648, :697).  Codes beyond the read's end read as 0. */
int64_t or_candidates(const or_seed *seeds, int nseeds, const int32_t *const *first,
                      const int32_t *const *map, const uint8_t *read, int L, int I,
                      int32_t *out, int64_t cap) {
  int64_t n = 0, alloc = 1024;
  int32_t *all = malloc(sizeof(int32_t) * (size_t)alloc);
  uint8_t padded[(STORMGPU_MAX_READ_LEN + STORMGPU_MAX_SPAN + 256) / 4 + 16];
  memset(padded, 0, sizeof(padded));
  memcpy(padded, read, (size_t)((L + 3) / 4));
  if (L & 3) padded[L >> 2] &= (uint8_t)((1u << (2 * (L & 3))) - 1);
  for (int si = 0; si < nseeds; ++si) {
    const or_seed *s = &seeds[si];
    int np = s->n_positions ? s->n_positions : (L - s->span + 1);
    for (int t = 0; t < np; ++t) {
      int rp = s->n_positions ? s->positions[t] : t;
      if (rp < 0 || rp >= L) continue;
      uint32_t key = or_seed_key(s, padded, rp);
      for (int32_t a = first[si][key]; a < first[si][key + 1]; ++a) {
        if (n == alloc) { alloc *= 2; all = realloc(all, sizeof(int32_t) * (size_t)alloc); }
        all[n++] = map[si][a] - rp;
      }
    }
  }
  qsort(all, (size_t)n, sizeof(int32_t), cmp_i32);
  int64_t m = 0;
  int32_t prev = -I;
  for (int64_t t = 0; t < n; ++t) {
    if (all[t] > prev) {
      if (m < cap) out[m] = all[t];
      m++;
    }
    prev = all[t];
  }
  free(all);
  return m;
}

/* ------------------------------------------------------------------------------ filter */

/* Mask table of alignment_avx2__setlength_* (alignment_simd.c:2282-2507), one W-byte lane
 * group as a bit set (bit k = byte k): step 0 keeps only byte W-1; at even steps l <= 2(W-1)
 * the next lower byte is added; at even steps l >= prlength - 2(W-1) the group is shifted
 * down one byte.  prlength = 2(L + W - 1). */
static void filter_masks(int W, int L, uint32_t *m, int prlength) {
  uint32_t full = (W == 32) ? 0xffffffffu : ((1u << W) - 1);
  m[0] = 1u << (W - 1);
  for (int l = 1; l < prlength; ++l) {
    m[l] = m[l - 1];
    if (!(l & 1)) {
      if (l >= prlength - (W - 1) * 2) m[l] = (m[l] >> 1) & full;
      else if (l <= (W - 1) * 2) m[l] = m[l - 1] | ((m[l] >> 1) & full);
    }
  }
}

static inline int sat_u8(int x) { return x < 0 ? 0 : (x > 255 ? 255 : x); }

/* alignment_avx2__align_{pair,quad,octa,hexa} (alignment_simd.c:2613-3404).  One hit is a
 * group of W byte cells.  Before the loop the genome register holds codes 0..W-1 of the
 * window (byte k = code W-1-k); at odd steps one more genome code enters byte 0 (the others
 * move up a byte), at even steps one more read code enters byte W-1 (the others move down).
 * Per step, per byte: M = subs(adds(M[l-2], match if equal), mismatch if different);
 * I = max(subs(max(I[l-1], I[l-1] moved), ext), subs(max(M[l-1], M[l-1] moved), open)),
 * "moved" = the neighbour byte (from below at odd steps, from above at even steps, zero at
 * the group edge); M = max(M, I) & mask[l]; Max = max(Max, M).  Pass iff Max > thr. */
int or_sw_filter(int W, int L, uint32_t match, uint32_t mismatch, uint32_t gapopen,
                 uint32_t gapext, uint32_t threshold, const uint8_t *genome, int64_t pos,
                 const uint8_t *read) {
  int ma = match & 0xff, mi = mismatch & 0xff, go = gapopen & 0xff, ge = gapext & 0xff;
  int thr = threshold >= 255 ? 254 : (int)threshold;
  int prlength = 2 * (L + W - 1);
  uint32_t *mask = malloc(sizeof(uint32_t) * (size_t)prlength);
  filter_masks(W, L, mask, prlength);
  int A[32] = {0}, B[32] = {0}, M1[32] = {0}, M2[32] = {0}, I1[32] = {0}, Max = 0;
  int64_t g = pos;                 /* next genome code */
  int r = 0;                       /* next read code */
  for (int d = 0; d < W; ++d) {    /* init: B = codes 0..W-1, byte k = code W-1-k */
    for (int k = W - 1; k > 0; --k) B[k] = B[k - 1];
    B[0] = code_at(genome, g++);
  }
  for (int l = 0; l < prlength; ++l) {
    if (l & 1) {
      for (int k = W - 1; k > 0; --k) B[k] = B[k - 1];
      B[0] = code_at(genome, g++);
    } else {
      for (int k = 0; k < W - 1; ++k) A[k] = A[k + 1];
      A[W - 1] = code_at(read, r++);
    }
    int M[32], I[32];
    for (int k = 0; k < W; ++k) {
      int eq = A[k] == B[k];
      M[k] = sat_u8(sat_u8(M2[k] + (eq ? ma : 0)) - (eq ? 0 : mi));
      int Im, Mm;
      if (l & 1) {
        int Is = k > 0 ? I1[k - 1] : 0, Ms = k > 0 ? M1[k - 1] : 0;
        Im = I1[k] > Is ? I1[k] : Is;
        Mm = M1[k] > Ms ? M1[k] : Ms;
      } else {
        int Is = k < W - 1 ? I1[k + 1] : 0, Ms = k < W - 1 ? M1[k + 1] : 0;
        Im = I1[k] > Is ? I1[k] : Is;
        Mm = M1[k] > Ms ? M1[k] : Ms;
      }
      int i1 = sat_u8(Im - ge), i2 = sat_u8(Mm - go);
      I[k] = i1 > i2 ? i1 : i2;
      if (I[k] > M[k]) M[k] = I[k];
      if (!((mask[l] >> k) & 1)) M[k] = 0;
      if (M[k] > Max) Max = M[k];
    }
    for (int k = 0; k < W; ++k) { M2[k] = M1[k]; M1[k] = M[k]; I1[k] = I[k]; }
  }
  free(mask);
  return Max > thr;
}

/* ------------------------------------------------------------------------------ DP */

typedef struct cellt {
  int score;
  int from;          /* bit1: from top (I_MASK), bit0: from left (J_MASK); 3 = corner */
  int indels;
  int chk, ac, fr;   /* colour checksum, auto-correct code, mismatch freshness */
} cellt;

/* SCALE_SCORE (alignment.h:30) */
static int scale_score(int s, int lvl) { return (int)(((s) * (lvl + 1) + 0.) / 4); }

/* alignment.c:465-468 */
static int colour_adjust(int prev, int crt, int ref, int s) {
  return (prev && (((prev ^ crt) == 0) || ((prev ^ crt) == ref)) && s != MINS && s < 0) ? -2 * s : s;
}

/* alignment.c:326-360 (init), :488-632 (DP), :642-734 (traceback).  Rows i = read codes,
 * row i covers window codes i..i+2I; corner (i-1, c), top (i-1, c+1), left (i, c-1) in band
 * coordinates c = j - i; the band edges are MIN_SCORE cells with indels = I. */
void or_align(const stormgpu_params *p, const uint8_t *read_packed, const uint8_t *levels_packed,
              int L, const uint8_t *genome, const uint8_t *mask, int64_t win, or_align_out *o) {
  const int I = p->allowed_indels, BW = 2 * I + 1, colour = p->colour;
  int pair[2][4];
  for (int l = 0; l < 4; ++l) {
    pair[0][l] = scale_score(p->match, l);
    pair[1][l] = scale_score(p->mismatch, l);
  }
  const int gap_open = p->gap_open, gap_ext = p->gap_extend;
  int *rd = malloc(sizeof(int) * (size_t)L), *q = malloc(sizeof(int) * (size_t)L);
  int RL = L + 2 * I;
  int *rf = malloc(sizeof(int) * (size_t)RL), *mk = malloc(sizeof(int) * (size_t)RL);
  for (int i = 0; i < L; ++i) {
    rd[i] = code_at(read_packed, i);
    q[i] = levels_packed ? code_at(levels_packed, i) : 3;
  }
  for (int j = 0; j < RL; ++j) {
    rf[j] = code_at(genome, win + j);
    mk[j] = code_at(mask, win + j);
  }
  cellt *m = malloc(sizeof(cellt) * (size_t)L * (size_t)BW);
#define C(i, c) m[(size_t)(i) * BW + (c)]
  for (int k = 0; k < L; ++k)
    for (int c = 0; c < BW; ++c) {
      int j = k + c;
      cellt *x = &C(k, c);
      if (mk[j] == 0) {
        if (colour) {
          x->ac = x->chk = rd[k] ^ rf[j];
          x->fr = x->ac ? q[k] : 0;
          x->score = pair[x->chk ? 1 : 0][q[k]];
        } else {
          x->chk = x->ac = x->fr = 0;
          x->score = pair[rd[k] != rf[j]][q[k]];
        }
      } else {
        x->chk = x->ac = x->fr = 0;
        x->score = MINS;
      }
      x->from = 3;
      x->indels = 0;
    }
  cellt border = {MINS, 3, I, 0, 0, 0};
  int best_possible = (colour ? (L - 2) : L) * pair[0][3];
  long bound = 0x7fffffff;
  for (int i = 1; i < L; ++i) {
    int max_on_line = MINS;
    for (int c = 0; c < BW; ++c) {
      int j = i + c;
      cellt *crt = &C(i, c);
      const cellt *corner = &C(i - 1, c);
      const cellt *top = (c + 1 < BW) ? &C(i - 1, c + 1) : &border;
      const cellt *left = (c > 0) ? &C(i, c - 1) : &border;
      int ms = colour ? colour_adjust(corner->chk, crt->chk, corner->ac, crt->score) : crt->score;
      int score = corner->score + ms;
      int it = 0, tmp;
      if (top->indels < I && (tmp = top->score + ((top->from ^ 2) ? gap_open : gap_ext)) > score) {
        it = 1;
        score = tmp;
      }
      if (left->indels < I && (tmp = left->score + ((left->from ^ 1) ? gap_open : gap_ext)) > score) {
        it = 2;
        score = tmp;
      }
      crt->score = score;
      if (it == 0) {
        crt->indels = corner->indels;
        if (colour) {
          int chk = crt->chk ^ corner->chk;
          crt->chk = chk;
          if (corner->chk != chk) {
            if (corner->chk == 0) {
              crt->ac = chk;
              crt->fr = q[i];
            } else if (chk == corner->ac) {
              crt->ac = 0; crt->chk = 0; crt->fr = 0;
            } else if (chk == 0) {
              if (corner->fr - 1 > 0) { crt->ac = corner->ac; crt->fr = corner->fr - 1; }
              else { crt->ac = 0; crt->fr = 0; }
            } else {
              if (corner->fr - 1 > 0) { crt->ac = corner->ac; crt->fr = corner->fr - 1; }
              else { crt->ac = chk; crt->fr = q[i]; }
            }
          } else {
            if (corner->ac != 0) {
              if (corner->fr - 1 > 0) {
                if (chk == 0) { crt->ac = 0; crt->fr = 0; }
                else { crt->ac = corner->ac; crt->fr = corner->fr - 1; }
              }
            } else {
              crt->chk = 0; crt->ac = 0; crt->fr = 0;
            }
          }
        }
      } else if (it == 1) {
        crt->from = 2;
        crt->indels = top->indels + 1;
        if (colour) {
          crt->chk = top->chk ^ rd[i];
          if (top->fr - 1 > 0) { crt->fr = top->fr - 1; crt->ac = corner->ac; }
        }
      } else {
        crt->from = 1;
        crt->indels = left->indels + 1;
        if (colour) {
          crt->chk = left->chk ^ rf[j];
          if (left->fr - 1 > 0) { crt->fr = left->fr - 1; crt->ac = corner->ac; }
        }
      }
      if (max_on_line < crt->score) max_on_line = crt->score;
    }
    if ((long)max_on_line + best_possible < bound) bound = (long)max_on_line + best_possible;
    best_possible -= pair[0][3];
  }
  int best = MINS, bi = -1, bj = -1;
  for (int c = 0; c < BW; ++c)
    if (best < C(L - 1, c).score) { best = C(L - 1, c).score; bi = L - 1; bj = L - 1 + c; }
  o->score = best;
  o->bound = bound > 0x7fffffffL ? 0x7fffffff : (int32_t)bound;
  o->best_i = (int16_t)bi;
  o->best_j = (int16_t)bj;
  o->best_i0 = (int16_t)bi;
  o->best_j0 = (int16_t)bj;
  o->tb_len = 0;
  memset(o->tb, 0, sizeof(o->tb));
  if (bi >= 0) {
    int i = bi, j = bj, colr = 0;
    while (i >= 0 && i < L && j >= i && j <= i + 2 * I) {
      const cellt *x = &C(i, j - i);
      o->best_i0 = (int16_t)i;
      o->best_j0 = (int16_t)j;
      int di = (x->from & 2) ? -1 : 0, dj = (x->from & 1) ? -1 : 0, op;
      if (di && !dj) op = 0xC | rd[i];
      else if (dj && !di) op = 0x1;
      else if (rd[i] != rf[j]) {
        if (!colour) op = 0x4 | rd[i];
        else if (colr || (i != 0 && j != 0 && x->score > C(i - 1, j - i).score)) {
          op = 0x8 | rd[i];
          colr ^= rd[i] ^ rf[j];
        } else op = 0x4 | rd[i];
      } else op = 0x3;
      int t = o->tb_len++;
      if (t & 1) o->tb[t >> 1] = (uint8_t)((o->tb[t >> 1] & 0xF0) | op);
      else o->tb[t >> 1] = (uint8_t)((o->tb[t >> 1] & 0x0F) | (op << 4));
      i += di;
      j += dj;
    }
  }
#undef C
  free(m); free(rd); free(q); free(rf); free(mk);
}

/* ------------------------------------------------------------------------------ top-4 */

static inline int tb_get(const uint8_t *t, int i) { return (t[i >> 1] >> ((i & 1) ? 0 : 4)) & 0xF; }
static inline void tb_set(uint8_t *t, int i, int v) {
  if (i & 1) t[i >> 1] = (uint8_t)((t[i >> 1] & 0xF0) | (v & 0xF));
  else t[i >> 1] = (uint8_t)((t[i >> 1] & 0x0F) | ((v << 4) & 0xF0));
}

/* hit_map.c:50-144: dedupe on equal (ref, start, read_start) or (ref, end, read_end), keep
 * the four best by strict '>', insert below equal scores, traceback stored reversed. */
int or_hitmap_update(stormgpu_hit *slot, uint8_t *tb, int64_t tb_stride, uint8_t *mapped,
                     int ref_id, int ref_pos, const or_align_out *a, int sense) {
  if (!*mapped) {
    for (int k = 0; k < 4; ++k) {
      memset(&slot[k], 0, sizeof(slot[k]));
      slot[k].score = MINS;
      slot[k].ref_id = slot[k].ref_start = slot[k].ref_end = -1;
      slot[k].read_start = slot[k].read_end = -1;
    }
    *mapped = 1;
  }
  int score = a->score;
  int k;
  for (k = 0; k < 4 && slot[k].ref_id != -1; ++k) {
    if (slot[k].ref_id == ref_id &&
        ((slot[k].ref_start == ref_pos + a->best_j0 && slot[k].read_start == a->best_i0) ||
         (slot[k].ref_end == ref_pos + a->best_j && slot[k].read_end == a->best_i))) {
      if (score > slot[k].score) break;
      return -1;
    }
  }
  if (k == 4) k--;
  int i = k;
  while (i >= 0 && score > slot[i].score) i--;
  if (i == 3) return -1;
  /* the tb buffer of slot k is the one freed (hit_map.c:116-119); keep buffers with slots */
  uint8_t *keep = malloc((size_t)tb_stride);
  memcpy(keep, tb + (size_t)k * tb_stride, (size_t)tb_stride);
  for (int j = k; j > i + 1; --j) {
    slot[j] = slot[j - 1];
    memcpy(tb + (size_t)j * tb_stride, tb + (size_t)(j - 1) * tb_stride, (size_t)tb_stride);
  }
  free(keep);
  stormgpu_hit *h = &slot[i + 1];
  h->score = score;
  h->ref_id = ref_id;
  h->ref_start = ref_pos + a->best_j0;
  h->ref_end = ref_pos + a->best_j;
  h->read_start = a->best_i0;
  h->read_end = a->best_i;
  h->sense = sense;
  h->tb_len = a->tb_len;
  uint8_t *t = tb + (size_t)(i + 1) * tb_stride;
  memset(t, 0, (size_t)tb_stride);
  for (int p = 0; p < a->tb_len; ++p) tb_set(t, p, tb_get(a->tb, a->tb_len - 1 - p));
  return i + 1;
}

/* ------------------------------------------------------------------------------ reads */

/* reads_data.c:9-35, codes.c:429-439, read_quality.c:226-243 */
void or_reverse_read(int colour, const uint8_t *codes, const uint8_t *levels, int L,
                     uint8_t first_level, uint8_t *rcodes, uint8_t *rlevels) {
  memset(rcodes, 0, (size_t)(L + 3) / 4);
  for (int i = 0; i < L; ++i) {
    int c = code_at(codes, i);
    int v = colour ? c : (3 - c);
    rcodes[(L - 1 - i) >> 2] |= (uint8_t)(v << (((L - 1 - i) & 3) << 1));
  }
  if (levels && rlevels) {
    memset(rlevels, 0, (size_t)(L + 3) / 4);
    if (!colour) {
      for (int i = 0; i < L; ++i)
        rlevels[i >> 2] |= (uint8_t)(code_at(levels, L - 1 - i) << ((i & 3) << 1));
    } else {
      rlevels[(L - 1) >> 2] |= (uint8_t)((first_level & 3) << (((L - 1) & 3) << 1));
      for (int i = 0; i < L - 1; ++i)
        rlevels[i >> 2] |= (uint8_t)(code_at(levels, L - 2 - i) << ((i & 3) << 1));
    }
  }
}

/* ------------------------------------------------------------------------------ mapping */

static int filter_width(int is) { return is <= 1 ? 2 : is <= 3 ? 4 : is <= 7 ? 8 : 16; }

/* run.c:764-994 + run.c:555-747 */
int or_map(const stormgpu_params *p, const char *seeds_str, const or_ref *refs, int nrefs,
           const stormgpu_reads *reads, stormgpu_results *out, int64_t *counters) {
  or_seed seeds[STORMGPU_MAX_SEEDS];
  int ns = or_parse_seeds(seeds_str, seeds, STORMGPU_MAX_SEEDS);
  if (ns <= 0) return STORMGPU_EINVAL;
  const int I = p->allowed_indels, Is = I < 15 ? I : 15, W = filter_width(Is);
  const uint32_t fm = (uint32_t)abs(p->match), fx = (uint32_t)abs(p->mismatch);
  const uint32_t fo = (uint32_t)abs(p->gap_open), fe = (uint32_t)abs(p->gap_extend);
  const uint32_t fz = (uint32_t)p->min_score_filter;
  memset(out->mapped, 0, (size_t)reads->n);
  for (int64_t r = 0; r < reads->n; ++r)
    for (int k = 0; k < 4; ++k) {
      stormgpu_hit *h = &out->hits[r * 4 + k];
      memset(h, 0, sizeof(*h));
      h->score = MINS;
      h->ref_id = h->ref_start = h->ref_end = -1;
      h->read_start = h->read_end = -1;
    }
  memset(out->tb, 0, (size_t)(reads->n * 4 * out->tb_stride));
  int64_t cnt_cand = 0, cnt_pass = 0, cnt_align = 0;
  int64_t cap = 1 << 20;
  int32_t *cand = malloc(sizeof(int32_t) * (size_t)cap);
  uint8_t rc[STORMGPU_MAX_READ_LEN / 4 + 16], rl[STORMGPU_MAX_READ_LEN / 4 + 16];
  for (int ref_id = 0; ref_id < nrefs; ++ref_id) {
    const or_ref *R = &refs[ref_id];
    int32_t *first[STORMGPU_MAX_SEEDS], *map[STORMGPU_MAX_SEEDS];
    for (int si = 0; si < ns; ++si) {
      first[si] = malloc(sizeof(int32_t) * (((size_t)1 << (2 * seeds[si].weight)) + 1));
      map[si] = malloc(sizeof(int32_t) * (size_t)(R->n_codes + R->nreg + 1));
      or_index_build(&seeds[si], p->stdev_distance, R->codes, R->n_codes, R->rs, R->re, R->nreg,
                     first[si], map[si], R->n_codes + R->nreg + 1);
    }
    for (int strand = 0; strand < 2; ++strand) {
      if (!(p->senses & (1 << strand))) continue;
      for (int64_t r = 0; r < reads->n; ++r) {
        int L = reads->lengths[r];
        const uint8_t *codes = reads->codes + r * reads->code_stride;
        const uint8_t *levels = reads->levels ? reads->levels + r * reads->level_stride : NULL;
        if (strand == 1) {
          uint8_t fl = reads->first_levels ? reads->first_levels[r] : 3;
          or_reverse_read(p->colour, codes, levels, L, fl, rc, levels ? rl : NULL);
          codes = rc;
          levels = levels ? rl : NULL;
        }
        int64_t nc;
        for (;;) {
          nc = or_candidates(seeds, ns, (const int32_t *const *)first, (const int32_t *const *)map,
                             codes, L, I, cand, cap);
          if (nc <= cap) break;
          cap = nc;
          cand = realloc(cand, sizeof(int32_t) * (size_t)cap);
        }
        cnt_cand += nc;
        int T = p->min_score;
        stormgpu_hit *slots = &out->hits[r * 4];
        uint8_t *tb = out->tb + (size_t)r * 4 * out->tb_stride;
        for (int64_t t = 0; t < nc; ++t) {
          int d = cand[t];
          if (!or_sw_filter(W, L, fm, fx, fo, fe, fz, R->codes, (int64_t)d - Is, codes)) continue;
          cnt_pass++;
          int win = d - I > -Is ? d - I : -Is;
          or_align_out a;
          or_align(p, codes, levels, L, R->codes, R->mask, win, &a);
          cnt_align++;
          int aborted = a.bound < T;
          int ret = aborted ? MINS : a.score;
          if (ret > T) {
            or_hitmap_update(slots, tb, out->tb_stride, &out->mapped[r], ref_id, win, &a,
                             strand ? -1 : 1);
            if (slots[3].score > T) T = slots[3].score;
          }
        }
      }
    }
    for (int si = 0; si < ns; ++si) { free(first[si]); free(map[si]); }
  }
  free(cand);
  if (counters) { counters[0] = cnt_cand; counters[1] = cnt_pass; counters[2] = cnt_align; }
  return 0;
}
