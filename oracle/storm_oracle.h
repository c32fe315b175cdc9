/*
 * storm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C, single-threaded restatement of the reference mapper's hot path (SToRM,
 * laurentnoe/storm), used by tests/ and by bench.py's CPU-baseline leg as the checker of
 * the CUDA path.  Nothing in the product links, loads or calls this code.  Each function
 * cites the reference file:line it restates.  Parity of this oracle is pinned against the
 * reference itself, compiled from its own sources into oracle/_ref (see oracle/Makefile),
 * by the known-answer tests in tests/test_oracle_pin.py.
 */
#ifndef STORM_ORACLE_H
#define STORM_ORACLE_H

#include <stdint.h>
#include "../include/stormgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_seed {
  int weight;                 /* number of '#' */
  int span;                   /* pattern length */
  uint8_t care[STORMGPU_MAX_SPAN];
  int n_positions;            /* 0: every read position */
  int positions[256];
} or_seed;

/* seed.c:97-135 + seed.c:25-88.  Returns the number of seeds, or -1 if invalid. */
int or_parse_seeds(const char *list, or_seed *out, int max_seeds);

/* seed.c:203-213 */
uint32_t or_seed_key(const or_seed *s, const uint8_t *packed, int64_t pos);

/* index.c:19-195.  first must hold 4^w + 1 ints; map_capacity >= n_codes.  Returns the
 * number of positions in map (first[4^w]), or -1. */
int64_t or_index_build(const or_seed *s, int stdev_distance, const uint8_t *codes,
                       int64_t n_codes, const int32_t *rs, const int32_t *re, int nreg,
                       int32_t *first, int32_t *map, int64_t map_capacity);

/* run.c:577-698 (heap merge of the CSR lists, accept rule of run.c:617 and :648):
 * ascending accepted diagonals of one read-strand.  Returns the count (<= cap). */
int64_t or_candidates(const or_seed *seeds, int nseeds, const int32_t *const *first,
                      const int32_t *const *map, const uint8_t *read, int L, int I,
                      int32_t *out, int64_t cap);

/* alignment_simd.c:2282-3404 (AVX2 family; identical semantics for every ISA). */
int or_sw_filter(int W, int L, uint32_t match, uint32_t mismatch, uint32_t gapopen,
                 uint32_t gapext, uint32_t threshold, const uint8_t *genome, int64_t pos,
                 const uint8_t *read);

/* alignment.c:255-285, :326-360, :488-632, :642-734.  Window = codes [win, win+L+2I). */
typedef struct or_align_out {
  int32_t score;              /* best score on the last row (no abort) */
  int32_t bound;              /* min over rows 1..L-1 of max_on_line + best_possible */
  int16_t best_i, best_j, best_i0, best_j0;
  int32_t tb_len;
  uint8_t tb[(STORMGPU_MAX_READ_LEN + STORMGPU_MAX_INDELS + 2) / 2];  /* end-to-start */
} or_align_out;

void or_align(const stormgpu_params *p, const uint8_t *read_packed, const uint8_t *levels_packed,
              int L, const uint8_t *genome, const uint8_t *mask, int64_t win, or_align_out *o);

/* hit_map.c:50-144 on one read's four slots (tb slots of tb_stride bytes). */
int or_hitmap_update(stormgpu_hit *slots, uint8_t *tb, int64_t tb_stride, uint8_t *mapped,
                     int ref_id, int ref_pos, const or_align_out *a, int sense);

/* Whole mapping (run.c:764-994 with process_read run.c:555-747), single thread.
 * refs: packed codes / masks with >= `pad` readable codes around each sequence. */
typedef struct or_ref {
  const uint8_t *codes;
  const uint8_t *mask;
  int64_t n_codes;
  const int32_t *rs, *re;
  int nreg;
} or_ref;

int or_map(const stormgpu_params *p, const char *seeds, const or_ref *refs, int nrefs,
           const stormgpu_reads *reads, stormgpu_results *out, int64_t *counters);

/* reads_data.c:9-35 (read__reverse): reversed read codes and levels. */
void or_reverse_read(int colour, const uint8_t *codes, const uint8_t *levels, int L,
                     uint8_t first_level, uint8_t *rcodes, uint8_t *rlevels);

#ifdef __cplusplus
}
#endif
#endif
