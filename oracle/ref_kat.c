/* Test infrastructure: flat entry points over single functions of the reference mapper,
 * compiled together with the reference's own sources (read in place, see oracle/Makefile)
 * into oracle/_ref/libref_{nuc,col}.so, so that known-answer tests can compare the oracle
 * and the CUDA kernels with the reference function by function.  This file only calls the
 * reference's public functions; it contains none of their logic. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "alignment.h"
#include "alignment_simd.h"
#include "index.h"
#include "seed.h"
#include "reference_data.h"

extern int FILTER_REPEATS;
extern int ACCEPTED_STDEV_DISTANCE;
extern int VERBOSITY;

/* SIMD filter: init + one align call on W-byte groups (alignment_simd.c AVX2 family).
 * pos has 32/W entries (one per hit of the call).  Returns the pass bitmask. */
unsigned kat_filter(int W, unsigned match, unsigned mismatch, unsigned gapopen, unsigned gapext,
                    unsigned threshold, unsigned readlength, unsigned char *genome, int *pos,
                    unsigned char *read) {
  VERBOSITY = 0;
  unsigned r = 0;
  switch (W) {
  case 2:
    alignment_avx2__init_hexa(match, mismatch, gapopen, gapext, threshold, readlength);
    r = alignment_avx2__align_hexa(genome, pos, read);
    break;
  case 4:
    alignment_avx2__init_octa(match, mismatch, gapopen, gapext, threshold, readlength);
    r = alignment_avx2__align_octa(genome, pos, read);
    break;
  case 8:
    alignment_avx2__init_quad(match, mismatch, gapopen, gapext, threshold, readlength);
    r = alignment_avx2__align_quad(genome, pos, read);
    break;
  case 16:
    alignment_avx2__init_pair(match, mismatch, gapopen, gapext, threshold, readlength);
    r = alignment_avx2__align_pair(genome, pos, read);
    break;
  }
  alignment_avx2__clean();
  return r;
}

/* Full alignment (alignment.c:488-632) then traceback (alignment.c:642-734) of one read
 * against the window of ref_len = L + 2I codes starting at `offset`.  out[0..5] = returned
 * score, best_i, best_j, best_i0, best_j0, traceback length; tb receives the raw traceback. */
void kat_align(int L, int I, int match, int mismatch, int gap_open, int gap_extend,
               unsigned char *read, unsigned char *quality, unsigned char *ref,
               unsigned char *ref_masked, int offset, int threshold, int *out, unsigned char *tb) {
  VERBOSITY = 0;
  AlignmentType al;
  alignment__init(&al, (short)L, (short)(L + 2 * I), (short)I);
  alignment__set_params(&al, (short)match, (short)mismatch, (short)gap_open, (short)gap_extend);
  alignment__reset_with_compressed(&al, read, quality, ref, ref_masked, offset);
  int score = alignment__align(&al, threshold);
  out[0] = score;
  out[1] = al.best_i;
  out[2] = al.best_j;
  al.traceback_seq_len = 0;
  if (al.best_i >= 0) alignment__traceback(&al);
  out[3] = al.best_i0;
  out[4] = al.best_j0;
  out[5] = al.traceback_seq_len;
  memcpy(tb, al.traceback, (size_t)TRACEBACK_SEQ_SIZE(L + I));
  alignment__destroy(&al);
}

/* Index of one sequence for the first seed of `seed_list` (index.c:19-195).  `seq` points at
 * code 0 of a packed sequence readable beyond its end.  Copies first[0..4^w] and the map. */
long kat_index(const char *seed_list, int stdev_distance, unsigned char *seq, int size,
               const int *rs, const int *re, int nreg, int *first_out, int *map_out, long cap) {
  VERBOSITY = 0;
  FILTER_REPEATS = stdev_distance > 0;
  ACCEPTED_STDEV_DISTANCE = stdev_distance > 0 ? stdev_distance : 0;
  SeedType **seeds = NULL;
  if (seed__parse_list(seed_list, &seeds) <= 0) return -1;
  ReferenceDBType db;
  memset(&db, 0, sizeof(db));
  db.name = "kat";
  db.size = size;
  db.sequence = seq;
  MaskedRegionType *head = NULL, *tail = NULL;
  for (int k = 0; k < nreg; ++k) {
    MaskedRegionType *m = calloc(1, sizeof(MaskedRegionType));
    m->start = rs[k];
    m->end = re[k];
    if (tail) tail->next = m; else head = m;
    tail = m;
  }
  db.masked_regions = head;
  IndexType *idx = index__build_reference(&db, seeds[0]);
  long n = 0;
  if (idx->map_size > 0 && idx->first) {
    memcpy(first_out, idx->first, sizeof(int) * (size_t)(idx->index_size + 1));
    n = idx->first[idx->index_size];
    if (n > cap) n = -2;
    else memcpy(map_out, idx->map, sizeof(int) * (size_t)n);
    index__destroy(idx);
  }
  free(idx);
  while (head) { MaskedRegionType *t = head->next; free(head); head = t; }
  return n;
}
