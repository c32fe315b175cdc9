/* TEST INFRASTRUCTURE ONLY: the storm-nucleotide / storm-color front end of the product
 * (storm_b200/csrc/host) driven by the single-threaded oracle mapper instead of the GPU, so
 * that the whole chain loader -> mapping -> SAM writer can be compared byte for byte with
 * the reference binary on the CPU.  Never shipped, never called by the product. */
#include <stdlib.h>
#include <string.h>

#include "../storm_b200/csrc/host/storm_cli.h"
#include "storm_oracle.h"

static int oracle_map(void *user, const stormgpu_params *p, const char *seeds, const sh_refs *refs,
                      const sh_reads *reads, stormgpu_results *out, char *err, int errlen) {
  (void)user;
  or_ref *R = calloc((size_t)refs->n, sizeof(or_ref));
  for (int s = 0; s < refs->n; ++s) {
    R[s].codes = refs->codes[s];
    R[s].mask = refs->masks[s];
    R[s].n_codes = refs->sizes[s];
    R[s].rs = refs->rs[s];
    R[s].re = refs->re[s];
    R[s].nreg = refs->nreg[s];
  }
  stormgpu_reads v;
  sh_reads_view(reads, &v);
  int rc = or_map(p, seeds, R, refs->n, &v, out, NULL);
  if (rc == STORMGPU_EINVAL) strncpy(err, "invalid seed list", (size_t)errlen - 1);
  free(R);
  return rc;
}

/* the same in pieces, each piece's results handed to chunk() before the next maps (the front
 * end's pipelined SAM output, exercised on the CPU) */
static int oracle_map_chunked(void *user, const stormgpu_params *p, const char *seeds, const sh_refs *refs,
                              const sh_reads *reads, stormgpu_results *out, int64_t piece, storm_chunk_fn chunk,
                              void *chunk_user, char *err, int errlen) {
  if (piece <= 0 || piece >= reads->n) piece = reads->n > 0 ? reads->n : 1;
  for (int64_t first = 0; first < reads->n; first += piece) {
    const int64_t n = reads->n - first < piece ? reads->n - first : piece;
    sh_reads pr = *reads;
    pr.n = n;
    pr.codes += first * reads->code_stride;
    if (pr.levels) pr.levels += first * reads->level_stride;
    pr.lengths += first;
    if (pr.first_level) pr.first_level += first;
    stormgpu_results po = *out;
    po.hits += 4 * first;
    po.tb += 4 * first * out->tb_stride;
    po.mapped += first;
    const int rc = oracle_map(user, p, seeds, refs, &pr, &po, err, errlen);
    if (rc) return rc;
    chunk(chunk_user, first, n);
  }
  return 0;
}

/* greedy placement, restated: reads in read order, kept iff their rank-0 alignment exists (and
 * leads rank 1 by the -u threshold), then a stable insertion into (sequence, start) order
 * (genome_map.c:187-214, printed position-major by genome_map.c:551-796) */
static int oracle_place_greedy(void *user, const sh_refs *refs, const stormgpu_results *res, int64_t n,
                               int uniqueness_threshold, sh_placement *out, int64_t *n_out, char *err, int errlen) {
  (void)user; (void)refs; (void)err; (void)errlen;
  int64_t k = 0;
  for (int64_t r = 0; r < n; ++r) {
    const stormgpu_hit *h = &res->hits[r * 4];
    if (!res->mapped[r] || h[0].ref_start == -1) continue;
    if (uniqueness_threshold > 0 && !(h[0].score - h[1].score >= uniqueness_threshold)) continue;
    int64_t j = k++;
    while (j > 0) {  /* stable: move only past strictly later positions */
      const stormgpu_hit *p = &res->hits[(int64_t)out[j - 1].read * 4];
      if (p->ref_id < h[0].ref_id || (p->ref_id == h[0].ref_id && p->ref_start <= h[0].ref_start)) break;
      out[j] = out[j - 1];
      --j;
    }
    out[j] = (sh_placement){(int32_t)r, 0};
  }
  *n_out = k;
  return 0;
}

int main(int argc, char **argv) {
  storm_mapper m = {"oracle", oracle_map, oracle_place_greedy, NULL, NULL, NULL, oracle_map_chunked, NULL};
  return storm_cli_main(argc, argv, STORM_COLOUR, &m);
}
