/* storm-nucleotide / storm-color: the reference's command line over the CUDA mapping library
 * (include/stormgpu.h).  There is no CPU fallback: without a usable GPU the mapping step
 * fails with a clear error. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "storm_cli.h"

/* the context stays open after mapping: the greedy placement reads its device results */
typedef struct gpu_state {
  stormgpu_ctx *ctx;
} gpu_state;

/* context creation (the device's start-up) while the command line loads its inputs */
static void gpu_prepare(void *user, const stormgpu_params *p, const char *seeds) {
  gpu_state *gs = (gpu_state *)user;
  if (stormgpu_open(p, seeds, &gs->ctx) != 0) gs->ctx = NULL;  /* gpu_map opens again and reports */
}

/* reads [first, first + n) of v, and their part of the results */
static void piece_views(const stormgpu_reads *v, const stormgpu_results *out, int64_t first, int64_t n,
                        stormgpu_reads *pv, stormgpu_results *po) {
  *pv = *v;
  *po = *out;
  pv->n = n;
  pv->codes += first * v->code_stride;
  if (pv->levels) pv->levels += first * v->level_stride;
  pv->lengths += first;
  if (pv->first_levels) pv->first_levels += first;
  po->hits += 4 * first;
  po->tb += 4 * first * out->tb_stride;
  po->mapped += first;
}

static int gpu_map_chunked(void *user, const stormgpu_params *p, const char *seeds, const sh_refs *refs,
                           const sh_reads *reads, stormgpu_results *out, int64_t piece, storm_chunk_fn chunk,
                           void *chunk_user, char *err, int errlen) {
  gpu_state *gs = (gpu_state *)user;
  stormgpu_ctx *ctx = gs->ctx;
  gs->ctx = NULL;
  int rc = ctx ? 0 : stormgpu_open(p, seeds, &ctx);
  if (rc) goto fail;
  for (int s = 0; s < refs->n; ++s) {
    rc = stormgpu_add_reference(ctx, refs->codes[s], refs->masks[s], refs->sizes[s], refs->rs[s],
                                refs->re[s], refs->nreg[s]);
    if (rc) goto fail;
  }
  rc = stormgpu_build_index(ctx);
  if (rc) goto fail;
  stormgpu_reads v;
  sh_reads_view(reads, &v);
  if (piece <= 0 || piece >= reads->n) piece = reads->n;
  for (int64_t first = 0; first < reads->n || first == 0; first += piece) {
    const int64_t n = reads->n - first < piece ? reads->n - first : piece;
    stormgpu_reads pv;
    stormgpu_results po;
    piece_views(&v, out, first, n, &pv, &po);
    rc = stormgpu_map(ctx, &pv, &po);
    if (rc) goto fail;
    if (chunk) chunk(chunk_user, first, n);
    if (reads->n == 0) break;
  }
  gs->ctx = ctx;
  return 0;
fail:
  snprintf(err, (size_t)errlen, "%s", stormgpu_last_error());
  if (ctx) stormgpu_close(ctx);
  return rc;
}

/* the whole read set in one call (the greedy placement reads the context's device results) */
static int gpu_map(void *user, const stormgpu_params *p, const char *seeds, const sh_refs *refs,
                   const sh_reads *reads, stormgpu_results *out, char *err, int errlen) {
  return gpu_map_chunked(user, p, seeds, refs, reads, out, 0, NULL, NULL, err, errlen);
}

static int gpu_place_greedy(void *user, const sh_refs *refs, const stormgpu_results *res, int64_t n,
                            int uniqueness_threshold, sh_placement *out, int64_t *n_out, char *err, int errlen) {
  (void)refs; (void)res;
  gpu_state *gs = (gpu_state *)user;
  int32_t *order = malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
  int rc = stormgpu_genome_map_greedy(gs->ctx, uniqueness_threshold, order, n_out);
  if (rc) snprintf(err, (size_t)errlen, "%s", stormgpu_last_error());
  else
    for (int64_t i = 0; i < *n_out; ++i) out[i] = (sh_placement){order[i], 0};
  free(order);
  return rc;
}

static int gpu_place_contextual(void *user, const sh_refs *refs, const stormgpu_results *res, int64_t n,
                                int uniqueness, int uniqueness_threshold, sh_placement *out, int64_t *n_out,
                                char *err, int errlen) {
  (void)refs; (void)res;
  gpu_state *gs = (gpu_state *)user;
  int32_t *rd = malloc(sizeof(int32_t) * (size_t)(n ? n : 1)), *rk = malloc(sizeof(int32_t) * (size_t)(n ? n : 1));
  int rc = rd && rk ? stormgpu_genome_map_contextual(gs->ctx, uniqueness, uniqueness_threshold, rd, rk, n_out)
                    : STORMGPU_ENOMEM;
  if (rc) snprintf(err, (size_t)errlen, "%s", rd && rk ? stormgpu_last_error() : "host allocation failed");
  else
    for (int64_t i = 0; i < *n_out; ++i) out[i] = (sh_placement){rd[i], rk[i]};
  free(rd);
  free(rk);
  return rc;
}

static void gpu_finish(void *user) {
  gpu_state *gs = (gpu_state *)user;
  if (gs->ctx) stormgpu_close(gs->ctx);
  gs->ctx = NULL;
}

int main(int argc, char **argv) {
  gpu_state gs = {NULL};
  storm_mapper m = {"cuda", gpu_map, gpu_place_greedy, gpu_finish, &gs, gpu_prepare, gpu_map_chunked,
                    gpu_place_contextual};
  return storm_cli_main(argc, argv, STORM_COLOUR, &m);
}
