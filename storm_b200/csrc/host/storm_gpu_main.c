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

static int gpu_map(void *user, const stormgpu_params *p, const char *seeds, const sh_refs *refs,
                   const sh_reads *reads, stormgpu_results *out, char *err, int errlen) {
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
  rc = stormgpu_map(ctx, &v, out);
  if (rc) goto fail;
  gs->ctx = ctx;
  return 0;
fail:
  snprintf(err, (size_t)errlen, "%s", stormgpu_last_error());
  if (rc == STORMGPU_EINVAL && strstr(err, "seed") == NULL && strstr(err, "invalid") != NULL) {}
  if (ctx) stormgpu_close(ctx);
  return rc;
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

static void gpu_finish(void *user) {
  gpu_state *gs = (gpu_state *)user;
  if (gs->ctx) stormgpu_close(gs->ctx);
  gs->ctx = NULL;
}

int main(int argc, char **argv) {
  gpu_state gs = {NULL};
  storm_mapper m = {"cuda", gpu_map, gpu_place_greedy, gpu_finish, &gs, gpu_prepare};
  return storm_cli_main(argc, argv, STORM_COLOUR, &m);
}
