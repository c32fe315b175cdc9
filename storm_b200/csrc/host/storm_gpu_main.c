/* storm-nucleotide / storm-color: the reference's command line over the CUDA mapping library
 * (include/stormgpu.h).  There is no CPU fallback: without a usable GPU the mapping step
 * fails with a clear error. */
#include <stdlib.h>
#include <string.h>

#include "storm_cli.h"

static int gpu_map(void *user, const stormgpu_params *p, const char *seeds, const sh_refs *refs,
                   const sh_reads *reads, stormgpu_results *out, char *err, int errlen) {
  (void)user;
  stormgpu_ctx *ctx = NULL;
  int rc = stormgpu_open(p, seeds, &ctx);
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
  stormgpu_close(ctx);
  return 0;
fail:
  snprintf(err, (size_t)errlen, "%s", stormgpu_last_error());
  if (rc == STORMGPU_EINVAL && strstr(err, "seed") == NULL && strstr(err, "invalid") != NULL) {}
  if (ctx) stormgpu_close(ctx);
  return rc;
}

int main(int argc, char **argv) {
  storm_mapper m = {"cuda", gpu_map, NULL};
  return storm_cli_main(argc, argv, STORM_COLOUR, &m);
}
