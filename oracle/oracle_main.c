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

int main(int argc, char **argv) {
  storm_mapper m = {"oracle", oracle_map, NULL};
  return storm_cli_main(argc, argv, STORM_COLOUR, &m);
}
