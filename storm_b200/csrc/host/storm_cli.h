/*
 * storm_cli.h -- the storm-nucleotide / storm-color command line (main.c:174-463 and the
 * driver reads_against_references, run.c:764-1109), parameterised by the mapper that fills
 * the per-read results, so that the same front end drives the CUDA library.
 */
#ifndef STORM_CLI_H
#define STORM_CLI_H

#include "storm_host.h"

#ifdef __cplusplus
extern "C" {
#endif

/* called by a chunked map once the results of reads [first, first + count) are in `out` */
typedef void (*storm_chunk_fn)(void *chunk_user, int64_t first, int64_t count);

typedef struct storm_mapper {
  const char *name;
  /* fill `out` (already allocated for reads->n reads) for all reads against all sequences;
   * return 0 or a negative error code (message through `err`). */
  int (*map)(void *user, const stormgpu_params *p, const char *seeds, const sh_refs *refs,
             const sh_reads *reads, stormgpu_results *out, char *err, int errlen);
  /* greedy genome_map placement (no -M, -G) of the results of the last map call: placed reads
   * in position-major order (rank 0); uniqueness_threshold 0 = no -u. */
  int (*place_greedy)(void *user, const sh_refs *refs, const stormgpu_results *res, int64_t n,
                      int uniqueness_threshold, sh_placement *out, int64_t *n_out, char *err, int errlen);
  /* release what map kept (may be NULL) */
  void (*finish)(void *user);
  void *user;
  /* may be NULL; else called once at start-up, from another thread, while the inputs load:
   * device set-up that needs only the parameters and the seeds (map must still work, and report
   * the error, if it failed) */
  void (*prepare)(void *user, const stormgpu_params *p, const char *seeds);
  /* may be NULL; else the same as map, in consecutive pieces of about `piece` reads, calling
   * chunk() after each piece's results are in `out` and before the next piece maps (the
   * command line writes a piece's SAM records while the next one maps) */
  int (*map_chunked)(void *user, const stormgpu_params *p, const char *seeds, const sh_refs *refs,
                     const sh_reads *reads, stormgpu_results *out, int64_t piece, storm_chunk_fn chunk,
                     void *chunk_user, char *err, int errlen);
  /* may be NULL (then the host's sh_genome_map_contextual); else the contextual placement
   * (no -M, no -G) of the results of the last map call, as sh_genome_map_contextual */
  int (*place_contextual)(void *user, const sh_refs *refs, const stormgpu_results *res, int64_t n, int uniqueness,
                          int uniqueness_threshold, sh_placement *out, int64_t *n_out, char *err, int errlen);
} storm_mapper;

int storm_cli_main(int argc, char **argv, int colour, const storm_mapper *mapper);

#ifdef __cplusplus
}
#endif
#endif
