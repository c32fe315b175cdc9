/*
 * storm_host.h -- host side of the storm-nucleotide / storm-color drop-in: input loading,
 * read ordering and SAM / FASTQ output, in plain C.  The mapping itself is done by the CUDA
 * library behind include/stormgpu.h; this layer never maps anything.
 *
 * It reproduces the reference's file semantics byte for byte:
 *   reference FASTA  -> reference_data.c:14-252
 *   reads FASTQ      -> reads_data.c:351-566     (FASTA/CSFASTA + .qual: reads_data.c:73-345)
 *   tag and order    -> reads_data.c:249-257, :494-502, :41-67
 *   SAM output       -> hit_map.c:197-504, alignment.c:749-887
 *   unmapped FASTQ   -> hit_map.c:514-579
 */
#ifndef STORM_HOST_H
#define STORM_HOST_H

#include <stdint.h>
#include <stdio.h>

#include "../../../include/stormgpu.h"

#ifdef __cplusplus
extern "C" {
#endif

#define SH_PAD_BYTES 512   /* bytes of padding around each packed reference sequence */

typedef struct sh_refs {
  int       n;
  char    **names;         /* NULL when the FASTA chunk has no header */
  int64_t  *sizes;         /* codes (bases, or colours in colour space) */
  uint8_t **codes;         /* -> code 0; SH_PAD_BYTES of zero bytes before and after */
  uint8_t **masks;         /* -> code 0; padding bytes are 0x55 (every code masked) */
  int32_t **rs, **re;      /* masked regions [rs, re) */
  int32_t  *nreg;
  uint8_t  *first_base;    /* colour space: first base of each sequence */
  uint8_t **alloc_codes, **alloc_masks;
} sh_refs;

typedef struct sh_reads {
  int64_t   n;
  int       colour;
  int       min_len, max_len;
  int       has_quality;
  char     *db_name;       /* the @RG name (title line, or common name prefix) */
  char    **names;         /* per read (after sorting) */
  uint8_t  *codes;         /* n * code_stride packed codes */
  int64_t   code_stride;
  uint8_t  *levels;        /* n * level_stride packed levels (NULL without qualities) */
  int64_t   level_stride;
  int16_t  *lengths;
  uint64_t *tags;
  uint8_t  *first_base;    /* colour: real first base (TRANSFORM(primer, colour 1)) */
  uint8_t  *first_level;   /* colour: level of the first colour's quality */
  int64_t  *file_index;    /* original position in the file */
  char     *arena;         /* the names[] strings live here (one allocation) */
  uint8_t  *no_quality;    /* per read: 1 when its record has no quality line while others have
                              one (its levels are then all 3 and its QUAL is written as the
                              reference writes a NULL quality); NULL when there is no such read */
} sh_reads;

/* Status: 0 ok, negative on error (message in sh_last_error()). */
const char *sh_last_error(void);
/* Inputs of at least `bytes` take the loaders' threaded paths (default 64 MiB; the results do
 * not depend on it). */
void sh_set_parallel_min_bytes(size_t bytes);
/* 1 when the last error's message is the reference's whole message for a failure it reports
 * and exits on (print it alone), 0 when the caller adds its own line as the reference does */
int sh_last_error_final(void);

int  sh_load_reference(const char *path, int colour, int ignore_lowercase, sh_refs *out);
void sh_free_reference(sh_refs *r);

/* FASTQ by extension (.fastq .fq .fastq2 .fq2), FASTA / CSFASTA otherwise (reads_data.c:568).
 * quality_base is -b.  allow_mixed: accept reads of different lengths (the reference exits). */
int  sh_load_reads(const char *path, const char *qual_path, int colour, int quality_base,
                   int allow_mixed, sh_reads *out);
void sh_free_reads(sh_reads *r);

/* Stable sort by (length, tag): within one length, the order of the reference's qsort by tag
 * with ties in file order (reads_data.c:41-67).  0, or STORMGPU_ENOMEM (reads unchanged). */
int sh_sort_reads(sh_reads *r);

/* The reads as the C ABI expects them. */
void sh_reads_view(const sh_reads *r, stormgpu_reads *view);

typedef struct sh_sam_opts {
  int    colour;
  int    max_rank;          /* -M */
  int    print_all;         /* -A */
  int    uniqueness;        /* -u given */
  int    uniqueness_threshold;
  int    min_score;         /* -t */
  int    delta_m;           /* match - mismatch */
  int    quality_base;      /* -b */
  int    argc;
  char **argv;              /* echoed in @PG CL */
} sh_sam_opts;

int sh_write_sam(FILE *f, const sh_sam_opts *o, const sh_refs *refs, const sh_reads *reads,
                 const stormgpu_results *res, int64_t first, int64_t count, int header);
int sh_write_unmapped_fastq(FILE *f, const sh_sam_opts *o, const sh_reads *reads,
                            const stormgpu_results *res);
/* The same into the file at `path` (created or truncated; the SAM with its header). */
int sh_write_sam_path(const char *path, const sh_sam_opts *o, const sh_refs *refs, const sh_reads *reads,
                      const stormgpu_results *res);
int sh_write_unmapped_fastq_path(const char *path, const sh_sam_opts *o, const sh_reads *reads,
                                 const stormgpu_results *res);

/* genome_map (the mapping without -M): the reads placed on the references, in the order
 * genome_map__generate_SAM_output prints them (sequence, position, then placement order),
 * each with the rank of its alignment that was placed. */
typedef struct sh_placement {
  int32_t read;
  int32_t rank;
} sh_placement;

/* Contextual placement (the default, genome_map.c:253-536): reads by descending best score
 * (a stable sort on the unsigned value, as the reference's radix sort); every alignment of the
 * read rescored against the consensus of the reads placed so far (6-bit counters per code that
 * wrap, genome_map.c:37-48), the best placed and the consensus updated along its traceback.
 * out holds n entries; *n_out receives the number placed.  The restatement the oracle front end
 * places with (the CUDA command line places on the device, stormgpu_genome_map_contextual). */
int sh_genome_map_contextual(const sh_refs *refs, const stormgpu_results *res, int64_t n, int colour, int indels,
                             int match, int mismatch, int uniqueness, int uniqueness_threshold,
                             sh_placement *out, int64_t *n_out);

/* Order placements by (sequence, position of the placed alignment), keeping their order
 * within a position. */
void sh_sort_placements(const stormgpu_results *res, sh_placement *pl, int64_t n);

/* The SAM of a genome map (genome_map.c:551-796): @HD SO:coordinate, records position-major. */
int sh_write_genome_map_sam(FILE *f, const sh_sam_opts *o, const sh_refs *refs, const sh_reads *reads,
                            const stormgpu_results *res, const sh_placement *pl, int64_t n_pl);

/* alignment.c:749-887 (exposed for tests). */
int sh_traceback_to_cigar(const uint8_t *tb, int tb_len, const uint8_t *ref_codes,
                          int64_t ref_start, int colour, int ref_start_symbol, char *cigar,
                          char *seq);
/* hit_map.c:384-403 (exposed for tests). */
int sh_mapq(int rank, int score0, int score1, int score_rank, int min_score, int delta_m);

#ifdef __cplusplus
}
#endif
#endif
