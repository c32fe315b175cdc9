/*
 * stormgpu.h -- C ABI of the B200 mapping library (libstormgpu.so).
 *
 * The reference mapper (SToRM) has no plugin API: its hot path is the static function
 * process_read() in run.c, driven by the per-reference, per-strand OpenMP read loops of
 * reads_against_references() (run.c:764-1109), with the SIMD filter reached through three
 * function pointers (run.c:15-221):
 *
 *     void     (*init)(unsigned match, unsigned mismatch, unsigned gapopen,
 *                      unsigned gapext, unsigned threshold, unsigned readlength);
 *     unsigned (*align)(unsigned char *genome, int *pos_genome, unsigned char *read);
 *     void     (*clean)(void);
 *
 * This header replaces that seam: the host driver hands the library the packed reference
 * and the packed, tag-sorted reads, and gets back for every read the MAP_DETAIL_SIZE (4)
 * best alignments in the exact semantics of HitInfoType (hit_map.h:17-40), from which it
 * formats the SAM output.  All integer, all bit-exact with the reference's CPU build.
 *
 * Conventions: plain pointers and sizes, no exceptions, every function returns 0 on
 * success or a negative STORMGPU_E* code; stormgpu_last_error() gives a message.  A
 * context owns its device memory; one context per thread (calls on a context are not
 * thread-safe, except stormgpu_submit/stormgpu_poll which the serving loop serialises).
 *
 * Codes are 2-bit, packed four per byte, first code in the low bits (codes.h:129-130):
 * nucleotides A,C,G,T = 0..3, colours 0..3.  Quality levels are 2-bit (0..3), packed the
 * same way (read_quality.h:129-133).
 */
#ifndef STORMGPU_H
#define STORMGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define STORMGPU_MAP_DETAIL   4        /* MAP_DETAIL_SIZE, util.h:30 */
#define STORMGPU_MIN_SCORE    (-16383) /* MIN_SCORE, alignment.h:48 */
#define STORMGPU_UNMAPPED     (-1)     /* UNMAPPED, hit_map.h:9 */
#define STORMGPU_MAX_SEEDS    16
#define STORMGPU_MAX_SPAN     64
#define STORMGPU_MAX_READ_LEN 1024
#define STORMGPU_MAX_INDELS   64

/* error codes */
#define STORMGPU_OK        0
#define STORMGPU_EINVAL  (-1)   /* bad argument (mirrors RETURN_INPUT_ERR, load_data.h:8) */
#define STORMGPU_ENOMEM  (-2)   /* device or host allocation failed (RETURN_MEM_ERR) */
#define STORMGPU_ECUDA   (-3)   /* a CUDA call failed, or no usable GPU */
#define STORMGPU_ESTATE  (-4)   /* call out of order (e.g. map before build_index) */
#define STORMGPU_ETIMEOUT (-5)  /* a bounded device wait ran out */

/* Mapping parameters: the reference's command-line options, same signs and defaults
 * (alignment.h:24-28, alignment.h:51-52, index.h:16, main.c:302-313). */
typedef struct stormgpu_params {
  int32_t colour;            /* 0: storm-nucleotide, 1: storm-color */
  int32_t match;             /* -m, > 0            (default  5) */
  int32_t mismatch;          /* -x, <= 0           (default -4) */
  int32_t gap_open;          /* -d, <= 0           (default -9) */
  int32_t gap_extend;        /* -e, <= 0           (default -4) */
  int32_t allowed_indels;    /* -i, >= 0           (default  3) */
  int32_t min_score;         /* -t                 (default 115) */
  int32_t min_score_filter;  /* -z                 (default 100) */
  int32_t stdev_distance;    /* -l; <= 0 disables the repeat filter (default 100) */
  int32_t senses;            /* bit 0: forward, bit 1: reverse complement (default 3) */
  int32_t device;            /* CUDA device ordinal */
} stormgpu_params;

/* One alignment of a read, the fields of HitInfoType (hit_map.h:17-40).  An empty slot has
 * ref_id = ref_start = UNMAPPED and score = MIN_SCORE, as hit_map__update initialises it. */
typedef struct stormgpu_hit {
  int32_t score;
  int32_t ref_id;
  int32_t ref_start;
  int32_t ref_end;
  int16_t read_start;
  int16_t read_end;
  int32_t sense;             /* +1 forward, -1 reverse complement, 0 empty */
  int32_t tb_len;            /* traceback length in 4-bit operations */
} stormgpu_hit;

/* A batch of reads, tag-sorted by the caller (reads_data.c:59-67).  Read r has lengths[r]
 * codes at codes + r*code_stride and quality levels at levels + r*level_stride (levels may
 * be NULL: every level is then 3, alignment.c:157-160). */
typedef struct stormgpu_reads {
  int64_t        n;
  const uint8_t *codes;
  int64_t        code_stride;
  const uint8_t *levels;
  int64_t        level_stride;
  const int16_t *lengths;
  const uint8_t *first_levels; /* colour space only: level of the primer colour (first_qual,
                                  reads_data.h:27), which read__reverse moves to the end of
                                  the reversed read (read_quality.c:238); NULL: level 3 */
} stormgpu_reads;

/* Per-read results.  hits[r*4 + k] is the rank-k alignment; traceback operations of that
 * slot are packed two per byte (high nibble first, alignment.h:81-83) at
 * tb + (r*4 + k)*tb_stride, already in start-to-end order (hit_map.c:137-141).
 * mapped[r] != 0 iff the read reached hit_map__update at least once (hit_map.c:53-74). */
typedef struct stormgpu_results {
  stormgpu_hit *hits;        /* n * 4 */
  uint8_t      *tb;          /* n * 4 * tb_stride */
  int64_t       tb_stride;   /* >= (max read length + allowed_indels + 1) / 2 */
  uint8_t      *mapped;      /* n */
} stormgpu_results;

typedef struct stormgpu_ctx stormgpu_ctx;

/* Library and device --------------------------------------------------------------------- */
const char *stormgpu_version(void);
const char *stormgpu_last_error(void);
/* 1 if a CUDA device is usable, 0 otherwise (never aborts). */
int stormgpu_device_available(void);

/* Context: parameters and the seed family.  `seeds` is the reference's -s syntax
 * ("#-##;1101:0 3", seed.c:25-135); an invalid list gives STORMGPU_EINVAL.
 * Replaces: the set-up half of reads_against_references (run.c:790-858). */
int  stormgpu_open(const stormgpu_params *params, const char *seeds, stormgpu_ctx **out);
void stormgpu_close(stormgpu_ctx *ctx);

/* Reference sequences, in file order.  `codes` holds n_codes packed codes; `mask` holds the
 * packed per-code masked flag (non-ACGT input, reference_data.c:115-126); masked regions are
 * [starts[k], ends[k]) in ascending order (reference_data.c:121-177).
 * Replaces: load_reference_db's output (reference_data.c:195-252). */
int stormgpu_add_reference(stormgpu_ctx *ctx, const uint8_t *codes, const uint8_t *mask,
                           int64_t n_codes, const int32_t *region_starts,
                           const int32_t *region_ends, int32_t n_regions);

/* Build the device-resident spaced-seed index of every reference sequence for every seed.
 * Replaces: index__build_reference (index.c:19-195), called per sequence per seed
 * (run.c:876-884). */
int stormgpu_build_index(stormgpu_ctx *ctx);

/* Map a batch: every read against every sequence, forward then reverse, the top-4 table
 * updated in the reference's order (sequence, strand, diagonal).  Host buffers in and out.
 * Replaces: the read loops of run.c:865-994 around process_read (run.c:555-747) and
 * hit_map__update (hit_map.c:50-144). */
int stormgpu_map(stormgpu_ctx *ctx, const stormgpu_reads *reads, stormgpu_results *out);

/* Device-resident variant for callers that already hold the reads in GPU memory:
 * every pointer in `reads` and `out` is a device pointer.  `stream` is a cudaStream_t
 * (NULL: the context's stream).  Asynchronous; stormgpu_sync() waits. */
int stormgpu_map_device(stormgpu_ctx *ctx, const stormgpu_reads *reads,
                        stormgpu_results *out, void *stream);
int stormgpu_sync(stormgpu_ctx *ctx);

/* Served mapping ----------------------------------------------------------------------------
 * The reference and the index of every step of an -O seed chain stay resident on the GPU;
 * batches are submitted from any thread and run concurrently on `slots` workers (own stream and
 * buffers each).  `budget_bytes` bounds the device memory of the batches besides the resident
 * sequences and indexes: half of it is the workers' mapping buffers (an equal share each, never
 * exceeded: a pass that would need more maps its reads in halves), the other half the chain
 * buffers of the batches in flight (reads, results; exactly sized, taken when a batch starts and
 * returned when it ends).  A batch is admitted, in arrival order, when a worker is free and its
 * chain buffers fit what the batches in flight leave of that half; a batch whose chain buffers
 * alone exceed it is refused by stormgpu_submit.  Host copies go through a pinned staging area
 * per worker.  Step k of a batch maps, with chain[k], the reads no earlier step mapped, in
 * their order: the reference run again on its own -O FASTQ output (README:97-101,
 * hit_map.c:514-579); every read gets the results of the step that mapped it.
 * No counterpart in the reference (one read file per process there). */
typedef struct stormgpu_server stormgpu_server;
int stormgpu_server_open(const stormgpu_params *params, const char *const *chain, int nsteps,
                         int slots, int64_t budget_bytes, stormgpu_server **out);
int stormgpu_server_add_reference(stormgpu_server *s, const uint8_t *codes, const uint8_t *mask,
                                  int64_t n_codes, const int32_t *region_starts,
                                  const int32_t *region_ends, int32_t n_regions);
/* Index every step, start the workers. */
int stormgpu_server_build(stormgpu_server *s);
/* Launch parameters of every worker slot (stormgpu_tuning, declared below; none changes a
 * result).  Before stormgpu_server_build only (the slots take them when they are built), else
 * STORMGPU_ESTATE.  No counterpart in the reference. */
struct stormgpu_tuning;
int stormgpu_server_set_tuning(stormgpu_server *s, const struct stormgpu_tuning *t);
/* Queue a batch (host buffers, which must stay valid until stormgpu_poll reports it done).
 * step[r] (optional, n bytes) receives the chain step that mapped read r, 255 if none did. */
int stormgpu_submit(stormgpu_server *s, const stormgpu_reads *reads, stormgpu_results *out,
                    uint8_t *step, int64_t *ticket);
/* 0: done (results in place, *latency_ms = submit to completion), 1: not yet after
 * timeout_ms (< 0: wait), < 0: the batch failed (message in stormgpu_last_error). */
int stormgpu_poll(stormgpu_server *s, int64_t ticket, int timeout_ms, double *latency_ms);
void stormgpu_server_close(stormgpu_server *s);

/* Greedy placement of the mapping without -M (-G; genome_map.c:187-214, order of
 * genome_map.c:551-796): the reads whose rank-0 alignment exists -- and, when
 * uniqueness_threshold > 0 (-u), whose rank-0 score leads the rank-1 score by at least that --
 * in (sequence, rank-0 start) order, reads of one position in read order.  Works on the results
 * of the last stormgpu_map call on ctx, which stay on the device; order (host) holds n int32,
 * *n_placed receives how many are placed. */
int stormgpu_genome_map_greedy(stormgpu_ctx *ctx, int32_t uniqueness_threshold, int32_t *order,
                               int64_t *n_placed);

/* Contextual placement of the mapping without -M and without -G (the default; genome_map.c:
 * 233-531, order of genome_map.c:551-796): the mapped reads in descending (unsigned) order of
 * their rank-0 score, ties in read order, each placed at the first of its ranks with the highest
 * score adjusted to the consensus of the reads placed before it (genome_map.c:366-424) -- when
 * uniqueness is set (-u), only if the adjusted rank-0 score leads the adjusted rank-1 score by
 * more than uniqueness_threshold -- whose counters it then updates.  Output in (sequence,
 * start) order, reads of one position in placement order: read[i] and the placed rank rank[i]
 * for i < *n_placed (read and rank hold n int32 on the host).  Works on the results of the last
 * stormgpu_map call on ctx, which stay on the device.
 * Replaces: genome_map__build_contextual (genome_map.c:432-531) and the position-major walk of
 * genome_map__generate_SAM_output (genome_map.c:551-796). */
int stormgpu_genome_map_contextual(stormgpu_ctx *ctx, int32_t uniqueness, int32_t uniqueness_threshold,
                                   int32_t *read, int32_t *rank, int64_t *n_placed);

/* Statistics of the last stormgpu_map* call. */
typedef struct stormgpu_stats {
  int64_t candidates;        /* diagonals produced by the hit gather */
  int64_t filter_passed;     /* diagonals passing the banded SW filter */
  int64_t aligned;           /* full alignments computed */
  int64_t seed_lookups;      /* (seed, read position) key lookups */
  int64_t hit_positions;     /* index positions read by the hit gather */
  int64_t filter_cells;      /* filter cell updates: W * 2 * (L + W - 1) per candidate, W = 2..16 */
  int64_t align_cells;       /* band cells the full alignment computed: 2*i+1 per row, L rows for
                                a candidate that runs to its last row, fewer for one that stops
                                once it can no longer be accepted */
  int64_t kernels;           /* kernel launches */
  int64_t filter_band_cells; /* band cells of the filtered diagonals: L * (2*min(i,15)+1) each */
  double  ms_index, ms_gather, ms_filter, ms_align, ms_replay, ms_total;
  int64_t passes;            /* strand passes run (one filter launch each; a batch cut into pieces
                                runs one per piece, sequence and strand) */
  int64_t graph_passes;      /* of them, passes that ran inside a CUDA graph (every pass of a call
                                captured as one graph and launched once, no host read between
                                its launches) */
  int64_t placement_waves;   /* waves of the last stormgpu_genome_map_contextual call on the
                                context (reads placed together in one wave share no position) */
} stormgpu_stats;
int stormgpu_get_stats(stormgpu_ctx *ctx, stormgpu_stats *out);

/* Launch parameters of the mapping stages.  None of them changes a result: they trade
 * occupancy, load balance and atomics against each other, and the best values depend on the
 * read lengths, the band and the index.  No counterpart in the reference (it has no GPU). */
typedef struct stormgpu_tuning {
  int32_t gather_warp_cap;        /* index positions one gather warp holds in shared memory (the
                                     hit bucket), 256..1536; reads with more go to a block per read */
  int32_t gather_reads_per_steal; /* reads a gather warp takes from the work cursor at a time, 1..64 */
  int32_t filter_rows;            /* rows of 256 candidates in a filter block's tile when
                                     filter_cursor is 1 (else 8), 1..64 */
  int32_t align_steal;            /* passing candidates an alignment warp takes at a time, 32..1024,
                                     a multiple of 32 */
  int32_t filter_cursor;          /* 1: the filter runs as a persistent grid whose blocks take tiles
                                     from a work cursor; 0: one block per tile */
  int32_t align_rounds;           /* 1..6: a read's passing candidates are aligned in this many
                                     rounds of increasing rank (the first 8, then up to 32, 128,
                                     512, 2048, then the rest), each followed by the replay of its
                                     ranks; a later round's alignment stops as soon as it cannot
                                     reach the read's running threshold.  1: one round */
} stormgpu_tuning;
/* CUDA graphs (default on, unless the environment sets STORMGPU_GRAPHS=0 when the context
 * opens): from the second mapping call of a context on, all strand passes of a call are
 * captured as one graph, with every list sized from the densest pass seen so far (+25 %), and
 * launched once; a call whose lists outgrow those sizes is run again as separate launches with
 * the host reading each list size (the results are the same either way).  0 turns them off. */
int stormgpu_set_graphs(stormgpu_ctx *ctx, int enable);
/* The context's parameters (defaults 768, 4, 8, 32, 0, 4). */
int stormgpu_get_tuning(stormgpu_ctx *ctx, stormgpu_tuning *out);
/* Set them; STORMGPU_EINVAL (nothing changed) if one is outside its range. */
int stormgpu_set_tuning(stormgpu_ctx *ctx, const stormgpu_tuning *t);
/* Autotuner: maps the reads (or `sample` of them, spread evenly over the batch, when
 * 0 < sample < n; a sample whose mapping takes under 50 ms is grown, up to the whole batch,
 * so that the stage times are not decided by fixed launch costs) once per candidate value of
 * each parameter,
 * stage by stage, times the stage it affects with CUDA events, and keeps the fastest value of
 * each (the result is in the context and, when `out` is not null, in *out).  The reads are
 * on the host, as for stormgpu_map.  Requires stormgpu_build_index.  Afterwards the context's
 * last results (used by stormgpu_genome_map_greedy) are those of the sample. */
int stormgpu_autotune(stormgpu_ctx *ctx, const stormgpu_reads *reads, int64_t sample, stormgpu_tuning *out);

/* Unit-level entry points (host buffers), one kernel each, used by the parity tests.
 * ------------------------------------------------------------------------------------- */

/* Banded SW filter (alignment_simd.c:2282-3404, semantics shared by every ISA): for each
 * i < n, pass[i] = 1 iff the saturating-u8 local band score of the read against the genome
 * window starting at code pos[i] exceeds min(threshold, 254).  W = 2,4,8,16 cells per hit.
 * `genome` points at code 0 of a packed sequence that is readable (zero) for `pad` codes
 * before and after its n_codes codes.  match..gapext are the absolute values that
 * run.c:839 passes to the init function. */
int stormgpu_sw_filter(int W, int read_len, uint32_t match, uint32_t mismatch,
                       uint32_t gapopen, uint32_t gapext, uint32_t threshold,
                       const uint8_t *genome, int64_t n_codes, int64_t pad,
                       const int32_t *pos, int64_t n, const uint8_t *read, uint8_t *pass);

/* Full banded alignment + traceback of one read against n windows (alignment.c:488-734).
 * Window k starts at code win[k] of `genome`/`mask` (same padding rule as above).  Outputs
 * per window: score (MIN_SCORE-free: the unaborted best score), abort bound (the smallest
 * max_on_line + best_possible over rows 1..L-1; the reference aborts iff bound < threshold),
 * best_i, best_j, best_i0, best_j0, traceback length and the traceback operations in the
 * reference's end-to-start order, packed two per byte at tb + k*tb_stride. */
int stormgpu_align(const stormgpu_params *params, const uint8_t *read, const uint8_t *levels,
                   int read_len, const uint8_t *genome, const uint8_t *mask, int64_t n_codes,
                   int64_t pad, const int32_t *win, int64_t n, int32_t *score, int32_t *bound,
                   int16_t *best, int32_t *tb_len, uint8_t *tb, int64_t tb_stride);

/* stormgpu_align for callers that cannot allocate device memory: callers whose device memory
 * belongs to another allocator (a framework's caching allocator, a pool reserved at start-up,
 * with no room for a cudaMalloc of its own) and callers that cannot afford the device-wide
 * synchronisation of cudaMalloc / cudaFree.  No counterpart in the reference (it has no GPU).
 *
 * Same computation and outputs as stormgpu_align, but every array is device memory of the
 * current device, owned by the caller, and nothing is allocated: read / levels are packed as
 * for stormgpu_align (levels may be NULL); genome / mask hold n_codes codes with no padding,
 * and every window must lie inside them (0 <= win[k], win[k] + read_len + 2 * allowed_indels
 * <= n_codes; otherwise STORMGPU_EINVAL, and every output buffer may have been overwritten,
 * the results of the valid windows included); win, score, bound, tb_len
 * hold n entries, best 4n, tb n * tb_stride bytes (zero-filled, then the traceback).
 * params->device is not consulted.  Runs on `stream` (a cudaStream_t; NULL: the default
 * stream) and returns when the results are in place.
 *
 * The kernel works in one fixed device array of STORMGPU_NOALLOC_SCRATCH_BYTES inside the
 * library, which every GPU that loads the library holds until the process exits.  A call
 * needs 4 * read_len * words_per_row * n bytes of it plus at most 8n + 768 of bookkeeping
 * (words_per_row = ceil((4I + 2) / 32), plus ceil((2I + 1) / 32) in colour space,
 * I = allowed_indels); larger calls fail with STORMGPU_EINVAL: split the windows.  Every call
 * looks up the array's device address on the current device (cudaGetSymbolAddress, which
 * allocates nothing); the first call on a device also loads the library's module there, so
 * make it before any stream capture.  Every call on a device shares that device's array, so
 * calls that overlap on the GPU race: serialise them. */
#define STORMGPU_NOALLOC_SCRATCH_BYTES (8ll << 20)
int stormgpu_align_noalloc(const stormgpu_params *params, const uint8_t *read, const uint8_t *levels,
                           int read_len, const uint8_t *genome, const uint8_t *mask, int64_t n_codes,
                           const int32_t *win, int64_t n, int32_t *score, int32_t *bound,
                           int16_t *best, int32_t *tb_len, uint8_t *tb, int64_t tb_stride,
                           void *stream);

/* CSR index of one sequence for one seed (index.c:19-195): first[4^w + 1] offsets and
 * map[first[4^w]] positions, ascending within each key. */
int stormgpu_index_one(const char *seed, int32_t stdev_distance, const uint8_t *codes,
                       int64_t n_codes, int64_t pad, const int32_t *region_starts,
                       const int32_t *region_ends, int32_t n_regions, int32_t *first,
                       int32_t *map, int64_t map_capacity, int64_t *map_len);

/* Measurement helper: the device's rate, in 32-bit lane instructions per second, for the
 * instruction mix of one step of the packed 16-bit filter recurrence (6.5 instructions per
 * register of two cells), run register-resident; the roofline denominator of the filter.
 * No counterpart in the reference (it has no GPU). */
int stormgpu_filter_peak(int device, double *ops_per_s, double *ms);

#ifdef __cplusplus
}
#endif
#endif /* STORMGPU_H */
