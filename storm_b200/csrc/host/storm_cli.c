/*
 * storm_cli.c -- command line of storm-nucleotide / storm-color.
 *
 * Same getopt string, defaults, checks and exit codes as the reference front end
 * (main.c:174-463); the driver steps of reads_against_references (run.c:764-1109): parse the
 * seeds, load and tag-sort the reads, load the reference, map, write the SAM and the
 * unmapped FASTQ.  Extension: reads of different lengths are accepted in one file; they are
 * mapped in one batch and reported grouped by length (ascending), each group in tag order,
 * i.e. exactly the concatenation of per-length runs of the reference.
 */
#include "storm_cli.h"

#include <getopt.h>
#include <pthread.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#define DEFAULT_SEEDS_NUC "####--#-#--##--####;#####--###-#-###;###-##-#######"
#define DEFAULT_SEEDS_COL "####----##--##-####;####-###--#----####;####-####-####"
#define DEFAULT_SEED_FILE_NUC "seeds/solexa_lossy-3-12.in"
#define DEFAULT_SEED_FILE_COL "seeds/solid_lossy-3-12.in"

static int verbosity = 1;

static void msg(int level, const char *fmt, ...) {
  if (level > verbosity) return;
  va_list ap;
  va_start(ap, fmt);
  vfprintf(stderr, fmt, ap);
  va_end(ap);
  fflush(stderr);
}

static void err(const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, "\033[31;1m");
  vfprintf(stderr, fmt, ap);
  fprintf(stderr, "\033[0m\n");
  va_end(ap);
  fflush(stderr);
}

static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* the reference load, run beside the reads load */
typedef struct ref_job {
  const char *path;
  int colour, ignore_lower, rc;
  sh_refs refs;
  char msg[512];
  double seconds;
} ref_job;

static void *ref_job_run(void *arg) {
  ref_job *j = (ref_job *)arg;
  const double t = now_s();
  j->rc = sh_load_reference(j->path, j->colour, j->ignore_lower, &j->refs);
  if (j->rc) snprintf(j->msg, sizeof(j->msg), "%s", sh_last_error());
  j->seconds = now_s() - t;
  return NULL;
}

/* the mapper's device set-up, run beside the loads */
typedef struct prep_job {
  const storm_mapper *m;
  const stormgpu_params *p;
  const char *seeds;
  double seconds;
} prep_job;

static void *prep_job_run(void *arg) {
  prep_job *j = (prep_job *)arg;
  const double t = now_s();
  j->m->prepare(j->m->user, j->p, j->seeds);
  j->seconds = now_s() - t;
  return NULL;
}

/* SAM records written by a second thread, piece after piece in read order, while the next
 * piece maps */
enum { SAM_PIPE_SLOTS = 64 };
typedef struct sam_pipe {
  pthread_mutex_t mu;
  pthread_cond_t cv;
  int64_t first[SAM_PIPE_SLOTS], count[SAM_PIPE_SLOTS];
  int head, tail, done, rc;
  char msg[512];
  FILE *f;
  const sh_sam_opts *so;
  const sh_refs *refs;
  const sh_reads *reads;
  const stormgpu_results *res;
} sam_pipe;

static void *sam_pipe_run(void *arg) {
  sam_pipe *q = (sam_pipe *)arg;
  for (;;) {
    pthread_mutex_lock(&q->mu);
    while (q->head == q->tail && !q->done) pthread_cond_wait(&q->cv, &q->mu);
    if (q->head == q->tail) {
      pthread_mutex_unlock(&q->mu);
      return NULL;
    }
    const int64_t first = q->first[q->head % SAM_PIPE_SLOTS], count = q->count[q->head % SAM_PIPE_SLOTS];
    pthread_mutex_unlock(&q->mu);
    if (q->rc == 0) {
      q->rc = sh_write_sam(q->f, q->so, q->refs, q->reads, q->res, first, count, first == 0);
      if (q->rc) snprintf(q->msg, sizeof(q->msg), "%s", sh_last_error());
    }
    pthread_mutex_lock(&q->mu);
    q->head++;
    pthread_cond_broadcast(&q->cv);
    pthread_mutex_unlock(&q->mu);
  }
}

/* storm_chunk_fn: queue the piece's records (waits while every slot is taken) */
static void sam_pipe_push(void *arg, int64_t first, int64_t count) {
  sam_pipe *q = (sam_pipe *)arg;
  pthread_mutex_lock(&q->mu);
  while (q->tail - q->head >= SAM_PIPE_SLOTS) pthread_cond_wait(&q->cv, &q->mu);
  q->first[q->tail % SAM_PIPE_SLOTS] = first;
  q->count[q->tail % SAM_PIPE_SLOTS] = count;
  q->tail++;
  pthread_cond_broadcast(&q->cv);
  pthread_mutex_unlock(&q->mu);
}

static void sam_pipe_finish(sam_pipe *q, pthread_t th) {
  pthread_mutex_lock(&q->mu);
  q->done = 1;
  pthread_cond_broadcast(&q->cv);
  pthread_mutex_unlock(&q->mu);
  pthread_join(th, NULL);
}

/* reads mapped in this many pieces when the SAM output is written beside the mapping */
enum { SAM_PIPE_PIECES = 4 };
#define SAM_PIPE_MIN_READS 200000

/* seed.c:140-179: one seed per line, '%' lines ignored, trailing blanks removed, ';' added */
static char *seeds_from_file(const char *path) {
  FILE *f = fopen(path, "r");
  if (!f) return NULL;
  size_t cap = 1024, n = 0;
  char *s = calloc(cap, 1);
  char line[65536];
  while (fgets(line, sizeof(line), f)) {
    if (line[0] == '%') continue;
    size_t l = strlen(line);
    while (l > 0 && (line[l - 1] == '\n' || line[l - 1] == '\r' || line[l - 1] == ' ' || line[l - 1] == '\t')) line[--l] = 0;
    if (n + l + 2 > cap) { cap = (n + l + 2) * 2; s = realloc(s, cap); }
    memcpy(s + n, line, l);
    n += l;
    s[n] = 0;
    if (n == 0 || s[n - 1] != ';') { s[n++] = ';'; s[n] = 0; }
  }
  fclose(f);
  return s;
}

static void usage(const char *prog, const char *seeds) {
  fprintf(stderr,
          "\nSToRM (B200 build)\n\nUSAGE: %s parameters\n\n"
          "Mandatory:\n  -g <genome_file>  reference (.fasta/.multifasta)\n"
          "  -r <reads_file>   reads (.fastq)\n\n"
          "Optional:\n  -s <seed list>  default: %s\n  -S <seed file>\n  -l <number>  repeat filter (stdev distance, <=0 disables)\n"
          "  -j  ignore lowercase   -F forward only   -R reverse only\n"
          "  -o <sam file>   -O <unmapped fastq>   -M <1..4>   -A\n"
          "  -m <match> -x <mismatch> -d <gap open> -e <gap extend> -i <indels>\n"
          "  -t <min score> -z <filter min score> -u <uniqueness> -b <quality base>\n"
          "  -v <verbosity>  -h\n", prog, seeds);
}

int storm_cli_main(int argc, char **argv, int colour, const storm_mapper *mapper) {
  const char *optstring = "g:r:q:s:S:a:b:f:p:m:x:d:e:t:z:T:i:v:o:O:l:u:M:N:jFRhcPHUGA";
  char *genome_file = NULL, *reads_file = NULL, *qual_file = NULL;
  char *single_read = NULL, *single_ref = NULL;
  int match = 5, mismatch = -4, gap_open = -9, gap_extend = -4;
  int allowed_indels = 3, simd_diags = 3, min_score = 115, min_score_filter = 100;
  int quality_base = 33, map_unordered = 0, print_all = 0, uniqueness = 0, uniq_thr = 0;
  int stdev = 100, ignore_lower = 0, senses = 3, map_greedy = 0;
  FILE *output = stdout, *unmapped = NULL;
  char *seeds = seeds_from_file(colour ? DEFAULT_SEED_FILE_COL : DEFAULT_SEED_FILE_NUC);
  if (!seeds) seeds = colour ? DEFAULT_SEEDS_COL : DEFAULT_SEEDS_NUC;
  int opt;
#define INTARG(v) do { if (sscanf(optarg, "%d", &(v)) != 1) { err("Mandatory numeric parameter missing for option %c.", opt); exit(1); } } while (0)
#define FATAL_VALUE(v, what) do { err("Invalid value %d for option %c. Expected: %s.", v, opt, what); exit(1); } while (0)
#define STRARG(t) do { if (strlen(optarg) == 2 && optarg[0] == '-' && optarg[1] != ':' && strchr(optstring, optarg[1])) { err("Mandatory parameter missing for option %c.", opt); exit(1); } t = optarg; } while (0)
  while ((opt = getopt(argc, argv, optstring)) != -1) {
    switch (opt) {
    case 'g':
      if (genome_file) { err("Genome file previously set with \"%s\".\nUnable to set it again.\n", genome_file); exit(1); }
      STRARG(genome_file);
      break;
    case 'r':
      if (reads_file) { err("Read file previously set with \"%s\".\nUnable to set it again.\n", reads_file); exit(1); }
      STRARG(reads_file);
      break;
    case 'q':
      if (qual_file) { err("Quality file previously set with \"%s\".\nUnable to set it again.\n", qual_file); exit(1); }
      STRARG(qual_file);
      break;
    case 'S': {
      char *t = seeds_from_file(optarg);
      if (!t) { err("Unable to read seeds input file %s.", optarg); exit(1); }
      seeds = t;
      break;
    }
    case 's': seeds = optarg; break;
    case 'm': INTARG(match); if (match <= 0) FATAL_VALUE(match, "a strictly positive integer"); break;
    case 'x': INTARG(mismatch); if (mismatch > 0) FATAL_VALUE(mismatch, "a negative value or zero"); break;
    case 'd': INTARG(gap_open); if (gap_open > 0) FATAL_VALUE(gap_open, "a negative value or zero"); break;
    case 'e': INTARG(gap_extend); if (gap_extend > 0) FATAL_VALUE(gap_extend, "a negative value or zero"); break;
    case 't': INTARG(min_score); break;
    case 'z': INTARG(min_score_filter); break;
    case 'b': INTARG(quality_base); break;
    case 'i':
      INTARG(allowed_indels);
      if (allowed_indels < 0) FATAL_VALUE(allowed_indels, "a positive value or zero");
      if (allowed_indels >= 16) {
        msg(1, "SToRM may not handle more than 15 indels in SIMD (local alignment) filter (16 diagonals).\n"
               "However final alignment does support this -i <%d> value...\n", allowed_indels);
        simd_diags = 15;
      } else simd_diags = allowed_indels;
      break;
    case 'a': single_read = optarg; break;
    case 'p': break;
    case 'f': single_ref = optarg; break;
    case 'o':
      if (!strcmp(optarg, "NULL") || !strcmp(optarg, "null")) output = NULL;
      else if (!(output = fopen(optarg, "w"))) { err("Could not open or create output file %s.\n", optarg); exit(1); }
      break;
    case 'O':
      if (!strcmp(optarg, "NULL") || !strcmp(optarg, "null")) unmapped = NULL;
      else if (!(unmapped = fopen(optarg, "w"))) { err("Could not open or create FASTQ output file %s.\n", optarg); exit(1); }
      break;
    case 'F': senses = 1; break;
    case 'R': senses = 2; break;
    case 'h': usage(argv[0], seeds); return 0;
    case 'G': map_greedy = 1; break;
    case 'M':
      INTARG(map_unordered);
      if (map_unordered <= 0) FATAL_VALUE(map_unordered, "a strictly positive integer");
      if (map_unordered > STORMGPU_MAP_DETAIL) FATAL_VALUE(map_unordered, "a value smaller than MAP_DETAIL_SIZE (4)");
      break;
    case 'A':
      if (!map_unordered) {
        err("The -A (output all reads in SAM) parameter is not available with the Ordered Mapping\n"
            "because not all mappable reads are already displayed in this mode.\n"
            "Please use the Unordered Mapping (-M <number>) before using -A.\n");
        exit(1);
      }
      print_all = 1;
      break;
    case 'v':
      INTARG(verbosity);
      if (verbosity < 0 || verbosity > 3) verbosity = 1;
      break;
    case 'P': case 'U': break;
    case 'H': { int w; INTARG(w); break; }
    case 'N': { int nt; INTARG(nt); if (nt <= 0) FATAL_VALUE(nt, "a strictly positive integer"); break; }
    case 'l':
      INTARG(stdev);
      if (stdev <= 0) stdev = 0;
      break;
    case 'j': ignore_lower = 1; break;
    case 'u':
      uniqueness = 1;
      INTARG(uniq_thr);
      if (uniq_thr <= 0) FATAL_VALUE(uniq_thr, "a positive integer");
      break;
    default:
      exit(1);
    }
  }
  (void)simd_diags;
  int delta_m = match - mismatch;
  if (single_read && single_ref) {
    err("The two-sequence alignment mode (-a/-f) is not part of this build.");
    exit(1);
  }
  if (!reads_file || !genome_file) {
    err("\nNot enough mandatory parameters provided.\n");
    usage(argv[0], seeds);
    return 0;
  }
  if (min_score < STORMGPU_MIN_SCORE) {
    err("-t below %d is not supported.", STORMGPU_MIN_SCORE);
    exit(1);
  }
  time_t t0 = time(NULL);
  stormgpu_params p;
  memset(&p, 0, sizeof(p));
  p.colour = colour;
  p.match = match; p.mismatch = mismatch; p.gap_open = gap_open; p.gap_extend = gap_extend;
  p.allowed_indels = allowed_indels; p.min_score = min_score; p.min_score_filter = min_score_filter;
  p.stdev_distance = stdev; p.senses = senses; p.device = 0;
  if (allowed_indels > STORMGPU_MAX_INDELS) { err("-i above %d is not supported.", STORMGPU_MAX_INDELS); exit(1); }

  /* the mapper's device set-up and the reference load run beside the reads load and sort;
   * errors are reported in the reference's order (reads first, run.c:812-835) */
  const double t_start = now_s();
  prep_job prep = {mapper, &p, seeds, 0.0};
  pthread_t prep_th, ref_th;
  const int prep_started = mapper->prepare && pthread_create(&prep_th, NULL, prep_job_run, &prep) == 0;
  ref_job rj;
  memset(&rj, 0, sizeof(rj));
  rj.path = genome_file;
  rj.colour = colour;
  rj.ignore_lower = ignore_lower;
  const int ref_started = pthread_create(&ref_th, NULL, ref_job_run, &rj) == 0;
  msg(1, "Loading reads database...\n");
  sh_reads reads;
  const int reads_rc = sh_load_reads(reads_file, qual_file, colour, quality_base, 1, &reads);
  char reads_msg[512];
  snprintf(reads_msg, sizeof(reads_msg), "%s", sh_last_error());
  const int reads_final = reads_rc != 0 && sh_last_error_final();
  const double t_reads = now_s();
  const int sort_rc = reads_rc == 0 ? sh_sort_reads(&reads) : 0;
  if (sort_rc != 0) snprintf(reads_msg, sizeof(reads_msg), "%s", sh_last_error());
  const double t_sort = now_s();
  if (ref_started) pthread_join(ref_th, NULL);
  else ref_job_run(&rj);
  if (reads_rc != 0 || sort_rc != 0) {
    err("%s", reads_msg);
    if (reads_rc == STORMGPU_ENOMEM || sort_rc == STORMGPU_ENOMEM) exit(1);  /* SAFE_FAILURE__ALLOC, util.h:70-80 */
    if (reads_final) exit(-1);  /* RETURN_INPUT_ERR from inside the loader */
    err("Reads could not be loaded. Exiting.");
    exit(-1);
  }
  msg(1, "Loaded %ld reads (read length %d..%d).\n", (long)reads.n, reads.min_len, reads.max_len);
  msg(1, "Loading reference database...\n");
  sh_refs refs = rj.refs;
  if (rj.rc != 0) {
    err("%s", rj.msg);
    if (rj.rc == STORMGPU_ENOMEM) exit(1);
    err("Reference could not be loaded. Exiting.");
    exit(-1);
  }
  msg(1, "Loaded %d reference sequence%s.\n", refs.n, refs.n == 1 ? "" : "s");
  if (prep_started) pthread_join(prep_th, NULL);
  msg(2, "Times: reads %.3f s, sort %.3f s, reference %.3f s (beside), device set-up %.3f s (beside).\n",
      t_reads - t_start, t_sort - t_reads, rj.seconds, prep.seconds);

  stormgpu_results res;
  res.tb_stride = ((reads.max_len + allowed_indels + 1) / 2 + 7) & ~7;
  res.hits = calloc((size_t)(reads.n ? reads.n : 1) * 4, sizeof(stormgpu_hit));
  res.tb = calloc((size_t)(reads.n ? reads.n : 1) * 4, (size_t)res.tb_stride);
  res.mapped = calloc((size_t)(reads.n ? reads.n : 1), 1);
  if (!res.hits || !res.tb || !res.mapped) {
    err("Not enough memory for the results of %ld reads.", (long)reads.n);
    exit(1);
  }
  sh_sam_opts so;
  memset(&so, 0, sizeof(so));
  so.colour = colour; so.max_rank = map_unordered; so.print_all = print_all;
  so.uniqueness = uniqueness; so.uniqueness_threshold = uniq_thr; so.min_score = min_score;
  so.delta_m = delta_m; so.quality_base = quality_base; so.argc = argc; so.argv = argv;
  static char obuf[1 << 22];
  if (map_unordered && output) setvbuf(output, obuf, _IOFBF, sizeof(obuf));

  /* with -M and a SAM file, a large read set maps in pieces and each piece's records are
   * written by a second thread while the next piece maps */
  int64_t pipe_min = SAM_PIPE_MIN_READS;  /* STORM_PIPE_MIN_READS lowers it (tests of small inputs) */
  if (getenv("STORM_PIPE_MIN_READS")) pipe_min = atoll(getenv("STORM_PIPE_MIN_READS"));
  const int pipelined = map_unordered && output && mapper->map_chunked && reads.n >= pipe_min && reads.n >= 2;
  sam_pipe pipe;
  pthread_t pipe_th;
  if (pipelined) {
    memset(&pipe, 0, sizeof(pipe));
    pthread_mutex_init(&pipe.mu, NULL);
    pthread_cond_init(&pipe.cv, NULL);
    pipe.f = output; pipe.so = &so; pipe.refs = &refs; pipe.reads = &reads; pipe.res = &res;
    if (pthread_create(&pipe_th, NULL, sam_pipe_run, &pipe) != 0) {
      err("Could not start the SAM output thread.");
      exit(1);
    }
  }
  char emsg[512] = {0};
  const double t_map = now_s();
  int rc = pipelined ? mapper->map_chunked(mapper->user, &p, seeds, &refs, &reads, &res,
                                           (reads.n + SAM_PIPE_PIECES - 1) / SAM_PIPE_PIECES, sam_pipe_push,
                                           &pipe, emsg, sizeof(emsg))
                     : mapper->map(mapper->user, &p, seeds, &refs, &reads, &res, emsg, sizeof(emsg));
  msg(2, "Times: index build and mapping %.3f s%s.\n", now_s() - t_map,
      pipelined ? " (SAM output of each piece beside the next)" : "");
  if (rc != 0 && pipelined) sam_pipe_finish(&pipe, pipe_th);
  if (rc == STORMGPU_EINVAL && strstr(emsg, "seed")) {
    err("The seed pattern is invalid: \"%s\".\nExpected: {0,1}+ or {-,#}+ with at least one '1'/'#' (seed separator ';').", seeds);
    exit(-1);
  }
  if (rc != 0) {
    err("Mapping failed (%s): %s", mapper->name, emsg);
    exit(2);
  }
  int64_t mapped = 0;
  for (int64_t r = 0; r < reads.n; ++r) mapped += res.mapped[r] != 0;
  msg(1, "\nAligned %ld of %ld reads (%5.2f%%) in %ld seconds.\n", (long)mapped, (long)reads.n,
      reads.n ? mapped * 100.0 / reads.n : 0.0, (long)(time(NULL) - t0));

  if (map_unordered) {
    if (output) {
      const double t_sam = now_s();
      if (pipelined) {
        sam_pipe_finish(&pipe, pipe_th);
        if (pipe.rc != 0) {
          err("%s", pipe.msg);
          exit(1);
        }
      } else if (sh_write_sam(output, &so, &refs, &reads, &res, 0, reads.n, 1) != 0) {
        err("%s", sh_last_error());
        exit(1);
      }
      fflush(output);
      msg(2, "Times: SAM output %.3f s%s.\n", now_s() - t_sam, pipelined ? " after the mapping" : "");
    } else {
      err("No file name provided for SAM output.");
    }
  } else {
    /* the per-position map (genome_map, run.c:1025-1061) */
    msg(1, "\n\nReference mapping...\n");
    sh_placement *pl = malloc(sizeof(sh_placement) * (size_t)(reads.n ? reads.n : 1));
    if (!pl) {
      err("Not enough memory for the placement of %ld reads.", (long)reads.n);
      exit(1);
    }
    int64_t npl = 0;
    const double t_place = now_s();
    if (map_greedy) {
      if (!mapper->place_greedy ||
          mapper->place_greedy(mapper->user, &refs, &res, reads.n, uniqueness ? uniq_thr : 0, pl, &npl, emsg,
                               sizeof(emsg)) != 0) {
        err("Mapping failed (%s): %s", mapper->name, emsg);
        exit(2);
      }
    } else if (mapper->place_contextual) {
      if (mapper->place_contextual(mapper->user, &refs, &res, reads.n, uniqueness, uniq_thr, pl, &npl, emsg,
                                   sizeof(emsg)) != 0) {
        err("Mapping failed (%s): %s", mapper->name, emsg);
        exit(2);
      }
    } else {
      sh_genome_map_contextual(&refs, &res, reads.n, colour, allowed_indels, match, mismatch, uniqueness, uniq_thr,
                               pl, &npl);
    }
    msg(2, "Times: placement of %ld reads %.3f s.\n", (long)npl, now_s() - t_place);
    if (output) {
      static char obuf2[1 << 22];
      setvbuf(output, obuf2, _IOFBF, sizeof(obuf2));
      const double t_sam = now_s();
      if (sh_write_genome_map_sam(output, &so, &refs, &reads, &res, pl, npl) != 0) {
        err("%s", sh_last_error());
        exit(1);
      }
      fflush(output);
      msg(2, "Times: SAM output %.3f s.\n", now_s() - t_sam);
    } else {
      err("No file name provided for SAM output.");
    }
    free(pl);
  }
  if (mapper->finish) mapper->finish(mapper->user);
  if (unmapped && sh_write_unmapped_fastq(unmapped, &so, &reads, &res) != 0) {
    err("%s", sh_last_error());
    exit(1);
  }
  if (output && output != stdout) fclose(output);
  if (unmapped) fclose(unmapped);
  free(res.hits); free(res.tb); free(res.mapped);
  sh_free_reads(&reads);
  sh_free_reference(&refs);
  return 0;
}
