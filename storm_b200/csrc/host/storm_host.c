/*
 * storm_host.c -- input loading, read ordering, SAM / FASTQ output (see storm_host.h).
 */
#include "storm_host.h"

#ifdef _OPENMP
#include <omp.h>
#endif

#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <sys/stat.h>
#include <unistd.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_err[512];  /* per thread: loads may run in parallel threads */
static __thread int g_err_final;   /* g_err is the reference's whole message before it exits */
const char *sh_last_error(void) { return g_err; }
int sh_last_error_final(void) { return g_err_final; }
static int fail(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  g_err_final = 0;
  return code;
}
/* "seams corrupt" at a line of a read file: the reference reports it and exits in the loader
 * (reads_data.c:429-432) */
static int fail_corrupt_line(int lineno) {
  snprintf(g_err, sizeof(g_err), "\nReads file seams corrupt at line %d. Exiting.\n", lineno);
  g_err_final = 1;
  return STORMGPU_EINVAL;
}

/* Quality levels (read_quality.h:83-91, read_quality.c:189-195) */
static const int LEVEL_UB[4] = {2, 7, 10, 93};
static inline int quality_level(int q) {
  int i = 0;
  while (i < 3 && LEVEL_UB[i] < q) ++i;
  return i;
}

/* inputs at least this large take the threaded paths of the loaders (a file read by ranges,
 * line starts and sequence measures by threads, a reference sequence filled by threads) */
static size_t g_parallel_min = (size_t)64 << 20;
void sh_set_parallel_min_bytes(size_t bytes) { g_parallel_min = bytes; }

static inline void put2(uint8_t *p, int64_t i, int v) {
  p[i >> 2] = (uint8_t)(p[i >> 2] | ((v & 3) << ((i & 3) << 1)));
}
static inline int get2(const uint8_t *p, int64_t i) { return (p[i >> 2] >> ((i & 3) << 1)) & 3; }

/* whole file in memory, NUL-terminated; one allocation of the file's size when it has one.
 * NULL when the file cannot be read; *oom is set when memory ran out. */
static char *slurp(const char *path, size_t *len, int *oom) {
  *oom = 0;
  FILE *f = fopen(path, "rb");
  if (!f) return NULL;
  struct stat st;
  size_t cap = 1 << 20, n = 0;
  /* one byte more than the file: the read that finds the end needs no larger buffer */
  if (fstat(fileno(f), &st) == 0 && S_ISREG(st.st_mode) && st.st_size > 0) cap = (size_t)st.st_size + 1;
  char *buf = malloc(cap + 1);
  if (!buf) { fclose(f); *oom = 1; return NULL; }
  if (cap > g_parallel_min && cap > 1) {
    /* a large regular file: the threads read equal ranges of it (the copy out of the page cache
     * and the buffer's first touch in parallel); the file's end is then confirmed as below */
    const size_t size = cap - 1;
    int nt = 1, bad = 0;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    if (nt > 64) nt = 64;
    const int fd = fileno(f);
#pragma omp parallel for schedule(static) num_threads(nt) reduction(|| : bad)
    for (int t = 0; t < nt; ++t) {
      size_t lo = size * (size_t)t / (size_t)nt;
      const size_t hi = size * (size_t)(t + 1) / (size_t)nt;
      while (lo < hi) {
        const ssize_t got = pread(fd, buf + lo, hi - lo, (off_t)lo);
        if (got <= 0) { bad = 1; break; }
        lo += (size_t)got;
      }
    }
    if (!bad && fseeko(f, (off_t)size, SEEK_SET) == 0) n = size;  /* else read it all again below */
    else rewind(f);
  }
  for (;;) {
    if (n == cap) {
      char *grown = realloc(buf, 2 * cap + 1);
      if (!grown) { free(buf); fclose(f); *oom = 1; return NULL; }
      buf = grown;
      cap *= 2;
    }
    size_t got = fread(buf + n, 1, cap - n, f);
    if (!got) break;
    n += got;
  }
  fclose(f);
  buf[n] = 0;
  *len = n;
  return buf;
}

static int read_failed(int oom, const char *path, const char *what) {
  if (oom) return fail(STORMGPU_ENOMEM, "Not enough memory to read %s (%s).", path, what);
  return fail(STORMGPU_EINVAL, "Failed to read input file %s (%s).", path, what);
}

/* ---------------------------------------------------------------------------- reference */

/* doubles the masked-region arrays; non-zero (arrays unchanged) when memory runs out */
static int grow_regions(int32_t **rs, int32_t **re, int32_t *cap) {
  int32_t *a = realloc(*rs, sizeof(int32_t) * (size_t)(2 * *cap));
  if (!a) return 1;
  *rs = a;
  int32_t *b = realloc(*re, sizeof(int32_t) * (size_t)(2 * *cap));
  if (!b) return 1;
  *re = b;
  *cap *= 2;
  return 0;
}

enum { REF_SPACE = 4, REF_HEADER = 5, REF_OTHER = 6 };

/* One reference sequence, the symbols of buf[p, q) (size of them not spaces), filled by threads
 * exactly as the one-pass loop of sh_load_reference fills it: every byte range counts its
 * symbols, masked symbols and last base first; the masked symbols' rand() & 3 codes are drawn
 * in order beforehand (nucleotide); the ranges then write their codes (whole bytes directly, the
 * bytes shared with a neighbour by atomic OR) and their masked runs, which are joined in order.
 * Symbol j is output position j, or j - 1 in colour space, where the first symbol only gives the
 * first base.  Returns 0, or 1 when memory runs out. */
typedef struct ref_range {
  size_t lo, hi;
  int64_t nsym, noth, nseg, sym0, oth0, seg0;
  int last, carry;  /* last base code of the range (-1: none); the code before the range */
} ref_range;

static int fill_sequence_threads(const char *buf, size_t p, size_t q, const uint8_t cls[256], int colour,
                                 int64_t size, uint8_t *cd, uint8_t *mk, uint8_t *first_base, int32_t **rs,
                                 int32_t **re, int32_t *rcap, int32_t *nr) {
  int nc = 1;
#ifdef _OPENMP
  nc = omp_get_max_threads();
#endif
  nc = nc < 1 ? 1 : nc > 256 ? 256 : nc;
  ref_range *rg = calloc((size_t)nc, sizeof(ref_range));
  if (!rg) return 1;
  for (int c = 0; c < nc; ++c) {
    rg[c].lo = p + (q - p) * (size_t)c / (size_t)nc;
    rg[c].hi = p + (q - p) * (size_t)(c + 1) / (size_t)nc;
  }
#pragma omp parallel for schedule(static) num_threads(nc)
  for (int c = 0; c < nc; ++c) {
    int64_t ns = 0, no = 0, nseg = 0;
    int last = -1, in_run = 0;
    for (size_t u = rg[c].lo; u < rg[c].hi; ++u) {
      const int k = cls[(unsigned char)buf[u]];
      if (k == REF_SPACE) continue;
      ns++;
      if (k == REF_OTHER) { no++; nseg += !in_run; in_run = 1; }
      else { last = k; in_run = 0; }
    }
    rg[c].nsym = ns; rg[c].noth = no; rg[c].nseg = nseg; rg[c].last = last;
  }
  int64_t sym = 0, oth = 0, seg = 0;
  int carry = 0;
  for (int c = 0; c < nc; ++c) {
    rg[c].sym0 = sym; rg[c].oth0 = oth; rg[c].seg0 = seg; rg[c].carry = carry;
    sym += rg[c].nsym; oth += rg[c].noth; seg += rg[c].nseg;
    if (rg[c].last >= 0) carry = rg[c].last;
  }
  uint8_t *rnd = colour || oth == 0 ? NULL : malloc((size_t)oth);
  int64_t *sj0 = malloc(sizeof(int64_t) * (size_t)(seg ? seg : 1)), *sj1 = malloc(sizeof(int64_t) * (size_t)(seg ? seg : 1));
  if ((!colour && oth && !rnd) || !sj0 || !sj1) { free(rnd); free(sj0); free(sj1); free(rg); return 1; }
  for (int64_t u = 0; rnd && u < oth; ++u) rnd[u] = (uint8_t)(rand() & 3);  /* in the loop's order */
#pragma omp parallel for schedule(static) num_threads(nc)
  for (int c = 0; c < nc; ++c) {
    int64_t j = rg[c].sym0, o = rg[c].oth0, sg = rg[c].seg0;
    int code_prev = rg[c].carry, in_run = 0;
    /* the output positions of the range: [ilo, ihi) */
    const int64_t ilo = colour ? (j > 0 ? j - 1 : 0) : j;
    const int64_t ihi = colour ? (j + rg[c].nsym > 0 ? j + rg[c].nsym - 1 : 0) : j + rg[c].nsym;
    int64_t cur = -1;
    unsigned cacc = 0, macc = 0;
#define SH_FLUSH()                                                                                 \
    do {                                                                                           \
      if (cur >= 0) {                                                                              \
        if (4 * cur >= ilo && 4 * cur + 4 <= ihi) cd[cur] = (uint8_t)cacc;                        \
        else if (cacc) __atomic_fetch_or(&cd[cur], (uint8_t)cacc, __ATOMIC_RELAXED);               \
        if (macc) __atomic_fetch_or(&mk[cur], (uint8_t)macc, __ATOMIC_RELAXED);                    \
      }                                                                                            \
    } while (0)
    for (size_t u = rg[c].lo; u < rg[c].hi; ++u) {
      const int k = cls[(unsigned char)buf[u]];
      if (k == REF_SPACE) continue;
      const int64_t i = colour ? (j > 0 ? j - 1 : 0) : j;
      if ((i >> 2) != cur) {
        SH_FLUSH();
        cur = i >> 2;
        cacc = macc = 0;
      }
      int code;
      if (k == REF_OTHER) {
        code = colour ? code_prev : rnd[o++];
        if (!in_run) { sj0[sg] = j; sj1[sg] = -1; sg++; in_run = 1; }
        macc |= 1u << ((i & 3) << 1);
      } else {
        code = k;
        if (in_run) { sj1[sg - 1] = j; in_run = 0; }
      }
      if (colour && j == 0) {
        *first_base = (uint8_t)code;
        code_prev = code;
        j++;
        continue;
      }
      cacc |= (unsigned)(colour ? code_prev ^ code : code) << ((i & 3) << 1);
      code_prev = code;
      j++;
    }
    SH_FLUSH();
#undef SH_FLUSH
  }
  /* the masked runs in order, a run open at the end of a range joined with the next range's */
  const int64_t total = sym;
  int64_t open = -1;
  int rc = 0;
  for (int c = 0; c < nc && !rc; ++c) {
    if (rg[c].nsym == 0) continue;
    int64_t s0 = rg[c].seg0, s1 = rg[c].seg0 + rg[c].nseg;
    int cont = open >= 0 && s0 < s1 && sj0[s0] == rg[c].sym0;
    if (open >= 0 && !cont) {
      const int64_t a = colour ? (open > 0 ? open - 1 : 0) : open, b = colour ? rg[c].sym0 - 1 : rg[c].sym0;
      if (*nr == *rcap && grow_regions(rs, re, rcap)) { rc = 1; break; }
      (*rs)[*nr] = (int32_t)a; (*re)[*nr] = (int32_t)b; (*nr)++;
      open = -1;
    }
    for (int64_t g = s0; g < s1; ++g) {
      const int64_t start = (g == s0 && cont) ? open : sj0[g];
      open = -1;
      if (sj1[g] < 0) { open = start; continue; }
      const int64_t a = colour ? (start > 0 ? start - 1 : 0) : start, b = colour ? sj1[g] - 1 : sj1[g];
      if (*nr == *rcap && grow_regions(rs, re, rcap)) { rc = 1; break; }
      (*rs)[*nr] = (int32_t)a; (*re)[*nr] = (int32_t)b; (*nr)++;
    }
  }
  if (!rc && open >= 0) {
    const int64_t a = colour ? (open > 0 ? open - 1 : 0) : open, b = colour ? (total > 0 ? total - 1 : 0) : total;
    if (*nr == *rcap && grow_regions(rs, re, rcap)) rc = 1;
    else { (*rs)[*nr] = (int32_t)a; (*re)[*nr] = (int32_t)b; (*nr)++; }
  }
  (void)size;
  free(rnd); free(sj0); free(sj1); free(rg);
  return rc;
}

/* reference_data.c:14-190: one FASTA chunk per '>' header; whitespace skipped; letters
 * upper-cased unless -j; non-ACGT letters are masked and coded rand()&3 (nucleotide) or as
 * the previous base (colour); colour space stores the XOR of consecutive bases and keeps
 * the first base apart; masked regions are the maximal runs of masked codes. */

/* Class of each input byte: 0-3 the base (upper-cased first unless -j), REF_SPACE (isspace),
 * REF_HEADER ('>'), REF_OTHER (masked). */
static void reference_classes(int ignore_lowercase, uint8_t cls[256]) {
  for (int c = 0; c < 256; ++c) {
    const int u = ignore_lowercase ? c : toupper(c);
    cls[c] = (uint8_t)(u == 'A' ? 0 : u == 'C' ? 1 : u == 'G' ? 2 : u == 'T' ? 3 : isspace(u) ? REF_SPACE
                       : u == '>' ? REF_HEADER : REF_OTHER);
  }
}

int sh_load_reference(const char *path, int colour, int ignore_lowercase, sh_refs *out) {
  memset(out, 0, sizeof(*out));
  uint8_t cls[256];
  reference_classes(ignore_lowercase, cls);
  size_t len;
  int oom;
  char *buf = slurp(path, &len, &oom);
  if (!buf) return read_failed(oom, path, "reference sequence");
  /* count chunks: lines starting with '>' (reference_data.c:210-220) */
  int nseq = len > 0 && buf[0] == '>';
#pragma omp parallel for schedule(static) reduction(+ : nseq) if (len > g_parallel_min)
  for (int64_t i = 1; i < (int64_t)len; ++i)
    if (buf[i] == '>' && buf[i - 1] == '\n') nseq++;
  int headerless = nseq == 0;
  if (headerless) nseq = 1;
  out->names = calloc((size_t)nseq, sizeof(char *));
  out->sizes = calloc((size_t)nseq, sizeof(int64_t));
  out->codes = calloc((size_t)nseq, sizeof(uint8_t *));
  out->masks = calloc((size_t)nseq, sizeof(uint8_t *));
  out->alloc_codes = calloc((size_t)nseq, sizeof(uint8_t *));
  out->alloc_masks = calloc((size_t)nseq, sizeof(uint8_t *));
  out->rs = calloc((size_t)nseq, sizeof(int32_t *));
  out->re = calloc((size_t)nseq, sizeof(int32_t *));
  out->nreg = calloc((size_t)nseq, sizeof(int32_t));
  out->first_base = calloc((size_t)nseq, 1);
  if (!out->names || !out->sizes || !out->codes || !out->masks || !out->alloc_codes || !out->alloc_masks ||
      !out->rs || !out->re || !out->nreg || !out->first_base) {
    free(buf);
    sh_free_reference(out);
    return fail(STORMGPU_ENOMEM, "Not enough memory for the reference sequences.");
  }
  size_t p = 0;
  int s;
  for (s = 0; s < nseq; ++s) {
    if (p >= len) break;
    /* header line */
    if (buf[p] == '>') {
      size_t e = p;
      while (e < len && buf[e] != '\n') e++;
      size_t nl = strcspn(buf + p + 1, " \r\n");
      if (nl > e - p - 1) nl = e - p - 1;
      if (nl == 0) { free(buf); return fail(STORMGPU_EINVAL, "Empty fasta header line in the reference sequence."); }
      out->names[s] = malloc(nl + 1);
      if (!out->names[s]) { free(buf); out->n = s; sh_free_reference(out); return fail(STORMGPU_ENOMEM, "Not enough memory for the reference sequences."); }
      memcpy(out->names[s], buf + p + 1, nl);
      out->names[s][nl] = 0;
      if (out->names[s][0] == '=' || out->names[s][0] == '*') out->names[s][0] = '-';
      p = (e < len) ? e + 1 : e;
    }
    /* measure: the symbols up to the next '>' that are not spaces */
    const char *hq = memchr(buf + p, '>', len - p);
    const size_t q = hq ? (size_t)(hq - buf) : len;
    int64_t size = 0;
#pragma omp parallel for schedule(static) reduction(+ : size) if (q - p > g_parallel_min)
    for (int64_t u = (int64_t)p; u < (int64_t)q; ++u) size += cls[(unsigned char)buf[u]] != REF_SPACE;
    if (size == 0) break; /* reference_data.c:67-70, load_reference_db:241-246 */
    int64_t nbytes = (size + 3) / 4 + 1;
    int64_t tot = nbytes + 2 * SH_PAD_BYTES;
    uint8_t *ca = calloc((size_t)tot, 1), *ma = calloc((size_t)tot, 1);
    int32_t rcap = 16, nr = 0;
    int32_t *rs = malloc(sizeof(int32_t) * (size_t)rcap), *re = malloc(sizeof(int32_t) * (size_t)rcap);
    if (!ca || !ma || !rs || !re) {
      free(ca); free(ma); free(rs); free(re); free(buf);
      out->n = s + 1;  /* the name of this sequence is freed with the others */
      sh_free_reference(out);
      return fail(STORMGPU_ENOMEM, "Not enough memory for the reference sequences.");
    }
    memset(ma, 0x55, SH_PAD_BYTES);
    uint8_t *cd = ca + SH_PAD_BYTES, *mk = ma + SH_PAD_BYTES;
    int64_t i = 0, mstart = -1;
    int code_prev = 0, have_first = 0;
    unsigned cacc = 0; /* the codes of the byte being filled */
    if (q - p > g_parallel_min) {
      if (fill_sequence_threads(buf, p, q, cls, colour, size, cd, mk, &out->first_base[s], &rs, &re, &rcap, &nr)) {
        free(ca); free(ma); free(rs); free(re); free(buf);
        out->n = s + 1;
        sh_free_reference(out);
        return fail(STORMGPU_ENOMEM, "Not enough memory for the reference sequences.");
      }
      i = colour ? (size > 0 ? size - 1 : 0) : size;
      p = q;
    }
    while (p < len) {
      const int k = cls[(unsigned char)buf[p]];
      if (k == REF_HEADER) break;
      p++;
      if (k == REF_SPACE) continue;
      int code;
      if (k == REF_OTHER) {
        code = colour ? code_prev : (rand() & 3);
        if (mstart == -1) mstart = i;
        put2(mk, i, 1);
      } else {
        code = k;
        if (mstart != -1) {
          if (nr == rcap && grow_regions(&rs, &re, &rcap)) {
            free(ca); free(ma); free(rs); free(re); free(buf);
            out->n = s + 1;
            sh_free_reference(out);
            return fail(STORMGPU_ENOMEM, "Not enough memory for the masked regions of the reference.");
          }
          rs[nr] = (int32_t)mstart; re[nr] = (int32_t)i; nr++;
          mstart = -1;
        }
      }
      if (colour && !have_first) {
        have_first = 1;
        code_prev = code;
        out->first_base[s] = (uint8_t)code;
        continue;
      }
      cacc |= (unsigned)(colour ? code_prev ^ code : code) << ((i & 3) << 1);
      if ((i & 3) == 3) { cd[i >> 2] = (uint8_t)cacc; cacc = 0; }
      i++;
      code_prev = code;
    }
    if ((i & 3) && cacc) cd[i >> 2] = (uint8_t)cacc;
    if (mstart != -1) {
      if (nr == rcap && grow_regions(&rs, &re, &rcap)) {
        free(ca); free(ma); free(rs); free(re); free(buf);
        out->n = s + 1;
        sh_free_reference(out);
        return fail(STORMGPU_ENOMEM, "Not enough memory for the masked regions of the reference.");
      }
      rs[nr] = (int32_t)mstart; re[nr] = (int32_t)i; nr++;
    }
    out->sizes[s] = i;
    /* mask the rest of the last byte and everything after (reference_data.c:183-188) */
    for (int64_t k = i; k & 3; ++k) put2(mk, k, 1);
    memset(mk + ((i + 3) >> 2), 0x55, (size_t)(tot - SH_PAD_BYTES - ((i + 3) >> 2)));
    out->alloc_codes[s] = ca; out->alloc_masks[s] = ma;
    out->codes[s] = cd; out->masks[s] = mk;
    out->rs[s] = rs; out->re[s] = re; out->nreg[s] = nr;
    if (headerless && s == 0 && out->names[s] == NULL) {
      fprintf(stderr, "No fasta header line in the reference sequence.\n");
    }
    if (i == 0) { s++; break; }
  }
  out->n = s;
  free(buf);
  if (out->n <= 0) return fail(STORMGPU_EINVAL, "Reference could not be loaded.");
  return 0;
}

void sh_free_reference(sh_refs *r) {
  for (int s = 0; s < r->n; ++s) {
    free(r->names ? r->names[s] : NULL);
    if (r->alloc_codes) free(r->alloc_codes[s]);
    if (r->alloc_masks) free(r->alloc_masks[s]);
    if (r->rs) free(r->rs[s]);
    if (r->re) free(r->re[s]);
  }
  free(r->names); free(r->sizes); free(r->codes); free(r->masks); free(r->alloc_codes);
  free(r->alloc_masks); free(r->rs); free(r->re); free(r->nreg); free(r->first_base);
  memset(r, 0, sizeof(*r));
}

/* ---------------------------------------------------------------------------- reads */

typedef struct growbuf { char *p; size_t n, cap; int oom; } growbuf;
static void gb_put(growbuf *g, const void *src, size_t n) {
  if (g->oom) return;
  if (g->n + n > g->cap) {
    const size_t cap = (g->n + n) * 2 + 4096;
    char *p = realloc(g->p, cap);
    if (!p) { g->oom = 1; return; }
    g->p = p;
    g->cap = cap;
  }
  memcpy(g->p + g->n, src, n);
  g->n += n;
}

typedef struct rawread {
  size_t name_off, seq_off, qual_off;
  int name_len, seq_len, qual_len;
  int has_qual;
} rawread;

/* doubles the raw-record array; non-zero (array unchanged) when memory runs out */
static int grow_raw(rawread **rr, int64_t *cap) {
  rawread *p = realloc(*rr, sizeof(rawread) * (size_t)(2 * *cap));
  if (!p) return 1;
  *rr = p;
  *cap *= 2;
  return 0;
}

/* reads_data.c:538-564: printable common prefix of the first and last read names */
static char *common_name(const char *a, const char *b) {
  int l = 0, t = 0;
  while (a[l] && b[l] && a[l] == b[l]) {
    char c = a[l];
    if ((t == 0 && ((c >= '!' && c <= ')') || (c >= '+' && c <= '<') || (c >= '>' && c <= '~'))) ||
        (t > 0 && c >= '!' && c <= '~'))
      t = l + 1;
    l++;
  }
  if (t <= 0) return NULL;
  char *s = malloc((size_t)t + 1);
  memcpy(s, a, (size_t)t);
  s[t] = 0;
  return s;
}

static int next_line(const char *buf, size_t len, size_t *pos, const char **line, size_t *ll) {
  if (*pos >= len) return 0;
  size_t s = *pos;
  const char *nl = memchr(buf + s, '\n', len - s);
  size_t e = nl ? (size_t)(nl - buf) : len;
  *line = buf + s;
  *ll = e - s;  /* without '\n' */
  *pos = (e < len) ? e + 1 : e;
  return 1;
}

/* name of a header line: after the marker, up to the first char outside '!'..'~' or '@',
 * at most 255 chars (reads_data.c:466-478) */
static int header_name_len(const char *line, size_t ll) {
  int n = 1;
  while ((size_t)n < ll && (signed char)line[n] > ' ' && (signed char)line[n] <= '~' && line[n] != '@') {
    n++;
    if (n >= 256) break;
  }
  return n - 1;
}

/* Read i of the batch (its raw record r) into out: name, codes, tag, qualities.  Returns 0, or
 * STORMGPU_EINVAL for a negative quality value, with the message only when `report` is set.
 * qv: scratch of maxl + 2 shorts. */
static int fill_one(sh_reads *out, const char *buf, const rawread *r, int64_t i, int colour, int quality_base,
                    int any_qual, int maxl, short *qv, int report) {
  out->file_index[i] = i;
  out->names[i] = out->arena + r->name_off;  /* NUL-terminated in the arena by fill_reads */
  const char *sq = buf + r->seq_off;
  int L = r->seq_len - (colour ? 2 : 0);
  out->lengths[i] = (int16_t)L;
  uint8_t *cd = out->codes + i * out->code_stride;
  if (!colour) {
    for (int k = 0; k < L; ++k) {
      char c = sq[k];
      put2(cd, k, c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : c == 'T' ? 3 : 0);
    }
  } else {
    /* reads_data.c:488-491: real first base = TRANSFORM(primer, first colour) */
    int c0 = sq[0];
    int b = ((c0 & 0x4) >> 1) | (((c0 & 0x4) >> 2) ^ ((c0 & 0x2) >> 1));
    out->first_base[i] = (uint8_t)((b ^ (sq[1] & 3)) & 3);
    for (int k = 0; k < L; ++k) put2(cd, k, sq[k + 2] & 3);
  }
  /* tag: maximum of the rolling 64-bit window, codes remapped to a,t,g,c order */
  uint64_t tag = 0, ct = 0;
  for (int k = 0; k < L; ++k) {
    ct = (ct << 2) | (uint64_t)((((unsigned)get2(cd, k) + 1) & 3) ^ 1);
    if (ct > tag) tag = ct;
  }
  out->tags[i] = tag;
  if (any_qual && r->has_qual) {
    const char *ql = buf + r->qual_off;
    int qlen = r->qual_len;
    memset(qv, 0, sizeof(short) * ((size_t)maxl + 2));
    if (colour) {
      int v = (int)(signed char)(qlen > 0 ? ql[0] : '\n') - quality_base;
      if (v < 0) return report ? fail(STORMGPU_EINVAL, "Quality level char induces a negative value (read #%ld).", (long)i + 1) : STORMGPU_EINVAL;
      out->first_level[i] = (uint8_t)quality_level(v > 93 ? 93 : v);
    }
    int lim = L < qlen ? L : qlen;
    for (int k = colour ? 1 : 0; k < lim; ++k) {
      int v = (int)(signed char)ql[k] - quality_base;
      if (v < 0) return report ? fail(STORMGPU_EINVAL, "Quality level char \"%c\" induces a negative value (read #%ld).", ql[k], (long)i + 1) : STORMGPU_EINVAL;
      qv[k] = (short)(v > 93 ? 93 : v);
    }
    uint8_t *lv = out->levels + i * out->level_stride;
    /* colour: level of colour k is the quality of file colour k+1 (compress shift 1); the
     * last one reads one past the parsed qualities, which is 0 (read_quality.c:31-41) */
    for (int k = 0; k < L; ++k) put2(lv, k, quality_level(colour ? (k + 1 < L ? qv[k + 1] : 0) : qv[k]));
  } else if (any_qual) {
    /* a record without its quality line (the file's last, cut short): the reference keeps a NULL
     * quality for it (reads_data.c:479), aligned at level 3 (alignment.c:157-160) */
    uint8_t *lv = out->levels + i * out->level_stride;
    for (int k = 0; k < L; ++k) put2(lv, k, 3);
    out->first_level[i] = 3;
    out->no_quality[i] = 1;
  }
  return 0;
}

/* buf: the loaded text, which becomes the reads' name arena (each name is NUL-terminated in
 * place: the byte after a name is a separator of its header line, read by nothing later). */
static int fill_reads(sh_reads *out, char *buf, rawread *rr, int64_t n, int colour,
                      int quality_base, int allow_mixed, int any_qual) {
  int minl = 1 << 30, maxl = 0;
  for (int64_t i = 0; i < n; ++i) {
    int L = rr[i].seq_len - (colour ? 2 : 0);
    if (L <= 0) return fail(STORMGPU_EINVAL, "Reads file seams corrupt: the read #%ld length is %d.", (long)i + 1, L);
    if (L > STORMGPU_MAX_READ_LEN) return fail(STORMGPU_EINVAL, "Read #%ld is longer than %d.", (long)i + 1, STORMGPU_MAX_READ_LEN);
    if (L < minl) minl = L;
    if (L > maxl) maxl = L;
  }
  if (!allow_mixed && n && minl != maxl)
    return fail(STORMGPU_EINVAL, "The reads do not all have the same length (%d..%d). All the reads must be of equal length for the parallel processing.", minl, maxl);
  out->n = n;
  out->colour = colour;
  out->min_len = n ? minl : 0;
  out->max_len = n ? maxl : 0;
  out->has_quality = any_qual;
  out->code_stride = ((maxl + 3) / 4 + 7) & ~7;
  out->level_stride = out->code_stride;
  out->codes = calloc((size_t)(n ? n : 1), (size_t)out->code_stride);
  out->levels = any_qual ? calloc((size_t)(n ? n : 1), (size_t)out->level_stride) : NULL;
  out->lengths = calloc((size_t)(n ? n : 1), sizeof(int16_t));
  out->tags = calloc((size_t)(n ? n : 1), sizeof(uint64_t));
  out->names = calloc((size_t)(n ? n : 1), sizeof(char *));
  out->first_base = calloc((size_t)(n ? n : 1), 1);
  out->first_level = calloc((size_t)(n ? n : 1), 1);
  out->file_index = calloc((size_t)(n ? n : 1), sizeof(int64_t));
  out->arena = buf;
  if (!out->codes || (any_qual && !out->levels) || !out->lengths || !out->tags || !out->names || !out->first_base ||
      !out->first_level || !out->file_index)
    return fail(STORMGPU_ENOMEM, "Not enough memory for %ld reads.", (long)n);
  if (any_qual) {
    int64_t missing = 0;
    for (int64_t i = 0; i < n; ++i) missing += !rr[i].has_qual;
    if (missing && !(out->no_quality = calloc((size_t)n, 1)))
      return fail(STORMGPU_ENOMEM, "Not enough memory for %ld reads.", (long)n);
  }
  for (int64_t i = 0; i < n; ++i) buf[rr[i].name_off + (size_t)rr[i].name_len] = 0;
  /* reads are independent: filled in parallel; the first failing read (in file order) is filled
   * again alone to report its message, as a sequential pass would */
  int64_t first_bad = n;
  int nomem = 0;
#pragma omp parallel reduction(|| : nomem)
  {
    short *qv = calloc((size_t)maxl + 2, sizeof(short));
    if (!qv) nomem = 1;
#pragma omp for schedule(static) reduction(min : first_bad)
    for (int64_t i = 0; i < n; ++i)
      if (qv && fill_one(out, buf, &rr[i], i, colour, quality_base, any_qual, maxl, qv, 0)) first_bad = i < first_bad ? i : first_bad;
    free(qv);
  }
  if (nomem) return fail(STORMGPU_ENOMEM, "Not enough memory for %ld reads.", (long)n);
  if (first_bad < n) {
    short *qv = calloc((size_t)maxl + 2, sizeof(short));
    if (!qv) return fail(STORMGPU_ENOMEM, "Not enough memory for %ld reads.", (long)n);
    const int rc = fill_one(out, buf, &rr[first_bad], first_bad, colour, quality_base, any_qual, maxl, qv, 1);
    free(qv);
    return rc;
  }
  return 0;
}

/* The start of every line of buf[from, len), as next_line walks them (a line after each '\n'
 * that is not the buffer's last byte), found by the threads over equal byte ranges.  Returns 0,
 * or 1 when memory runs out. */
static int line_starts(const char *buf, size_t len, size_t from, size_t **out, int64_t *n_out) {
  *out = NULL;
  *n_out = 0;
  if (from >= len) return 0;
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  if (len - from < g_parallel_min / 64) nt = 1;
  if (nt > 256) nt = 256;
  int64_t cnt[257] = {0};
  /* '\n' at p, with p + 1 < len, in thread t's range [lo, hi) */
#define SH_RANGE(t, lo, hi)                                                   \
  const size_t lo = from + (len - from) * (size_t)(t) / (size_t)nt;          \
  const size_t hi = from + (len - from) * (size_t)((t) + 1) / (size_t)nt;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int t = 0; t < nt; ++t) {
    SH_RANGE(t, lo, hi)
    int64_t c = 0;
    for (const char *p = buf + lo, *e = buf + hi; (p = memchr(p, '\n', (size_t)(e - p))) != NULL; ++p)
      if ((size_t)(p - buf) + 1 < len) c++;
    cnt[t + 1] = c;
  }
  for (int t = 0; t < nt; ++t) cnt[t + 1] += cnt[t];
  const int64_t n = 1 + cnt[nt];
  size_t *ls = malloc(sizeof(size_t) * (size_t)n);
  if (!ls) return 1;
  ls[0] = from;
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int t = 0; t < nt; ++t) {
    SH_RANGE(t, lo, hi)
    int64_t k = 1 + cnt[t];
    for (const char *p = buf + lo, *e = buf + hi; (p = memchr(p, '\n', (size_t)(e - p))) != NULL; ++p)
      if ((size_t)(p - buf) + 1 < len) ls[k++] = (size_t)(p - buf) + 1;
  }
#undef SH_RANGE
  *out = ls;
  *n_out = n;
  return 0;
}

static int load_fastq(const char *path, int colour, int quality_base, int allow_mixed, sh_reads *out) {
  size_t len;
  int oom;
  memset(out, 0, sizeof(*out));
  char *buf = slurp(path, &len, &oom);
  if (!buf) return read_failed(oom, path, "read sequences");
  size_t pos = 0;
  const char *line;
  size_t ll;
  char *title = NULL;
  /* leading comments (reads_data.c:374-392) */
  size_t rec_start = 0;
  int lineno = 0;
  while (1) {
    rec_start = pos;
    if (!next_line(buf, len, &pos, &line, &ll)) { free(buf); return fail(STORMGPU_EINVAL, "Failed to read input file %s (read sequences) first line.", path); }
    if (ll >= 9 && !title && strncmp(line, "# Title: ", 9) == 0) {
      size_t nl = strcspn(line + 9, "\r\n");
      if (nl > ll - 9) nl = ll - 9;
      title = malloc(nl + 1);
      if (!title) { free(buf); return fail(STORMGPU_ENOMEM, "Not enough memory to read %s.", path); }
      memcpy(title, line + 9, nl);
      title[nl] = 0;
    }
    if (ll > 0 && line[0] == '#') { lineno++; continue; }
    break;
  }
  /* the lines from rec_start: their starts found in parallel, then the record structure in one
   * pass over them (the reference's line types and its error line numbers), then each record's
   * name and sequence lengths in parallel */
  size_t *ls = NULL;
  int64_t nl = 0;
  if (line_starts(buf, len, rec_start, &ls, &nl)) { free(buf); free(title); return fail(STORMGPU_ENOMEM, "Not enough memory to read %s.", path); }
  int64_t cap = nl / 4 + 2, n = 0;
  rawread *rr = malloc(sizeof(rawread) * (size_t)cap);
  if (!rr) { free(ls); free(buf); free(title); return fail(STORMGPU_ENOMEM, "Not enough memory to read %s.", path); }
  int any_qual = 0;
  int state = 0; /* 0 header, 1 seq, 2 plus, 3 qual */
  const size_t last_end = len > 0 && buf[len - 1] == '\n' ? len - 1 : len;
  for (int64_t i = 0; i < nl; ++i) {
    line = buf + ls[i];
    ll = (i + 1 < nl ? ls[i + 1] - 1 : last_end) - ls[i];  /* without '\n' */
    size_t l2 = ll;
    while (l2 > 0 && line[l2 - 1] == '\r') l2--;
    if (state == 0) {
      if (ll == 0 || line[0] != '@') { free(ls); free(rr); free(buf); free(title); return fail_corrupt_line(lineno + 1); }
      if (n == cap && grow_raw(&rr, &cap)) { free(ls); free(rr); free(buf); free(title); return fail(STORMGPU_ENOMEM, "Not enough memory to read %s.", path); }
      rr[n].name_off = ls[i] + 1;
      rr[n].name_len = (int)(l2 < INT32_MAX ? l2 : INT32_MAX);  /* the header's length for now */
      rr[n].has_qual = 0;
      rr[n].qual_len = 0;
      state = 1;
    } else if (state == 1) {
      if (ll == 0) { free(ls); free(rr); free(buf); free(title); return fail_corrupt_line(lineno + 1); }
      rr[n].seq_off = ls[i];
      rr[n].seq_len = (int)(ll < INT32_MAX ? ll : INT32_MAX);  /* the line's length for now */
      n++;
      state = 2;
    } else if (state == 2) {
      if (ll == 0 || line[0] != '+') { free(ls); free(rr); free(buf); free(title); return fail_corrupt_line(lineno + 1); }
      state = 3;
    } else {
      rr[n - 1].qual_off = ls[i];
      rr[n - 1].qual_len = (int)l2;
      rr[n - 1].has_qual = 1;
      any_qual = 1;
      state = 0;
    }
    lineno++;
  }
  free(ls);
  /* the name: after the '@', up to the first char outside '!'..'~' or '@' (at most 255); the
   * sequence: up to the first '\r' (or the line's end) */
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    rr[i].name_len = header_name_len(buf + rr[i].name_off - 1, (size_t)rr[i].name_len);
    const size_t sl = strcspn(buf + rr[i].seq_off, "\r\n");
    if (sl < (size_t)rr[i].seq_len) rr[i].seq_len = (int)sl;
  }
  if (n == 0) { free(rr); free(buf); free(title); return fail(STORMGPU_EINVAL, "Reads could not be loaded."); }
  int rc = fill_reads(out, buf, rr, n, colour, quality_base, allow_mixed, any_qual);
  if (rc == 0) {
    if (title) out->db_name = title;
    else out->db_name = common_name(out->names[0], out->names[n - 1]);
  } else {
    free(title);
    if (!out->arena) free(buf);
    sh_free_reads(out);
  }
  free(rr);
  return rc;
}

/* FASTA reads, or CSFASTA (a primer base, then colours) with an optional quality file of
 * space-separated integers (reads_data.c:73-345).  After leading '#' comments (a "# Title: "
 * names the read set), a record is a '>' header and one or more sequence lines; a header not
 * followed by sequence lines leaves its name to the next record (the reference overwrites it).
 * Quality lines are the quality file's lines that are neither comments nor headers, one per read
 * in order; a short line keeps the values of the previous read for the missing positions (the
 * reference parses into one buffer reused across reads, load_data.c:15-33). */
/* The quality file of a FASTA / CSFASTA read set (reads_data.c:73-345): its lines that are
 * neither empty, comments nor headers, one per read in order, each a list of integers split on
 * spaces; a short line keeps, for the positions it lacks, the values of the reads before it (the
 * reference parses into one buffer kept across reads, load_data.c:15-33).  Lines are found and
 * parsed by threads, the positions a short line lacks then taken from the latest read before it
 * that had them, and the levels written by threads.  out->levels is allocated (zeroed).  Returns
 * 0, or 1 when memory runs out. */
static int parse_quality_lines(const char *qb, size_t qlen, int colour, sh_reads *out, int64_t n) {
  if (!out->levels) return 1;
  size_t *qls = NULL;
  int64_t nql = 0;
  if (line_starts(qb, qlen, 0, &qls, &nql)) return 1;
  const size_t qend = qlen > 0 && qb[qlen - 1] == '\n' ? qlen - 1 : qlen;
  int64_t *keep = malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
  if (!keep) { free(qls); return 1; }
  int64_t nq = 0;
  size_t maxll = 0;
  for (int64_t t = 0; t < nql && nq < n; ++t) {
    const char *line = qb + qls[t];
    const size_t ll = (t + 1 < nql ? qls[t + 1] - 1 : qend) - qls[t];
    if (ll == 0 || line[0] == '\r' || line[0] == '#' || line[0] == '>') continue;
    keep[nq++] = t;
    if (ll > maxll) maxll = ll;
  }
  const int need = out->max_len + (colour ? 1 : 0);
  short *pv = malloc(sizeof(short) * (size_t)(nq ? nq : 1) * (size_t)(need ? need : 1));
  int *pc = malloc(sizeof(int) * (size_t)(nq ? nq : 1));
  int nomem = !pv || !pc;
#pragma omp parallel reduction(|| : nomem)
  {
    char *tmp = nomem ? NULL : malloc(maxll + 1);
    if (!tmp) nomem = 1;
#pragma omp for schedule(static)
    for (int64_t i = 0; i < nq; ++i) {
      if (!tmp) continue;
      const int64_t t = keep[i];
      const size_t ll = (t + 1 < nql ? qls[t + 1] - 1 : qend) - qls[t];
      memcpy(tmp, qb + qls[t], ll);
      tmp[ll] = 0;
      const int want = out->lengths[i] + (colour ? 1 : 0);
      short *row = pv + (size_t)i * (size_t)need;
      char *save = NULL, *tok = strtok_r(tmp, " ", &save);
      int j = 0;
      for (; j < want && tok; ++j, tok = strtok_r(NULL, " ", &save)) row[j] = (short)atoi(tok);
      pc[i] = j;
    }
    free(tmp);
  }
  int64_t short_lines = 0;
  for (int64_t i = 0; !nomem && i < nq; ++i) short_lines += pc[i] < out->lengths[i] + (colour ? 1 : 0);
  if (!nomem && short_lines) {
    /* the positions a short line lacks: the buffer's value then, the reads replayed in order */
    short *qv = calloc((size_t)need + 1, sizeof(short));
    if (!qv) nomem = 1;
    for (int64_t i = 0; qv && i < nq; ++i) {
      const int want = out->lengths[i] + (colour ? 1 : 0);
      short *row = pv + (size_t)i * (size_t)need;
      for (int j = pc[i]; j < want; ++j) row[j] = qv[j];
      memcpy(qv, row, sizeof(short) * (size_t)pc[i]);
    }
    free(qv);
  }
  if (!nomem) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < nq; ++i) {
      const int L = out->lengths[i];
      const short *row = pv + (size_t)i * (size_t)need;
      uint8_t *lv = out->levels + i * out->level_stride;
      if (colour) out->first_level[i] = (uint8_t)quality_level(row[0]);
      for (int k = 0; k < L; ++k) put2(lv, k, quality_level(row[k + (colour ? 1 : 0)]));
    }
  }
  free(pv); free(pc); free(keep); free(qls);
  return nomem;
}

static int load_fasta(const char *path, const char *qual_path, int colour, int allow_mixed, sh_reads *out) {
  size_t len;
  int oom;
  memset(out, 0, sizeof(*out));
  char *buf = slurp(path, &len, &oom);
  if (!buf) return read_failed(oom, path, "read sequences");
  size_t pos = 0;
  const char *line;
  size_t ll;
  char *title = NULL;
  size_t rec_start = 0;
  while (1) {
    rec_start = pos;
    if (!next_line(buf, len, &pos, &line, &ll)) { free(buf); return fail(STORMGPU_EINVAL, "Failed to read input file %s (read sequences) first line.", path); }
    if (ll >= 9 && !title && strncmp(line, "# Title: ", 9) == 0) {
      size_t nl = strcspn(line + 9, "\r\n");
      if (nl > ll - 9) nl = ll - 9;
      title = malloc(nl + 1);
      if (!title) { free(buf); return fail(STORMGPU_ENOMEM, "Not enough memory to read %s.", path); }
      memcpy(title, line + 9, nl);
      title[nl] = 0;
    }
    if (ll > 0 && line[0] == '#') continue;
    break;
  }
  pos = rec_start;
  /* sequences may span lines: gather each record's sequence into one contiguous copy */
  growbuf seq = {0};
  int64_t cap = 1 << 16, n = 0;
  rawread *rr = malloc(sizeof(rawread) * (size_t)cap);
  if (!rr) { free(buf); free(title); return fail(STORMGPU_ENOMEM, "Not enough memory to read %s.", path); }
  size_t name_off = 0;
  int name_len = -1;
  int in_seq = 0;
  while (next_line(buf, len, &pos, &line, &ll)) {
    size_t l2 = ll;
    while (l2 > 0 && (line[l2 - 1] == '\r' || line[l2 - 1] == '\n')) l2--;
    const int type = ll == 0 || line[0] == '\r' ? 0 : line[0] == '#' ? 0 : line[0] == '>' ? 1 : 2;
    if (type == 2 && name_len >= 0) {
      if (!in_seq) {
        if (n == cap && grow_raw(&rr, &cap)) {
          free(rr); free(buf); free(seq.p); free(title);
          return fail(STORMGPU_ENOMEM, "Not enough memory to read %s.", path);
        }
        rr[n].name_off = name_off;
        rr[n].name_len = name_len;
        rr[n].seq_off = seq.n;
        rr[n].seq_len = 0;
        rr[n].has_qual = 0;
        rr[n].qual_len = 0;
        n++;
        in_seq = 1;
      }
      gb_put(&seq, line, l2);
      rr[n - 1].seq_len += (int)l2;
    } else {
      in_seq = 0;
      if (type == 1) {
        name_off = (size_t)(line - buf) + 1;
        name_len = header_name_len(line, l2);
      }
    }
  }
  if (n == 0) { free(rr); free(buf); free(seq.p); free(title); return fail(STORMGPU_EINVAL, "Reads could not be loaded."); }
  /* names live in buf, sequences in seq: copy the names next to the sequences, each followed by
   * a byte for its terminating NUL */
  for (int64_t i = 0; i < n; ++i) {
    const size_t o = seq.n;
    gb_put(&seq, buf + rr[i].name_off, (size_t)rr[i].name_len + 1);
    rr[i].name_off = o;
  }
  if (seq.oom) {
    free(rr); free(buf); free(seq.p); free(title);
    return fail(STORMGPU_ENOMEM, "Not enough memory to read %s.", path);
  }
  int rc = fill_reads(out, seq.p, rr, n, colour, 33, allow_mixed, 0);
  if (rc && !out->arena) free(seq.p);
  seq.p = NULL;
  if (rc == 0 && qual_path) {
    size_t qlen;
    char *qb = slurp(qual_path, &qlen, &oom);
    if (!qb) rc = read_failed(oom, qual_path, "quality of read sequences");
    else {
      out->has_quality = 1;
      out->levels = calloc((size_t)n, (size_t)out->level_stride);
      rc = parse_quality_lines(qb, qlen, colour, out, n) ? fail(STORMGPU_ENOMEM, "Not enough memory to read %s.", qual_path) : 0;
      free(qb);
    }
  }
  if (rc == 0) {
    if (title) out->db_name = title;
    else out->db_name = common_name(out->names[0], out->names[n - 1]);
  } else {
    free(title);
    sh_free_reads(out);
  }
  free(rr);
  free(buf);
  return rc;
}

int sh_load_reads(const char *path, const char *qual_path, int colour, int quality_base,
                  int allow_mixed, sh_reads *out) {
  const char *dot = strrchr(path, '.');
  if (dot && (!strcmp(dot, ".fastq") || !strcmp(dot, ".fq") || !strcmp(dot, ".fastq2") || !strcmp(dot, ".fq2")))
    return load_fastq(path, colour, quality_base, allow_mixed, out);
  return load_fasta(path, qual_path, colour, allow_mixed, out);
}

void sh_free_reads(sh_reads *r) {
  free(r->arena);
  free(r->names); free(r->codes); free(r->levels); free(r->lengths); free(r->tags);
  free(r->first_base); free(r->first_level); free(r->file_index); free(r->db_name); free(r->no_quality);
  memset(r, 0, sizeof(*r));
}

/* ---------------------------------------------------------------------------- ordering */

/* order: length, then tag, then file position */
typedef struct sortkey { uint64_t tag; uint32_t idx; uint16_t len; } sortkey;

/* One stable counting pass on digit d (8 bits) of every key, from `a` into `b`: each thread
 * counts its contiguous block, the counts are laid out bucket-major (bucket, thread), and every
 * thread scatters its block in order, so equal digits keep their order. */
static void radix_pass(const sortkey *a, sortkey *b, int64_t n, int d, int nt, int64_t *cnt) {
#define SK_DIGIT(x) (d < 8 ? (int)(((x).tag >> (8 * d)) & 0xff) : (int)(((x).len >> (8 * (d - 8))) & 0xff))
  memset(cnt, 0, sizeof(int64_t) * 256 * (size_t)nt);
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num();
    const int64_t lo = n * t / nt, hi = n * (t + 1) / nt;
    int64_t *c = cnt + 256 * t;
    for (int64_t i = lo; i < hi; ++i) c[SK_DIGIT(a[i])]++;
#pragma omp barrier
#pragma omp single
    {
      int64_t acc = 0;
      for (int v = 0; v < 256; ++v)
        for (int u = 0; u < nt; ++u) {
          const int64_t x = cnt[256 * u + v];
          cnt[256 * u + v] = acc;
          acc += x;
        }
    }
    for (int64_t i = lo; i < hi; ++i) b[c[SK_DIGIT(a[i])]++] = a[i];
  }
#undef SK_DIGIT
}

/* reads_data.c:59-67 (a stable sort by tag) per read length, lengths ascending: a stable LSD
 * radix sort on (length, tag) from file order, 8-bit digits, parallel passes; digits that are
 * the same for every read are skipped.  The read arrays are then permuted in parallel.
 * Returns 0, or STORMGPU_ENOMEM (reads unchanged). */
int sh_sort_reads(sh_reads *r) {
  const int64_t n = r->n;
  if (n <= 1) return 0;
  if (n > (int64_t)UINT32_MAX) return fail(STORMGPU_EINVAL, "More than %u reads in one file.", UINT32_MAX);
  int nt = 1;
#ifdef _OPENMP
  nt = omp_get_max_threads();
#endif
  if (nt > 64) nt = 64;
  if (n < 65536) nt = 1;
  sortkey *k = malloc(sizeof(sortkey) * (size_t)n), *t = malloc(sizeof(sortkey) * (size_t)n);
  int64_t *cnt = malloc(sizeof(int64_t) * 256 * (size_t)nt);
  uint8_t *codes = malloc((size_t)n * (size_t)r->code_stride);
  uint8_t *levels = r->levels ? malloc((size_t)n * (size_t)r->level_stride) : NULL;
  int16_t *lengths = malloc(sizeof(int16_t) * (size_t)n);
  uint64_t *tags = malloc(sizeof(uint64_t) * (size_t)n);
  char **names = malloc(sizeof(char *) * (size_t)n);
  uint8_t *fb = malloc((size_t)n), *fl = malloc((size_t)n);
  uint8_t *nq = r->no_quality ? malloc((size_t)n) : NULL;
  int64_t *fi = malloc(sizeof(int64_t) * (size_t)n);
  if (!k || !t || !cnt || !codes || (r->levels && !levels) || !lengths || !tags || !names || !fb || !fl || !fi ||
      (r->no_quality && !nq)) {
    free(k); free(t); free(cnt); free(codes); free(levels); free(lengths); free(tags); free(names);
    free(fb); free(fl); free(fi); free(nq);
    return fail(STORMGPU_ENOMEM, "Not enough memory to sort %ld reads.", (long)n);
  }
  uint64_t vt = 0;
  uint16_t vl = 0;
#pragma omp parallel for schedule(static) reduction(| : vt, vl) num_threads(nt)
  for (int64_t i = 0; i < n; ++i) {
    k[i].tag = r->tags[i];
    k[i].len = (uint16_t)r->lengths[i];
    k[i].idx = (uint32_t)i;
    vt |= r->tags[i] ^ r->tags[0];
    vl |= (uint16_t)(r->lengths[i] ^ r->lengths[0]);
  }
  for (int d = 0; d < 10; ++d) {
    const int varies = d < 8 ? ((vt >> (8 * d)) & 0xff) != 0 : ((vl >> (8 * (d - 8))) & 0xff) != 0;
    if (!varies) continue;
    radix_pass(k, t, n, d, nt, cnt);
    sortkey *sw = k; k = t; t = sw;
  }
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t i = 0; i < n; ++i) {
    const int64_t s = k[i].idx;
    memcpy(codes + i * r->code_stride, r->codes + s * r->code_stride, (size_t)r->code_stride);
    if (levels) memcpy(levels + i * r->level_stride, r->levels + s * r->level_stride, (size_t)r->level_stride);
    lengths[i] = r->lengths[s]; tags[i] = r->tags[s]; names[i] = r->names[s];
    fb[i] = r->first_base[s]; fl[i] = r->first_level[s]; fi[i] = r->file_index[s];
    if (nq) nq[i] = r->no_quality[s];
  }
  free(r->codes); free(r->levels); free(r->lengths); free(r->tags); free(r->names);
  free(r->first_base); free(r->first_level); free(r->file_index); free(r->no_quality);
  r->codes = codes; r->levels = levels; r->lengths = lengths; r->tags = tags; r->names = names;
  r->first_base = fb; r->first_level = fl; r->file_index = fi; r->no_quality = nq;
  free(k); free(t); free(cnt);
  return 0;
}

void sh_reads_view(const sh_reads *r, stormgpu_reads *v) {
  v->n = r->n;
  v->codes = r->codes;
  v->code_stride = r->code_stride;
  v->levels = r->levels;
  v->level_stride = r->level_stride;
  v->lengths = r->lengths;
  v->first_levels = r->colour ? r->first_level : NULL;
}

/* ---------------------------------------------------------------------------- SAM */

static inline int tb_get(const uint8_t *t, int i) { return (t[i >> 1] >> ((i & 1) ? 0 : 4)) & 0xF; }

/* alignment.c:749-887 */
int sh_traceback_to_cigar(const uint8_t *tb, int tb_len, const uint8_t *ref, int64_t ref_start,
                          int colour, int ref_start_symbol, char *cigar, char *seq) {
  int edit = 0, span = colour ? 1 : 0, prev = 0x3, slen = 0;
  int64_t ri = 0;
  int ref_hist = 0, read_hist = 0;
  char *cp = cigar;
  *cp = 0;
  uint8_t sq[2 * STORMGPU_MAX_READ_LEN + 8];
  if (colour) sq[slen++] = 0;
  for (int i = 0; i < tb_len; ++i) {
    int cell = tb_get(tb, i);
    int type;
    if ((cell & 0xC) == 0x4) type = 0x4;
    else if (colour && (cell & 0xC) == 0x8) type = 0x8;
    else if ((cell & 0xC) == 0xC) type = 0xC;
    else type = cell;
    int code = cell & 3;
    switch (type) {
    case 0x3:
      edit--;
      if (!colour) code = get2(ref, ref_start + ri);
      /* fall through */
    case 0x4:
      edit++;
      if (colour) {
        ref_hist ^= get2(ref, ref_start + ri);
        code = ref_hist ^ read_hist;
      }
      sq[slen++] = (uint8_t)code;
      if (colour) read_hist ^= code;
      ri++;
      break;
    case 0x8:
      if (colour) {
        edit++;
        sq[slen++] = (uint8_t)code;
        read_hist ^= code;
        ref_hist ^= get2(ref, ref_start + ri);
        ri++;
      }
      break;
    case 0xC:
      edit++;
      sq[slen++] = (uint8_t)code;
      if (colour) read_hist ^= code;
      break;
    case 0x1:
      edit++;
      if (colour) ref_hist ^= get2(ref, ref_start + ri);
      ri++;
      break;
    default:
      break;
    }
    int crt = (type == 0x1 || type == 0xC) ? type : 0x3;
    if (crt == prev) span++;
    else {
      if (span) cp += sprintf(cp, "%d%c", span, prev == 0x3 ? 'M' : prev == 0xC ? 'I' : prev == 0x1 ? 'D' : '?');
      span = 1;
      prev = crt;
    }
  }
  if (span) sprintf(cp, "%d%c", span, prev == 0x3 ? 'M' : prev == 0xC ? 'I' : prev == 0x1 ? 'D' : '?');
  static const char B[4] = {'A', 'C', 'G', 'T'};
  if (!colour) {
    for (int u = 0; u < slen; ++u) seq[u] = B[sq[u] & 3];
  } else {
    int c = ref_start_symbol;
    for (int u = 0; u < slen; ++u) { c = (c ^ sq[u]) & 3; seq[u] = B[c]; }
  }
  seq[slen] = 0;
  return edit;
}

/* hit_map.c:384-403 */
int sh_mapq(int rank, int score0, int score1, int score_rank, int min_score, int delta_m) {
  double n;
  if (rank == 0) {
    int s2 = score1 > min_score ? score1 : min_score;
    n = (double)(score0 - s2) / (double)delta_m;
  } else {
    n = (double)(score_rank - score0) / (double)delta_m;
  }
  int mapq = (int)(-4.343 * (n * log(.3)));
  mapq = (int)(mapq - 4.343 * log(.3));
  if (mapq < 0) mapq = 0;
  if (mapq > 254) mapq = 254;
  return mapq;
}

/* whether read r's record had qualities (the reference writes "*", or the maximal quality in
 * the unmapped FASTQ, for a read whose quality is NULL) */
static inline int has_quality(const sh_reads *reads, int64_t r) {
  return reads->levels && !(reads->no_quality && reads->no_quality[r]);
}

/* base of sequence s at position pos in colour space, from its first base and colours */

typedef struct colour_cursor { int seq; int64_t pos; int base; } colour_cursor;

/* colour space: base of each sequence at every multiple of SYM_STEP positions (the first
 * base transformed by the colours before it), so that a record's reference base needs at most
 * SYM_STEP - 1 more steps */
#define SYM_STEP 64
static uint8_t **symbol_checkpoints(const sh_refs *refs) {
  uint8_t **chk = calloc((size_t)refs->n, sizeof(uint8_t *));
  if (!chk) return NULL;
  for (int s = 0; s < refs->n; ++s) {
    const int64_t nck = refs->sizes[s] / SYM_STEP + 2;
    chk[s] = malloc((size_t)nck);
    if (!chk[s]) {
      for (int t = 0; t < s; ++t) free(chk[t]);
      free(chk);
      return NULL;
    }
    int b = refs->first_base[s];
    for (int64_t p = 0, k = 0; k < nck; ++k) {
      chk[s][k] = (uint8_t)b;
      for (int64_t e = (k + 1) * SYM_STEP; p < e && p < refs->sizes[s]; ++p) b ^= get2(refs->codes[s], p);
    }
  }
  return chk;
}

static int symbol_at(const sh_refs *refs, uint8_t *const *chk, int s, int64_t pos) {
  const int64_t ck = pos / SYM_STEP;
  int b = chk[s][ck];
  for (int64_t p = ck * SYM_STEP; p < pos && p < refs->sizes[s]; ++p) b ^= get2(refs->codes[s], p);
  return b & 3;
}

/* decimal text of v at p (as printf's %ld); returns the end */
static inline char *put_long(char *p, long v) {
  char t[24];
  int k = 0;
  unsigned long u = v < 0 ? 0ul - (unsigned long)v : (unsigned long)v;
  do { t[k++] = (char)('0' + u % 10); u /= 10; } while (u);
  if (v < 0) *p++ = '-';
  while (k) *p++ = t[--k];
  return p;
}
static inline char *put_str(char *p, const char *s) {
  const size_t n = strlen(s);
  memcpy(p, s, n);
  return p + n;
}

/* the records of reads [first, first + count) (hit_map.c:197-504); a mapped record's line is
 * formatted in a buffer (the fields of the reference's fprintf, hit_map.c:291-340) and written
 * at once.  Returns 0, or STORMGPU_ENOMEM when a line buffer cannot be allocated. */
static int write_sam_records(FILE *f, const sh_sam_opts *o, const sh_refs *refs, const sh_reads *reads,
                              const stormgpu_results *res, int64_t first, int64_t count, uint8_t *const *chk) {
  const int colour = o->colour;
  char cigar[4 * STORMGPU_MAX_READ_LEN + 64], seq[2 * STORMGPU_MAX_READ_LEN + 8];
  static const char B[4] = {'A', 'C', 'G', 'T'};
  char *qbuf = malloc((size_t)reads->max_len + 8);
  size_t lcap = 4096;
  char *line = malloc(lcap);
  if (!qbuf || !line) { free(qbuf); free(line); return STORMGPU_ENOMEM; }
  for (int64_t r = first; r < first + count; ++r) {
    const stormgpu_hit *h = &res->hits[r * 4];
    int L = reads->lengths[r];
    if (res->mapped[r]) {
      int M = o->max_rank;
#define REPORTABLE(k) ((k) < M && h[k].ref_start != -1 && \
   ((o->uniqueness == 0) || (((k) + 1 < M) && ((h[k].score - h[(k) + 1].score) >= o->uniqueness_threshold)) || ((k) + 1 == M)))
      int nrep = 0;
      for (int k = 0; REPORTABLE(k); ++k) nrep++;
      for (int k = 0; REPORTABLE(k); ++k) {
        int rev = (h[k].sense & 2) != 0;  /* sense is +1/-1; -1 & ALIGNMENT_SENSE_REVERSE */
        int flag = (rev ? 0x10 : 0) | (k ? 0x100 : 0);
        int ref_id = h[k].ref_id;
        int64_t ref_start = h[k].ref_start;
        int mapq = sh_mapq(k, h[0].score, h[1].score, h[k].score, o->min_score, o->delta_m);
        int sym = 0;
        if (colour) {
          sym = symbol_at(refs, chk, ref_id, ref_start >= 0 ? ref_start : 0);
        }
        int ed = sh_traceback_to_cigar(res->tb + (size_t)(r * 4 + k) * (size_t)res->tb_stride, h[k].tb_len,
                                       refs->codes[ref_id], ref_start, colour, sym, cigar, seq);
        const char *rname = refs->names[ref_id] ? refs->names[ref_id] : "*";
        const size_t need = strlen(reads->names[r]) + strlen(rname) + strlen(cigar) + strlen(seq) + (size_t)L + 160;
        if (need > lcap) {
          char *grown = realloc(line, 2 * need);
          if (!grown) { free(line); free(qbuf); return STORMGPU_ENOMEM; }
          line = grown;
          lcap = 2 * need;
        }
        char *p = line;
        p = put_str(p, reads->names[r]); *p++ = '\t';
        p = put_long(p, flag); *p++ = '\t';
        p = put_str(p, rname); *p++ = '\t';
        p = put_long(p, (long)(ref_start + 1)); *p++ = '\t';
        p = put_long(p, mapq); *p++ = '\t';
        p = put_str(p, cigar);
        p = put_str(p, "\t*\t0\t0\t");
        p = put_str(p, seq); *p++ = '\t';
        if (has_quality(reads, r)) {
          const uint8_t *lv = reads->levels + r * reads->level_stride;
          if (rev) {
            for (int q = L - 1; q >= 0; --q) { int c = o->quality_base + LEVEL_UB[get2(lv, q)]; *p++ = (char)(c < 126 ? c : 126); }
            if (colour) { int c = o->quality_base + LEVEL_UB[reads->first_level[r]]; *p++ = (char)(c < 126 ? c : 126); }
          } else {
            if (colour) { int c = o->quality_base + LEVEL_UB[reads->first_level[r]]; *p++ = (char)(c < 126 ? c : 126); }
            for (int q = 0; q < L; ++q) { int c = o->quality_base + LEVEL_UB[get2(lv, q)]; *p++ = (char)(c < 126 ? c : 126); }
          }
        } else {
          *p++ = '*';
        }
        p = put_str(p, "\tAS:i:"); p = put_long(p, h[k].score);
        p = put_str(p, "\tNM:i:"); p = put_long(p, ed);
        p = put_str(p, "\tNH:i:"); p = put_long(p, nrep);
        *p++ = '\n';
        fwrite(line, 1, (size_t)(p - line), f);
      }
#undef REPORTABLE
    } else if (o->print_all) {
      if (colour) {
        fprintf(f, "%s\t4\t*\t0\t255\t*\t*\t0\t0\t*\t*\n", reads->names[r]);
      } else {
        fprintf(f, "%s\t4\t*\t0\t255\t*\t*\t0\t0\t", reads->names[r]);
        const uint8_t *cd = reads->codes + r * reads->code_stride;
        for (int q = 0; q < L; ++q) qbuf[q] = B[get2(cd, q)];
        fwrite(qbuf, 1, (size_t)L, f);
        fputc('\t', f);
        if (has_quality(reads, r)) {
          const uint8_t *lv = reads->levels + r * reads->level_stride;
          for (int q = 0; q < L; ++q) { int c = o->quality_base + LEVEL_UB[get2(lv, q)]; qbuf[q] = (char)(c < 126 ? c : 126); }
          fwrite(qbuf, 1, (size_t)L, f);
        } else fputc('*', f);
        fputc('\n', f);
      }
    }
  }
  free(line);
  free(qbuf);
  return 0;
}

int sh_write_sam(FILE *f, const sh_sam_opts *o, const sh_refs *refs, const sh_reads *reads,
                 const stormgpu_results *res, int64_t first, int64_t count, int header) {
  const int colour = o->colour;
  if (header) {
    fprintf(f, "@HD\tVN:1.4\tSO:unsorted\n");
    for (int s = 0; s < refs->n; ++s)
      fprintf(f, "@SQ\tSN:%s\tLN:%ld\n", refs->names[s] ? refs->names[s] : "*",
              (long)(refs->sizes[s] + (colour ? 1 : 0)));
    const char *rg = reads->db_name ? reads->db_name : "*";
    fprintf(f, "@RG\tID:%s\tSM:%s\n", rg, rg);
    fprintf(f, "@PG\tID:%s\tVN:%s\tCL:\"", "SToRM", "0.0101");
    for (int i = 0; i < o->argc; ++i) fprintf(f, "%s ", o->argv[i]);
    fprintf(f, "\"\n");
  }
  /* records formatted in chunks, several chunks at once, written in read order */
  uint8_t **chk = colour ? symbol_checkpoints(refs) : NULL;
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  int64_t CH = count / (4 * (int64_t)nthreads);
  CH = CH < 256 ? 256 : CH > 16384 ? 16384 : CH;
  const int64_t per_round = CH * nthreads * 2;
  char **bufs = calloc((size_t)nthreads * 2, sizeof(char *));
  size_t *lens = calloc((size_t)nthreads * 2, sizeof(size_t));
  int nomem = !bufs || !lens || (colour && !chk);
  for (int64_t lo = first; !nomem && lo < first + count; lo += per_round) {
    const int64_t hi = lo + per_round < first + count ? lo + per_round : first + count;
    const int nchunks = (int)((hi - lo + CH - 1) / CH);
#pragma omp parallel for schedule(dynamic, 1) reduction(|| : nomem)
    for (int c = 0; c < nchunks; ++c) {
      const int64_t a = lo + (int64_t)c * CH, e = a + CH < hi ? a + CH : hi;
      FILE *m = open_memstream(&bufs[c], &lens[c]);
      if (!m) { nomem = 1; continue; }
      if (write_sam_records(m, o, refs, reads, res, a, e - a, chk)) nomem = 1;
      fclose(m);
    }
    for (int c = 0; c < nchunks; ++c) {
      if (!nomem) fwrite(bufs[c], 1, lens[c], f);
      free(bufs[c]);
      bufs[c] = NULL;
    }
  }
  free(bufs);
  free(lens);
  if (chk) {
    for (int s = 0; s < refs->n; ++s) free(chk[s]);
    free(chk);
  }
  if (nomem) return fail(STORMGPU_ENOMEM, "Out of memory while writing the SAM output.");
  return 0;
}

/* hit_map.c:514-579 */
/* ------------------------------------------------------------------------------ genome_map */

#define GM_CODES 4                 /* BASE_CODE_COUNT / COLOR_CODE_COUNT (codes.h:25-29) */
#define GM_NO_CODE GM_CODES        /* genome_map.c:26 */
#define GM_BLOCK 4096

/* 6-bit counters, one per code and the no-code symbol, packed in 32 bits (genome_map.c:37-48) */
static inline int gm_get(uint32_t c, int code) { return (int)((c >> (code * 6)) & 0x3F); }
static inline uint32_t gm_inc(uint32_t c, int code) {
  const uint32_t v = (uint32_t)((gm_get(c, code) + 1) & 0x3F);
  return (c & ~(0x3Fu << (code * 6))) | (v << (code * 6));
}

/* per-position data, created lazily in blocks of GM_BLOCK positions */
typedef struct gm_block {
  uint8_t created[GM_BLOCK];
  uint32_t aligned[GM_BLOCK];
  uint32_t *inserted;  /* indels * GM_BLOCK */
} gm_block;

typedef struct gm_map {
  int nref, indels;
  int64_t *npos;
  gm_block ***blocks;
} gm_map;

static gm_block *gm_block_of(gm_map *m, int ref, int64_t pos, int create) {
  gm_block **b = &m->blocks[ref][pos / GM_BLOCK];
  if (!*b && create) {
    *b = calloc(1, sizeof(gm_block));
    if (m->indels) (*b)->inserted = calloc((size_t)m->indels * GM_BLOCK, sizeof(uint32_t));
  }
  return *b;
}

/* genome_map__create_position_data */
static void gm_create(gm_map *m, int ref, int64_t pos) {
  gm_block *b = gm_block_of(m, ref, pos, 1);
  b->created[pos % GM_BLOCK] = 1;
}

/* genome_map__get_direct_consensus_code (genome_map.c:312-337) */
static int gm_consensus(gm_map *m, int ref, int64_t pos, int offset, int ref_code) {
  gm_block *b = gm_block_of(m, ref, pos, 0);
  if (!b || !b->created[pos % GM_BLOCK]) return ref_code;
  const uint32_t counts = offset < 0 ? b->aligned[pos % GM_BLOCK]
                                     : b->inserted[(size_t)offset * GM_BLOCK + (size_t)(pos % GM_BLOCK)];
  int best = ref_code;
  for (int i = 0; i <= GM_CODES; ++i)
    if (gm_get(counts, i) > gm_get(counts, best)) best = i;
  if (gm_get(counts, best) == 0) best = GM_NO_CODE;
  return best;
}

/* genome_map__update_consensus_code (genome_map.c:346-356) */
static void gm_update(gm_map *m, int ref, int64_t pos, int offset, int code) {
  gm_create(m, ref, pos);
  gm_block *b = gm_block_of(m, ref, pos, 0);
  if (offset >= 0) {
    uint32_t *c = &b->inserted[(size_t)offset * GM_BLOCK + (size_t)(pos % GM_BLOCK)];
    *c = gm_inc(*c, code);
  } else {
    b->aligned[pos % GM_BLOCK] = gm_inc(b->aligned[pos % GM_BLOCK], code);
  }
}

/* GET_PAIR_TYPE (alignment.h:87-94) */
static inline int pair_type(int code, int colour) {
  if ((code & 0xC) == 0x4) return 0x4;
  if (colour && (code & 0xC) == 0x8) return 0x8;
  if ((code & 0xC) == 0xC) return 0xC;
  return code;
}

/* genome_map__compute_adjusted_score (genome_map.c:366-424) */
static int gm_adjusted(gm_map *m, const sh_refs *refs, const stormgpu_hit *h, const uint8_t *tb, int colour,
                       int match, int mismatch) {
  if (h->ref_start == -1) return STORMGPU_MIN_SCORE;
  int score = 0, indel = 0, ref = h->ref_id;
  int64_t pos = h->ref_start;
  for (int i = 0; i < h->tb_len; ++i) {
    const int cell = tb_get(tb, i);
    switch (pair_type(cell, colour)) {
    case 0x3: {
      const int rc = get2(refs->codes[ref], pos);
      score += rc == gm_consensus(m, ref, pos, -1, rc) ? match : mismatch;
      ++pos;
      indel = 0;
      break;
    }
    case 0x1:
      score += gm_consensus(m, ref, pos, -1, GM_NO_CODE) == GM_NO_CODE ? match : mismatch;
      ++pos;
      indel = 0;
      break;
    case 0x4:
    case 0x8: {
      const int c = cell & 3;
      score += c == gm_consensus(m, ref, pos, -1, c) ? match : mismatch;
      ++pos;
      indel = 0;
      break;
    }
    case 0xC: {
      const int c = cell & 3;
      score += c == gm_consensus(m, ref, pos, indel, c) ? match : mismatch;
      ++indel;
      break;
    }
    default:
      break;
    }
  }
  return score;
}

int sh_genome_map_contextual(const sh_refs *refs, const stormgpu_results *res, int64_t n, int colour, int indels,
                             int match, int mismatch, int uniqueness, int uniqueness_threshold,
                             sh_placement *out, int64_t *n_out) {
  *n_out = 0;
  gm_map m;
  m.nref = refs->n;
  m.indels = indels;
  m.npos = calloc((size_t)refs->n, sizeof(int64_t));
  m.blocks = calloc((size_t)refs->n, sizeof(gm_block **));
  for (int s = 0; s < refs->n; ++s) {
    m.npos[s] = refs->sizes[s] + 1;  /* GENOME_MAP_SIZE */
    m.blocks[s] = calloc((size_t)(m.npos[s] / GM_BLOCK + 1), sizeof(gm_block *));
  }
  /* mapped reads in read order, then a stable sort by descending unsigned best score
   * (genome_map.c:233-299: 4-bit digits, bucket 15 - digit) */
  int64_t nm = 0;
  for (int64_t r = 0; r < n; ++r) nm += res->mapped[r] != 0;
  int32_t *idx = malloc(sizeof(int32_t) * (size_t)(nm ? nm : 1)), *tmp = malloc(sizeof(int32_t) * (size_t)(nm ? nm : 1));
  for (int64_t r = 0, j = 0; r < n; ++r)
    if (res->mapped[r]) idx[j++] = (int32_t)r;
  for (int d = 0; d < 8; ++d) {
    int64_t count[16] = {0}, index[16];
    for (int64_t j = 0; j < nm; ++j) count[15 - (((uint32_t)res->hits[(int64_t)idx[j] * 4].score >> (4 * d)) & 15)]++;
    index[0] = 0;
    for (int b = 1; b < 16; ++b) index[b] = index[b - 1] + count[b - 1];
    for (int64_t j = 0; j < nm; ++j)
      tmp[index[15 - (((uint32_t)res->hits[(int64_t)idx[j] * 4].score >> (4 * d)) & 15)]++] = idx[j];
    int32_t *sw = tmp; tmp = idx; idx = sw;
  }
  for (int64_t j = 0; j < nm; ++j) {
    const int64_t r = idx[j];
    const stormgpu_hit *h = &res->hits[r * 4];
    int adj[STORMGPU_MAP_DETAIL];
    for (int k = 0; k < STORMGPU_MAP_DETAIL; ++k) adj[k] = STORMGPU_MIN_SCORE;
    int best_rank = -1, best = STORMGPU_MIN_SCORE;
    for (int k = 0; k < STORMGPU_MAP_DETAIL && h[k].ref_start != -1; ++k) {
      adj[k] = gm_adjusted(&m, refs, &h[k], res->tb + (size_t)(r * 4 + k) * (size_t)res->tb_stride, colour, match,
                           mismatch);
      if (adj[k] > best) { best = adj[k]; best_rank = k; }
    }
    if (best_rank < 0 || (uniqueness && !(adj[0] - adj[1] > uniqueness_threshold))) continue;
    const stormgpu_hit *b = &h[best_rank];
    const int ref = b->ref_id;
    int64_t pos = b->ref_start;
    gm_create(&m, ref, pos);
    out[(*n_out)++] = (sh_placement){(int32_t)r, best_rank};
    const uint8_t *tb = res->tb + (size_t)(r * 4 + best_rank) * (size_t)res->tb_stride;
    int insertions = -1;
    for (int k = 0; k < b->tb_len; ++k) {
      const int cell = tb_get(tb, k);
      switch (pair_type(cell, colour)) {
      case 0xC: insertions++; gm_update(&m, ref, pos, insertions, cell & 3); break;
      case 0x3: insertions = -1; gm_update(&m, ref, pos, -1, get2(refs->codes[ref], pos)); break;
      case 0x4: insertions = -1; gm_update(&m, ref, pos, -1, cell & 3); break;
      case 0x1: insertions = -1; gm_update(&m, ref, pos, -1, GM_NO_CODE); break;
      case 0x8: insertions = -1; gm_update(&m, ref, pos, -1, cell & 3); break;
      default: break;
      }
      for (int p = insertions + 1; p < indels; ++p) gm_update(&m, ref, pos, p, GM_NO_CODE);
      if (insertions < 0) pos++;
    }
  }
  free(idx);
  free(tmp);
  for (int s = 0; s < refs->n; ++s) {
    for (int64_t k = 0; k <= m.npos[s] / GM_BLOCK; ++k)
      if (m.blocks[s][k]) { free(m.blocks[s][k]->inserted); free(m.blocks[s][k]); }
    free(m.blocks[s]);
  }
  free(m.blocks);
  free(m.npos);
  sh_sort_placements(res, out, *n_out);
  return 0;
}

typedef struct { int32_t ref; int64_t pos; int64_t seq; sh_placement p; } gm_key;
static int gm_key_cmp(const void *a, const void *b) {
  const gm_key *x = a, *y = b;
  if (x->ref != y->ref) return x->ref < y->ref ? -1 : 1;
  if (x->pos != y->pos) return x->pos < y->pos ? -1 : 1;
  return x->seq < y->seq ? -1 : x->seq > y->seq;
}

void sh_sort_placements(const stormgpu_results *res, sh_placement *pl, int64_t n) {
  if (n <= 1) return;
  gm_key *k = malloc(sizeof(gm_key) * (size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    const stormgpu_hit *h = &res->hits[(int64_t)pl[i].read * 4 + pl[i].rank];
    k[i] = (gm_key){h->ref_id, h->ref_start, i, pl[i]};
  }
  qsort(k, (size_t)n, sizeof(gm_key), gm_key_cmp);
  for (int64_t i = 0; i < n; ++i) pl[i] = k[i].p;
  free(k);
}

/* the records of placements [first, first + count) (genome_map.c:551-796): each line formatted
 * in a buffer (the fields of the reference's fprintf) and written at once.  In colour space the
 * reference's running reference symbol (the first base transformed by every colour before the
 * start; placements come in (sequence, position) order) is the symbol at the start.  Returns 0,
 * or STORMGPU_ENOMEM when a line buffer cannot be allocated. */
static int write_placement_records(FILE *f, const sh_sam_opts *o, const sh_refs *refs, const sh_reads *reads,
                                   const stormgpu_results *res, const sh_placement *pl, int64_t first,
                                   int64_t count, uint8_t *const *chk) {
  const int colour = o->colour;
  char cigar[4 * STORMGPU_MAX_READ_LEN + 64], seq[2 * STORMGPU_MAX_READ_LEN + 8];
  size_t lcap = 4096;
  char *line = malloc(lcap);
  if (!line) return STORMGPU_ENOMEM;
  for (int64_t i = first; i < first + count; ++i) {
    const int64_t r = pl[i].read;
    const int k = pl[i].rank;
    const stormgpu_hit *h = &res->hits[r * 4];
    const int ref = h[k].ref_id;
    const int64_t start = h[k].ref_start;
    const int sym = colour ? symbol_at(refs, chk, ref, start) : 0;
    const int rev = (h[k].sense & 2) != 0;
    const int mapq = sh_mapq(k, h[0].score, h[1].score, h[k].score, o->min_score, o->delta_m);
    const int ed = sh_traceback_to_cigar(res->tb + (size_t)(r * 4 + k) * (size_t)res->tb_stride, h[k].tb_len,
                                         refs->codes[ref], start, colour, sym, cigar, seq);
    const char *rname = refs->names[ref] ? refs->names[ref] : "*";
    const int L = reads->lengths[r];
    const size_t need = strlen(reads->names[r]) + strlen(rname) + strlen(cigar) + strlen(seq) + (size_t)L + 160;
    if (need > lcap) {
      char *grown = realloc(line, 2 * need);
      if (!grown) { free(line); return STORMGPU_ENOMEM; }
      line = grown;
      lcap = 2 * need;
    }
    char *p = line;
    p = put_str(p, reads->names[r]); *p++ = '\t';
    p = put_long(p, rev ? 0x10 : 0); *p++ = '\t';
    p = put_str(p, rname); *p++ = '\t';
    p = put_long(p, (long)(start + 1)); *p++ = '\t';
    p = put_long(p, mapq); *p++ = '\t';
    p = put_str(p, cigar);
    p = put_str(p, "\t*\t0\t0\t");
    p = put_str(p, seq); *p++ = '\t';
    if (has_quality(reads, r)) {
      const uint8_t *lv = reads->levels + r * reads->level_stride;
      if (rev) {
        for (int q = L - 1; q >= 0; --q) { int c = o->quality_base + LEVEL_UB[get2(lv, q)]; *p++ = (char)(c < 126 ? c : 126); }
        if (colour) { int c = o->quality_base + LEVEL_UB[reads->first_level[r]]; *p++ = (char)(c < 126 ? c : 126); }
      } else {
        if (colour) { int c = o->quality_base + LEVEL_UB[reads->first_level[r]]; *p++ = (char)(c < 126 ? c : 126); }
        for (int q = 0; q < L; ++q) { int c = o->quality_base + LEVEL_UB[get2(lv, q)]; *p++ = (char)(c < 126 ? c : 126); }
      }
    } else {
      *p++ = '*';
    }
    p = put_str(p, "\tAS:i:"); p = put_long(p, h[k].score);
    p = put_str(p, "\tNM:i:"); p = put_long(p, ed);
    *p++ = '\n';
    fwrite(line, 1, (size_t)(p - line), f);
  }
  free(line);
  return 0;
}

int sh_write_genome_map_sam(FILE *f, const sh_sam_opts *o, const sh_refs *refs, const sh_reads *reads,
                            const stormgpu_results *res, const sh_placement *pl, int64_t n_pl) {
  const int colour = o->colour;
  fprintf(f, "@HD\tVN:1.4\tSO:coordinate\n");
  for (int s = 0; s < refs->n; ++s)
    fprintf(f, "@SQ\tSN:%s\tLN:%ld\n", refs->names[s] ? refs->names[s] : "*", (long)(refs->sizes[s] + (colour ? 1 : 0)));
  const char *rg = reads->db_name ? reads->db_name : "*";
  fprintf(f, "@RG\tID:%s\tSM:%s\n", rg, rg);
  fprintf(f, "@PG\tID:%s\tVN:%s\tCL:\"", "SToRM", "0.0101");
  for (int i = 0; i < o->argc; ++i) fprintf(f, "%s ", o->argv[i]);
  fprintf(f, "\"\n");
  /* records formatted in chunks, several chunks at once, written in placement order */
  uint8_t **chk = colour ? symbol_checkpoints(refs) : NULL;
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  int64_t CH = n_pl / (4 * (int64_t)nthreads);
  CH = CH < 256 ? 256 : CH > 16384 ? 16384 : CH;
  const int64_t per_round = CH * nthreads * 2;
  char **bufs = calloc((size_t)nthreads * 2, sizeof(char *));
  size_t *lens = calloc((size_t)nthreads * 2, sizeof(size_t));
  int nomem = !bufs || !lens || (colour && !chk);
  for (int64_t lo = 0; !nomem && lo < n_pl; lo += per_round) {
    const int64_t hi = lo + per_round < n_pl ? lo + per_round : n_pl;
    const int nchunks = (int)((hi - lo + CH - 1) / CH);
#pragma omp parallel for schedule(dynamic, 1) reduction(|| : nomem)
    for (int c = 0; c < nchunks; ++c) {
      const int64_t a = lo + (int64_t)c * CH, e = a + CH < hi ? a + CH : hi;
      FILE *m = open_memstream(&bufs[c], &lens[c]);
      if (!m) { nomem = 1; continue; }
      if (write_placement_records(m, o, refs, reads, res, pl, a, e - a, chk)) nomem = 1;
      fclose(m);
    }
    for (int c = 0; c < nchunks; ++c) {
      if (!nomem) fwrite(bufs[c], 1, lens[c], f);
      free(bufs[c]);
      bufs[c] = NULL;
    }
  }
  free(bufs);
  free(lens);
  if (chk) {
    for (int s = 0; s < refs->n; ++s) free(chk[s]);
    free(chk);
  }
  if (nomem) return fail(STORMGPU_ENOMEM, "Out of memory while writing the SAM output.");
  return 0;
}

/* the unmapped reads among [first, first + count), each record formatted in a buffer and written
 * at once.  Returns 0, or STORMGPU_ENOMEM when the buffer cannot be allocated. */
static int write_unmapped_records(FILE *f, const sh_sam_opts *o, const sh_reads *reads,
                                  const stormgpu_results *res, int64_t first, int64_t count) {
  static const char B[4] = {'A', 'C', 'G', 'T'}, CL[4] = {'0', '1', '2', '3'};
  size_t lcap = 4096;
  char *line = malloc(lcap);
  if (!line) return STORMGPU_ENOMEM;
  for (int64_t r = first; r < first + count; ++r) {
    if (res->mapped[r]) continue;
    const int L = reads->lengths[r];
    const size_t need = 2 * strlen(reads->names[r]) + 2 * (size_t)L + 16;
    if (need > lcap) {
      char *grown = realloc(line, 2 * need);
      if (!grown) { free(line); return STORMGPU_ENOMEM; }
      line = grown;
      lcap = 2 * need;
    }
    char *p = line;
    *p++ = '@';
    p = put_str(p, reads->names[r]);
    *p++ = '\n';
    const uint8_t *cd = reads->codes + r * reads->code_stride;
    if (!o->colour) {
      for (int k = 0; k < L; ++k) *p++ = B[get2(cd, k)];
    } else {
      *p++ = B[reads->first_base[r] & 3];
      for (int k = 0; k < L; ++k) *p++ = CL[get2(cd, k)];
    }
    *p++ = '\n';
    *p++ = '+';
    p = put_str(p, reads->names[r]);
    *p++ = '\n';
    if (has_quality(reads, r)) {
      const uint8_t *lv = reads->levels + r * reads->level_stride;
      if (o->colour) { int c = o->quality_base + LEVEL_UB[reads->first_level[r]]; *p++ = (char)(c < 126 ? c : 126); }
      for (int q = 0; q < L; ++q) { int c = o->quality_base + LEVEL_UB[get2(lv, q)]; *p++ = (char)(c < 126 ? c : 126); }
    } else {
      const int c = o->quality_base + 93;  /* MAX_READ_QUALITY for a NULL quality (hit_map.c:565-571) */
      if (o->colour) *p++ = (char)(c < 126 ? c : 126);
      for (int q = 0; q < L; ++q) *p++ = (char)(c < 126 ? c : 126);
    }
    *p++ = '\n';
    fwrite(line, 1, (size_t)(p - line), f);
  }
  free(line);
  return 0;
}

/* hit_map.c:514-579: records formatted in chunks, several chunks at once, written in read order */
int sh_write_unmapped_fastq(FILE *f, const sh_sam_opts *o, const sh_reads *reads,
                            const stormgpu_results *res) {
  const int64_t count = reads->n;
  int nthreads = 1;
#ifdef _OPENMP
  nthreads = omp_get_max_threads();
#endif
  int64_t CH = count / (4 * (int64_t)nthreads);
  CH = CH < 1024 ? 1024 : CH > 65536 ? 65536 : CH;
  const int64_t per_round = CH * nthreads * 2;
  char **bufs = calloc((size_t)nthreads * 2, sizeof(char *));
  size_t *lens = calloc((size_t)nthreads * 2, sizeof(size_t));
  int nomem = !bufs || !lens;
  for (int64_t lo = 0; !nomem && lo < count; lo += per_round) {
    const int64_t hi = lo + per_round < count ? lo + per_round : count;
    const int nchunks = (int)((hi - lo + CH - 1) / CH);
#pragma omp parallel for schedule(dynamic, 1) reduction(|| : nomem)
    for (int c = 0; c < nchunks; ++c) {
      const int64_t a = lo + (int64_t)c * CH, e = a + CH < hi ? a + CH : hi;
      FILE *m = open_memstream(&bufs[c], &lens[c]);
      if (!m) { nomem = 1; continue; }
      if (write_unmapped_records(m, o, reads, res, a, e - a)) nomem = 1;
      fclose(m);
    }
    for (int c = 0; c < nchunks; ++c) {
      if (!nomem) fwrite(bufs[c], 1, lens[c], f);
      free(bufs[c]);
      bufs[c] = NULL;
    }
  }
  free(bufs);
  free(lens);
  if (nomem) return fail(STORMGPU_ENOMEM, "Out of memory while writing the unmapped reads.");
  return 0;
}

/* writers into a named file, for callers without a FILE * (language bindings) */
int sh_write_sam_path(const char *path, const sh_sam_opts *o, const sh_refs *refs, const sh_reads *reads,
                      const stormgpu_results *res) {
  FILE *f = fopen(path, "w");
  if (!f) return fail(STORMGPU_EINVAL, "Cannot open %s for writing.", path);
  char *obuf = malloc(1 << 22);
  if (obuf) setvbuf(f, obuf, _IOFBF, 1 << 22);
  const int rc = sh_write_sam(f, o, refs, reads, res, 0, reads->n, 1);
  const int closed = fclose(f);
  free(obuf);
  if (closed != 0 && rc == 0) return fail(STORMGPU_EINVAL, "Cannot write %s.", path);
  return rc;
}

int sh_write_unmapped_fastq_path(const char *path, const sh_sam_opts *o, const sh_reads *reads,
                                 const stormgpu_results *res) {
  FILE *f = fopen(path, "w");
  if (!f) return fail(STORMGPU_EINVAL, "Cannot open %s for writing.", path);
  const int rc = sh_write_unmapped_fastq(f, o, reads, res);
  if (fclose(f) != 0 && rc == 0) return fail(STORMGPU_EINVAL, "Cannot write %s.", path);
  return rc;
}
