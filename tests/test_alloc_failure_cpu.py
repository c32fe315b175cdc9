"""Allocation failure in the host front end, injected on the host: a preloaded allocator that
refuses the requests of a given size range (a fake of malloc / calloc / realloc), under the
command line's front end (the oracle build of storm-nucleotide, which shares it with the GPU
binary).  Where the reference prints a message and exits with status 1 (SAFE_FAILURE__ALLOC,
util.h:70-80), the front end must do the same: no crash, no partial output passed off as a
result.  The refused sizes are windows chosen so that the first refused request is, in turn,
the read file's buffer, the per-read arrays and the result arrays; with no window the run
maps normally."""
import os
import subprocess

import pytest

from storm_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_CLI = os.path.join(ROOT, "oracle", "storm-oracle-nucleotide")

SHIM = r"""
#include <errno.h>
#include <stddef.h>
#include <stdlib.h>
extern void *__libc_malloc(size_t);
extern void *__libc_calloc(size_t, size_t);
extern void *__libc_realloc(void *, size_t);
/* STORM_TEST_ALLOC_REFUSE="lo:hi": requests of lo..hi bytes fail */
static int refused(size_t n) {
  static size_t lo = 1, hi = 0;
  static int init;
  if (!init) {
    const char *s = getenv("STORM_TEST_ALLOC_REFUSE");
    if (s) {
      char *e;
      lo = (size_t)strtoull(s, &e, 10);
      hi = *e == ':' ? (size_t)strtoull(e + 1, 0, 10) : 0;
    }
    init = 1;
  }
  return n >= lo && n <= hi;
}
void *malloc(size_t n) { if (refused(n)) { errno = ENOMEM; return NULL; } return __libc_malloc(n); }
void *calloc(size_t a, size_t b) {
  if (b && a <= ((size_t)-1) / b && refused(a * b)) { errno = ENOMEM; return NULL; }
  return __libc_calloc(a, b);
}
void *realloc(void *p, size_t n) { if (refused(n)) { errno = ENOMEM; return NULL; } return __libc_realloc(p, n); }
"""


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    d = tmp_path_factory.mktemp("shim")
    src = d / "failalloc.c"
    src.write_text(SHIM)
    so = d / "libfailalloc.so"
    subprocess.run(["gcc", "-O2", "-shared", "-fPIC", "-o", str(so), str(src)], check=True)
    return str(so)


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    d = tmp_path_factory.mktemp("inputs")
    genome = synth.make_genome([200000], 61)
    synth.write_fasta(str(d / "ref.fa"), genome)
    seqs, quals = synth.simulate_nucleotide_reads(genome, 20000, 150, 62)
    synth.write_fastq(str(d / "reads.fq"), seqs, quals)
    return d


def _run(shim, d, window):
    env = dict(os.environ, LD_PRELOAD=shim, OMP_NUM_THREADS="2")
    if window:
        env["STORM_TEST_ALLOC_REFUSE"] = "%d:%d" % window
    return subprocess.run([ORACLE_CLI, "-g", "ref.fa", "-r", "reads.fq", "-o", "out.sam", "-M", "1", "-i", "3",
                           "-z", "100", "-t", "100", "-v", "0"], cwd=str(d), env=env, capture_output=True, timeout=600)


@pytest.mark.skipif(not os.path.exists(ORACLE_CLI), reason="oracle CLI not built (make -C oracle)")
def test_refused_allocations_end_with_status_1_and_a_message(shim, inputs):
    size = os.path.getsize(inputs / "reads.fq")
    n = 20000
    # the read file's buffer (its size + 2); the packed codes (n * 40 bytes: 150 codes in a
    # stride of 40); the traceback rows of the results (n * 4 rows of 80 bytes at -i 3)
    for window, what in (((size + 2, size + 2), b"Not enough memory to read"),
                         ((n * 40, n * 40), b"Not enough memory for 20000 reads"),
                         ((n * 4 * 80, n * 4 * 80), b"Not enough memory for the results")):
        p = _run(shim, inputs, window)
        assert p.returncode == 1, (window, p.returncode, p.stderr[-400:])
        assert what in p.stderr, (window, p.stderr[-400:])


@pytest.mark.skipif(not os.path.exists(ORACLE_CLI), reason="oracle CLI not built (make -C oracle)")
def test_without_refusals_the_run_maps(shim, inputs):
    p = _run(shim, inputs, None)
    assert p.returncode == 0, p.stderr[-400:]
    recs = [l for l in (inputs / "out.sam").read_bytes().split(b"\n") if l and not l.startswith(b"@")]
    assert len(recs) > 15000
