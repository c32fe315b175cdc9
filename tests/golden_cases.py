"""Shared helpers for the golden-fixture tests: rebuild the inputs of a case, run a CLI on
them, and compare its SAM records and -O FASTQ with the fixture."""
import gzip
import json
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
sys.path.insert(0, GOLDEN)

import make_golden  # noqa: E402


def meta():
    return json.load(open(os.path.join(GOLDEN, "golden.json")))


def check_case(name, tmpdir, exe_for_mode):
    m = meta()[name]
    w, ref, reads = make_golden.make_inputs(name, tmpdir)
    assert make_golden.digest(ref, reads) == m["inputs_sha256_16"], "synthetic generator drifted"
    exe = exe_for_mode(w["mode"])
    sam, fq = os.path.join(tmpdir, "g.sam"), os.path.join(tmpdir, "g.fq")
    p = subprocess.run([exe, "-g", ref, "-r", reads, "-o", sam, "-O", fq, "-v", "0"] + w["args"],
                       cwd=tmpdir, capture_output=True, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    body = b"".join(l + b"\n" for l in open(sam, "rb").read().split(b"\n") if l and not l.startswith(b"@"))
    exp = gzip.open(os.path.join(GOLDEN, name + ".sam.gz")).read()
    if body != exp:
        a, b = body.split(b"\n"), exp.split(b"\n")
        for i, (x, y) in enumerate(zip(a, b)):
            if x != y:
                raise AssertionError("%s: record %d differs\n got %r\n exp %r" % (name, i, x, y))
        raise AssertionError("%s: %d records vs %d expected" % (name, len(a), len(b)))
    assert open(fq, "rb").read() == gzip.open(os.path.join(GOLDEN, name + ".unmapped.fq.gz")).read()
    return body.count(b"\n")
