"""Generate the golden fixtures of tests/golden from the reference itself.

For each case, the inputs are regenerated deterministically by storm_b200.synth (seeded), the
reference binary built from its own sources by oracle/Makefile (oracle/_ref) is run on them
with MALLOC_PERTURB_=255 (zero-filled allocations, see tests/test_e2e_cpu.py), and the SAM
records (header lines dropped: they echo file names and argv) and the -O FASTQ are stored
gzip-compressed, with a digest of the inputs so that generator drift is detected.

    python tests/golden/make_golden.py            # needs oracle/_ref (the reference sources)

Mixed read lengths: the reference accepts one read length per run (reads_data.c:418-426), so
the golden output of a mixed-length case is the concatenation, in ascending length order, of
one reference run per length on the reads of that length (file order kept)."""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from storm_b200 import synth  # noqa: E402

CASES = {
    "nuc_small": dict(cfg=0, scale=0.01),
    "col_small": dict(cfg=1, scale=0.0005),
    "mixed_small": dict(cfg=2, scale=0.0001, ref_scale=0.0005),
}


def make_inputs(name, d):
    c = CASES[name]
    w = synth.workload(c["cfg"], c["scale"])
    if "ref_scale" in c:
        w["ref_sizes"] = [int(s * c["ref_scale"] / c["scale"]) for s in w["ref_sizes"]]
    genome = synth.make_genome(w["ref_sizes"], w["ref_seed"], w["gc"], w["repeat"])
    ref = os.path.join(d, "ref.fa")
    reads = os.path.join(d, "reads.fq")
    synth.write_fasta(ref, genome)
    if w["mode"] == "colour":
        pr, cols, q = synth.simulate_colour_reads(genome, w["reads"], w["lengths"], w["read_seed"])
        synth.write_colour_fastq(reads, pr, cols, q)
    else:
        seqs, quals = synth.simulate_nucleotide_reads(genome, w["reads"], w["lengths"], w["read_seed"])
        synth.write_fastq(reads, seqs, quals)
    return w, ref, reads


def digest(*paths):
    h = hashlib.sha256()
    for p in paths:
        h.update(open(p, "rb").read())
    return h.hexdigest()[:16]


def split_by_length(reads_path, d):
    lines = open(reads_path, "rb").read().split(b"\n")
    by_len = {}
    for k in range(0, len(lines) - 3, 4):
        by_len.setdefault(len(lines[k + 1]), []).extend(lines[k:k + 4])
    out = []
    for L in sorted(by_len):
        p = os.path.join(d, "reads_%d.fq" % L)
        open(p, "wb").write(b"\n".join(by_len[L]) + b"\n")
        out.append(p)
    return out


def run_reference(w, ref, reads, d, exe):
    body, unmapped = b"", b""
    parts = split_by_length(reads, d) if isinstance(w["lengths"], list) else [reads]
    for p in parts:
        sam, fq = os.path.join(d, "o.sam"), os.path.join(d, "o.fq")
        cmd = [exe, "-g", ref, "-r", p, "-o", sam, "-O", fq, "-v", "0"] + w["args"]
        subprocess.run(cmd, check=True, env=dict(os.environ, MALLOC_PERTURB_="255"), cwd=d)
        body += b"".join(l + b"\n" for l in open(sam, "rb").read().split(b"\n") if l and not l.startswith(b"@"))
        unmapped += open(fq, "rb").read()
    return body, unmapped


def main():
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    meta = {}
    for name in CASES:
        with tempfile.TemporaryDirectory() as d:
            w, ref, reads = make_inputs(name, d)
            exe = os.path.join(ref_dir, "storm-color" if w["mode"] == "colour" else "storm-nucleotide")
            body, unmapped = run_reference(w, ref, reads, d, exe)
            with gzip.open(os.path.join(HERE, name + ".sam.gz"), "wb", compresslevel=9) as f:
                f.write(body)
            with gzip.open(os.path.join(HERE, name + ".unmapped.fq.gz"), "wb", compresslevel=9) as f:
                f.write(unmapped)
            meta[name] = dict(args=w["args"], mode=w["mode"], inputs_sha256_16=digest(ref, reads),
                              records=body.count(b"\n"))
            print(name, meta[name])
    json.dump(meta, open(os.path.join(HERE, "golden.json"), "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
