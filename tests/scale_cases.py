"""The at-scale parity cases: the benchmarked workloads at their full reference sizes, with
the reads (or a stated sample of them) that the reference maps here in bounded time.

Each case writes its inputs deterministically from the workload's seeds (storm_b200.synth),
so that the GPU box regenerates exactly the inputs whose reference outputs are pinned, as
SHA-256 digests, in tests/golden/scale_digests.json (written by
tests/golden/make_scale_digests.py).  A case runs as one or more runs of the command line:

  single  one run on the read file;
  buckets one run per read length, the reads of that length in file order (the reference maps
          one read length per run, reads_data.c:418-426);
  chain   per read length, the runs of an -O chain: run k maps the -O FASTQ of run k - 1 with
          the k-th seed family (README:97-101, hit_map.c:514-579); a chain stops when a run
          leaves no read unmapped (the reference refuses an empty read file).
"""
from __future__ import annotations

import hashlib
import os

import numpy as np

from storm_b200 import synth

CASES = {
    # colour workload, all 2M reads of 49 colours, 10 Mbp
    "colour_10M_2M": dict(cfg=1, scale=1.0, kind="single"),
    # mixed-length workload at full size: 100 Mbp, the first chunk (100k reads) of the 10M
    "mixed_100M_chunk0": dict(cfg=2, scale=1.0, kind="buckets", chunk=0, n=synth.CHUNK_READS),
    # served chain: 100 Mbp, 20k reads of its read model through the three-step -O chain
    "chain_100M_20k": dict(cfg=3, scale=1.0, kind="chain", chunk=0, n=20000),
    # mixed-length workload at a tenth of its size: 10 Mbp (45 % repeats), 1M reads of 35-150 bp
    "mixed_10M_1M": dict(cfg=2, scale=0.1, kind="buckets"),
    # large workload: 3.1 Gbp in 24 sequences, 10k reads of 100 bp
    "large_3G_10k": dict(cfg=4, scale=1.0, kind="single", chunk=0, n=10000),
}


def make_inputs(name: str, d: str):
    """Write the case's reference FASTA and reads FASTQ into directory d (once); returns
    (workload dict, reference path, reads path)."""
    c = CASES[name]
    w = synth.workload(c["cfg"], c["scale"])
    ref, reads = os.path.join(d, "ref.fa"), os.path.join(d, "reads.fq")
    done = os.path.join(d, "inputs.done")
    if not os.path.exists(done):
        os.makedirs(d, exist_ok=True)
        if "chunk" in c:
            genome = synth.genome_of(w)
            synth.write_fasta(ref, genome)
            seqs, quals = synth.reads_chunk(w, genome, c["chunk"], c["n"])
            synth.write_fastq(reads, seqs, quals)
        else:
            synth.generate(c["cfg"], c["scale"], ref, reads)
        open(done, "w").write("ok")
    return w, ref, reads


def split_by_length(reads: str, d: str):
    """Per read length, a FASTQ of the reads of that length in file order; returns
    [(length, path)] in ascending length."""
    files, out = {}, []
    with open(reads, "rb") as f:
        while True:
            rec = [f.readline() for _ in range(4)]
            if not rec[0]:
                break
            L = len(rec[1].rstrip(b"\n"))
            if L not in files:
                files[L] = open(os.path.join(d, "len%d.fq" % L), "wb")
            files[L].write(b"".join(rec))
    for L in sorted(files):
        files[L].close()
        out.append((L, os.path.join(d, "len%d.fq" % L)))
    return out


def runs(name: str, w, reads: str, d: str):
    """The command-line runs of the case: [(label, reads file, seeds or None, sam, unmapped
    fastq)], in the order they must run (a chain's run reads the -O output of the run before
    it)."""
    c = CASES[name]
    if c["kind"] == "single":
        return [("all", reads, None, os.path.join(d, "all.sam"), os.path.join(d, "all.un.fq"))]
    out = []
    for L, path in split_by_length(reads, d):
        if c["kind"] == "buckets":
            out.append(("len%d" % L, path, None, os.path.join(d, "len%d.sam" % L), os.path.join(d, "len%d.un.fq" % L)))
        else:
            src = path
            for k, seeds in enumerate(w["chain"]):
                lab = "len%d.step%d" % (L, k)
                out.append((lab, src, seeds, os.path.join(d, lab + ".sam"), os.path.join(d, lab + ".un.fq")))
                src = os.path.join(d, lab + ".un.fq")
    return out


def skip_run(path: str) -> bool:
    """A chain's run whose input, the previous run's -O FASTQ, is empty or was never written
    (the chain stopped earlier) does not run."""
    return not os.path.exists(path) or os.path.getsize(path) == 0


def command_args(w, seeds, reads: str, sam: str, unmapped: str, ref: str):
    """The run's options after the program name (the workload's options; a chain step's seed
    family replaces -s)."""
    args = list(w["args"])
    if seeds is not None:
        if "-s" in args:
            i = args.index("-s")
            del args[i:i + 2]
        args += ["-s", seeds]
    return ["-g", ref, "-r", reads, "-o", sam, "-O", unmapped, "-v", "0"] + args


def digest_sam(path: str):
    """(sha256 of the SAM without its @PG line, which echoes the command line; record count)."""
    h = hashlib.sha256()
    n = 0
    with open(path, "rb") as f:
        for line in f:
            if line.startswith(b"@PG"):
                continue
            if not line.startswith(b"@"):
                n += 1
            h.update(line)
    return h.hexdigest(), n


def digest_file(path: str):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for block in iter(lambda: f.read(1 << 20), b""):
            h.update(block)
    return h.hexdigest()


def inputs_digest(ref: str, reads: str) -> str:
    """Short digest of the input files: a drifted generator shows here first."""
    h = hashlib.sha256()
    for p in (ref, reads):
        h.update(digest_file(p).encode())
    return h.hexdigest()[:16]


def sample_sizes(reads: str):
    """Read count per length of a FASTQ."""
    lens = []
    with open(reads, "rb") as f:
        for k, line in enumerate(f):
            if k % 4 == 1:
                lens.append(len(line.rstrip(b"\n")))
    u, c = np.unique(np.array(lens), return_counts=True)
    return {int(a): int(b) for a, b in zip(u, c)}
