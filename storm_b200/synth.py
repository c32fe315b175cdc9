"""Seeded synthetic references and reads for the mapping workloads.

No public dataset is used by the mapper's own benchmarks, so every workload is generated
here, deterministically from its seed:

* references: i.i.d. bases with a given GC content, optionally with a fraction of their
  length overwritten by mutated copies of other segments (repeats);
* Illumina-like reads: uniform start on either strand, substitution rate rising linearly
  along the read, rare indels, Phred qualities from a normal whose mean falls along the read;
* SOLiD colour-space reads: a primer base followed by colours, with i.i.d. colour errors
  (higher over the last colours) and true SNPs, which appear as two adjacent colour changes.

Codes are 0..3 for A, C, G, T (colours 0..3 are the XOR of adjacent base codes).
"""
from __future__ import annotations

import dataclasses
import numpy as np

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
COLOURS = np.frombuffer(b"0123", dtype=np.uint8)


@dataclasses.dataclass
class ReadModel:
    sub_lo: float = 0.005          # substitution rate at the 5' end
    sub_hi: float = 0.04           # substitution rate at the 3' end
    indel_rate: float = 0.0005     # per-base probability of an indel
    indel_max: int = 1             # indel lengths are uniform in 1..indel_max
    q_hi: float = 35.0             # mean Phred at the 5' end
    q_lo: float = 20.0             # mean Phred at the 3' end
    q_sd: float = 5.0
    q_min: int = 2
    q_max: int = 40


@dataclasses.dataclass
class ColourModel:
    err: float = 0.03              # i.i.d. colour error rate
    err_tail: float = 0.06         # colour error rate over the last `tail` colours
    tail: int = 10
    snp: float = 0.001             # true SNP rate (a base change = two colour changes)


def random_bases(rng: np.random.Generator, n: int, gc: float = 0.5) -> np.ndarray:
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    return rng.choice(4, size=n, p=p).astype(np.uint8)


def random_bases_fast(rng: np.random.Generator, n: int, gc: float = 0.5, chunk: int = 1 << 24) -> np.ndarray:
    """Like random_bases, for genomes of billions of codes: 16-bit uniforms through a table of
    the base probabilities (quantised to 1/65536), in chunks, without 64-bit temporaries."""
    p = np.array([(1 - gc) / 2, gc / 2, gc / 2, (1 - gc) / 2])
    edges = np.rint(np.cumsum(p) * 65536).astype(np.int64)
    lut = np.searchsorted(edges, np.arange(65536), side="right").astype(np.uint8)
    out = np.empty(n, np.uint8)
    for a in range(0, n, chunk):
        e = min(n, a + chunk)
        out[a:e] = lut[rng.integers(0, 65536, size=e - a, dtype=np.uint16)]
    return out


def make_reference(size: int, seed: int, gc: float = 0.5, repeat_frac: float = 0.0,
                   seg_min: int = 300, seg_max: int = 6000, mut_min: float = 0.05,
                   mut_max: float = 0.15, fast: bool = False) -> np.ndarray:
    """One reference sequence of `size` codes; `repeat_frac` of it is made of mutated copies.
    `fast` draws the bases with random_bases_fast (another sequence for the same seed)."""
    rng = np.random.default_rng(seed)
    seq = random_bases_fast(rng, size, gc) if fast else random_bases(rng, size, gc)
    if repeat_frac > 0 and size > 2 * seg_max:
        covered = 0
        target = int(repeat_frac * size)
        while covered < target:
            ln = int(rng.integers(seg_min, seg_max + 1))
            src = int(rng.integers(0, size - ln))
            dst = int(rng.integers(0, size - ln))
            seg = seq[src:src + ln].copy()
            rate = rng.uniform(mut_min, mut_max)
            m = rng.random(ln) < rate
            seg[m] = (seg[m] + rng.integers(1, 4, size=int(m.sum()))) % 4
            seq[dst:dst + ln] = seg
            covered += ln
    return seq


def make_genome(sizes, seed: int, gc: float = 0.5, repeat_frac: float = 0.0, fast: bool = False):
    """Several named sequences ("chr1", ...) with independent seeds derived from `seed`."""
    return [("chr%d" % (i + 1), make_reference(int(s), seed * 1000 + i, gc, repeat_frac, fast=fast))
            for i, s in enumerate(sizes)]


def _qualities(rng, n, L, model: ReadModel) -> np.ndarray:
    pos = np.arange(L, dtype=np.float64) / max(L - 1, 1)
    mean = model.q_hi + (model.q_lo - model.q_hi) * pos
    q = rng.normal(mean[None, :], model.q_sd, size=(n, L))
    return np.clip(np.rint(q), model.q_min, model.q_max).astype(np.uint8)


def _sample_fragments(rng, genome, n, flen):
    """Pick n fragments of length flen (uniform chromosome by length, uniform start, random strand)."""
    lens = np.array([len(s) for _, s in genome], dtype=np.int64)
    w = (lens - flen).clip(min=0).astype(np.float64)
    chrom = rng.choice(len(genome), size=n, p=w / w.sum())
    frags = np.empty((n, flen), dtype=np.uint8)
    starts = np.empty(n, dtype=np.int64)
    for c in range(len(genome)):
        idx = np.nonzero(chrom == c)[0]
        if idx.size == 0:
            continue
        st = rng.integers(0, lens[c] - flen + 1, size=idx.size)
        starts[idx] = st
        frags[idx] = genome[c][1][st[:, None] + np.arange(flen)[None, :]]
    rev = rng.random(n) < 0.5
    frags[rev] = (frags[rev][:, ::-1]) ^ 3
    return frags, chrom, starts, rev


def _apply_indels(rng, frags, L, model: ReadModel):
    """Return an (n, L) array: each row is its fragment with indels applied, cut to L."""
    n, flen = frags.shape
    out = frags[:, :L].copy()
    n_ev = rng.binomial(L, model.indel_rate, size=n)
    for r in np.nonzero(n_ev)[0]:
        s = list(frags[r])
        for _ in range(int(n_ev[r])):
            p = int(rng.integers(1, L - 1))
            k = int(rng.integers(1, model.indel_max + 1))
            if rng.random() < 0.5:
                s[p:p] = list(rng.integers(0, 4, size=k).astype(np.uint8))
            else:
                del s[p:p + k]
        s = s + [0] * max(0, L - len(s))
        out[r] = np.array(s[:L], dtype=np.uint8)
    return out


def simulate_nucleotide_reads(genome, n: int, lengths, seed: int, model: ReadModel | None = None):
    """Illumina-like reads.  `lengths` is an int or a sequence of lengths drawn uniformly.

    Returns (seqs, quals): lists of uint8 code arrays and Phred arrays (one per read)."""
    model = model or ReadModel()
    rng = np.random.default_rng(seed)
    if np.isscalar(lengths):
        lens = np.full(n, int(lengths), dtype=np.int64)
    else:
        lens = rng.choice(np.asarray(lengths, dtype=np.int64), size=n)
    seqs, quals = [None] * n, [None] * n
    for L in np.unique(lens):
        idx = np.nonzero(lens == L)[0]
        L = int(L)
        slack = 4 * model.indel_max + 8
        frags, _, _, _ = _sample_fragments(rng, genome, idx.size, L + slack)
        reads = _apply_indels(rng, frags, L, model)
        rate = model.sub_lo + (model.sub_hi - model.sub_lo) * np.arange(L) / max(L - 1, 1)
        m = rng.random(reads.shape) < rate[None, :]
        reads[m] = (reads[m] + rng.integers(1, 4, size=int(m.sum()))) % 4
        q = _qualities(rng, idx.size, L, model)
        for j, r in enumerate(idx):
            seqs[r] = reads[j]
            quals[r] = q[j]
    return seqs, quals


def simulate_colour_reads(genome, n: int, n_colours: int, seed: int,
                          model: ReadModel | None = None, cmodel: ColourModel | None = None,
                          primer: int = 3):
    """SOLiD reads: returns (primers, colour arrays of n_colours, Phred arrays of n_colours)."""
    model = model or ReadModel()
    cmodel = cmodel or ColourModel()
    rng = np.random.default_rng(seed)
    frags, _, _, _ = _sample_fragments(rng, genome, n, n_colours)
    snp = rng.random(frags.shape) < cmodel.snp
    frags[snp] = (frags[snp] + rng.integers(1, 4, size=int(snp.sum()))) % 4
    prev = np.concatenate([np.full((n, 1), primer, dtype=np.uint8), frags[:, :-1]], axis=1)
    cols = prev ^ frags
    rate = np.full(n_colours, cmodel.err)
    rate[-cmodel.tail:] = cmodel.err_tail
    m = rng.random(cols.shape) < rate[None, :]
    cols[m] = (cols[m] + rng.integers(1, 4, size=int(m.sum()))) % 4
    q = _qualities(rng, n, n_colours, model)
    return np.full(n, primer, dtype=np.uint8), cols, q


# ----------------------------------------------------------------------------- file writers

def write_fasta(path, genome, width: int = 60):
    with open(path, "wb") as f:
        for name, seq in genome:
            f.write(b">" + name.encode() + b"\n")
            s = BASES[seq].tobytes()
            for i in range(0, len(s), width):
                f.write(s[i:i + width] + b"\n")


def write_fastq(path, seqs, quals, offset: int = 33, prefix: str = "r"):
    with open(path, "wb") as f:
        for k, (s, q) in enumerate(zip(seqs, quals)):
            f.write(b"@%s%d\n%s\n+\n%s\n" % (prefix.encode(), k, BASES[s].tobytes(),
                                            (q.astype(np.uint8) + offset).tobytes()))


def write_colour_fastq(path, primers, cols, quals, offset: int = 33, prefix: str = "r"):
    with open(path, "wb") as f:
        for k in range(len(cols)):
            f.write(b"@%s%d\n%c%s\n+\n%s\n" % (prefix.encode(), k, BASES[primers[k]],
                                              COLOURS[cols[k]].tobytes(),
                                              (quals[k].astype(np.uint8) + offset).tobytes()))


# ----------------------------------------------------------------------------- workloads
# The five workloads the mapper is measured on, with their default sizes.  `scale` shrinks
# the read count and reference length together for tests and CPU samples.

def workload(cfg: int, scale: float = 1.0):
    """Return a dict describing workload `cfg` (0..4), scaled by `scale`."""
    if cfg == 0:
        return dict(mode="nucleotide", ref_sizes=[int(1_000_000 * scale)], gc=0.5, repeat=0.0,
                    ref_seed=1, reads=int(100_000 * scale), lengths=50, read_seed=11,
                    args=["-M", "1", "-z", "100", "-t", "100", "-i", "3", "-b", "33"])
    if cfg == 1:
        return dict(mode="colour", ref_sizes=[int(10_000_000 * scale)], gc=0.41, repeat=0.20,
                    ref_seed=2, reads=int(2_000_000 * scale), lengths=50, read_seed=12,
                    args=["-M", "1", "-z", "105", "-t", "120", "-i", "7", "-s",
                          "####-##-#-####;###-#--##-##--###;####-#---#----#--####"])
    if cfg == 2:
        return dict(mode="nucleotide", ref_sizes=[int(100_000_000 * scale)], gc=0.41, repeat=0.45,
                    ref_seed=3, reads=int(10_000_000 * scale), lengths=[35, 50, 75, 100, 150],
                    read_seed=13,
                    args=["-i", "15", "-M", "1", "-z", "100", "-t", "100", "-s",
                          "##-##-###-###;###--#-#--#--####;####--#--#---#---###"])
    if cfg == 3:
        return dict(mode="nucleotide", ref_sizes=[int(100_000_000 * scale)], gc=0.41, repeat=0.45,
                    ref_seed=3, reads=int(1_000_000 * scale), lengths=[35, 50, 75, 100, 150],
                    read_seed=7,
                    chain=["###-##--#-##-#-###", "####-#-#--##-###", "#####-##-###"],
                    args=["-i", "15", "-M", "1", "-z", "100", "-t", "100"])
    if cfg == 4:
        rng = np.random.default_rng(4)
        sizes = np.exp(rng.uniform(np.log(50e6), np.log(250e6), size=24))
        sizes = (sizes * (3.1e9 / sizes.sum()) * scale).astype(np.int64)
        return dict(mode="nucleotide", ref_sizes=[int(s) for s in sizes], gc=0.41, repeat=0.50,
                    ref_seed=4, reads=int(100_000_000 * scale), lengths=100, read_seed=14,
                    model=dict(indel_rate=0.002, indel_max=20), fast_genome=True,
                    args=["-i", "20", "-z", "85", "-t", "100", "-M", "1"])
    raise ValueError(cfg)


def genome_of(w):
    """The reference sequences of workload `w` (a workload() dict)."""
    return make_genome(w["ref_sizes"], w["ref_seed"], w["gc"], w["repeat"], fast=w.get("fast_genome", False))


CHUNK_READS = 100_000


def reads_chunk(w, genome, chunk: int, n: int = CHUNK_READS):
    """Reads [chunk * CHUNK_READS, chunk * CHUNK_READS + n) of workload `w`'s read set, when the
    set is drawn in independent chunks of CHUNK_READS reads (so that any chunk can be made
    without the others): chunk c draws from seed read_seed * 100003 + c.  Nucleotide workloads
    only; returns (seqs, quals) as simulate_nucleotide_reads."""
    if w["mode"] != "nucleotide":
        raise ValueError("chunked reads are drawn for nucleotide workloads")
    model = ReadModel(**w.get("model", {}))
    return simulate_nucleotide_reads(genome, n, w["lengths"], w["read_seed"] * 100003 + chunk, model)


def generate(cfg: int, scale: float, ref_path, reads_path):
    """Write the reference FASTA and the reads FASTQ of workload `cfg` at `scale`."""
    w = workload(cfg, scale)
    genome = genome_of(w)
    write_fasta(ref_path, genome)
    model = ReadModel(**w.get("model", {}))
    if w["mode"] == "colour":
        pr, cols, q = simulate_colour_reads(genome, w["reads"], w["lengths"], w["read_seed"], model)
        write_colour_fastq(reads_path, pr, cols, q)
    else:
        seqs, quals = simulate_nucleotide_reads(genome, w["reads"], w["lengths"], w["read_seed"], model)
        write_fastq(reads_path, seqs, quals)
    return w
