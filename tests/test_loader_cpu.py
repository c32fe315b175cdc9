"""The host read loader on a file large enough for its parallel paths (read by ranges in
threads, lines found by threads): the same reads as two halves of the file loaded on their own."""
import numpy as np
import pytest

from storm_b200 import build, host, synth


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


@pytest.mark.parametrize("colour", [0, 1])
def test_large_file_loads_like_its_halves(tmp_path, colour):
    genome = synth.make_genome([200000], 61)
    n = 700000 if colour else 450000
    if colour:
        pr, cols, q = synth.simulate_colour_reads(genome, n, 49, 62)
        synth.write_colour_fastq(str(tmp_path / "all.fq"), pr, cols, q)
    else:
        seqs, quals = synth.simulate_nucleotide_reads(genome, n, [35, 75, 150], 62)
        synth.write_fastq(str(tmp_path / "all.fq"), seqs, quals)
    data = (tmp_path / "all.fq").read_bytes()
    assert len(data) > 70 << 20  # above the size the loader reads by ranges
    lines = data.split(b"\n")
    cut = 4 * (n // 2)
    (tmp_path / "a.fq").write_bytes(b"\n".join(lines[:cut]) + b"\n")
    (tmp_path / "b.fq").write_bytes(b"\n".join(lines[cut:]))
    whole = host.ReadSet(str(tmp_path / "all.fq"), colour, sort=False)
    a = host.ReadSet(str(tmp_path / "a.fq"), colour, sort=False)
    b = host.ReadSet(str(tmp_path / "b.fq"), colour, sort=False)
    assert whole.n == n and a.n + b.n == n
    w = whole.codes.shape[1]
    for field in ("codes", "levels"):
        got = getattr(whole, field)
        want = np.concatenate([getattr(a, field)[:, :w] if getattr(a, field).shape[1] >= w else
                               np.pad(getattr(a, field), ((0, 0), (0, w - getattr(a, field).shape[1]))),
                               getattr(b, field)[:, :w] if getattr(b, field).shape[1] >= w else
                               np.pad(getattr(b, field), ((0, 0), (0, w - getattr(b, field).shape[1])))])
        assert np.array_equal(got, want), field
    assert np.array_equal(whole.lengths, np.concatenate([a.lengths, b.lengths]))
    assert np.array_equal(whole.first_levels, np.concatenate([a.first_levels, b.first_levels]))


def _refs_snapshot(ref):
    import ctypes as C
    s = ref._s
    out = []
    for k in range(s.n):
        size = int(s.sizes[k])
        nb = (size + 3) // 4 + 4
        rs = C.cast(s.rs[k], C.POINTER(C.c_int32))
        re_ = C.cast(s.re[k], C.POINTER(C.c_int32))
        regions = [(rs[r], re_[r]) for r in range(int(s.nreg[k]))]
        out.append((s.names[k], size, C.string_at(s.codes[k], nb), C.string_at(s.masks[k], nb), regions,
                    int(s.first_base[k])))
    return out


def _random_fasta(rng, nseq):
    parts = []
    for k in range(nseq):
        n = int(rng.integers(1, 40000)) if k else int(rng.integers(20000, 60000))
        seq = np.frombuffer(b"ACGTacgt", np.uint8)[rng.integers(0, 8, size=n)].copy()
        for _ in range(int(rng.integers(0, 12))):  # masked runs: N, other letters, at either end too
            a = int(rng.integers(0, n))
            b = min(n, a + int(rng.integers(1, 3000)))
            seq[a:b] = np.frombuffer(b"NNNNRYn-", np.uint8)[rng.integers(0, 8, size=b - a)]
        if rng.random() < 0.3:
            seq[0] = ord("N")
        text = bytearray()
        u = 0
        while u < n:
            w = int(rng.integers(1, 120))
            text += seq[u:u + w].tobytes()
            u += w
            text += b"\r\n" if rng.random() < 0.1 else b" \t\n" if rng.random() < 0.05 else b"\n"
        parts.append(b">seq%d some text\n" % k + bytes(text))
    return b"".join(parts)


@pytest.mark.parametrize("colour,ignore_lowercase,seed", [(0, 0, 1), (0, 1, 2), (1, 0, 3), (1, 1, 4), (0, 0, 5)])
def test_reference_filled_by_threads_like_one_pass(tmp_path, colour, ignore_lowercase, seed):
    """A reference FASTA loaded with the threaded paths forced on every sequence (read by ranges,
    headers and sizes counted by threads, codes, masks and masked runs filled by threads, the
    masked symbols' rand() codes drawn in order) gives what the one-pass loader gives."""
    import ctypes as C
    libc = C.CDLL(None)
    L = host.hostlib()
    L.sh_set_parallel_min_bytes.argtypes = [C.c_size_t]
    rng = np.random.default_rng(seed)
    (tmp_path / "ref.fa").write_bytes(_random_fasta(rng, 5))
    try:
        libc.srand(1)
        one = _refs_snapshot(host.Reference(str(tmp_path / "ref.fa"), colour, ignore_lowercase))
        L.sh_set_parallel_min_bytes(1)
        libc.srand(1)
        threads = _refs_snapshot(host.Reference(str(tmp_path / "ref.fa"), colour, ignore_lowercase))
    finally:
        L.sh_set_parallel_min_bytes(64 << 20)
    assert len(one) == 5 and sum(len(r[4]) for r in one) > 5
    for a, b in zip(one, threads):
        assert a == b


@pytest.mark.parametrize("layout", ["plain", "crlf", "comments", "cut_short", "corrupt"])
def test_reads_loaded_by_threads_like_one_pass(tmp_path, layout):
    """A FASTQ file loaded with the threaded paths forced (read by ranges, line starts found by
    threads) gives the one-pass loader's reads, or its error message and line number."""
    import ctypes as C
    L = host.hostlib()
    L.sh_set_parallel_min_bytes.argtypes = [C.c_size_t]
    genome = synth.make_genome([30000], 71)
    seqs, quals = synth.simulate_nucleotide_reads(genome, 3000, [35, 50, 100], 72)
    synth.write_fastq(str(tmp_path / "r.fq"), seqs, quals)
    lines = (tmp_path / "r.fq").read_bytes().split(b"\n")
    if layout == "crlf":
        lines = [l + b"\r" if l else l for l in lines]
    elif layout == "comments":
        lines = [b"# Title: threads", b"# comment"] + lines
    elif layout == "cut_short":
        lines = lines[:-2]
    elif layout == "corrupt":
        lines[4 * 2345 + 2] = b"x"
    (tmp_path / "r.fq").write_bytes(b"\n".join(lines))

    def load():
        try:
            r = host.ReadSet(str(tmp_path / "r.fq"), 0, sort=True)
        except Exception as e:  # the loader's message
            return str(e)
        return (r.n, r.codes.tobytes(), None if r.levels is None else r.levels.tobytes(), r.lengths.tobytes())

    try:
        one = load()
        L.sh_set_parallel_min_bytes(1)
        threads = load()
    finally:
        L.sh_set_parallel_min_bytes(64 << 20)
    assert one == threads
    if layout == "corrupt":
        assert "line %d" % (4 * 2345 + 3) in one
    else:
        assert one[0] == 3000
