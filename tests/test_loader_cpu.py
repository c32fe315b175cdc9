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
