"""Parity at the benchmarked sizes: the storm-nucleotide / storm-color binaries (CUDA library
behind the reference's command line) on the at-scale cases of scale_cases.py -- full genome
sizes, the benchmarked read sets or stated samples of them -- against digests of the
reference's own SAM and -O FASTQ for the same runs (tests/golden/scale_digests.json, written
by tests/golden/make_scale_digests.py from the reference compiled from its sources).

Every case regenerates its inputs from the workload's seeds and first checks their digest, so
that a drifted generator fails as such and not as a mapping difference.  The runs are the
reference's: one per read file, one per read length for the mixed-length workload (the
reference maps one length per run), and per length the three runs of the -O chain, each on the
previous run's unmapped FASTQ.  The mixed-length cases also map the whole mixed file in one run
and check that its records and unmapped reads are the per-length runs' ones, in ascending
length.
"""
import json
import os
import subprocess

import pytest

import scale_cases
from storm_b200 import build

pytestmark = pytest.mark.gpu

DIGESTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scale_digests.json")


def _digests():
    return json.load(open(DIGESTS)) if os.path.exists(DIGESTS) else {}


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _exe(mode):
    return os.path.join(build.BIN_DIR, "storm-color" if mode == "colour" else "storm-nucleotide")


def _records(path):
    with open(path, "rb") as f:
        return b"".join(x for x in f if not x.startswith(b"@"))


@pytest.mark.parametrize("name", [n for n in scale_cases.CASES if n != "large_3G_10k"])
def test_cli_matches_reference_at_scale(name, tmp_path):
    _run_case(name, str(tmp_path))


@pytest.mark.parametrize("name", ["large_3G_10k"])
def test_cli_matches_reference_on_the_large_genome(name, tmp_path):
    """3.1 Gbp in 24 sequences, -i 20 (filter band clipped at 15, alignment band 41)."""
    _run_case(name, str(tmp_path))


def _run_case(name, d):
    exp = _digests().get(name)
    if exp is None:
        pytest.skip("no reference digests for %s" % name)
    w, ref, reads = scale_cases.make_inputs(name, d)
    assert scale_cases.inputs_digest(ref, reads) == exp["inputs_sha256_16"], "synthetic generator drifted"
    assert scale_cases.sample_sizes(reads) == {int(k): v for k, v in exp["reads_per_length"].items()}
    exe = _exe(w["mode"])
    bad = []
    plan = scale_cases.runs(name, w, reads, d)
    done = []
    for lab, src, seeds, sam, un in plan:
        if scale_cases.skip_run(src):
            continue
        done.append(lab)
        p = subprocess.run([exe] + scale_cases.command_args(w, seeds, src, sam, un, ref), cwd=d, capture_output=True,
                           timeout=3600)
        assert p.returncode == 0, (lab, p.stderr[-3000:])
        h, n = scale_cases.digest_sam(sam)
        e = exp["runs"][lab]
        if h != e["sam_sha256"] or n != e["records"]:
            bad.append((lab, "sam", n, e["records"]))
        if scale_cases.digest_file(un) != e["unmapped_fastq_sha256"]:
            bad.append((lab, "unmapped fastq"))
    assert not bad, bad
    assert sorted(done) == sorted(exp["runs"]), (done, sorted(exp["runs"]))
    if scale_cases.CASES[name]["kind"] == "buckets":
        mixed_sam, mixed_un = os.path.join(d, "mixed.sam"), os.path.join(d, "mixed.un.fq")
        p = subprocess.run([exe] + scale_cases.command_args(w, None, reads, mixed_sam, mixed_un, ref), cwd=d,
                           capture_output=True, timeout=3600)
        assert p.returncode == 0, p.stderr[-3000:]
        assert _records(mixed_sam) == b"".join(_records(sam) for _, _, _, sam, _ in plan)
        with open(mixed_un, "rb") as f:
            mixed_unmapped = f.read()
        parts = []
        for _, _, _, _, un in plan:
            with open(un, "rb") as f:
                parts.append(f.read())
        assert mixed_unmapped == b"".join(parts)
