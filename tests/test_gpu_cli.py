"""End to end on the GPU: the storm-nucleotide / storm-color binaries (CUDA library behind the
reference's command line) against the golden SAM / FASTQ produced by the reference itself,
and, when oracle/_ref is present, against a live reference run on a larger input."""
import os
import subprocess

import pytest

import ffi
import golden_cases
from storm_b200 import api, build, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()


def _exe(mode):
    return os.path.join(build.BIN_DIR, "storm-color" if mode == "colour" else "storm-nucleotide")


@pytest.mark.parametrize("name", sorted(golden_cases.meta()))
def test_gpu_cli_matches_golden(name, tmp_path):
    assert golden_cases.check_case(name, str(tmp_path), _exe) > 0


@pytest.mark.skipif(not ffi.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("cfg,scale,extra", [(0, 0.2, []), (1, 0.02, []), (0, 0.05, ["-M", "4", "-A", "-i", "20", "-z", "70"])])
def test_gpu_cli_matches_reference(cfg, scale, extra, tmp_path):
    _live(cfg, scale, extra, tmp_path)


def _without_m(args):
    out, i = [], 0
    while i < len(args):
        if args[i] == "-M":
            i += 2
            continue
        out.append(args[i])
        i += 1
    return out


@pytest.mark.skipif(not ffi.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("cfg,scale,extra", [(0, 0.2, []), (0, 0.2, ["-G"]), (0, 0.05, ["-G", "-u", "5", "-i", "7"]),
                                             (0, 0.05, ["-u", "5", "-i", "7"]), (1, 0.02, []), (1, 0.05, ["-u", "3"]),
                                             (1, 0.02, ["-G"])])
def test_gpu_cli_genome_map_matches_reference(cfg, scale, extra, tmp_path):
    """Without -M: the per-position map (greedy placement by a device sort, contextual placement
    in device waves), SAM written position-major."""
    _live(cfg, scale, extra, tmp_path, strip_m=True)


@pytest.mark.skipif(not ffi.ref_available(), reason="oracle/_ref not built")
def test_gpu_cli_contextual_placement_of_piled_reads(tmp_path):
    """Reads piled on repeated and overlapping positions (40 kbp, half of it repeats, 4,000 reads
    with indels): the contextual rescoring against the consensus decides between copies, and the
    device waves run long chains of reads that share positions."""
    genome = synth.make_genome([40000], 12, 0.45, 0.5)
    synth.write_fasta(str(tmp_path / "ref.fa"), genome)
    seqs, quals = synth.simulate_nucleotide_reads(genome, 4000, 50, 13, synth.ReadModel(indel_rate=0.01, indel_max=2))
    synth.write_fastq(str(tmp_path / "reads.fq"), seqs, quals)
    outs = {}
    for tag, exe in (("ref", os.path.join(ffi.REF_DIR, "storm-nucleotide")), ("gpu", _exe("nucleotide"))):
        p = subprocess.run([exe, "-g", "ref.fa", "-r", "reads.fq", "-o", tag + ".sam", "-v", "0", "-i", "5", "-z", "90",
                            "-t", "95"], cwd=str(tmp_path), env=dict(os.environ, MALLOC_PERTURB_="255"),
                           capture_output=True, timeout=600)
        assert p.returncode == 0, p.stderr[-3000:]
        outs[tag] = [l for l in (tmp_path / (tag + ".sam")).read_bytes().split(b"\n") if not l.startswith(b"@PG")]
    assert outs["gpu"] == outs["ref"]
    assert sum(1 for l in outs["gpu"] if l and not l.startswith(b"@")) > 1000


def _live(cfg, scale, extra, tmp_path, strip_m=False):
    w = synth.generate(cfg, scale, str(tmp_path / "ref.fa"), str(tmp_path / "reads.fq"))
    args = (_without_m(w["args"]) if strip_m else w["args"]) + extra
    colour = w["mode"] == "colour"
    outs = {}
    for tag, exe in (("ref", os.path.join(ffi.REF_DIR, "storm-color" if colour else "storm-nucleotide")),
                     ("gpu", _exe(w["mode"]))):
        p = subprocess.run([exe, "-g", "ref.fa", "-r", "reads.fq", "-o", tag + ".sam", "-O", tag + ".fq", "-v", "0"] + args,
                           cwd=str(tmp_path), env=dict(os.environ, MALLOC_PERTURB_="255"), capture_output=True,
                           timeout=1800)
        assert p.returncode == 0, p.stderr[-3000:]
        lines = (tmp_path / (tag + ".sam")).read_bytes().split(b"\n")
        outs[tag] = [l for l in lines if not l.startswith(b"@PG")], (tmp_path / (tag + ".fq")).read_bytes()
    assert outs["gpu"][0] == outs["ref"][0]
    assert outs["gpu"][1] == outs["ref"][1]


@pytest.mark.parametrize("cfg,scale,extra", [(0, 0.05, []), (1, 0.01, []), (0, 0.05, ["-M", "3", "-A", "-i", "7"])])
def test_resident_front_end_matches_cli(cfg, scale, extra, tmp_path):
    """storm_b200.pipeline.ResidentMapper (reference and index resident, read file in, SAM out):
    the same records and unmapped reads as the command line, on two read files in a row."""
    from storm_b200 import pipeline
    w = synth.generate(cfg, scale, str(tmp_path / "ref.fa"), str(tmp_path / "reads.fq"))
    args = _without_m(w["args"]) + (extra if "-M" in extra else ["-M", "1"] + extra)
    colour = w["mode"] == "colour"
    seeds = None if "-s" in args else (synth_default_seeds(colour))
    half = tmp_path / "half.fq"
    with open(tmp_path / "reads.fq", "rb") as f, open(half, "wb") as o:
        lines = f.readlines()
        o.writelines(lines[:4 * (len(lines) // 8)])
    rm = pipeline.ResidentMapper(str(tmp_path / "ref.fa"), args, colour=int(colour), default_seeds=seeds)
    try:
        for name in ("reads.fq", "half.fq"):
            p = subprocess.run([_exe(w["mode"]), "-g", "ref.fa", "-r", name, "-o", "cli.sam", "-O", "cli.fq",
                                "-v", "0"] + args, cwd=str(tmp_path), capture_output=True, timeout=600)
            assert p.returncode == 0, p.stderr[-2000:]
            rm.map_file(str(tmp_path / name), str(tmp_path / "res.sam"), str(tmp_path / "res.fq"))
            body = [(tmp_path / x).read_bytes().split(b"\n") for x in ("cli.sam", "res.sam")]
            assert [l for l in body[0] if not l.startswith(b"@PG")] == [l for l in body[1] if not l.startswith(b"@PG")]
            assert (tmp_path / "cli.fq").read_bytes() == (tmp_path / "res.fq").read_bytes()
    finally:
        rm.close()


def synth_default_seeds(colour):
    """The command line's default seed family when no seeds file is found (seed.h:22-33)."""
    return ("####----##--##-####;####-###--#----####;####-####-####" if colour
            else "####--#-#--##--####;#####--###-#-###;###-##-#######")


def _write_csfasta(tmp_path, n=1500):
    genome = synth.make_genome([40000], 19)
    synth.write_fasta(str(tmp_path / "ref.fa"), genome)
    pr, cols, q = synth.simulate_colour_reads(genome, n, 50, 20)
    with open(tmp_path / "reads.csfasta", "wb") as f:
        f.write(b"# Title: solid set\n")
        for k in range(len(cols)):
            f.write(b">r%d_F3\n%c%s\n" % (k, synth.BASES[pr[k]], synth.COLOURS[cols[k]].tobytes()))
    with open(tmp_path / "reads.qual", "wb") as f:
        f.write(b"# qualities\n")
        for k in range(len(cols)):
            v = [int(x) for x in q[k]]
            if k % 50 == 3:
                v[5] = -1
            if k == 77:
                v = v[:30]  # short line: the rest keeps the previous read's values
            f.write(b">r%d_F3\n%s\n" % (k, b" ".join(b"%d" % x for x in v)))


def _both(tmp_path, colour, args, tags=("ref", "gpu")):
    """Run the reference binary and the GPU binary with the same arguments in tmp_path; returns
    {tag: (SAM lines without @PG, -O FASTQ bytes)}."""
    outs = {}
    for tag in tags:
        exe = (os.path.join(ffi.REF_DIR, "storm-color" if colour else "storm-nucleotide") if tag == "ref"
               else _exe("colour" if colour else "nucleotide"))
        p = subprocess.run([exe, "-o", tag + ".sam", "-O", tag + ".fq", "-v", "0"] + args, cwd=str(tmp_path),
                           env=dict(os.environ, MALLOC_PERTURB_="255"), capture_output=True, timeout=1800)
        assert p.returncode == 0, (tag, p.stderr[-3000:])
        lines = (tmp_path / (tag + ".sam")).read_bytes().split(b"\n")
        outs[tag] = [l for l in lines if not l.startswith(b"@PG")], (tmp_path / (tag + ".fq")).read_bytes()
    return outs


@pytest.mark.skipif(not ffi.ref_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("with_qual", [True, False])
def test_gpu_cli_csfasta_matches_reference(with_qual, tmp_path):
    """Colour reads as CSFASTA with an integer .qual file (-q; a negative value, a short line)
    or without qualities (reads_data.c:73-345), through the GPU binary and the reference."""
    _write_csfasta(tmp_path)
    args = ["-g", "ref.fa", "-r", "reads.csfasta", "-M", "2", "-z", "90", "-t", "100", "-i", "5"] + \
        (["-q", "reads.qual"] if with_qual else [])
    outs = _both(tmp_path, True, args)
    assert outs["gpu"] == outs["ref"]
    assert sum(1 for l in outs["ref"][0] if l and not l.startswith(b"@")) > 500


@pytest.mark.skipif(not ffi.ref_available(), reason="oracle/_ref not built")
def test_gpu_cli_colour_chain_matches_reference(tmp_path):
    """Colour -O chain: each step maps the previous step's unmapped FASTQ, which has lost one
    colour (hit_map.c:541-547), with a stricter seed family; GPU and reference, step by step."""
    synth.generate(1, 0.01, str(tmp_path / "ref.fa"), str(tmp_path / "reads.fq"))
    src = "reads.fq"
    # a contiguous w15 seed at read position 0 only, then w14 at positions 0 and 5, then a
    # spaced w11 seed: about half the reads, then a third of the rest, stay unmapped
    for k, seeds in enumerate(["###############:0", "##############:0 5", "####-##-#-####"]):
        args = ["-g", "ref.fa", "-r", src, "-M", "1", "-z", "100", "-t", "115", "-i", "7", "-s", seeds]
        outs = _both(tmp_path, True, args)
        assert outs["gpu"] == outs["ref"], k
        assert sum(1 for l in outs["ref"][0] if l and not l.startswith(b"@")) > 1000, k
        if k < 2:
            assert outs["ref"][1].count(b"\n") > 4000, k
        nxt = "step%d.fq" % k
        (tmp_path / nxt).write_bytes(outs["ref"][1])
        src = nxt
