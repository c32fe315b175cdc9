"""End-to-end parity on the CPU: the reference binary (oracle/_ref, built from its sources)
against the product's front end (loader, tag sort, SAM and FASTQ writers) driven by the
oracle mapper (oracle/storm-oracle-*), on small seeded inputs over the option surface.

The reference is run with MALLOC_PERTURB_=255 (every malloc returns zeroed memory): in colour
space its SAM writer ORs bits into an uninitialised buffer (hit_map.c:243-251) and the
quality loader reads one past the parsed qualities (read_quality.c:38), so without it the
reference's own output changes from run to run.  The @PG line (argv echo) is compared with
the binary name normalised."""
import os
import subprocess

import numpy as np
import pytest

import ffi
from storm_b200 import synth

pytestmark = pytest.mark.skipif(not ffi.ref_available(), reason="oracle/_ref not built")

ORACLE_BIN = {0: os.path.join(ffi.ORACLE_DIR, "storm-oracle-nucleotide"),
              1: os.path.join(ffi.ORACLE_DIR, "storm-oracle-color")}
REF_BIN = {0: os.path.join(ffi.REF_DIR, "storm-nucleotide"), 1: os.path.join(ffi.REF_DIR, "storm-color")}


def _build():
    subprocess.run(["make", "-s", "-C", ffi.ORACLE_DIR, "storm-oracle-nucleotide",
                    "storm-oracle-color"], check=True)


def run_pair(tmp, colour, args, ref="ref.fa", reads="reads.fq", outputs=("out.sam", "un.fq")):
    _build()
    res = {}
    for name, exe in (("ref", REF_BIN[colour]), ("new", ORACLE_BIN[colour])):
        cmd = [exe, "-g", ref, "-r", reads, "-o", name + "_" + outputs[0], "-v", "0"] + list(args)
        if "-O" not in args and outputs[1]:
            cmd += ["-O", name + "_" + outputs[1]]
        env = dict(os.environ, MALLOC_PERTURB_="255")
        p = subprocess.run(cmd, cwd=tmp, env=env, capture_output=True, timeout=600)
        res[name] = p
    for name in ("ref", "new"):
        assert res[name].returncode == res["ref"].returncode, (name, res[name].stderr[-2000:])
    if res["ref"].returncode != 0:
        return None
    out = {}
    for name in ("ref", "new"):
        with open(os.path.join(tmp, name + "_" + outputs[0]), "rb") as f:
            lines = f.read().split(b"\n")
        out[name] = [l for l in lines if not l.startswith(b"@PG")]
        pg = [l for l in lines if l.startswith(b"@PG")]
        assert len(pg) == 1
        out[name + "_pg"] = pg[0].split(b"-g", 1)[1].replace(name.encode() + b"_", b"X_")
    assert out["ref"] == out["new"], _first_diff(out["ref"], out["new"])
    assert out["ref_pg"] == out["new_pg"]
    if outputs[1]:
        a = open(os.path.join(tmp, "ref_" + outputs[1]), "rb").read()
        b = open(os.path.join(tmp, "new_" + outputs[1]), "rb").read()
        assert a == b
    return out["ref"]


def _first_diff(a, b):
    for i, (x, y) in enumerate(zip(a, b)):
        if x != y:
            return "line %d:\nref %r\nnew %r" % (i, x, y)
    return "lengths %d vs %d" % (len(a), len(b))


def _mapped(lines):
    return sum(1 for l in lines if l and not l.startswith(b"@"))


@pytest.fixture(scope="module")
def nuc_data(tmp_path_factory):
    d = tmp_path_factory.mktemp("nuc")
    synth.generate(0, 0.05, str(d / "ref.fa"), str(d / "reads.fq"))
    return str(d)


@pytest.mark.parametrize("args", [
    ["-M", "1", "-z", "100", "-t", "100", "-i", "3", "-b", "33"],
    ["-M", "4", "-A", "-z", "90", "-t", "95"],
    ["-M", "2", "-F"],
    ["-M", "3", "-R", "-u", "5"],
    ["-M", "4", "-i", "0", "-z", "60", "-t", "60"],
    ["-M", "1", "-i", "1"],
    ["-M", "4", "-i", "7", "-z", "80"],
    ["-M", "4", "-i", "15", "-z", "80"],
    ["-M", "4", "-i", "20", "-z", "70", "-t", "90"],
    ["-M", "4", "-l", "3"],
    ["-M", "4", "-l", "0", "-s", "#####-##-###;####--##-####"],
    ["-M", "4", "-s", "###-##-#######:0 5 10 20 30"],
    ["-M", "1", "-m", "3", "-x", "-2", "-d", "-5", "-e", "-1", "-t", "60", "-z", "60"],
    ["-M", "1", "-b", "30"],
])
def test_nucleotide_options(nuc_data, args):
    lines = run_pair(nuc_data, 0, args)
    assert _mapped(lines) > 0


def test_bad_quality_base_fails_like_reference(nuc_data):
    """Quality characters below -b are an input error (read_quality.c:197-208): exit -1."""
    assert run_pair(nuc_data, 0, ["-M", "1", "-b", "48"]) is None


@pytest.fixture(scope="module")
def col_data(tmp_path_factory):
    d = tmp_path_factory.mktemp("col")
    synth.generate(1, 0.004, str(d / "ref.fa"), str(d / "reads.fq"))
    return str(d)


@pytest.mark.parametrize("args", [
    ["-M", "1", "-z", "105", "-t", "120", "-i", "7", "-s",
     "####-##-#-####;###-#--##-##--###;####-#---#----#--####"],
    ["-M", "4", "-A", "-i", "3"],
    ["-M", "2", "-i", "10", "-z", "90", "-t", "100"],
])
def test_colour_options(col_data, args):
    lines = run_pair(col_data, 1, args)
    assert _mapped(lines) > 0


def test_masked_multi_sequence(tmp_path):
    """N runs in the reference (masked regions, rand()&3 codes), several sequences, an N at the
    very start and end, lowercase letters, and N / lowercase bases inside reads."""
    rng = np.random.default_rng(5)
    genome = synth.make_genome([30000, 12000, 5000], 9)
    text = []
    for name, seq in genome:
        s = bytearray(synth.BASES[seq].tobytes())
        for _ in range(6):
            a = int(rng.integers(0, len(s) - 50))
            s[a:a + int(rng.integers(1, 40))] = b"N" * len(s[a:a + int(rng.integers(1, 40))])
        s[0:3] = b"NNN"
        s[-2:] = b"NN"
        low = int(rng.integers(0, len(s) - 100))
        s[low:low + 60] = s[low:low + 60].lower()
        text.append(b">" + name.encode() + b" some description\n" +
                    b"\n".join(bytes(s[i:i + 70]) for i in range(0, len(s), 70)) + b"\n")
    (tmp_path / "ref.fa").write_bytes(b"".join(text))
    seqs, quals = synth.simulate_nucleotide_reads(genome, 3000, 50, 8)
    synth.write_fastq(str(tmp_path / "reads.fq"), seqs, quals)
    raw = bytearray((tmp_path / "reads.fq").read_bytes())
    lines = raw.split(b"\n")
    for k in range(1, len(lines), 40):
        if k % 4 == 1 and len(lines[k]) > 10:
            lines[k] = lines[k][:5] + b"N" + lines[k][6:8].lower() + lines[k][8:]
    (tmp_path / "reads.fq").write_bytes(b"\n".join(lines))
    run_pair(str(tmp_path), 0, ["-M", "4", "-A", "-z", "90", "-t", "95"])
    run_pair(str(tmp_path), 0, ["-M", "4", "-j", "-z", "90", "-t", "95"])


@pytest.mark.parametrize("args", [
    ["-z", "100", "-t", "100", "-i", "3"],          # contextual placement (default without -M)
    ["-G", "-z", "100", "-t", "100", "-i", "3"],    # greedy placement
    ["-i", "7", "-z", "80", "-t", "90"],            # more indels: inserted-code counters
    ["-u", "5", "-z", "90", "-t", "95"],
    ["-G", "-u", "5", "-z", "90", "-t", "95"],
    ["-i", "0", "-z", "60", "-t", "60"],
])
def test_genome_map_nucleotide(nuc_data, args):
    """The mapping without -M (genome_map.c): reads placed per reference position, SAM written
    position-major."""
    lines = run_pair(nuc_data, 0, args)
    assert _mapped(lines) > 0


@pytest.mark.parametrize("args", [
    ["-z", "105", "-t", "120", "-i", "7"],
    ["-G", "-i", "3"],
])
def test_genome_map_colour(col_data, args):
    lines = run_pair(col_data, 1, args)
    assert _mapped(lines) > 0


def test_genome_map_repeats_stack_reads(tmp_path):
    """Reads piled on repeated and overlapping positions, so that the contextual rescoring
    against the consensus decides between copies."""
    genome = synth.make_genome([40000], 12, 0.45, 0.5)
    synth.write_fasta(str(tmp_path / "ref.fa"), genome)
    seqs, quals = synth.simulate_nucleotide_reads(genome, 4000, 50, 13,
                                                  synth.ReadModel(indel_rate=0.01, indel_max=2))
    synth.write_fastq(str(tmp_path / "reads.fq"), seqs, quals)
    lines = run_pair(str(tmp_path), 0, ["-i", "5", "-z", "90", "-t", "95"])
    assert _mapped(lines) > 1000


def test_fasta_reads(tmp_path):
    """Nucleotide reads as FASTA (no qualities): some sequences wrapped over two lines, a header
    without a sequence (its name passes to the next record), comments and a title first."""
    genome = synth.make_genome([30000], 17)
    synth.write_fasta(str(tmp_path / "ref.fa"), genome)
    seqs, _ = synth.simulate_nucleotide_reads(genome, 1500, 50, 18)
    with open(tmp_path / "reads.fa", "wb") as f:
        f.write(b"# Title: fasta reads\n# another comment\n")
        for k, s in enumerate(seqs):
            b = synth.BASES[s].tobytes()
            if k == 10:
                f.write(b">orphan header\n")
            f.write(b">r%d some text\n" % k)
            f.write(b[:20] + b"\n" + b[20:] + b"\n" if k % 7 == 0 else b + b"\n")
    lines = run_pair(str(tmp_path), 0, ["-M", "2", "-z", "90", "-t", "95"], reads="reads.fa")
    assert _mapped(lines) > 500


@pytest.mark.parametrize("with_qual", [True, False])
def test_csfasta_reads(tmp_path, with_qual):
    """Colour reads as CSFASTA (primer base + colours), with the qualities in a .qual file of
    integers (-q): comments and headers there too, a negative value, and short lines."""
    genome = synth.make_genome([40000], 19)
    synth.write_fasta(str(tmp_path / "ref.fa"), genome)
    pr, cols, q = synth.simulate_colour_reads(genome, 1500, 50, 20)
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
            if k % 7 in (5, 6):
                v = v[:len(v) - 1 - k % 5]  # more short lines, two in a row
            if k % 97 == 11:
                v = v[:3]
            f.write(b">r%d_F3\n%s\n" % (k, b" ".join(b"%d" % x for x in v)))
    args = ["-M", "2", "-z", "90", "-t", "100", "-i", "5"] + (["-q", "reads.qual"] if with_qual else [])
    lines = run_pair(str(tmp_path), 1, args, reads="reads.csfasta")
    assert _mapped(lines) > 500


@pytest.mark.parametrize("colour,args", [
    (0, ["-M", "4", "-A", "-z", "90", "-t", "95"]),
    (1, ["-M", "2", "-i", "7", "-z", "105", "-t", "110"]),
])
def test_pipelined_sam_output_is_the_same(nuc_data, col_data, colour, args):
    """The front end maps a large read set in pieces and writes each piece's SAM records from a
    second thread while the next maps (STORM_PIPE_MIN_READS lowers the size at which it does so):
    the SAM and -O files are those of the one-piece run, byte for byte."""
    _build()
    d = col_data if colour else nuc_data
    outs = {}
    for tag, env_extra in (("whole", {}), ("pieces", {"STORM_PIPE_MIN_READS": "2"})):
        env = dict(os.environ, MALLOC_PERTURB_="255", **env_extra)
        cmd = [ORACLE_BIN[colour], "-g", "ref.fa", "-r", "reads.fq", "-o", tag + ".sam", "-O", tag + ".un.fq",
               "-v", "0"] + args
        p = subprocess.run(cmd, cwd=d, env=env, capture_output=True, timeout=600)
        assert p.returncode == 0, p.stderr[-2000:]
        with open(os.path.join(d, tag + ".sam"), "rb") as f:
            sam = [l for l in f.read().split(b"\n") if not l.startswith(b"@PG")]
        with open(os.path.join(d, tag + ".un.fq"), "rb") as f:
            outs[tag] = (sam, f.read())
    assert _mapped(outs["whole"][0]) > 0
    assert outs["pieces"] == outs["whole"]


def _fastq_text(seqs, quals, names=None):
    out = []
    for k, (s, q) in enumerate(zip(seqs, quals)):
        out.append(b"@" + (names[k] if names else b"r%d extra words" % k) + b"\n")
        out.append(synth.BASES[s].tobytes() + b"\n+\n" + bytes(int(v) + 33 for v in q) + b"\n")
    return b"".join(out)


@pytest.mark.parametrize("colour,case", [(0, "header_without_at"), (0, "missing_plus"), (0, "empty_sequence"),
                                         (0, "crlf"), (0, "title_comments"), (0, "last_record_without_quality"),
                                         (0, "last_record_without_quality_unmapped"),
                                         (0, "blank_line_between_records"), (1, "last_record_without_quality"),
                                         (1, "last_record_without_quality_unmapped"), (1, "missing_plus")])
def test_fastq_layouts_and_errors_like_reference(tmp_path, colour, case):
    """FASTQ read files of unusual layout, valid or not (reads_data.c:351-566): the exit code, the
    error message, and for a valid file the SAM and unmapped FASTQ must be the reference's (a
    record cut short before its quality line keeps a NULL quality there)."""
    genome = synth.make_genome([20000], 23)
    synth.write_fasta(str(tmp_path / "ref.fa"), genome)
    if colour:
        pr, cols, q = synth.simulate_colour_reads(genome, 400, 49, 24)
        synth.write_colour_fastq(str(tmp_path / "col.fq"), pr, cols, q)
        text = (tmp_path / "col.fq").read_bytes()
    else:
        seqs, quals = synth.simulate_nucleotide_reads(genome, 400, 50, 24)
        text = _fastq_text(seqs, quals)
    recs = text.split(b"\n")  # 4 lines per record
    if case == "last_record_without_quality_unmapped":  # a read that maps nowhere, then cut short
        rnd = np.random.default_rng(25).integers(0, 4, size=len(recs[-4]))
        recs[-4] = (recs[-4][:1] + bytes(b"0123"[v] for v in rnd[1:])) if colour else bytes(b"ACGT"[v] for v in rnd)
        case = "last_record_without_quality"
    if case == "header_without_at":
        recs[4 * 37] = recs[4 * 37][1:]
    elif case == "missing_plus":
        del recs[4 * 51 + 2]
    elif case == "empty_sequence":
        recs[4 * 12 + 1] = b""
    elif case == "crlf":
        recs = [l + b"\r" if l else l for l in recs]
    elif case == "title_comments":
        recs = [b"# Title: layout test", b"# a comment"] + recs
    elif case == "last_record_without_quality":
        recs = recs[:-2]
    elif case == "blank_line_between_records":
        recs.insert(4 * 20, b"")
    (tmp_path / "reads.fq").write_bytes(b"\n".join(recs))
    _build()
    res = {}
    for name, exe in (("ref", REF_BIN[colour]), ("new", ORACLE_BIN[colour])):
        p = subprocess.run([exe, "-g", "ref.fa", "-r", "reads.fq", "-o", name + ".sam", "-O", name + ".fq", "-v", "0",
                            "-M", "1", "-z", "90", "-t", "95"] + (["-i", "7"] if colour else []), cwd=str(tmp_path),
                           env=dict(os.environ, MALLOC_PERTURB_="255"), capture_output=True, timeout=600)
        res[name] = p
    assert res["new"].returncode == res["ref"].returncode, (res["ref"].stderr[-500:], res["new"].stderr[-500:])
    if res["ref"].returncode != 0:
        assert res["new"].stderr == res["ref"].stderr
        return
    for ext in (".sam", ".fq"):
        a = [l for l in (tmp_path / ("ref" + ext)).read_bytes().split(b"\n") if not l.startswith(b"@PG")]
        b = [l for l in (tmp_path / ("new" + ext)).read_bytes().split(b"\n") if not l.startswith(b"@PG")]
        assert a == b, _first_diff(a, b)
