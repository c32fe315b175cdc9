"""The device placements of the mapping without -M (genome_map.c) against the host restatement
(storm_host.c sh_genome_map_contextual, pinned to the reference by tests/test_e2e_cpu.py), on the
same device records: reads piled on a half-repeated genome, so that the contextual rescoring
decides between copies and the device waves run long chains of reads sharing positions."""
import ctypes as C

import numpy as np
import pytest

from storm_b200 import api, build, host, multi, pipeline, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    build.build()
    if not api.device_available():
        pytest.fail("no CUDA device: GPU tests need a B200")


class Placement(C.Structure):
    _fields_ = [("read", C.c_int32), ("rank", C.c_int32)]


def _host_contextual(rm, reads, res, uniq):
    L = host.hostlib()
    L.sh_genome_map_contextual.argtypes = [C.POINTER(host.ShRefs), C.POINTER(api.Results), C.c_int64, C.c_int,
                                           C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                           C.POINTER(C.c_int64)]
    out = (Placement * max(1, reads.n))()
    npl = C.c_int64(0)
    p = rm.params
    rr = res.cstruct()
    assert L.sh_genome_map_contextual(C.byref(rm.reference._s), C.byref(rr), reads.n, p.colour, p.allowed_indels,
                                      p.match, p.mismatch, 0 if uniq is None else 1, uniq or 0, out,
                                      C.byref(npl)) == 0
    got = np.frombuffer(out, dtype=np.int32).reshape(-1, 2)[:npl.value]
    return got[:, 0].copy(), got[:, 1].copy()


@pytest.mark.parametrize("colour,uniq", [(0, None), (0, 4), (1, None)])
def test_device_placements_match_the_host_restatement(tmp_path, colour, uniq):
    genome = synth.make_genome([40000], 12 + colour, 0.45, 0.5)
    synth.write_fasta(str(tmp_path / "ref.fa"), genome)
    if colour:
        pr, cols, q = synth.simulate_colour_reads(genome, 4000, 50, 14)
        synth.write_colour_fastq(str(tmp_path / "reads.fq"), pr, cols, q)
        args = ["-i", "5", "-z", "90", "-t", "110", "-M", "1"]
    else:
        seqs, quals = synth.simulate_nucleotide_reads(genome, 4000, 50, 13,
                                                      synth.ReadModel(indel_rate=0.01, indel_max=2))
        synth.write_fastq(str(tmp_path / "reads.fq"), seqs, quals)
        args = ["-i", "5", "-z", "90", "-t", "95", "-M", "1"]
    rm = pipeline.ResidentMapper(str(tmp_path / "ref.fa"), args, colour=colour,
                                 default_seeds=multi.DEFAULT_SEEDS[colour])
    reads = host.ReadSet(str(tmp_path / "reads.fq"), colour)
    tbs = ((reads.max_len + rm.params.allowed_indels + 1) // 2 + 7) & ~7
    res = rm.mapper.map(reads.batch(), tbs)
    d_read, d_rank = rm.mapper.genome_map(reads.n, uniqueness_threshold=uniq)
    waves = rm.mapper.stats()["placement_waves"]
    g_read, _ = rm.mapper.genome_map(reads.n, greedy=True, uniqueness_threshold=uniq)
    h_read, h_rank = _host_contextual(rm, reads, res, uniq)
    rm.close()
    assert len(h_read) > 1000
    assert np.array_equal(d_read, h_read) and np.array_equal(d_rank, h_rank)
    if uniq is None:  # (with -u the reads left are those whose best rank leads clearly)
        assert (h_rank > 0).sum() > 0  # some reads placed at a rank other than their best
    assert waves > 5, waves
    # greedy: every read at its rank-0 start (and its uniqueness test), positions in order, read order within one
    ok = res.hits["ref_start"].reshape(-1, 4)[:, 0] != -1
    ok &= res.mapped != 0
    if uniq is not None:
        sc = res.hits["score"].reshape(-1, 4)
        ok &= sc[:, 0] - sc[:, 1] >= uniq
    idx = np.nonzero(ok)[0]
    h0 = res.hits.reshape(-1, 4)[idx, 0]
    order = np.lexsort((idx, h0["ref_start"], h0["ref_id"]))
    assert np.array_equal(g_read, idx[order])
