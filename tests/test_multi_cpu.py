"""The read-sharded path for several GPUs (storm_b200.multi), covered on CPU: the shard split,
and two gloo ranks under torchrun that each map their slice (the oracle mapper standing in for
the GPU) and gather the records to rank 0 in order; the SAM rank 0 writes must equal the
single-process oracle CLI's, byte for byte outside the @PG line."""
import os
import socket
import subprocess
import sys

import pytest

import ffi
from storm_b200 import multi, synth

HERE = os.path.dirname(os.path.abspath(__file__))


def test_shard_range_partitions_contiguously():
    for n in (0, 1, 7, 100, 101, 1000003):
        for world in (1, 2, 3, 8):
            spans = [multi.shard_range(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            for (a, b), (c, _) in zip(spans, spans[1:]):
                assert b == c
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        multi.shard_range(10, 2, 2)


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.mark.parametrize("colour", [0, 1])
def test_two_ranks_gather_in_order_and_match_the_oracle_cli(tmp_path, colour):
    ffi.ensure_built()
    subprocess.run(["make", "-s", "-C", ffi.ORACLE_DIR, "storm-oracle-nucleotide", "storm-oracle-color"],
                   check=True)
    d = str(tmp_path)
    genome = synth.make_genome([30000, 12000], 21 + colour)
    synth.write_fasta(os.path.join(d, "ref.fa"), genome)
    if colour:
        pr, cols, q = synth.simulate_colour_reads(genome, 301, 50, 5)
        synth.write_colour_fastq(os.path.join(d, "reads.fq"), pr, cols, q)
    else:
        seqs, quals = synth.simulate_nucleotide_reads(genome, 301, 50, 5)
        synth.write_fastq(os.path.join(d, "reads.fq"), seqs, quals)
    args = ["-g", "ref.fa", "-r", "reads.fq", "-M", "2", "-z", "100", "-t", "100", "-i", "3"]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_port()), os.path.join(HERE, "multi_worker.py"), d]
    cmd += (["--colour"] if colour else []) + args + ["-o", "multi.sam"]
    p = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-3000:] + p.stderr[-3000:]
    exe = os.path.join(ffi.ORACLE_DIR, "storm-oracle-color" if colour else "storm-oracle-nucleotide")
    q = subprocess.run([exe] + args + ["-o", "single.sam", "-v", "0"], cwd=d, capture_output=True, timeout=600)
    assert q.returncode == 0, q.stderr[-2000:]

    def body(name):
        with open(os.path.join(d, name), "rb") as f:
            return [l for l in f.read().split(b"\n") if not l.startswith(b"@PG")]
    single, sharded = body("single.sam"), body("multi.sam")
    assert len(single) > 300
    assert single == sharded
