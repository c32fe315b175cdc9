"""Test infrastructure: one rank of the read-sharded mapping path (storm_b200.multi), run on
CPU under torchrun with the gloo backend; the oracle mapper stands in for the GPU mapper.

    torchrun --nproc-per-node 2 tests/multi_worker.py <dir> <args...>

Rank 0 checks that the ordered gather equals the single-process result and writes the SAM
from it to <dir>/multi.sam."""
import argparse
import ctypes as C
import datetime
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import numpy as np  # noqa: E402
import torch.distributed as dist  # noqa: E402

import ffi  # noqa: E402
from storm_b200 import api, host, multi  # noqa: E402


def oracle_mapper(reference, prm, seeds):
    orc = ffi.oracle()
    seqs = list(reference.sequences())
    keep = []
    refs = (ffi.OrRef * len(seqs))()
    for k, (codes, mask, n, regs) in enumerate(seqs):
        rs = np.array([a for a, _ in regs] or [0], np.int32)
        re = np.array([b for _, b in regs] or [0], np.int32)
        keep += [rs, re]
        refs[k] = ffi.OrRef(codes, mask, n, rs.ctypes.data, re.ctypes.data, len(regs))

    def run(batch, tbs):
        res = api.MapResults(batch.n, tbs)
        rd = ffi.ReadsT(batch.n, batch.codes.ctypes.data, batch.codes.shape[1],
                        batch.levels.ctypes.data if batch.levels is not None else None,
                        batch.levels.shape[1] if batch.levels is not None else 0, batch.lengths.ctypes.data,
                        batch.first_levels.ctypes.data if batch.first_levels is not None else None)
        out = ffi.ResultsT(res.hits.ctypes.data, res.tb.ctypes.data, tbs, res.mapped.ctypes.data)
        assert orc.or_map(C.byref(prm), seeds.encode(), refs, len(seqs), C.byref(rd), C.byref(out), None) == 0
        return res
    run.keep = (keep, refs)
    return run


def main():
    d = sys.argv[1]
    a = multi._parse(sys.argv[2:])
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
    rank = dist.get_rank()
    colour = 1 if a.colour else 0
    reads = host.ReadSet(os.path.join(d, a.r), colour, quality_base=a.b)
    reference = host.Reference(os.path.join(d, a.g), colour)
    prm = ffi.make_params(colour=colour, match=a.m, mismatch=a.x, gap_open=a.d, gap_extend=a.e, indels=a.i,
                          min_score=a.t, min_score_filter=a.z, stdev=a.l)
    seeds = a.s or multi.DEFAULT_SEEDS[colour]
    map_fn = oracle_mapper(reference, prm, seeds)
    tbs = ((reads.max_len + a.i + 1) // 2 + 7) & ~7
    res = multi.map_sharded(map_fn, reads.batch(), tbs)
    if rank == 0:
        whole = map_fn(reads.batch(), tbs)
        assert res.hits.tobytes() == whole.hits.tobytes()
        assert res.tb.tobytes() == whole.tb.tobytes()
        assert res.mapped.tobytes() == whole.mapped.tobytes()
        multi.write_sam(os.path.join(d, a.o), reference, reads, res, colour, a,
                        ["storm", "-g"] + sys.argv[3:])
    dist.barrier()
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
