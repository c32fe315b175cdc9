"""Read-sharded mapping on several GPUs of one node.

One process per GPU (torchrun); every rank loads the reference and the reads, maps the
contiguous slice of the tag-sorted reads that `shard_range` gives it against its own replica
of the reference and index, and rank 0 gathers the per-read records in rank order and writes
the SAM.  Reads are independent (the top-4 table of a read depends on that read alone), so the
data path has no collective; the one exchange is the final ordered gather of results, whose
concatenation in rank order is the single-GPU result.

    python -m torch.distributed.run --nproc-per-node N --master-addr 127.0.0.1 \\
        -m storm_b200.multi [--colour] -g ref.fa -r reads.fq -o out.sam [-M k -s seeds -z -t -i ...]
"""
from __future__ import annotations

import argparse
import ctypes as C
import os
import sys

import numpy as np

from . import api


def shard_range(n: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced slice [lo, hi) of n reads for `rank` of `world` (sizes differ by <= 1)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank %d of %d" % (rank, world))
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def slice_batch(batch: api.ReadBatch, lo: int, hi: int) -> api.ReadBatch:
    return api.ReadBatch(batch.codes[lo:hi], batch.lengths[lo:hi],
                         None if batch.levels is None else batch.levels[lo:hi],
                         None if batch.first_levels is None else batch.first_levels[lo:hi])


def gather_in_order(res: api.MapResults, group=None) -> api.MapResults | None:
    """Rank 0 receives the results of every rank concatenated in rank order (others: None)."""
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    parts = [None] * world if rank == 0 else None
    dist.gather_object((res.hits, res.tb, res.mapped), parts, dst=0, group=group)
    if rank != 0:
        return None
    hits = np.concatenate([p[0] for p in parts])
    tb = np.concatenate([p[1] for p in parts])
    mapped = np.concatenate([p[2] for p in parts])
    return api.MapResults(len(mapped), res.tb_stride, (hits, tb, mapped))


def map_sharded(map_fn, batch: api.ReadBatch, tb_stride: int, group=None) -> api.MapResults | None:
    """map_fn(sub_batch, tb_stride) -> MapResults on this rank's slice; rank 0 returns the whole."""
    import torch.distributed as dist
    lo, hi = shard_range(batch.n, dist.get_world_size(group), dist.get_rank(group))
    local = map_fn(slice_batch(batch, lo, hi), tb_stride)
    return gather_in_order(local, group)


# ------------------------------------------------------------------------------- command line

class ShSamOpts(C.Structure):
    _fields_ = [("colour", C.c_int), ("max_rank", C.c_int), ("print_all", C.c_int), ("uniqueness", C.c_int),
                ("uniqueness_threshold", C.c_int), ("min_score", C.c_int), ("delta_m", C.c_int),
                ("quality_base", C.c_int), ("argc", C.c_int), ("argv", C.POINTER(C.c_char_p))]


def _parse(argv):
    ap = argparse.ArgumentParser(prog="storm_b200.multi", add_help=True)
    ap.add_argument("--colour", action="store_true", help="storm-color (default: storm-nucleotide)")
    ap.add_argument("-g", required=True)
    ap.add_argument("-r", required=True)
    ap.add_argument("-o", required=True)
    ap.add_argument("-M", type=int, default=1)
    ap.add_argument("-s", default=None)
    ap.add_argument("-m", type=int, default=5)
    ap.add_argument("-x", type=int, default=-4)
    ap.add_argument("-d", type=int, default=-9)
    ap.add_argument("-e", type=int, default=-4)
    ap.add_argument("-i", type=int, default=3)
    ap.add_argument("-t", type=int, default=115)
    ap.add_argument("-z", type=int, default=100)
    ap.add_argument("-l", type=int, default=100)
    ap.add_argument("-b", type=int, default=33)
    ap.add_argument("-A", action="store_true")
    return ap.parse_args(argv)


DEFAULT_SEEDS = ("####--#-#--##--####;#####--###-#-###;###-##-#######",
                 "####----##--##-####;####-###--#----####;####-####-####")


def main(argv=None) -> int:
    import datetime

    import torch
    import torch.distributed as dist

    from . import build, host
    a = _parse(sys.argv[1:] if argv is None else argv)
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    rank = dist.get_rank()
    if rank == 0:
        build.build()
    dist.barrier()
    colour = 1 if a.colour else 0
    prm = api.params(colour=colour, match=a.m, mismatch=a.x, gap_open=a.d, gap_extend=a.e, indels=a.i,
                     min_score=a.t, min_score_filter=a.z, stdev=a.l, device=local)
    reads = host.ReadSet(a.r, colour, quality_base=a.b)
    reference = host.Reference(a.g, colour)
    mapper = api.Mapper(prm, a.s or DEFAULT_SEEDS[colour])
    reference.add_to(mapper)
    mapper.build_index()
    tbs = ((reads.max_len + a.i + 1) // 2 + 7) & ~7
    res = map_sharded(lambda b, t: mapper.map(b, t), reads.batch(), tbs)
    mapper.close()
    if rank == 0:
        write_sam(a.o, reference, reads, res, colour, a, ["storm_b200.multi"] + list(argv or sys.argv[1:]))
    dist.barrier()
    dist.destroy_process_group()
    return 0


def write_sam(path, reference, reads, res: api.MapResults, colour, a, args):
    """The reference's SAM for `res` (host library sh_write_sam, the writer of the CLI)."""
    from . import host
    L = host.hostlib()
    libc = C.CDLL(None)
    libc.fopen.restype = C.c_void_p
    libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
    libc.fclose.argtypes = [C.c_void_p]
    L.sh_write_sam.argtypes = [C.c_void_p, C.POINTER(ShSamOpts), C.c_void_p, C.c_void_p,
                               C.POINTER(api.Results), C.c_int64, C.c_int64, C.c_int]
    argv_c = (C.c_char_p * len(args))(*[s.encode() for s in args])
    so = ShSamOpts(colour, a.M, 1 if a.A else 0, 0, 0, a.t, a.m - a.x, a.b, len(args), argv_c)
    f = libc.fopen(path.encode(), b"w")
    if not f:
        raise OSError("cannot open %s" % path)
    rr = res.cstruct()
    rc = L.sh_write_sam(f, C.byref(so), C.addressof(reference._s), C.addressof(reads._s), C.byref(rr),
                        0, reads.n, 1)
    libc.fclose(f)
    if rc:
        raise api.StormError(L.sh_last_error().decode())


if __name__ == "__main__":
    sys.exit(main())
