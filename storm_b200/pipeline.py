"""The command line's work per read file with the reference and its index kept resident:
read file in, SAM (and the -O FASTQ of unmapped reads) out, as storm-nucleotide /
storm-color -M k write them, for a stream of read files mapped against one reference.

The reference's command line loads the reference and builds its indexes on every run
(run.c:831-884); a caller with many read files pays that once here.  Each map_file call does
what the command line does after that: load and tag-sort the reads (reads_data.c:351-566,
:59-67; reads of several lengths are kept, grouped by length), map them on the GPU with host
buffers in and out (stormgpu_map), and write the SAM (hit_map.c:197-504) and the -O FASTQ
(hit_map.c:514-579).  The records are the command line's for the same file and options.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import api, host

# options of main.c:188 this front end takes, with the stormgpu_params field each sets
_INT_OPTS = {"-m": "match", "-x": "mismatch", "-d": "gap_open", "-e": "gap_extend", "-i": "indels",
             "-t": "min_score", "-z": "min_score_filter", "-l": "stdev"}


class ShSamOpts(C.Structure):
    _fields_ = [("colour", C.c_int), ("max_rank", C.c_int), ("print_all", C.c_int), ("uniqueness", C.c_int),
                ("uniqueness_threshold", C.c_int), ("min_score", C.c_int), ("delta_m", C.c_int),
                ("quality_base", C.c_int), ("argc", C.c_int), ("argv", C.POINTER(C.c_char_p))]


def parse_options(args):
    """(params keyword arguments, seeds or None, -M, -b, -A, -u threshold or None) of a
    storm command line's mapping options (main.c:229-433 semantics for these options)."""
    p = dict(match=5, mismatch=-4, gap_open=-9, gap_extend=-4, indels=3, min_score=115, min_score_filter=100,
             stdev=100, senses=3)
    seeds, max_rank, qbase, print_all, uniq = None, 0, 33, 0, None
    i = 0
    while i < len(args):
        a = args[i]
        v = args[i + 1] if i + 1 < len(args) else None
        if a in _INT_OPTS:
            p[_INT_OPTS[a]] = int(v)
            i += 2
        elif a == "-s":
            seeds, i = v, i + 2
        elif a == "-M":
            max_rank, i = int(v), i + 2
        elif a == "-b":
            qbase, i = int(v), i + 2
        elif a == "-u":
            uniq, i = int(v), i + 2
        elif a == "-A":
            print_all, i = 1, i + 1
        else:
            raise ValueError("option %s is not taken by the resident front end" % a)
    if not 1 <= max_rank <= 4:
        raise ValueError("-M must be 1..4 (the top-k output)")
    return p, seeds, max_rank, qbase, print_all, uniq


def _bind():
    L = host.hostlib()
    if not hasattr(L, "_pipeline_bound"):
        L.sh_write_sam_path.argtypes = [C.c_char_p, C.POINTER(ShSamOpts), C.POINTER(host.ShRefs),
                                        C.POINTER(host.ShReads), C.POINTER(api.Results)]
        L.sh_write_unmapped_fastq_path.argtypes = [C.c_char_p, C.POINTER(ShSamOpts), C.POINTER(host.ShReads),
                                                   C.POINTER(api.Results)]
        L._pipeline_bound = True
    return L


class ResidentMapper:
    """A reference with its index resident on the GPU, mapping read files into SAM files.

    `args` are the command line's mapping options (-M 1..4 is required: the top-k output);
    `default_seeds` is used when they give no -s."""

    def __init__(self, reference_path: str, args, colour: int = 0, default_seeds: str | None = None,
                 device: int = 0, program: str | None = None):
        self.colour = colour
        p, seeds, self.max_rank, self.qbase, self.print_all, self.uniq = parse_options(list(args))
        self.seeds = seeds or default_seeds
        if not self.seeds:
            raise ValueError("no seed family (-s) given")
        self.params = api.params(colour=colour, device=device, **p)
        self.reference = host.Reference(reference_path, colour)
        self.mapper = api.Mapper(self.params, self.seeds)
        self.reference.add_to(self.mapper)
        self.mapper.build_index()
        prog = program or ("storm-color" if colour else "storm-nucleotide")
        self._argv = [prog.encode()] + [a.encode() for a in ["-g", reference_path] + list(args)]
        self._pinned = {}

    def _buffers(self, n: int, tb_stride: int):
        """Pinned host result buffers, kept and grown across calls (pinned memory makes the
        device-to-host copies asynchronous and at full PCIe speed)."""
        import torch
        have = self._pinned.get("shape")
        if have is None or have[0] < n or have[1] != tb_stride:
            cap = max(n, int(1.25 * have[0]) if have else n)
            self._pinned = {"shape": (cap, tb_stride),
                            "hits": torch.empty(cap * 4 * api.HIT_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True),
                            "tb": torch.empty(cap * 4 * tb_stride, dtype=torch.uint8, pin_memory=True),
                            "mapped": torch.empty(cap, dtype=torch.uint8, pin_memory=True)}
        b = self._pinned
        hits = b["hits"].numpy()[:n * 4 * api.HIT_DTYPE.itemsize].view(api.HIT_DTYPE)
        tb = b["tb"].numpy()[:n * 4 * tb_stride].reshape(n * 4, tb_stride)
        mapped = b["mapped"].numpy()[:n]
        return api.MapResults(n, tb_stride, (hits, tb, mapped))

    def map_file(self, reads_path: str, sam_path: str, unmapped_path: str | None = None,
                 quality_path: str | None = None) -> dict:
        """Map one read file; write its SAM (and -O FASTQ).  Returns counts."""
        L = _bind()
        reads = host.ReadSet(reads_path, self.colour, quality_base=self.qbase, allow_mixed=1,
                             quality_path=quality_path)
        tbs = ((reads.max_len + self.params.allowed_indels + 1) // 2 + 7) & ~7
        res = self._buffers(reads.n, tbs)
        self.mapper.map(reads.batch(), out=res)
        argv = self._argv + [b"-r", reads_path.encode(), b"-o", sam_path.encode()]
        if unmapped_path:
            argv += [b"-O", unmapped_path.encode()]
        cargv = (C.c_char_p * len(argv))(*argv)
        o = ShSamOpts(self.colour, self.max_rank, self.print_all, 1 if self.uniq is not None else 0,
                      self.uniq or 0, self.params.min_score, self.params.match - self.params.mismatch, self.qbase,
                      len(argv), cargv)
        rr = res.cstruct()
        rc = L.sh_write_sam_path(sam_path.encode(), C.byref(o), C.byref(self.reference._s), C.byref(reads._s),
                                 C.byref(rr))
        if rc:
            raise api.StormError(L.sh_last_error().decode())
        if unmapped_path:
            rc = L.sh_write_unmapped_fastq_path(unmapped_path.encode(), C.byref(o), C.byref(reads._s), C.byref(rr))
            if rc:
                raise api.StormError(L.sh_last_error().decode())
        return {"reads": int(reads.n), "mapped": int(np.count_nonzero(res.mapped[:reads.n]))}

    def close(self):
        self.mapper.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
