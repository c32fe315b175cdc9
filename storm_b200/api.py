"""Python bindings of the B200 mapping library (storm_b200/lib/libstormgpu.so, C ABI in
include/stormgpu.h), mirroring the reference's mapping interface: parameters as its command
line options, seeds in its -s syntax, packed 2-bit codes, per-read top-4 results.

There is no CPU fallback: if the CUDA library is missing or no GPU is usable, the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libstormgpu.so")
MIN_SCORE = -16383


class StormError(RuntimeError):
    pass


class Params(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("colour", "match", "mismatch", "gap_open", "gap_extend",
                                         "allowed_indels", "min_score", "min_score_filter",
                                         "stdev_distance", "senses", "device")]


class Hit(C.Structure):
    _fields_ = [("score", C.c_int32), ("ref_id", C.c_int32), ("ref_start", C.c_int32),
                ("ref_end", C.c_int32), ("read_start", C.c_int16), ("read_end", C.c_int16),
                ("sense", C.c_int32), ("tb_len", C.c_int32)]


HIT_DTYPE = np.dtype([("score", "<i4"), ("ref_id", "<i4"), ("ref_start", "<i4"), ("ref_end", "<i4"),
                      ("read_start", "<i2"), ("read_end", "<i2"), ("sense", "<i4"), ("tb_len", "<i4")])


class Reads(C.Structure):
    _fields_ = [("n", C.c_int64), ("codes", C.c_void_p), ("code_stride", C.c_int64),
                ("levels", C.c_void_p), ("level_stride", C.c_int64), ("lengths", C.c_void_p),
                ("first_levels", C.c_void_p)]


class Results(C.Structure):
    _fields_ = [("hits", C.c_void_p), ("tb", C.c_void_p), ("tb_stride", C.c_int64),
                ("mapped", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("candidates", "filter_passed", "aligned", "seed_lookups",
                                         "hit_positions", "filter_cells", "align_cells", "kernels",
                                         "filter_band_cells")] + \
               [(n, C.c_double) for n in ("ms_index", "ms_gather", "ms_filter", "ms_align",
                                          "ms_replay", "ms_total")] + [("passes", C.c_int64), ("graph_passes", C.c_int64),
                                                                 ("placement_waves", C.c_int64)]


class Tuning(C.Structure):
    """stormgpu_tuning: launch parameters of the stages (none changes a result)."""
    _fields_ = [(n, C.c_int32) for n in ("gather_warp_cap", "gather_reads_per_steal", "filter_rows", "align_steal",
                                         "filter_cursor", "align_rounds")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


DEFAULT_TUNING = dict(gather_warp_cap=768, gather_reads_per_steal=4, filter_rows=8, align_steal=32, filter_cursor=0,
                      align_rounds=4)

_lib = None


def lib():
    """Load libstormgpu.so (build it first with storm_b200.build.build())."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise StormError("libstormgpu.so is not built (%s); run storm_b200.build.build()" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        L.stormgpu_version.restype = C.c_char_p
        L.stormgpu_last_error.restype = C.c_char_p
        L.stormgpu_open.argtypes = [C.POINTER(Params), C.c_char_p, C.POINTER(C.c_void_p)]
        L.stormgpu_close.argtypes = [C.c_void_p]
        L.stormgpu_close.restype = None
        L.stormgpu_add_reference.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                             C.c_void_p, C.c_int32]
        L.stormgpu_build_index.argtypes = [C.c_void_p]
        L.stormgpu_map.argtypes = [C.c_void_p, C.POINTER(Reads), C.POINTER(Results)]
        L.stormgpu_map_device.argtypes = [C.c_void_p, C.POINTER(Reads), C.POINTER(Results), C.c_void_p]
        L.stormgpu_sync.argtypes = [C.c_void_p]
        L.stormgpu_get_stats.argtypes = [C.c_void_p, C.POINTER(Stats)]
        L.stormgpu_get_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
        L.stormgpu_set_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
        L.stormgpu_set_graphs.argtypes = [C.c_void_p, C.c_int]
        L.stormgpu_genome_map_greedy.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.POINTER(C.c_int64)]
        L.stormgpu_genome_map_contextual.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                                     C.POINTER(C.c_int64)]
        L.stormgpu_autotune.argtypes = [C.c_void_p, C.POINTER(Reads), C.c_int64, C.POINTER(Tuning)]
        L.stormgpu_server_set_tuning.argtypes = [C.c_void_p, C.POINTER(Tuning)]
        L.stormgpu_sw_filter.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                         C.c_uint32, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p,
                                         C.c_int64, C.c_void_p, C.c_void_p]
        L.stormgpu_align.argtypes = [C.POINTER(Params), C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                     C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int64,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_int64]
        L.stormgpu_server_open.argtypes = [C.POINTER(Params), C.POINTER(C.c_char_p), C.c_int, C.c_int, C.c_int64,
                                           C.POINTER(C.c_void_p)]
        L.stormgpu_server_add_reference.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p,
                                                    C.c_void_p, C.c_int32]
        L.stormgpu_server_build.argtypes = [C.c_void_p]
        L.stormgpu_submit.argtypes = [C.c_void_p, C.POINTER(Reads), C.POINTER(Results), C.c_void_p,
                                      C.POINTER(C.c_int64)]
        L.stormgpu_poll.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.POINTER(C.c_double)]
        L.stormgpu_server_close.argtypes = [C.c_void_p]
        L.stormgpu_server_close.restype = None
        L.stormgpu_align_noalloc.argtypes = [C.POINTER(Params), C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                             C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                             C.c_void_p]
        L.stormgpu_index_one.argtypes = [C.c_char_p, C.c_int32, C.c_void_p, C.c_int64, C.c_int64,
                                         C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                         C.c_int64, C.POINTER(C.c_int64)]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise StormError("stormgpu error %d: %s" % (rc, lib().stormgpu_last_error().decode()))


def device_available() -> bool:
    return bool(lib().stormgpu_device_available())


def params(colour=0, match=5, mismatch=-4, gap_open=-9, gap_extend=-4, indels=3, min_score=115,
           min_score_filter=100, stdev=100, senses=3, device=0) -> Params:
    """Defaults are the reference's (alignment.h:24-28, :51-52, index.h:16)."""
    return Params(colour, match, mismatch, gap_open, gap_extend, indels, min_score,
                  min_score_filter, stdev, senses, device)


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class ReadBatch:
    """Packed reads (tag order is the caller's business): codes/levels (n, stride) uint8."""

    def __init__(self, codes, lengths, levels=None, first_levels=None):
        self.codes = np.ascontiguousarray(codes, dtype=np.uint8)
        self.lengths = np.ascontiguousarray(lengths, dtype=np.int16)
        self.levels = None if levels is None else np.ascontiguousarray(levels, dtype=np.uint8)
        self.first_levels = None if first_levels is None else np.ascontiguousarray(first_levels, dtype=np.uint8)
        self.n = len(self.lengths)

    def cstruct(self) -> Reads:
        return Reads(self.n, _p(self.codes), self.codes.shape[1], _p(self.levels),
                     0 if self.levels is None else self.levels.shape[1], _p(self.lengths),
                     _p(self.first_levels))


class MapResults:
    """Per-read results; `buffers` = (hits, tb, mapped) arrays to write into (e.g. views of
    pinned host memory reused across batches), else fresh ones."""

    def __init__(self, n, tb_stride, buffers=None):
        if buffers is None:
            self.hits = np.zeros(n * 4, dtype=HIT_DTYPE)
            self.tb = np.zeros((n * 4, tb_stride), dtype=np.uint8)
            self.mapped = np.zeros(n, dtype=np.uint8)
        else:
            self.hits, self.tb, self.mapped = buffers
            if (self.hits.dtype != HIT_DTYPE or self.hits.shape != (n * 4,) or self.tb.shape != (n * 4, tb_stride)
                    or self.mapped.shape != (n,) or not all(a.flags.c_contiguous for a in buffers)):
                raise ValueError("result buffers of the wrong shape or type")
        self.tb_stride = tb_stride

    def cstruct(self) -> Results:
        return Results(_p(self.hits), _p(self.tb), self.tb_stride, _p(self.mapped))


class Mapper:
    """One mapping context: stormgpu_open / add_reference / build_index / map / close."""

    def __init__(self, prm: Params, seeds: str):
        self._ctx = C.c_void_p()
        self.params = prm
        _check(lib().stormgpu_open(C.byref(prm), seeds.encode(), C.byref(self._ctx)))

    def add_reference(self, codes, mask, n_codes, regions=()):
        codes = np.ascontiguousarray(codes, dtype=np.uint8)
        mask = np.ascontiguousarray(mask, dtype=np.uint8)
        rs = np.array([a for a, _ in regions] or [0], dtype=np.int32)
        re = np.array([b for _, b in regions] or [0], dtype=np.int32)
        _check(lib().stormgpu_add_reference(self._ctx, _p(codes), _p(mask), n_codes, _p(rs), _p(re),
                                            len(regions)))

    def build_index(self):
        _check(lib().stormgpu_build_index(self._ctx))

    def map(self, batch: ReadBatch, tb_stride=None, out: MapResults | None = None) -> MapResults:
        if out is not None:
            tb_stride = out.tb_stride
        elif tb_stride is None:
            tb_stride = ((int(batch.lengths.max()) + self.params.allowed_indels + 1) // 2 + 7) & ~7
        res = out if out is not None else MapResults(batch.n, tb_stride)
        rs, rr = batch.cstruct(), res.cstruct()
        _check(lib().stormgpu_map(self._ctx, C.byref(rs), C.byref(rr)))
        return res

    def map_device(self, reads: Reads, results: Results, stream=None):
        _check(lib().stormgpu_map_device(self._ctx, C.byref(reads), C.byref(results),
                                         C.c_void_p(stream) if stream else None))

    def sync(self):
        _check(lib().stormgpu_sync(self._ctx))

    def tuning(self) -> dict:
        t = Tuning()
        _check(lib().stormgpu_get_tuning(self._ctx, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = Tuning()
        _check(lib().stormgpu_get_tuning(self._ctx, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        _check(lib().stormgpu_set_tuning(self._ctx, C.byref(t)))

    def genome_map(self, n: int, greedy: bool = False, uniqueness_threshold: int | None = None):
        """Placement of the last `map` call's n reads without -M (genome_map.c): the placed reads
        in position order and the rank each is placed at (greedy: always rank 0)."""
        read = np.zeros(max(n, 1), np.int32)
        rank = np.zeros(max(n, 1), np.int32)
        npl = C.c_int64(0)
        thr = 0 if uniqueness_threshold is None else int(uniqueness_threshold)
        if greedy:
            _check(lib().stormgpu_genome_map_greedy(self._ctx, thr, read.ctypes.data, C.byref(npl)))
        else:
            _check(lib().stormgpu_genome_map_contextual(self._ctx, 0 if uniqueness_threshold is None else 1, thr,
                                                        read.ctypes.data, rank.ctypes.data, C.byref(npl)))
        return read[:npl.value], rank[:npl.value]

    def set_graphs(self, enable: bool):
        """CUDA graphs for the strand passes (on by default; the results are the same)."""
        _check(lib().stormgpu_set_graphs(self._ctx, 1 if enable else 0))

    def autotune(self, batch: ReadBatch, sample: int = 200000) -> dict:
        """Pick the launch parameters by timing them on (up to `sample` of) the batch."""
        t = Tuning()
        rs = batch.cstruct()
        _check(lib().stormgpu_autotune(self._ctx, C.byref(rs), int(sample), C.byref(t)))
        return t.as_dict()

    def stats(self) -> dict:
        s = Stats()
        _check(lib().stormgpu_get_stats(self._ctx, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def close(self):
        if self._ctx:
            lib().stormgpu_close(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sw_filter(W, L, match, mismatch, gapopen, gapext, threshold, genome_packed, n_codes, pos, read_packed):
    pos = np.ascontiguousarray(pos, dtype=np.int32)
    out = np.zeros(len(pos), dtype=np.uint8)
    g = np.ascontiguousarray(genome_packed, dtype=np.uint8)
    r = np.ascontiguousarray(read_packed, dtype=np.uint8)
    _check(lib().stormgpu_sw_filter(W, L, match, mismatch, gapopen, gapext, threshold, _p(g), n_codes, 0,
                                    _p(pos), len(pos), _p(r), _p(out)))
    return out


def align(prm: Params, read_packed, levels_packed, L, genome_packed, mask_packed, n_codes, wins):
    wins = np.ascontiguousarray(wins, dtype=np.int32)
    n = len(wins)
    tbs = ((L + prm.allowed_indels + 1) // 2 + 7) & ~7
    score = np.zeros(n, np.int32)
    bound = np.zeros(n, np.int32)
    best = np.zeros((n, 4), np.int16)
    tbl = np.zeros(n, np.int32)
    tb = np.zeros((n, tbs), np.uint8)
    r = np.ascontiguousarray(read_packed, dtype=np.uint8)
    q = None if levels_packed is None else np.ascontiguousarray(levels_packed, dtype=np.uint8)
    g = np.ascontiguousarray(genome_packed, dtype=np.uint8)
    m = np.ascontiguousarray(mask_packed, dtype=np.uint8)
    _check(lib().stormgpu_align(C.byref(prm), _p(r), _p(q), L, _p(g), _p(m), n_codes, 0, _p(wins), n,
                                _p(score), _p(bound), _p(best), _p(tbl), _p(tb), tbs))
    return score, bound, best, tbl, tb


class Server:
    """stormgpu_server_*: a resident -O chain (one seed family per step) serving batches
    submitted from any thread; `slots` batches run at once within `budget_bytes` of device memory."""

    def __init__(self, prm: Params, chain, slots: int = 2, budget_bytes: int = 16 << 30):
        self.params = prm
        self._h = C.c_void_p()
        arr = (C.c_char_p * len(chain))(*[c.encode() for c in chain])
        _check(lib().stormgpu_server_open(C.byref(prm), arr, len(chain), slots, budget_bytes, C.byref(self._h)))
        self._live = {}

    def add_reference(self, codes, mask, n_codes, regions=()):
        rs = np.array([a for a, _ in regions] or [0], np.int32)
        re = np.array([b for _, b in regions] or [0], np.int32)
        _check(lib().stormgpu_server_add_reference(self._h, C.c_void_p(codes) if isinstance(codes, int) else _p(codes),
                                                   C.c_void_p(mask) if isinstance(mask, int) else _p(mask), n_codes,
                                                   _p(rs), _p(re), len(regions)))

    def set_tuning(self, **kw):
        """Launch parameters of every slot (before build); unnamed ones keep their defaults."""
        t = Tuning(**DEFAULT_TUNING)
        for k, v in kw.items():
            setattr(t, k, int(v))
        _check(lib().stormgpu_server_set_tuning(self._h, C.byref(t)))

    def build(self):
        _check(lib().stormgpu_server_build(self._h))

    def submit(self, batch: ReadBatch, tb_stride=None) -> int:
        if tb_stride is None:
            tb_stride = ((int(batch.lengths.max()) + self.params.allowed_indels + 1) // 2 + 7) & ~7
        res = MapResults(batch.n, tb_stride)
        step = np.zeros(max(batch.n, 1), np.uint8)
        rs, rr = batch.cstruct(), res.cstruct()
        t = C.c_int64(0)
        _check(lib().stormgpu_submit(self._h, C.byref(rs), C.byref(rr), _p(step), C.byref(t)))
        self._live[t.value] = (batch, res, step, rs, rr)  # kept alive until done
        return t.value

    def poll(self, ticket: int, timeout_ms: int = -1):
        """(results, step per read, latency ms) when done; None if not done within timeout_ms."""
        lat = C.c_double(0)
        rc = lib().stormgpu_poll(self._h, ticket, timeout_ms, C.byref(lat))
        if rc == 1:
            return None
        batch, res, step, _, _ = self._live.pop(ticket)
        _check(rc)
        return res, step[:batch.n], lat.value

    def close(self):
        if self._h:
            lib().stormgpu_server_close(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def align_noalloc(prm: Params, read, levels, L, genome, mask, n_codes, win, n, score, bound, best, tb_len, tb,
                  tb_stride, stream=0):
    """stormgpu_align_noalloc: every buffer argument is a device address (int) of the current
    device, owned by the caller (levels may be 0); nothing is allocated.  For callers that
    cannot allocate device memory themselves at this point (a memory pool owned by another
    allocator, or no tolerance for the synchronisation of an allocation)."""
    _check(lib().stormgpu_align_noalloc(C.byref(prm), read, levels or None, L, genome, mask, n_codes, win, n,
                                        score, bound, best, tb_len, tb, tb_stride, stream or None))


def index_one(seed: str, stdev: int, codes_packed, n_codes, regions=()):
    w = seed.split(":")[0].count("#") + seed.split(":")[0].count("1")
    first = np.zeros((1 << (2 * w)) + 1, np.int32)
    mp = np.zeros(n_codes + len(regions) + 1, np.int32)
    rs = np.array([a for a, _ in regions] or [0], dtype=np.int32)
    re = np.array([b for _, b in regions] or [0], dtype=np.int32)
    nl = C.c_int64(0)
    g = np.ascontiguousarray(codes_packed, dtype=np.uint8)
    _check(lib().stormgpu_index_one(seed.encode(), stdev, _p(g), n_codes, 0, _p(rs), _p(re), len(regions),
                                    _p(first), _p(mp), len(mp), C.byref(nl)))
    return first, mp[:nl.value]
