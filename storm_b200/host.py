"""ctypes bindings of the host front end (storm_b200/lib/libstormhost.so): the reference's
FASTA / FASTQ loading and read ordering, as the storm-nucleotide / storm-color binaries use
them, so that Python callers feed the mapping library exactly what the command line would."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import api

HOST_LIB = os.path.join(api.PKG, "lib", "libstormhost.so")


class ShRefs(C.Structure):
    _fields_ = [("n", C.c_int), ("names", C.POINTER(C.c_char_p)), ("sizes", C.POINTER(C.c_int64)),
                ("codes", C.POINTER(C.c_void_p)), ("masks", C.POINTER(C.c_void_p)),
                ("rs", C.POINTER(C.c_void_p)), ("re", C.POINTER(C.c_void_p)), ("nreg", C.POINTER(C.c_int32)),
                ("first_base", C.POINTER(C.c_uint8)), ("alloc_codes", C.c_void_p), ("alloc_masks", C.c_void_p)]


class ShReads(C.Structure):
    _fields_ = [("n", C.c_int64), ("colour", C.c_int), ("min_len", C.c_int), ("max_len", C.c_int),
                ("has_quality", C.c_int), ("db_name", C.c_char_p), ("names", C.c_void_p),
                ("codes", C.c_void_p), ("code_stride", C.c_int64), ("levels", C.c_void_p),
                ("level_stride", C.c_int64), ("lengths", C.c_void_p), ("tags", C.c_void_p),
                ("first_base", C.c_void_p), ("first_level", C.c_void_p), ("file_index", C.c_void_p),
                ("arena", C.c_void_p), ("no_quality", C.c_void_p)]


_h = None


def hostlib():
    global _h
    if _h is None:
        if not os.path.exists(HOST_LIB):
            raise api.StormError("libstormhost.so is not built; run storm_b200.build.build()")
        L = C.CDLL(HOST_LIB)
        L.sh_last_error.restype = C.c_char_p
        L.sh_load_reference.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(ShRefs)]
        L.sh_free_reference.argtypes = [C.POINTER(ShRefs)]
        L.sh_load_reads.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(ShReads)]
        L.sh_free_reads.argtypes = [C.POINTER(ShReads)]
        L.sh_sort_reads.argtypes = [C.POINTER(ShReads)]
        _h = L
    return _h


class Reference:
    """Loaded reference: per sequence packed codes and masks (padded), masked regions."""

    def __init__(self, path: str, colour: int, ignore_lowercase: int = 0):
        self._s = ShRefs()
        rc = hostlib().sh_load_reference(path.encode(), colour, ignore_lowercase, C.byref(self._s))
        if rc:
            raise api.StormError(hostlib().sh_last_error().decode())
        self.n = self._s.n

    def sequences(self):
        s = self._s
        for k in range(s.n):
            n = s.sizes[k]
            nr = s.nreg[k]
            rs = np.ctypeslib.as_array(C.cast(s.rs[k], C.POINTER(C.c_int32)), shape=(max(nr, 1),))[:nr]
            re = np.ctypeslib.as_array(C.cast(s.re[k], C.POINTER(C.c_int32)), shape=(max(nr, 1),))[:nr]
            yield s.codes[k], s.masks[k], n, list(zip(rs.tolist(), re.tolist()))

    def add_to(self, mapper: api.Mapper):
        for codes, mask, n, regs in self.sequences():
            rs = np.array([a for a, _ in regs] or [0], np.int32)
            re = np.array([b for _, b in regs] or [0], np.int32)
            api._check(api.lib().stormgpu_add_reference(mapper._ctx, C.c_void_p(codes), C.c_void_p(mask), n,
                                                        C.c_void_p(rs.ctypes.data), C.c_void_p(re.ctypes.data),
                                                        len(regs)))

    def add_to_server(self, server: api.Server):
        for codes, mask, n, regs in self.sequences():
            server.add_reference(codes, mask, n, regs)

    def __del__(self):
        try:
            hostlib().sh_free_reference(C.byref(self._s))
        except Exception:
            pass


class ReadSet:
    """Loaded and tag-sorted reads, viewable as a stormgpu_reads batch (no copy)."""

    def __init__(self, path: str, colour: int, quality_base: int = 33, allow_mixed: int = 1, sort: bool = True,
                 quality_path: str | None = None):
        self._s = ShReads()
        rc = hostlib().sh_load_reads(path.encode(), quality_path.encode() if quality_path else None, colour,
                                     quality_base, allow_mixed, C.byref(self._s))
        if rc:
            raise api.StormError(hostlib().sh_last_error().decode())
        if sort:
            rc = hostlib().sh_sort_reads(C.byref(self._s))
            if rc:
                raise api.StormError(hostlib().sh_last_error().decode())
        s = self._s
        self.n = s.n
        self.max_len = s.max_len
        self.codes = np.ctypeslib.as_array(C.cast(s.codes, C.POINTER(C.c_uint8)), shape=(s.n, s.code_stride))
        self.levels = None if not s.levels else np.ctypeslib.as_array(
            C.cast(s.levels, C.POINTER(C.c_uint8)), shape=(s.n, s.level_stride))
        self.lengths = np.ctypeslib.as_array(C.cast(s.lengths, C.POINTER(C.c_int16)), shape=(s.n,))
        self.first_levels = np.ctypeslib.as_array(C.cast(s.first_level, C.POINTER(C.c_uint8)), shape=(s.n,))
        self.colour = colour

    def batch(self) -> api.ReadBatch:
        return api.ReadBatch(self.codes, self.lengths, self.levels, self.first_levels if self.colour else None)

    def __del__(self):
        try:
            hostlib().sh_free_reads(C.byref(self._s))
        except Exception:
            pass
