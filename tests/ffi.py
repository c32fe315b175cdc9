"""ctypes bindings used by the tests: the oracle (oracle/liboracle.so), the reference's own
functions (oracle/_ref/libref_*.so, built from the reference sources by oracle/Makefile) and
small packing helpers.  Test infrastructure only."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
REF_DIR = os.path.join(ORACLE_DIR, "_ref")

MIN_SCORE = -16383


def pack2(codes, pad_bytes: int = 0, fill: int = 0) -> np.ndarray:
    """Pack 0..3 codes four per byte (first code in the low bits), with pad_bytes of `fill`
    bytes before and after."""
    codes = np.asarray(codes, dtype=np.uint8)
    n = len(codes)
    nb = (n + 3) // 4
    c = np.zeros(nb * 4, dtype=np.uint8)
    c[:n] = codes
    c = c.reshape(-1, 4)
    body = (c[:, 0] | (c[:, 1] << 2) | (c[:, 2] << 4) | (c[:, 3] << 6)).astype(np.uint8)
    if pad_bytes:
        pad = np.full(pad_bytes, fill, dtype=np.uint8)
        return np.concatenate([pad, body, pad])
    return body


def unpack2(packed, n: int) -> np.ndarray:
    p = np.asarray(packed, dtype=np.uint8)
    out = np.stack([p & 3, (p >> 2) & 3, (p >> 4) & 3, (p >> 6) & 3], axis=1).reshape(-1)
    return out[:n]


def ptr(a: np.ndarray, off: int = 0, t=C.c_uint8):
    return C.cast(a.ctypes.data + off * a.itemsize, C.POINTER(t))


def ensure_built():
    """Build the oracle (and, when the reference sources are present, oracle/_ref)."""
    if not os.path.exists(os.path.join(ORACLE_DIR, "liboracle.so")):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


_oracle = None


def oracle():
    global _oracle
    if _oracle is None:
        ensure_built()
        lib = C.CDLL(os.path.join(ORACLE_DIR, "liboracle.so"))
        lib.or_sw_filter.restype = C.c_int
        lib.or_sw_filter.argtypes = [C.c_int, C.c_int, C.c_uint32, C.c_uint32, C.c_uint32,
                                     C.c_uint32, C.c_uint32, C.c_void_p, C.c_int64, C.c_void_p]
        lib.or_index_build.restype = C.c_int64
        lib.or_index_build.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p,
                                       C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int64]
        lib.or_align.restype = None
        lib.or_align.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                 C.c_void_p, C.c_int64, C.c_void_p]
        lib.or_map.argtypes = [C.c_void_p, C.c_char_p, C.c_void_p, C.c_int, C.c_void_p,
                               C.c_void_p, C.c_void_p]
        lib.or_parse_seeds.argtypes = [C.c_char_p, C.c_void_p, C.c_int]
        lib.or_candidates.restype = C.c_int64
        lib.or_parse_seeds.restype = C.c_int
        lib.or_map.restype = C.c_int
        _oracle = lib
    return _oracle


_refs = {}


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f)) for f in
               ("libref_nuc.so", "libref_col.so", "storm-nucleotide", "storm-color"))


def reflib(colour: bool):
    key = "col" if colour else "nuc"
    if key not in _refs:
        lib = C.CDLL(os.path.join(REF_DIR, "libref_%s.so" % key))
        lib.kat_filter.restype = C.c_uint
        lib.kat_filter.argtypes = [C.c_int, C.c_uint, C.c_uint, C.c_uint, C.c_uint, C.c_uint,
                                   C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.kat_align.restype = None
        lib.kat_align.argtypes = [C.c_int] * 6 + [C.c_void_p] * 4 + [C.c_int, C.c_int,
                                                                      C.c_void_p, C.c_void_p]
        lib.kat_index.restype = C.c_long
        lib.kat_index.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                  C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_long]
        _refs[key] = lib
    return _refs[key]


class ParamsT(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("colour", "match", "mismatch", "gap_open", "gap_extend",
                                         "allowed_indels", "min_score", "min_score_filter",
                                         "stdev_distance", "senses", "device")]


class HitT(C.Structure):
    _fields_ = [("score", C.c_int32), ("ref_id", C.c_int32), ("ref_start", C.c_int32),
                ("ref_end", C.c_int32), ("read_start", C.c_int16), ("read_end", C.c_int16),
                ("sense", C.c_int32), ("tb_len", C.c_int32)]


class ReadsT(C.Structure):
    _fields_ = [("n", C.c_int64), ("codes", C.c_void_p), ("code_stride", C.c_int64),
                ("levels", C.c_void_p), ("level_stride", C.c_int64), ("lengths", C.c_void_p),
                ("first_levels", C.c_void_p)]


class ResultsT(C.Structure):
    _fields_ = [("hits", C.c_void_p), ("tb", C.c_void_p), ("tb_stride", C.c_int64),
                ("mapped", C.c_void_p)]


class OrAlignOut(C.Structure):
    _fields_ = [("score", C.c_int32), ("bound", C.c_int32), ("best_i", C.c_int16),
                ("best_j", C.c_int16), ("best_i0", C.c_int16), ("best_j0", C.c_int16),
                ("tb_len", C.c_int32), ("tb", C.c_uint8 * ((1024 + 64 + 2) // 2))]


class OrRef(C.Structure):
    _fields_ = [("codes", C.c_void_p), ("mask", C.c_void_p), ("n_codes", C.c_int64),
                ("rs", C.c_void_p), ("re", C.c_void_p), ("nreg", C.c_int)]


def make_params(colour=0, match=5, mismatch=-4, gap_open=-9, gap_extend=-4, indels=3,
                min_score=115, min_score_filter=100, stdev=100, senses=3, device=0):
    return ParamsT(colour, match, mismatch, gap_open, gap_extend, indels, min_score,
                   min_score_filter, stdev, senses, device)
