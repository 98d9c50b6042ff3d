"""ctypes bindings of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by
bench.py's CPU-baseline leg.  The product never imports this module.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import List, Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"

MAX_SIZE = 32


class OrcResult(C.Structure):
    _fields_ = [("found", C.c_int), ("size", C.c_int), ("op", C.c_int),
                ("rank", C.c_uint64), ("postfix", C.c_char * (MAX_SIZE + 1)),
                ("candidates", C.c_uint64), ("per_size", C.c_uint64 * (MAX_SIZE + 1))]


class OrcVfbResult(C.Structure):
    _fields_ = [("found", C.c_int), ("size", C.c_int), ("op", C.c_int),
                ("postfix", C.c_char * 256), ("cache_full", C.c_int),
                ("candidates", C.c_uint64), ("rows_per_size", C.c_int64 * 101),
                ("rows_total", C.c_int64)]


_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = C.CDLL(str(LIB_PATH))
        u64p = C.POINTER(C.c_uint64)
        L.orc_count_table.argtypes = [C.c_int, C.c_int, u64p]
        L.orc_unrank.argtypes = [C.c_uint64, C.c_int, u64p, C.c_char_p]
        L.orc_eval1.argtypes = [C.c_char_p, C.c_int, C.c_int, u64p]
        L.orc_eval1.restype = C.c_uint64
        L.orc_check.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, u64p, u64p]
        L.orc_search.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, C.c_int, C.c_int,
                                 C.c_int, C.POINTER(OrcResult)]
        L.orc_search_rtid.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_void_p]
        L.orc_rtid_multiplier.argtypes = [C.c_uint64]
        L.orc_rtid_multiplier.restype = C.c_uint64
        L.orc_scan_range.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, C.c_int,
                                     C.c_uint64, C.c_uint64, C.c_int, u64p, u64p]
        L.orc_scan_range.restype = C.c_int64
        L.orc_vfb.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, C.c_int, C.c_int64,
                              C.c_int, C.POINTER(OrcVfbResult)]
        L.orc_vfb_fingerprint32.argtypes = [C.POINTER(C.c_uint32), C.c_int]
        L.orc_vfb_fingerprint32.restype = C.c_uint64
        L.orc_max_threads.restype = C.c_int
        L.orc_ext_count_table.argtypes = [C.c_int, C.c_int, u64p]
        L.orc_ext_unrank.argtypes = [C.c_uint64, C.c_int, u64p, C.c_char_p]
        L.orc_ext_eval1.argtypes = [C.c_char_p, C.c_int, C.c_int, u64p]
        L.orc_ext_eval1.restype = C.c_uint64
        L.orc_ext_check.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int, u64p, u64p]
        L.orc_ext_search.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, C.c_int, C.c_int,
                                     C.c_int, C.POINTER(OrcResult)]
        L.orc_ext_vfb.argtypes = [C.c_int, C.c_int, C.c_int, u64p, u64p, C.c_int, C.c_int64,
                                  C.POINTER(OrcVfbResult)]
        _lib = L
    return _lib


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def count_table(max_size: int, n_terms: int) -> np.ndarray:
    t = np.zeros((max_size + 1) * 9, dtype=np.uint64)
    rc = lib().orc_count_table(max_size, n_terms, _p(t))
    if rc != 0:
        raise OverflowError("count table exceeds 64 bits")
    return t.reshape(max_size + 1, 9)


def unrank(rank: int, size: int, table: np.ndarray) -> str:
    buf = C.create_string_buffer(MAX_SIZE + 1)
    t = _u64(table).reshape(-1)
    lib().orc_unrank(rank, size, _p(t), buf)
    return buf.raw[:size].decode()


def eval1(postfix: str, row, word_bits: int = 64) -> int:
    r = _u64(row)
    return int(lib().orc_eval1(postfix.encode(), len(postfix), word_bits, _p(r)))


def check(postfix: str, inputs: np.ndarray, outputs: np.ndarray, word_bits: int = 64) -> bool:
    ins = _u64(inputs)
    outs = _u64(outputs)
    S, k = ins.shape
    return bool(lib().orc_check(postfix.encode(), len(postfix), word_bits, k, S,
                                _p(ins), _p(outs)))


def search(inputs, outputs, max_size: int, word_bits: int = 64, include_edges: bool = False,
           n_threads: int = 0) -> dict:
    ins = _u64(inputs)
    outs = _u64(outputs)
    S, k = ins.shape
    res = OrcResult()
    rc = lib().orc_search(word_bits, k, S, _p(ins), _p(outs), max_size, int(include_edges),
                          n_threads, C.byref(res))
    if rc < 0:
        raise ValueError(f"oracle search failed ({rc})")
    return {"found": bool(res.found), "size": res.size, "op": res.op, "rank": res.rank,
            "postfix": res.postfix[: res.size].decode() if res.found else "",
            "candidates": res.candidates, "per_size": list(res.per_size)}


def search_rtid(inputs, outputs, max_size: int, word_bits: int = 64, include_edges: bool = False,
                reference_map: bool = False, n_threads: int = 0) -> dict:
    """RTid-order search: the match with the smallest thread position t of
    the first operator block with a match.  reference_map=True restates the
    reference's own map (64-bit wrap, C not coprime to every N)."""
    ins = _u64(inputs)
    outs = _u64(outputs)
    S, k = ins.shape
    res = OrcResult()
    rc = lib().orc_search_rtid(word_bits, k, S, _p(ins), _p(outs), max_size, int(include_edges),
                               int(reference_map), n_threads, C.byref(res))
    if rc < 0:
        raise ValueError(f"oracle rtid search failed ({rc})")
    return {"found": bool(res.found), "size": res.size, "op": res.op, "rank": res.rank,
            "postfix": res.postfix[: res.size].decode() if res.found else "",
            "candidates": res.candidates, "per_size": list(res.per_size)}


def rtid_multiplier(n: int) -> int:
    return int(lib().orc_rtid_multiplier(C.c_uint64(n)))


def scan_range(inputs, outputs, size: int, lo: int, hi: int, word_bits: int = 64,
               n_threads: int = 0):
    ins = _u64(inputs)
    outs = _u64(outputs)
    S, k = ins.shape
    mr = C.c_uint64(0)
    nh = C.c_uint64(0)
    e = lib().orc_scan_range(word_bits, k, S, _p(ins), _p(outs), size, lo, hi, n_threads,
                             C.byref(mr), C.byref(nh))
    return int(e), int(mr.value), int(nh.value)


def vfb(inputs, outputs, max_len: int, word_bits: int = 64, cap_rows: int = 0,
        ref_inverted: bool = False) -> dict:
    ins = _u64(inputs)
    outs = _u64(outputs)
    S, k = ins.shape
    res = OrcVfbResult()
    rc = lib().orc_vfb(word_bits, k, S, _p(ins), _p(outs), max_len, cap_rows,
                       int(ref_inverted), C.byref(res))
    if rc < 0:
        raise ValueError(f"oracle vfb failed ({rc})")
    return {"found": bool(res.found), "size": res.size, "op": res.op,
            "postfix": res.postfix.decode() if res.found else "",
            "cache_full": bool(res.cache_full), "candidates": res.candidates,
            "rows_per_size": list(res.rows_per_size), "rows_total": res.rows_total}


def fingerprint32(vec) -> int:
    a = np.ascontiguousarray(np.asarray(vec, dtype=np.uint32))
    return int(lib().orc_vfb_fingerprint32(a.ctypes.data_as(C.POINTER(C.c_uint32)), len(a)))


def max_threads() -> int:
    return int(lib().orc_max_threads())


# Extended grammar (~ & | ^ << >> neg + - * / %), see oracle.c.
EXT_CHARS = "~&|^<>#+-*/%"


def ext_count_table(max_size: int, n_terms: int) -> np.ndarray:
    t = np.zeros((max_size + 1) * 13, dtype=np.uint64)
    if lib().orc_ext_count_table(max_size, n_terms, _p(t)) != 0:
        raise OverflowError("count table exceeds 64 bits")
    return t.reshape(max_size + 1, 13)


def ext_unrank(rank: int, size: int, table: np.ndarray) -> str:
    buf = C.create_string_buffer(MAX_SIZE + 1)
    t = _u64(table).reshape(-1)
    lib().orc_ext_unrank(rank, size, _p(t), buf)
    return buf.raw[:size].decode()


def ext_eval1(postfix: str, row, word_bits: int = 64) -> int:
    r = _u64(row)
    return int(lib().orc_ext_eval1(postfix.encode(), len(postfix), word_bits, _p(r)))


def ext_check(postfix: str, inputs, outputs, word_bits: int = 64) -> bool:
    ins = _u64(inputs)
    outs = _u64(outputs)
    S, k = ins.shape
    return bool(lib().orc_ext_check(postfix.encode(), len(postfix), word_bits, k, S,
                                    _p(ins), _p(outs)))


def ext_search(inputs, outputs, max_size: int, word_bits: int = 64, include_edges: bool = False,
               n_threads: int = 0) -> dict:
    ins = _u64(inputs)
    outs = _u64(outputs)
    S, k = ins.shape
    res = OrcResult()
    rc = lib().orc_ext_search(word_bits, k, S, _p(ins), _p(outs), max_size, int(include_edges),
                              n_threads, C.byref(res))
    if rc < 0:
        raise ValueError(f"oracle ext search failed ({rc})")
    return {"found": bool(res.found), "size": res.size, "op": res.op, "rank": res.rank,
            "postfix": res.postfix[: res.size].decode() if res.found else "",
            "candidates": res.candidates, "per_size": list(res.per_size)}


def ext_vfb(inputs, outputs, max_len: int, word_bits: int = 64, cap_rows: int = 0) -> dict:
    ins = _u64(inputs)
    outs = _u64(outputs)
    S, k = ins.shape
    res = OrcVfbResult()
    rc = lib().orc_ext_vfb(word_bits, k, S, _p(ins), _p(outs), max_len, cap_rows, C.byref(res))
    if rc < 0:
        raise ValueError(f"oracle ext vfb failed ({rc})")
    return {"found": bool(res.found), "size": res.size, "op": res.op,
            "postfix": res.postfix.decode() if res.found else "",
            "cache_full": bool(res.cache_full), "candidates": res.candidates,
            "rows_per_size": list(res.rows_per_size), "rows_total": res.rows_total}
