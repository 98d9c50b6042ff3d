"""simba_b200: B200-native SIMBA / VFB search for Mixed-Boolean-Arithmetic.

Python mirror of the C ABI in include/simba_b200.h (loaded with ctypes from
the in-tree ``libsimba_b200.so``).  The reference has no library API; its
interface is the two executables ``simba <instance.json> <maxLen>`` and
``vfb <instance.json> <maxLen>``.  :func:`solve` / :func:`vfb_solve` take the
same instance and max size and return the same expression, plus counters.

The product path is CUDA only: importing works without a GPU, but every
search call raises if the native library or a CUDA device is missing.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path
from typing import List, Optional, Sequence

import numpy as np

from .instances import (Instance, infix_to_postfix, make_instance,  # noqa: F401
                        postfix_to_infix)

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libsimba_b200.so"

OK, NOT_FOUND, BUDGET, CACHE_FULL = 0, 1, 2, 3
OP_NAMES = ["~", "&", "|", "^", "neg", "+", "-", "*", "leaf"]


class SimbaError(RuntimeError):
    pass


class _Instance(C.Structure):
    _fields_ = [("num_variables", C.c_int32), ("num_examples", C.c_int32),
                ("word_bits", C.c_int32), ("unit_log2", C.c_int32),
                ("inputs", C.POINTER(C.c_uint64)), ("outputs", C.POINTER(C.c_uint64))]


class _Options(C.Structure):
    _fields_ = [("device", C.c_int32), ("size_range", C.c_int32), ("verbose", C.c_int32),
                ("engine", C.c_int32), ("budget_seconds", C.c_double),
                ("table_bytes", C.c_int64), ("stream", C.c_uint64),
                ("vfb_cache_rows", C.c_int64), ("vfb_reference_dedup", C.c_int32),
                ("unit_log2", C.c_int32), ("class_prior", C.POINTER(C.c_float)),
                ("rank_order", C.c_int32), ("grammar", C.c_int32),
                ("lanes_log2", C.c_int32), ("filter_samples", C.c_int32)]


class _BatchResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("size", C.c_int32), ("op", C.c_int32),
                ("reserved", C.c_int32), ("rank", C.c_uint64), ("postfix", C.c_char * 64),
                ("seconds", C.c_double), ("candidates", C.c_uint64)]


class _BatchStats(C.Structure):
    _fields_ = [("seconds", C.c_double), ("device_ms", C.c_double), ("kernel_ms", C.c_double),
                ("alg_ops", C.c_double), ("candidates", C.c_uint64), ("evaluated", C.c_uint64),
                ("rounds", C.c_int32), ("launches", C.c_int32), ("solved", C.c_int32),
                ("reserved", C.c_int32)]


class _SizeResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("launches", C.c_int32), ("best_rank", C.c_uint64),
                ("candidates", C.c_uint64), ("evaluated", C.c_uint64),
                ("device_ms", C.c_double), ("kernel_ms", C.c_double)]


class _VfbResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("size", C.c_int32), ("op", C.c_int32),
                ("max_size_searched", C.c_int32), ("postfix", C.c_char * 256),
                ("expr", C.c_char * 2048), ("seconds", C.c_double), ("device_ms", C.c_double),
                ("candidates", C.c_uint64), ("rows_total", C.c_int64),
                ("rows_per_size", C.c_int64 * 101), ("cache_bytes", C.c_uint64),
                ("table_bytes", C.c_uint64), ("bytes_moved", C.c_double),
                ("launches", C.c_int32), ("reserved", C.c_int32)]


class _Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("size", C.c_int32), ("op", C.c_int32),
                ("table_size", C.c_int32), ("rank", C.c_uint64), ("postfix", C.c_char * 64),
                ("expr", C.c_char * 512), ("seconds", C.c_double), ("device_ms", C.c_double),
                ("candidates", C.c_uint64), ("evaluated", C.c_uint64),
                ("per_size", C.c_uint64 * 33), ("max_size_searched", C.c_int32),
                ("launches", C.c_int32), ("kernel_ms", C.c_double), ("alg_ops", C.c_uint64),
                ("join_ms", C.c_double), ("nested_ms", C.c_double),
                ("join_candidates", C.c_uint64), ("nested_candidates", C.c_uint64),
                ("join_bytes_streamed", C.c_double), ("join_table_bytes", C.c_double),
                ("nested_live_candidates", C.c_uint64)]


_lib = None


def lib():
    """Load libsimba_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise SimbaError(f"native library missing: {LIB_PATH} (run python -m simba_b200.build)")
    L = C.CDLL(str(LIB_PATH))
    P = C.POINTER
    L.simba_solve.argtypes = [P(_Instance), C.c_int, P(_Options), P(_Result)]
    L.simba_session_create.argtypes = [P(_Instance), P(_Options), P(C.c_void_p)]
    L.simba_session_solve.argtypes = [C.c_void_p, C.c_int, P(_Result)]
    L.simba_session_sweep.argtypes = [C.c_void_p, C.c_int, C.c_int, P(_Result)]
    L.simba_session_destroy.argtypes = [C.c_void_p]
    L.simba_session_destroy.restype = None
    L.simba_count_table.argtypes = [C.c_int, C.c_int, P(C.c_uint64)]
    L.simba_unrank.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_char_p]
    L.simba_rank_of.argtypes = [C.c_char_p, C.c_int, P(C.c_uint64)]
    L.simba_format.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int]
    L.simba_instance_load.argtypes = [C.c_char_p, P(_Instance)]
    L.simba_instance_free.argtypes = [P(_Instance)]
    L.simba_instance_free.restype = None
    for f in ("simba_version", "simba_status_string", "simba_last_error"):
        getattr(L, f).restype = C.c_char_p
    L.simba_status_string.argtypes = [C.c_int]
    L.simba_device_count.restype = C.c_int
    L.simba_int_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    L.simba_alu_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    L.vfb_solve.argtypes = [P(_Instance), C.c_int, P(_Options), P(_VfbResult)]
    L.simba_solve_noalloc.argtypes = [P(_Instance), C.c_int, P(_Options), P(_Result)]
    L.simba_solve_batch.argtypes = [P(_Instance), C.c_int, C.c_int, P(_Options),
                                    P(_BatchResult), P(_BatchStats)]
    L.simba_session_search_size.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                            P(_SizeResult)]
    _lib = L
    return L


@dataclass
class Result:
    status: int
    size: int = 0
    op: int = -1
    rank: int = 0
    postfix: str = ""
    expr: str = "Not found !"
    seconds: float = 0.0
    device_ms: float = 0.0
    candidates: int = 0
    evaluated: int = 0
    per_size: List[int] = field(default_factory=list)
    table_size: int = 0
    max_size_searched: int = 0
    launches: int = 0
    kernel_ms: float = 0.0
    alg_ops: int = 0
    join_ms: float = 0.0
    nested_ms: float = 0.0
    join_candidates: int = 0
    nested_candidates: int = 0
    join_bytes_streamed: float = 0.0
    join_table_bytes: float = 0.0
    nested_live_candidates: int = 0

    @property
    def found(self) -> bool:
        return self.status == OK


def _res(r: _Result) -> Result:
    return Result(r.status, r.size, r.op, r.rank, r.postfix.decode(), r.expr.decode(),
                  r.seconds, r.device_ms, r.candidates, r.evaluated, list(r.per_size),
                  r.table_size, r.max_size_searched, r.launches, r.kernel_ms, r.alg_ops,
                  r.join_ms, r.nested_ms, r.join_candidates, r.nested_candidates,
                  r.join_bytes_streamed, r.join_table_bytes, r.nested_live_candidates)


class _Arrays:
    """Keeps the numpy buffers alive while the C struct points at them."""

    def __init__(self, inst: Instance):
        self.ins = np.ascontiguousarray(inst.inputs, dtype=np.uint64).reshape(-1)
        self.outs = np.ascontiguousarray(inst.outputs, dtype=np.uint64).reshape(-1)
        self.c = _Instance(inst.num_variables, inst.num_examples, inst.word_bits,
                           int(getattr(inst, "unit_log2", 0) or 0),
                           self.ins.ctypes.data_as(C.POINTER(C.c_uint64)),
                           self.outs.ctypes.data_as(C.POINTER(C.c_uint64)))


def _opts(device=0, complete=False, verbose=False, naive=False, budget=0.0,
          table_bytes=0, stream=0, cache_rows=0, reference_dedup=False,
          unit_log2=0, class_prior=None, rtid=False, extended=False, lanes_log2=0,
          filter_samples=0) -> _Options:
    o = _Options()
    o.device = device
    o.size_range = 1 if complete else 0
    o.verbose = 1 if verbose else 0
    o.engine = 1 if naive else 0
    o.budget_seconds = float(budget)
    o.table_bytes = int(table_bytes)
    o.stream = int(stream)
    o.vfb_cache_rows = int(cache_rows)
    o.vfb_reference_dedup = 1 if reference_dedup else 0
    o.unit_log2 = int(unit_log2)
    o.rank_order = 1 if rtid else 0
    o.grammar = 1 if extended else 0
    o.lanes_log2 = int(lanes_log2)
    o.filter_samples = int(filter_samples)
    if class_prior is not None:  # the caller keeps the array alive for the call
        o.class_prior = class_prior.ctypes.data_as(C.POINTER(C.c_float))
    return o


def _check(rc: int) -> None:
    if rc < 0:
        L = lib()
        raise SimbaError(f"{L.simba_status_string(rc).decode()}: {L.simba_last_error().decode()}")


def solve(inst: Instance, max_size: int, **kw) -> Result:
    """Plain SIMBA search (the reference's NoCache::solve, simba/src/nocache.cu:197-289).
    extended=True searches the extended grammar ~ & | ^ << >> neg + - * / %."""
    a = _Arrays(inst)
    r = _Result()
    rc = lib().simba_solve(C.byref(a.c), max_size, C.byref(_opts(**kw)), C.byref(r))
    _check(rc)
    return _res(r)


def solve_noalloc(inst: Instance, max_size: int, **kw) -> Result:
    """Same search as :func:`solve` with every scratch buffer in the library's
    static 64 MiB device array: for callers that cannot allocate device
    memory while they run.  Calls share that array; do not overlap them."""
    a = _Arrays(inst)
    r = _Result()
    rc = lib().simba_solve_noalloc(C.byref(a.c), max_size, C.byref(_opts(**kw)), C.byref(r))
    _check(rc)
    return _res(r)


def solve_batch(insts: Sequence[Instance], max_size: int, **kw):
    """Batched plain search: returns (per-instance Result list, stats dict).

    Each Result carries status, size, op, rank, postfix, expr, candidates and
    `seconds` = time to solution on the device clock from the batch's first
    kernel (guided: the first verified match; plain: the end of the
    instance's last work unit)."""
    n = len(insts)
    if kw.get("class_prior") is not None:
        cp = np.ascontiguousarray(kw["class_prior"], dtype=np.float32)
        if cp.shape != (n, 64):
            raise ValueError("batch class_prior must be n x 64")
        kw["class_prior"] = cp
    arrs = [_Arrays(i) for i in insts]
    carr = (_Instance * n)(*[a.c for a in arrs])
    res = (_BatchResult * max(n, 1))()
    st = _BatchStats()
    _check(lib().simba_solve_batch(carr, n, max_size, C.byref(_opts(**kw)), res, C.byref(st)))
    out = []
    for i in range(n):
        r = res[i]
        pf = r.postfix.decode()
        out.append(Result(r.status, r.size, r.op, r.rank, pf,
                          format_postfix(pf) if r.status == OK else "Not found !",
                          r.seconds, 0.0, r.candidates))
    stats = {k: getattr(st, k) for k, _ in _BatchStats._fields_ if k != "reserved"}
    return out, stats


@dataclass
class VfbResult:
    status: int
    size: int = 0
    op: int = -1
    postfix: str = ""
    expr: str = "Not found !"
    seconds: float = 0.0
    device_ms: float = 0.0
    candidates: int = 0
    rows_total: int = 0
    rows_per_size: List[int] = field(default_factory=list)
    cache_bytes: int = 0
    table_bytes: int = 0
    bytes_moved: float = 0.0
    launches: int = 0
    max_size_searched: int = 0

    @property
    def found(self) -> bool:
        return self.status == OK


def vfb_solve(inst: Instance, max_len: int, **kw) -> VfbResult:
    """VFB bottom-up search (the reference's MBA(), vfb/src/full-cache.cu:665-774)."""
    a = _Arrays(inst)
    r = _VfbResult()
    rc = lib().vfb_solve(C.byref(a.c), max_len, C.byref(_opts(**kw)), C.byref(r))
    _check(rc)
    return VfbResult(r.status, r.size, r.op, r.postfix.decode(), r.expr.decode(), r.seconds,
                     r.device_ms, r.candidates, r.rows_total, list(r.rows_per_size),
                     r.cache_bytes, r.table_bytes, r.bytes_moved, r.launches,
                     r.max_size_searched)


class Session:
    """Resident search session: samples and value tables stay in HBM."""

    def __init__(self, inst: Instance, **kw):
        self._a = _Arrays(inst)
        self._h = C.c_void_p()
        _check(lib().simba_session_create(C.byref(self._a.c), C.byref(_opts(**kw)),
                                          C.byref(self._h)))

    def solve(self, max_size: int) -> Result:
        r = _Result()
        _check(lib().simba_session_solve(self._h, max_size, C.byref(r)))
        return _res(r)

    def sweep(self, lo: int, hi: int) -> Result:
        r = _Result()
        _check(lib().simba_session_sweep(self._h, lo, hi, C.byref(r)))
        return _res(r)

    def search_size(self, size: int, shard: int = 0, nshards: int = 1) -> dict:
        """One size over work units u % nshards == shard; best_rank is the
        minimum matching rank in this shard (None if none)."""
        r = _SizeResult()
        _check(lib().simba_session_search_size(self._h, size, shard, nshards, C.byref(r)))
        return {"status": r.status, "best_rank": None if r.best_rank == 2 ** 64 - 1 else
                r.best_rank, "candidates": r.candidates, "evaluated": r.evaluated,
                "device_ms": r.device_ms, "kernel_ms": r.kernel_ms, "launches": r.launches}

    def close(self) -> None:
        if self._h:
            lib().simba_session_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def count_table(max_size: int, n_terms: int) -> np.ndarray:
    t = np.zeros((max_size + 1) * 9, dtype=np.uint64)
    _check(lib().simba_count_table(max_size, n_terms, t.ctypes.data_as(C.POINTER(C.c_uint64))))
    return t.reshape(max_size + 1, 9)


def unrank(rank: int, size: int, n_terms: int) -> str:
    buf = C.create_string_buffer(40)
    _check(lib().simba_unrank(rank, size, n_terms, buf))
    return buf.value.decode()


def rank_of(postfix: str, n_terms: int) -> int:
    r = C.c_uint64()
    _check(lib().simba_rank_of(postfix.encode(), n_terms, C.byref(r)))
    return r.value


def format_postfix(postfix: str, style: str = "simba", extended: bool = False) -> str:
    """Infix form in the SIMBA or VFB syntax; `extended` reads '<' '>' '/' '%'
    as the extended grammar's << >> / %."""
    buf = C.create_string_buffer(4096)
    code = (0 if style == "simba" else 1) + (2 if extended else 0)
    _check(lib().simba_format(postfix.encode(), code, buf, 4096))
    return buf.value.decode()


def load_instance(path: str) -> Instance:
    """Read an instance file through the native reader."""
    ci = _Instance()
    _check(lib().simba_instance_load(str(path).encode(), C.byref(ci)))
    try:
        S, k = ci.num_examples, ci.num_variables
        ins = np.ctypeslib.as_array(ci.inputs, shape=(S * k,)).copy().reshape(S, k)
        outs = np.ctypeslib.as_array(ci.outputs, shape=(S,)).copy()
    finally:
        lib().simba_instance_free(C.byref(ci))
    return Instance(k, ins, outs, ci.word_bits)


def int_peak(device: int = 0) -> float:
    """Measured int32 lane-operations per second of the device."""
    v = C.c_double()
    _check(lib().simba_int_peak(device, C.byref(v)))
    return v.value


def alu_peak(device: int = 0) -> float:
    """Measured ALU-pipe (LOP3) lane-operations per second of the device."""
    v = C.c_double()
    _check(lib().simba_alu_peak(device, C.byref(v)))
    return v.value


def release_device_cache() -> None:
    """Return the device memory the library keeps cached between calls."""
    _check(lib().simba_release_device_cache())


def device_count() -> int:
    return int(lib().simba_device_count())


def version() -> str:
    return lib().simba_version().decode()
