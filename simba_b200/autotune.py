"""Autotuner for the search kernels' launch shape.

The knob the engine exposes at run time is the work-unit size (log2 of the
candidates one CTA takes from the queue at a time, ``unit_log2``): small
units balance better across 148 SMs and retire early on a match, large ones
amortise the per-unit context setup.  For each (terminals, samples, word
width) bucket the tuner times a full sweep of one size of a probe instance
(an unsatisfiable target, so every candidate is evaluated) for each
candidate value and keeps the fastest.  Results are cached per GPU model in
``$SIMBA_CACHE`` (default ``~/.cache/simba_b200/autotune.json``).
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Dict, Iterable, Optional, Tuple

from . import Session, count_table
from .instances import make_instance

CANDIDATES = (18, 20, 22, 24)
_mem: Dict[str, int] = {}


def _cache_path() -> Path:
    root = Path(os.environ.get("SIMBA_CACHE", Path.home() / ".cache" / "simba_b200"))
    return root / "autotune.json"


def _gpu_name(device: int) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda"


def probe_size(n_terms: int, target: float = 3e9) -> int:
    """Largest size whose candidate count stays below `target`."""
    t = count_table(20, n_terms)
    s = 3
    while s < 20 and int(t[s + 1][8]) < target:
        s += 1
    return s


def tune_bucket(n_terms: int, n_samples: int, word_bits: int, device: int = 0,
                candidates: Iterable[int] = CANDIDATES, use_cache: bool = True) -> int:
    """Best unit_log2 for one (terminals, samples, word width) bucket."""
    key = f"{_gpu_name(device)}|k={n_terms}|S={n_samples}|w={word_bits}"
    if use_cache and key in _mem:
        return _mem[key]
    path = _cache_path()
    cache = {}
    if use_cache and path.exists():
        try:
            cache = json.loads(path.read_text())
        except Exception:
            cache = {}
        if key in cache:
            _mem[key] = int(cache[key]["unit_log2"])
            return _mem[key]
    nv = max(1, n_terms - 1)
    inst = make_instance(7, nv, n_samples, 0xA070 + n_terms, word_bits=word_bits,
                         const_one=n_terms > 1, unsat=True)
    s = probe_size(inst.num_variables)
    times = {}
    for u in candidates:
        with Session(inst, device=device, unit_log2=u) as ss:
            ss.sweep(s, s)                      # warm-up (tables)
            r = ss.sweep(s, s)
            times[u] = r.kernel_ms
    best = min(times, key=times.get)
    _mem[key] = best
    if use_cache:
        cache[key] = {"unit_log2": best, "probe_size": s,
                      "kernel_ms": {str(k): v for k, v in times.items()}}
        try:
            path.parent.mkdir(parents=True, exist_ok=True)
            path.write_text(json.dumps(cache, indent=1))
        except OSError:
            pass
    return best


def tune_batch(insts, device: int = 0, use_cache: bool = True) -> Dict[Tuple[int, int, int], int]:
    """unit_log2 per bucket present in a batch."""
    out = {}
    for i in insts:
        k = (i.num_variables, i.num_examples, i.word_bits)
        if k not in out:
            out[k] = tune_bucket(*k, device=device, use_cache=use_cache)
    return out
