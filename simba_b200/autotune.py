"""Autotuner for the search kernels' launch shape.

Knobs the engine exposes at run time, per (terminals, samples, word width)
bucket:

* ``unit_log2`` -- log2 of the candidates one CTA takes from the work queue
  at a time: small units balance better across 148 SMs and retire early on a
  match, large ones amortise the per-unit context setup;
* ``lanes_log2`` -- the split of a CTA's 256 threads between contexts and
  bottom values: every group of contexts keeps at least 2^lanes_log2 threads
  on the values (threads per context, from the bottom values' side);
* ``filter_samples`` -- how many samples besides sample 0 get value tables
  and filter sample-0 matches before verification (samples per candidate
  tested by table lookups instead of by evaluation).

For each bucket the tuner times a full size of a probe instance (an
unsatisfiable target, so every candidate is evaluated) and settles the knobs
one at a time (unit size first, then lanes, then filter samples), keeping the
fastest.  Results are cached per GPU model in ``$SIMBA_CACHE`` (default
``~/.cache/simba_b200/autotune.json``).
"""
from __future__ import annotations

import json
import os
from pathlib import Path
from typing import Dict, Iterable, Optional, Tuple

from . import Session, count_table
from .instances import make_instance

CANDIDATES = (18, 20, 22, 24)
LANES = (0, 2, 4)
FILTERS = (1, 3)
_mem: Dict[str, dict] = {}


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
                candidates: Iterable[int] = CANDIDATES, use_cache: bool = True,
                full: bool = False) -> int:
    """Best unit_log2 for one (terminals, samples, word width) bucket (see
    tune_bucket_knobs for all three knobs)."""
    return tune_bucket_knobs(n_terms, n_samples, word_bits, device, candidates, use_cache,
                             full)["unit_log2"]


def tune_bucket_knobs(n_terms: int, n_samples: int, word_bits: int, device: int = 0,
                      candidates: Iterable[int] = CANDIDATES, use_cache: bool = True,
                      full: bool = True) -> dict:
    """Best knobs for one bucket: {"unit_log2", "lanes_log2", "filter_samples"}.
    With full=False only the unit size is tuned (the others keep 0 = default)."""
    key = f"{_gpu_name(device)}|k={n_terms}|S={n_samples}|w={word_bits}|full={int(full)}"
    if use_cache and key in _mem:
        return _mem[key]
    path = _cache_path()
    cache = {}
    if use_cache and path.exists():
        try:
            cache = json.loads(path.read_text())
        except Exception:
            cache = {}
        if key in cache and "knobs" in cache[key]:
            _mem[key] = cache[key]["knobs"]
            return _mem[key]
    nv = max(1, n_terms - 1)
    inst = make_instance(7, nv, n_samples, 0xA070 + n_terms, word_bits=word_bits,
                         const_one=n_terms > 1, unsat=True)
    s = probe_size(inst.num_variables, 3e9 if not full else 1e9)
    times = {}

    def run(k: dict) -> float:
        tk = (k["unit_log2"], k["lanes_log2"], k["filter_samples"])
        if tk not in times:
            with Session(inst, device=device, **k) as ss:
                ss.sweep(s, s)                      # warm-up (tables)
                times[tk] = ss.sweep(s, s).kernel_ms
        return times[tk]

    best = {"unit_log2": 22, "lanes_log2": 0, "filter_samples": 0}
    best["unit_log2"] = min(candidates, key=lambda u: run(dict(best, unit_log2=u)))
    if full:
        best["lanes_log2"] = min(LANES, key=lambda l: run(dict(best, lanes_log2=l)))
        best["filter_samples"] = min(FILTERS, key=lambda f: run(dict(best, filter_samples=f)))
    _mem[key] = best
    if use_cache:
        cache[key] = {"knobs": best, "probe_size": s,
                      "kernel_ms": {",".join(map(str, k)): v for k, v in times.items()}}
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


def tune_batch_knobs(insts, device: int = 0, use_cache: bool = True):
    """Per-bucket knobs for a batch: sets each instance's unit_log2 and returns
    (per-bucket knobs, batch-wide options) -- lanes_log2 and filter_samples
    apply to a whole batch, so they come from its most populous bucket."""
    per = {}
    count: Dict[Tuple[int, int, int], int] = {}
    for i in insts:
        k = (i.num_variables, i.num_examples, i.word_bits)
        if k not in per:
            per[k] = tune_bucket_knobs(*k, device=device, use_cache=use_cache)
        count[k] = count.get(k, 0) + 1
        i.unit_log2 = per[k]["unit_log2"]
    top = max(count, key=count.get) if count else None
    opts = {} if top is None else {"lanes_log2": per[top]["lanes_log2"],
                                   "filter_samples": per[top]["filter_samples"]}
    return per, opts
