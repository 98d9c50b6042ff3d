"""Multi-GPU host logic: one process per GPU (torch.distributed plumbing).

Two ways to use several GPUs, neither with a collective on the data path:

* independent instances (``shard_instances``): each rank solves its own
  share of a batch; the only communication is the final gather of results
  and the max-over-ranks time.
* one instance over all GPUs (``solve_sharded``): every rank searches the work
  units ``u % world == rank`` of the current size
  (``Session.search_size``); the shards' minimum matching ranks meet in one
  8-byte MIN all-reduce per size, so every rank stops at the same size with
  the same answer -- the reference's per-size stop rule
  (simba/src/nocache.cu:246-276) across GPUs.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence

import numpy as np

NONE = (1 << 63) - 1  # "no match" in the int64 all-reduce


def shard_instances(n: int, rank: int, world: int) -> range:
    """Contiguous, balanced share of n independent instances for this rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    lo = n * rank // world
    hi = n * (rank + 1) // world
    return range(lo, hi)


def torch_allreduce_min(device=None) -> Callable[[int], int]:
    """MIN all-reduce of one int64 over the default process group."""
    import torch
    import torch.distributed as dist

    def f(x: int) -> int:
        t = torch.tensor([x], dtype=torch.int64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        return int(t.item())

    return f


def op_of_rank(counts: np.ndarray, size: int, rank: int) -> int:
    if size == 1:
        return 8
    off = 0
    for op in range(8):
        n = int(counts[size][op])
        if rank < off + n:
            return op
        off += n
    raise ValueError("rank outside the size")


def solve_sharded(session, max_size: int, rank: int, world: int,
                  allreduce_min: Callable[[int], int], counts: np.ndarray,
                  complete: bool = False) -> dict:
    """Plain search of one instance spread over `world` GPUs.

    `session` provides ``search_size(size, shard, nshards)`` (a
    :class:`simba_b200.Session`), `counts` the count table
    (``simba_b200.count_table(max_size, k)``).  Every rank returns the same
    dict: found / size / op / rank, the reference-rule candidate counts, and
    this rank's own evaluated count.
    """
    first = 1 if complete else 2
    last = max_size if complete else max_size - 1
    per_size = [0] * 33
    candidates = 0
    evaluated = 0
    for s in range(first, last + 1):
        r = session.search_size(s, rank, world)
        evaluated += int(r["evaluated"])
        local = NONE
        if r["best_rank"] is not None:
            local = int(r["best_rank"])
            if local >= NONE:
                raise OverflowError("rank does not fit the int64 all-reduce")
        best = allreduce_min(int(local))
        if best != NONE:
            op = op_of_rank(counts, s, best)
            c = best + 1 if s == 1 else int(sum(int(counts[s][q]) for q in range(op + 1)))
            per_size[s] = c
            candidates += c
            return {"found": True, "size": s, "op": op, "rank": best, "candidates": candidates,
                    "per_size": per_size, "evaluated": evaluated}
        per_size[s] = int(counts[s][8])
        candidates += int(counts[s][8])
    return {"found": False, "size": 0, "op": -1, "rank": None, "candidates": candidates,
            "per_size": per_size, "evaluated": evaluated}
