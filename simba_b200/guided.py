"""Learned proposal and guided search.

The proposal is the MLP of the C ABI (``simba_mlp_*``): it reads bit-level
features of an instance's samples and predicts a prior over the 64 shape
classes of the minimal expression (root operator x left-operand size or
root unary-chain length).  The guided search takes that prior: sizes are
still searched in increasing order and every smaller size is exhausted, so
the answer has the minimal size; inside a size the spines run in decreasing
prior and the search stops at the first verified match.  Nothing is pruned:
with a uniform prior the guided search degenerates to the plain order.

Training data comes from the plain search itself: instances are solved by
:func:`simba_b200.solve_batch` and labelled with the shape class of their
answer (:func:`shape_class`).
"""
from __future__ import annotations

import ctypes as C
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

from . import (OK, Result, SimbaError, _Arrays, _check, _Instance, lib, solve,
               solve_batch)
from .instances import Instance, iter_batch

N_CLASSES = 64
N_FEATURES = 8192


def shape_class(postfix: str) -> int:
    c = lib().simba_shape_class(postfix.encode())
    if c < 0:
        raise SimbaError(f"not an expression: {postfix!r}")
    return c


def _bind():
    L = lib()
    if getattr(L, "_mlp_bound", False):
        return L
    P = C.POINTER
    L.simba_shape_class.argtypes = [C.c_char_p]
    L.simba_mlp_param_count.restype = C.c_int64
    L.simba_mlp_create.argtypes = [C.c_int, C.c_uint64, P(C.c_void_p)]
    L.simba_mlp_destroy.argtypes = [C.c_void_p]
    L.simba_mlp_destroy.restype = None
    L.simba_mlp_train_step.argtypes = [C.c_void_p, P(_Instance), C.c_int, P(C.c_int32), C.c_float,
                                       P(C.c_float)]
    L.simba_mlp_gradients.argtypes = [C.c_void_p, P(_Instance), C.c_int, P(C.c_int32),
                                      P(C.c_float), P(C.c_float)]
    L.simba_mlp_apply.argtypes = [C.c_void_p, P(C.c_float), C.c_float]
    L.simba_mlp_predict.argtypes = [C.c_void_p, P(_Instance), C.c_int, P(C.c_float)]
    L.simba_mlp_features.argtypes = [C.c_void_p, P(_Instance), C.c_int, P(C.c_float)]
    L.simba_mlp_get_params.argtypes = [C.c_void_p, P(C.c_float)]
    L.simba_mlp_set_params.argtypes = [C.c_void_p, P(C.c_float)]
    L._mlp_bound = True
    return L


def _carr(insts: Sequence[Instance]):
    arrs = [_Arrays(i) for i in insts]
    return arrs, (_Instance * len(arrs))(*[a.c for a in arrs])


def _f32p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class Proposal:
    """The MLP proposal on one GPU."""

    def __init__(self, device: int = 0, seed: int = 0):
        L = _bind()
        self._h = C.c_void_p()
        _check(L.simba_mlp_create(device, seed, C.byref(self._h)))
        self.n_params = int(L.simba_mlp_param_count())

    def close(self):
        if self._h:
            lib().simba_mlp_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def train_step(self, insts: Sequence[Instance], labels: Sequence[int], lr: float = 1e-3) -> float:
        arrs, ca = _carr(insts)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        loss = C.c_float()
        _check(lib().simba_mlp_train_step(self._h, ca, len(insts),
                                          lab.ctypes.data_as(C.POINTER(C.c_int32)), lr,
                                          C.byref(loss)))
        return float(loss.value)

    def gradients(self, insts, labels) -> Tuple[np.ndarray, float]:
        arrs, ca = _carr(insts)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_float()
        _check(lib().simba_mlp_gradients(self._h, ca, len(insts),
                                         lab.ctypes.data_as(C.POINTER(C.c_int32)), _f32p(g),
                                         C.byref(loss)))
        return g, float(loss.value)

    def apply(self, grads: np.ndarray, lr: float = 1e-3) -> None:
        """One Adam step with the given gradients (the all-reduced mean in
        data-parallel training)."""
        g = np.ascontiguousarray(grads, dtype=np.float32)
        if g.size != self.n_params:
            raise ValueError("wrong gradient count")
        _check(lib().simba_mlp_apply(self._h, _f32p(g), lr))

    def predict(self, insts: Sequence[Instance]) -> np.ndarray:
        arrs, ca = _carr(insts)
        p = np.zeros((len(insts), N_CLASSES), dtype=np.float32)
        _check(lib().simba_mlp_predict(self._h, ca, len(insts), _f32p(p)))
        return p

    def features(self, insts: Sequence[Instance]) -> np.ndarray:
        arrs, ca = _carr(insts)
        x = np.zeros((len(insts), N_FEATURES), dtype=np.float32)
        _check(lib().simba_mlp_features(self._h, ca, len(insts), _f32p(x)))
        return x

    def get_params(self) -> np.ndarray:
        w = np.zeros(self.n_params, dtype=np.float32)
        _check(lib().simba_mlp_get_params(self._h, _f32p(w)))
        return w

    def set_params(self, w: np.ndarray) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.size != self.n_params:
            raise ValueError("wrong parameter count")
        _check(lib().simba_mlp_set_params(self._h, _f32p(w)))

    def save(self, path) -> None:
        np.save(path, self.get_params())

    def load(self, path) -> None:
        self.set_params(np.load(path))


def label_instances(insts: Sequence[Instance], max_size: int, budget: float = 0.0,
                    **kw) -> Tuple[List[Instance], np.ndarray]:
    """Solve with the plain batch search; keep the solved ones with labels."""
    res, _ = solve_batch(insts, max_size, budget=budget, **kw)
    keep, labels = [], []
    for inst, r in zip(insts, res):
        if r.status == OK:
            keep.append(inst)
            labels.append(shape_class(r.postfix))
    return keep, np.asarray(labels, dtype=np.int32)


def train(prop: Proposal, insts: Sequence[Instance], labels: np.ndarray, epochs: int = 3,
          batch: int = 256, lr: float = 1e-3, seed: int = 0) -> List[float]:
    """Minibatch Adam over (instances, labels); returns the loss per step."""
    rng = np.random.default_rng(seed)
    losses = []
    n = len(insts)
    for _ in range(epochs):
        order = rng.permutation(n)
        for s in range(0, n, batch):
            idx = order[s:s + batch]
            if len(idx) == 0:
                continue
            losses.append(prop.train_step([insts[i] for i in idx], labels[idx], lr))
    return losses


def torch_allreduce_mean(group=None):
    """All-reduce (mean over ranks) of a float32 vector through
    torch.distributed: NCCL over NVLink for GPU process groups, gloo on CPU."""
    import torch
    import torch.distributed as dist

    def reduce(x: np.ndarray) -> np.ndarray:
        world = dist.get_world_size(group)
        dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
        t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32)).to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        return (t / world).cpu().numpy()
    return reduce


def train_dp(prop, insts: Sequence[Instance], labels: np.ndarray, rank: int, world: int,
             allreduce_mean, epochs: int = 3, batch: int = 256, lr: float = 1e-3,
             seed: int = 0) -> List[float]:
    """Data-parallel minibatch Adam: every rank draws the same global
    minibatch order, computes gradients on its equal share of each
    minibatch, the shares' gradients are averaged by ``allreduce_mean`` and
    every rank applies the same Adam step, so the replicas stay identical.
    With equal shares the mean gradient is the full minibatch's.  Returns
    the mean loss per step."""
    rng = np.random.default_rng(seed)
    n = len(insts)
    per = batch // world
    if per == 0:
        raise ValueError("batch smaller than the number of ranks")
    losses = []
    for _ in range(epochs):
        order = rng.permutation(n)
        for s in range(0, n - per * world + 1, per * world):  # whole global minibatches only
            idx = order[s + rank * per: s + (rank + 1) * per]
            g, loss = prop.gradients([insts[i] for i in idx], labels[idx])
            g = allreduce_mean(g)
            losses.append(float(allreduce_mean(np.array([loss], dtype=np.float32))[0]))
            prop.apply(g, lr)
    return losses


def solve_guided(inst: Instance, max_size: int, prior: np.ndarray, **kw) -> Result:
    """Guided plain search of one instance with a 64-class prior."""
    pr = np.ascontiguousarray(prior, dtype=np.float32)
    if pr.size != N_CLASSES:
        raise ValueError("prior must have 64 entries")
    return solve(inst, max_size, class_prior=pr, **kw)


# ---------------------------------------------------------------------------
# The proposal's training and evaluation workloads (seeded, synthetic).

def training_set(n: int, seed0: int = 10 ** 6, max_size: int = 14, budget: float = 0.0,
                 device: int = 0) -> Tuple[List[Instance], np.ndarray]:
    """Instances for training the proposal: random targets of size 3-13 over
    1-4 variables (+ the constant 1), 64 uint64 samples, seeds seed0.., solved
    by the plain batch search and labelled with the shape class of the
    answer (unsolved ones are dropped)."""
    insts = list(iter_batch(n, seed0, sizes=range(3, 14), vars_=(1, 2, 3, 4), samples=(64,),
                            word_bits=64))
    return label_instances(insts, max_size, budget=budget, device=device)


def mixed_batch(n: int, seed0: int = 5 * 10 ** 6) -> List[Instance]:
    """The guided-and-batched workload: variables 2-5 (+ the constant 1),
    target size 7-19, samples {32, 64, 128}, uint64 words."""
    return list(iter_batch(n, seed0, sizes=range(7, 20), vars_=(2, 3, 4, 5),
                           samples=(32, 64, 128), word_bits=64))


def oracle_priors(results: Sequence[Result]) -> np.ndarray:
    """The best prior any proposal could give: all mass on the shape class of
    the answer the plain search found (uniform where it found none).  A guided
    run with these priors bounds what guidance can gain on that batch."""
    pri = np.full((len(results), N_CLASSES), 1.0 / N_CLASSES, dtype=np.float32)
    for i, r in enumerate(results):
        if r.status == OK:
            pri[i] = 1e-6
            pri[i, shape_class(r.postfix)] = 1.0
    return pri


def time_stats(results: Sequence[Result]) -> dict:
    """Solved fraction and time-to-solution percentiles (device clock);
    unsolved instances count as infinitely slow in the all-instance figures."""
    solved = sorted(r.seconds for r in results if r.status == OK)
    every = sorted([r.seconds if r.status == OK else float("inf") for r in results])

    def pct(xs, q):  # None where the percentile instance is unsolved
        if not xs:
            return None
        v = xs[min(len(xs) - 1, int(q * len(xs)))]
        return None if v == float("inf") else v
    return {"solved_frac": len(solved) / max(1, len(results)),
            "p50_s": pct(every, 0.5), "p95_s": pct(every, 0.95),
            "p50_solved_s": pct(solved, 0.5), "p95_solved_s": pct(solved, 0.95)}


def heldout_set(n: int = 1024, seed0: int = 3 * 10 ** 6) -> List[Instance]:
    """Held-out evaluation targets: random size 11-17 over 1-4 variables (+ the
    constant 1), 64 uint64 samples (seeds disjoint from the training set's)."""
    return list(iter_batch(n, seed0, sizes=range(11, 18), vars_=(1, 2, 3, 4), samples=(64,),
                           word_bits=64))


def label_in_chunks(insts: Sequence[Instance], max_size: int, chunk: int, budget: float,
                    device: int = 0) -> Tuple[List[Instance], np.ndarray]:
    """label_instances over consecutive chunks, each under its own budget."""
    keep: List[Instance] = []
    labels: List[int] = []
    for s in range(0, len(insts), chunk):
        k, l = label_instances(insts[s:s + chunk], max_size, budget=budget, device=device)
        keep += k
        labels += list(l)
    return keep, np.asarray(labels, dtype=np.int32)


def proposal_experiment(n_train: int = 200_000, n_eval: int = 1024, epochs: int = 4,
                        label_chunk: int = 16384, label_budget: float = 30.0,
                        eval_budget: float = 60.0, device: int = 0, seed: int = 0) -> dict:
    """The learned-proposal experiment: train on `n_train` instances solved by
    the plain batch search (training_set's distribution, max size 14), then
    search the held-out targets (max size 20) plain, guided by the trained
    proposal, and guided by the best possible prior (the plain answers'
    classes), each as one batch under `eval_budget` seconds.  Returns the
    timings, solved fractions, time-to-solution percentiles and the
    proposal's top-1 accuracy on the held-out answers."""
    import time
    t0 = time.perf_counter()
    train_insts = list(iter_batch(n_train, 10 ** 6, sizes=range(3, 14), vars_=(1, 2, 3, 4),
                                  samples=(64,), word_bits=64))
    keep, labels = label_in_chunks(train_insts, 14, label_chunk, label_budget, device)
    t_label = time.perf_counter() - t0
    prop = Proposal(device=device, seed=seed)
    t0 = time.perf_counter()
    losses = train(prop, keep, labels, epochs=epochs, batch=256, lr=1e-3, seed=seed)
    t_train = time.perf_counter() - t0
    ev = heldout_set(n_eval)
    plain, st_p = solve_batch(ev, 20, budget=eval_budget, device=device)
    pri = prop.predict(ev)
    guided, st_g = solve_batch(ev, 20, budget=eval_budget, device=device, class_prior=pri)
    best, st_b = solve_batch(ev, 20, budget=eval_budget, device=device,
                             class_prior=oracle_priors(plain))
    prop.close()
    cls = [shape_class(r.postfix) if r.status == OK else -1 for r in plain]
    top1 = [int(p.argmax()) == c for p, c in zip(pri, cls) if c >= 0]
    both = [(a, b) for a, b in zip(plain, guided) if a.status == OK and b.status == OK]
    out = {"train": {"instances": n_train, "labelled": len(keep), "label_s": t_label,
                     "train_s": t_train, "epochs": epochs,
                     "final_loss": float(np.mean(losses[-50:])) if losses else None},
           "eval": {"instances": n_eval, "top1": float(np.mean(top1)) if top1 else None,
                    "plain": time_stats(plain), "guided": time_stats(guided),
                    "oracle_prior": time_stats(best),
                    "same_minimal_size": all(a.size == b.size for a, b in both),
                    "kernel_s": {"plain": st_p["kernel_ms"] / 1e3, "guided": st_g["kernel_ms"] / 1e3,
                                 "oracle_prior": st_b["kernel_ms"] / 1e3}}}
    for k in ("guided", "oracle_prior"):
        a, b = out["eval"]["plain"]["p50_s"], out["eval"][k]["p50_s"]
        out["eval"][f"p50_ratio_plain_over_{k}"] = a / b if a and b else None
    return out


if __name__ == "__main__":  # python -m simba_b200.guided [n_train] > result.json
    import json
    import sys
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 200_000
    print(json.dumps(proposal_experiment(n_train=n), indent=1))
