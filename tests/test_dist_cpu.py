"""Multi-GPU host logic on CPU: world_size-2 gloo process groups.

The GPU side is replaced by a fake session whose per-(size, shard) minima
come from the oracle, so the per-size MIN all-reduce and stop rule of
simba_b200.dist.solve_sharded are checked without a GPU.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from simba_b200 import dist as D
from simba_b200.instances import make_instance


def free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class OracleShardSession:
    """search_size over ranks r with (r // unit) % world == shard, answered
    by the CPU oracle (stands in for the GPU work units)."""

    def __init__(self, inst, unit=64):
        from oracle import oracle as O
        self.O = O
        self.inst = inst
        self.unit = unit

    def search_size(self, size, shard, nshards):
        t = self.O.count_table(max(size, 2), self.inst.num_variables)
        n = int(t[size][8])
        best = None
        ev = 0
        u = shard
        while u * self.unit < n:
            lo, hi = u * self.unit, min(n, (u + 1) * self.unit)
            if size >= 2:
                e, mr, nh = self.O.scan_range(self.inst.inputs, self.inst.outputs, size, lo, hi,
                                              64, 1)
            else:
                e, mr, nh = hi - lo, 2 ** 64 - 1, 0
                for v in range(lo, hi):
                    if (self.inst.inputs[:, v] == self.inst.outputs).all():
                        mr, nh = v, 1
                        break
            ev += e
            if nh and (best is None or mr < best):
                best = mr
            u += nshards
        return {"best_rank": best, "evaluated": ev}


def _worker(rank, world, port, seed, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        inst = make_instance(6, 2, 16, seed, word_bits=64)
        from oracle import oracle as O
        counts = O.count_table(8, inst.num_variables)
        res = D.solve_sharded(OracleShardSession(inst), 8, rank, world,
                              D.torch_allreduce_min(), counts)
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_solve_sharded_two_ranks_matches_oracle(seed):
    from oracle import oracle as O
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, seed, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    inst = make_instance(6, 2, 16, seed, word_bits=64)
    ref = O.search(inst.inputs, inst.outputs, 8, 64)
    for r in (0, 1):
        assert out[r]["found"] == ref["found"]
        assert out[r]["candidates"] == ref["candidates"]
        if ref["found"]:
            assert (out[r]["size"], out[r]["op"], out[r]["rank"]) == (ref["size"], ref["op"],
                                                                    ref["rank"])
    # the shards split the work: together they evaluated the searched ranks once
    assert out[0]["evaluated"] > 0 and out[1]["evaluated"] > 0


def test_shard_instances_covers_everything_once():
    for n in (0, 1, 7, 4096):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                seen += list(D.shard_instances(n, r, world))
            assert seen == list(range(n))


def test_single_process_loop_without_collective():
    """world = 1 with an identity all-reduce gives the oracle answer."""
    from oracle import oracle as O
    inst = make_instance(7, 2, 16, 3, word_bits=64)
    counts = O.count_table(9, inst.num_variables)
    res = D.solve_sharded(OracleShardSession(inst), 9, 0, 1, lambda x: x, counts)
    ref = O.search(inst.inputs, inst.outputs, 9, 64)
    assert (res["found"], res["size"], res["rank"], res["candidates"]) == \
        (ref["found"], ref["size"], ref["rank"], ref["candidates"])


class OracleProposal:
    """Stands in for the GPU proposal on CPU: gradients from the numpy
    oracle of the network (small layer sizes), Adam in numpy; instances
    are row indices of a fixed feature matrix."""

    DIMS = (32, 16, 16, 8)

    def __init__(self, seed=0):
        from oracle import mlp_ref as R
        self.R = R
        rng = np.random.default_rng(seed)
        d = self.DIMS
        n = sum(d[i] * d[i + 1] + d[i + 1] for i in range(3))
        self.w = (rng.standard_normal(n) * 0.1).astype(np.float32)
        self.m = np.zeros(n, np.float32)
        self.v = np.zeros(n, np.float32)
        self.t = 0
        self.X = np.sign(np.random.default_rng(99).standard_normal((64, d[0]))).astype(np.float32)

    def gradients(self, rows, labels):
        loss, g, _ = self.R.forward_backward(self.w, self.X[list(rows)], np.asarray(labels),
                                             dims=self.DIMS, round_bf16=False)
        return np.asarray(g, np.float32), float(loss)

    def apply(self, g, lr):
        self.t += 1
        b1, b2 = 0.9, 0.999
        self.m = b1 * self.m + (1 - b1) * g
        self.v = b2 * self.v + (1 - b2) * g * g
        mh = self.m / (1 - b1 ** self.t)
        vh = self.v / (1 - b2 ** self.t)
        self.w = (self.w - lr * mh / (np.sqrt(vh) + 1e-8)).astype(np.float32)


def _dp_worker(rank, world, port, q):
    import torch.distributed as dist
    from simba_b200 import guided as G
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        prop = OracleProposal(seed=3)
        labels = np.arange(64, dtype=np.int32) % 8
        losses = G.train_dp(prop, list(range(64)), labels, rank, world, G.torch_allreduce_mean(),
                            epochs=3, batch=16, lr=1e-2)
        q.put((rank, prop.w, losses))
    finally:
        dist.destroy_process_group()


def test_data_parallel_training_two_ranks_equals_one():
    """The proposal's data-parallel training: two gloo ranks, each with half
    of every minibatch and a mean all-reduce of the gradients, end with the
    same parameters as one rank training on the whole minibatches."""
    from simba_b200 import guided as G
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_dp_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {r: (w, l) for r, w, l in (q.get(timeout=120) for _ in range(2))}
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    one = OracleProposal(seed=3)
    labels = np.arange(64, dtype=np.int32) % 8
    ref_losses = G.train_dp(one, list(range(64)), labels, 0, 1, lambda x: x, epochs=3, batch=16,
                            lr=1e-2)
    assert np.array_equal(out[0][0], out[1][0])  # replicas stay identical
    np.testing.assert_allclose(out[0][0], one.w, rtol=1e-4, atol=1e-6)
    np.testing.assert_allclose(out[0][1], ref_losses, rtol=1e-5)
    assert ref_losses[-1] < ref_losses[0]
