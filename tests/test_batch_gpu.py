"""Batched plain search on the GPU: every instance of a batch gets the answer
the single-instance search (and the oracle) gives it."""
import pytest

import simba_b200 as S
from simba_b200.instances import Instance, iter_batch, make_instance

pytestmark = pytest.mark.gpu


def test_batch_matches_oracle_per_instance(oracle):
    insts = list(iter_batch(48, 5000, sizes=range(3, 10), vars_=(1, 2, 3),
                            samples=(16, 32, 64, 128), word_bits=64))
    res, stats = S.solve_batch(insts, 10)
    assert stats["rounds"] >= 1 and stats["solved"] == sum(r.found for r in res)
    for inst, r in zip(insts, res):
        o = oracle.search(inst.inputs, inst.outputs, 10, 64)
        assert r.found == o["found"]
        assert r.candidates == o["candidates"]
        if o["found"]:
            assert (r.size, r.op, r.rank, r.postfix) == (o["size"], o["op"], o["rank"], o["postfix"])
            assert r.seconds > 0


def test_batch_u32_golden_equals_single_solves(golden):
    insts = [Instance.from_json(d) for d in golden["instances"][:60]]
    res, _ = S.solve_batch(insts, 11)
    for inst, r in zip(insts, res):
        one = S.solve(inst, 11)
        assert (r.status, r.size, r.rank, r.postfix, r.candidates) == \
            (one.status, one.size, one.rank, one.postfix, one.candidates)


def test_batch_small_tables_and_unsat_mix(oracle):
    insts = [make_instance(8, 2, 32, 90 + i, word_bits=64, unsat=(i % 3 == 0)) for i in range(9)]
    res, stats = S.solve_batch(insts, 9, table_bytes=1 << 12)
    for inst, r in zip(insts, res):
        o = oracle.search(inst.inputs, inst.outputs, 9, 64)
        assert (r.found, r.rank, r.candidates) == (o["found"], o["rank"], o["candidates"])


def test_batch_budget_retires_everything():
    insts = [make_instance(17, 4, 64, 300 + i, word_bits=64, unsat=True) for i in range(4)]
    res, stats = S.solve_batch(insts, 20, budget=0.5)
    assert all(r.status == S.BUDGET for r in res)


def test_empty_batch():
    res, stats = S.solve_batch([], 10)
    assert res == [] and stats["solved"] == 0


def test_autotuner_picks_a_candidate_and_caches(tmp_path, monkeypatch):
    from simba_b200 import autotune as A
    monkeypatch.setenv("SIMBA_CACHE", str(tmp_path))
    A._mem.clear()
    u = A.tune_bucket(3, 32, 64)
    assert u in A.CANDIDATES
    assert (tmp_path / "autotune.json").exists()
    A._mem.clear()
    assert A.tune_bucket(3, 32, 64) == u  # served from the cache file
    insts = list(iter_batch(12, 7000, sizes=range(3, 8), vars_=(2,), samples=(32,), word_bits=64))
    tuned = A.tune_batch(insts)
    for i in insts:
        i.unit_log2 = tuned[(i.num_variables, i.num_examples, i.word_bits)]
    res, _ = S.solve_batch(insts, 9)
    for inst, r in zip(insts, res):
        one = S.solve(inst, 9)
        assert (r.status, r.rank) == (one.status, one.rank)


def test_autotuned_knobs_keep_answers(tmp_path, monkeypatch):
    """All three tuned knobs (unit size, lanes per context group, filter
    samples) are chosen from their candidate sets, and searches run with any
    of them return the same answers as the defaults."""
    from simba_b200 import autotune as A
    monkeypatch.setenv("SIMBA_CACHE", str(tmp_path))
    A._mem.clear()
    k = A.tune_bucket_knobs(4, 64, 64)
    assert k["unit_log2"] in A.CANDIDATES and k["lanes_log2"] in A.LANES
    assert k["filter_samples"] in A.FILTERS
    insts = list(iter_batch(24, 9100, sizes=range(5, 11), vars_=(3,), samples=(64,), word_bits=64))
    base = [S.solve(i, 11) for i in insts]
    for lanes, filt in ((0, 1), (2, 3), (4, 2)):
        for inst, b in zip(insts, base):
            r = S.solve(inst, 11, lanes_log2=lanes, filter_samples=filt, table_bytes=1 << 24)
            assert (r.status, r.size, r.rank, r.postfix) == (b.status, b.size, b.rank, b.postfix)
    per, opts = A.tune_batch_knobs(insts)
    res, _ = S.solve_batch(insts, 11, **opts)
    for r, b in zip(res, base):
        assert (r.status, r.rank) == (b.status, b.rank)


def test_guided_batch_finds_minimal_sizes(oracle):
    """Guided batch with per-instance priors: same minimal size as the plain
    batch, every answer verified, in one launch per size round."""
    import numpy as np
    insts = list(iter_batch(40, 8000, sizes=range(4, 11), vars_=(1, 2, 3), samples=(32, 64),
                            word_bits=64))
    rng = np.random.default_rng(0)
    priors = rng.random((len(insts), 64)).astype(np.float32)
    plain, _ = S.solve_batch(insts, 11, table_bytes=1 << 16)
    guided, st = S.solve_batch(insts, 11, table_bytes=1 << 16, class_prior=priors)
    for inst, a, b in zip(insts, plain, guided):
        assert a.status == b.status
        if a.found:
            assert b.size == a.size
            assert oracle.check(b.postfix, inst.inputs, inst.outputs, 64)
