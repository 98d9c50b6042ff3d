"""Plain SIMBA search on the GPU, through the C ABI, against the oracle.

Parity bar: the minimum matching rank of the first (size, root-operator)
block that holds a match is bit-identical to the oracle's; the returned
expression therefore has the same size, the same block and evaluates to the
target on every sample; the reference-rule candidate counts are identical.
"""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import simba_b200 as S
from simba_b200.instances import Instance, infix_to_postfix, make_instance

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent
OPS = "~&|^#+-*"


def same_as_oracle(res, o):
    assert res.found == o["found"]
    if o["found"]:
        assert res.size == o["size"]
        assert res.op == o["op"]
        assert res.rank == o["rank"]
        assert res.postfix == o["postfix"]
    assert res.candidates == o["candidates"]
    assert list(res.per_size) == list(o["per_size"])


def test_golden_reference_instances(oracle, golden):
    """uint32 instances from the reference generator; answers vs the
    reference executable (same size/block) and the oracle (same rank)."""
    for r in golden["results"]["simba"]:
        d = golden["instances"][r["idx"]]
        inst = Instance.from_json(d)
        res = S.solve(inst, r["max_len"])
        o = oracle.search(inst.inputs, inst.outputs, r["max_len"], 32)
        same_as_oracle(res, o)
        ref = infix_to_postfix(r["expr"])
        assert res.size == len(ref) and res.op == OPS.index(ref[-1])
        assert oracle.check(res.postfix, inst.inputs, inst.outputs, 32)


@pytest.mark.parametrize("bits", [32, 64])
def test_random_instances_vs_oracle(oracle, bits):
    for seed in range(12):
        size = 3 + seed % 7
        nv = 1 + seed % 3
        ns = (8, 16, 32, 64)[seed % 4]
        inst = make_instance(size, nv, ns, 1000 + seed, word_bits=bits)
        res = S.solve(inst, 10)
        o = oracle.search(inst.inputs, inst.outputs, 10, bits)
        same_as_oracle(res, o)


def test_spine_engine_matches_naive_engine():
    for seed in range(4):
        inst = make_instance(11, 2, 32, 77 + seed, word_bits=64)
        a = S.solve(inst, 13)
        b = S.solve(inst, 13, naive=True)
        assert (a.status, a.size, a.rank, a.postfix) == (b.status, b.size, b.rank, b.postfix)


def test_small_tables_force_deep_spines(oracle):
    """A 1 MiB table cap forces spines of depth 3-6 with explicit levels."""
    for seed in range(4):
        inst = make_instance(9, 2, 16, 500 + seed, word_bits=64)
        a = S.solve(inst, 11, table_bytes=1 << 14)
        o = oracle.search(inst.inputs, inst.outputs, 11, 64)
        same_as_oracle(a, o)
        assert a.table_size <= 6


def test_unsat_sweep_counts():
    inst = make_instance(9, 3, 64, 9, word_bits=64, unsat=True)
    with S.Session(inst) as ss:
        r = ss.sweep(1, 10)
    t = S.count_table(10, inst.num_variables)
    assert r.status == S.NOT_FOUND
    assert r.candidates == int(t[1:11, 8].sum())
    # unary chains with the same affine map are tested once: evaluated <= candidates
    assert 0.9 * r.candidates <= r.evaluated <= r.candidates


def test_session_reuse_is_deterministic():
    inst = make_instance(10, 2, 32, 4, word_bits=64)
    with S.Session(inst) as ss:
        a = ss.solve(12)
        b = ss.solve(12)
    assert (a.status, a.size, a.rank) == (b.status, b.size, b.rank)


def test_edge_cases(oracle):
    # target = a bare variable: the reference never searches size 1
    inst = make_instance(1, 3, 16, 3, word_bits=64)
    r = S.solve(inst, 6)
    o = oracle.search(inst.inputs, inst.outputs, 6, 64)
    same_as_oracle(r, o)
    rc = S.solve(inst, 6, complete=True)
    assert rc.found and rc.size == 1 and rc.op == 8
    # constant-zero target: found as (v - v) at size 3
    z = make_instance(3, 2, 16, 1, word_bits=64)
    z.outputs[:] = 0
    r = S.solve(z, 6)
    o = oracle.search(z.inputs, z.outputs, 6, 64)
    same_as_oracle(r, o)
    assert r.size == 3
    # one variable, one sample, max size 1 and 2 (nothing searched)
    one = make_instance(2, 1, 1, 5, word_bits=32, const_one=False)
    for ms in (1, 2):
        r = S.solve(one, ms)
        assert r.status == S.NOT_FOUND and r.candidates == 0
    # 256 samples, 16 terminals (this build's limits)
    wide = make_instance(5, 15, 256, 8, word_bits=64)
    r = S.solve(wide, 7)
    o = oracle.search(wide.inputs, wide.outputs, 7, 64)
    same_as_oracle(r, o)


def test_budget_stops_a_long_search():
    inst = make_instance(17, 4, 64, 2, word_bits=64, unsat=True)
    r = S.solve(inst, 20, budget=0.5)
    assert r.status == S.BUDGET
    assert r.seconds < 10


def test_cli_dropin(tmp_path, oracle, golden):
    exe = ROOT / "simba_b200" / "bin" / "simba"
    for r in golden["results"]["simba"][:10]:
        d = golden["instances"][r["idx"]]
        p = tmp_path / f"inst_{r['idx']}.json"
        p.write_text(json.dumps(d))
        out = subprocess.run([str(exe), str(p), str(r["max_len"])], capture_output=True,
                             text=True, timeout=120)
        assert out.returncode == 0
        line = out.stdout.strip()
        path, expr, secs = line.rsplit(",", 2)
        assert path == str(p)
        float(secs)
        inst = Instance.from_json(d)
        o = oracle.search(inst.inputs, inst.outputs, r["max_len"], 32)
        assert expr == S.format_postfix(o["postfix"])
    out = subprocess.run([str(exe)], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout == "" and "maxLen" in out.stderr


def test_shards_of_a_size_combine_to_the_full_search(oracle):
    """Work units split across 3 shards (as over 3 GPUs): the minimum of the
    shards' best ranks is the single-GPU answer, size by size."""
    from simba_b200 import dist as D
    for seed in range(3):
        inst = make_instance(10, 2, 32, 60 + seed, word_bits=64)
        full = S.solve(inst, 12)
        counts = S.count_table(12, inst.num_variables)
        with S.Session(inst) as ss:
            res = [D.solve_sharded(ss, 12, shard, 3, lambda x: x, counts) for shard in range(3)]
        best = min((r["rank"] for r in res if r["found"]), default=None)
        if full.found:
            sizes = {r["size"] for r in res if r["found"]}
            assert min(sizes) == full.size
            # per size, only shards of the minimal size compete
            best = min(r["rank"] for r in res if r["found"] and r["size"] == full.size)
            assert best == full.rank
        with S.Session(inst) as ss:
            for size in range(2, 12):
                parts = [ss.search_size(size, sh, 3) for sh in range(3)]
                whole = ss.search_size(size, 0, 1)
                mins = [p["best_rank"] for p in parts if p["best_rank"] is not None]
                assert (min(mins) if mins else None) == whole["best_rank"]
                if whole["best_rank"] is not None:
                    break  # units above a match may be skipped differently
                assert sum(p["evaluated"] for p in parts) == whole["evaluated"]


@pytest.mark.parametrize("bits", [32, 64])
def test_rtid_order_matches_oracle(oracle, bits):
    """RTid order (simba_rtid): same size, block, candidate count and the same
    expression (the match of the smallest thread position) as the oracle."""
    for seed in range(12):
        inst = make_instance(5 + seed % 6, 1 + seed % 3, (16, 32, 64)[seed % 3], 5100 + seed,
                             word_bits=bits)
        r = S.solve(inst, 12, rtid=True)
        o = oracle.search_rtid(inst.inputs, inst.outputs, 12, bits)
        assert r.found == o["found"]
        assert r.candidates == o["candidates"]
        if o["found"]:
            assert (r.size, r.op, r.rank, r.postfix) == (o["size"], o["op"], o["rank"], o["postfix"])


def test_rtid_large_blocks_and_deep_spines(oracle):
    """Blocks of ~1e9 ranks (64-bit products in the position map) and small
    tables (explicit levels, fused spines): still the oracle's answer."""
    for seed in range(3):
        inst = make_instance(11, 3, 32, 5300 + seed, word_bits=64)
        for tb in (0, 1 << 16):
            r = S.solve(inst, 12, rtid=True, table_bytes=tb)
            o = oracle.search_rtid(inst.inputs, inst.outputs, 12, 64)
            assert (r.found, r.size, r.op, r.rank) == (o["found"], o["size"], o["op"], o["rank"])


def test_rtid_cli_dropin(tmp_path, oracle, golden):
    exe = ROOT / "simba_b200" / "bin" / "simba_rtid"
    for r in golden["results"]["simba"][:10]:
        d = golden["instances"][r["idx"]]
        p = tmp_path / f"inst_{r['idx']}.json"
        p.write_text(json.dumps(d))
        out = subprocess.run([str(exe), str(p), str(r["max_len"])], capture_output=True,
                             text=True, timeout=120)
        assert out.returncode == 0
        path, expr, secs = out.stdout.strip().rsplit(",", 2)
        inst = Instance.from_json(d)
        o = oracle.search_rtid(inst.inputs, inst.outputs, r["max_len"], 32)
        assert expr == (S.format_postfix(o["postfix"]) if o["found"] else "Not found !")


def test_rtid_matches_reference_rtid_executable(oracle):
    """The reference's simba_rtid on the golden instances: same size and
    operator block, and a verified match."""
    g = ROOT / "tests" / "golden"
    f = g / "ref_results_rtid_u32.json"
    if not f.exists():
        pytest.skip("reference RTid results not generated")
    insts = json.loads((g / "ref_instances_u32.json").read_text())
    for r in json.loads(f.read_text())["simba_rtid"]:
        inst = Instance.from_json(insts[r["idx"]])
        res = S.solve(inst, r["max_len"], rtid=True)
        if r["expr"] == "Not found !":
            assert not res.found
            continue
        p = infix_to_postfix(r["expr"])
        assert res.found and res.size == len(p) and res.postfix[-1] == p[-1]
        assert oracle.check(res.postfix, inst.inputs, inst.outputs, 32)
