"""VFB bottom-up search on the GPU, through the C ABI.

Parity bar: the found size, the operator block and found / not found are
those of the oracle; the returned expression evaluates to the target on
every sample.  With reference_dedup the reference's uniqueness test as
written is reproduced, and the found size matches the reference executable's
on every golden instance.
"""
import json
import subprocess
from pathlib import Path

import pytest

import simba_b200 as S
from simba_b200.instances import Instance, infix_to_postfix, make_instance

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent


def test_vfb_reference_dedup_matches_reference_executable(oracle, golden):
    for r in golden["results"]["vfb"]:
        d = golden["instances"][r["idx"]]
        inst = Instance.from_json(d)
        res = S.vfb_solve(inst, r["max_len"], reference_dedup=True)
        if r["expr"] in ("Not found !", ""):
            assert not res.found
            continue
        ref = infix_to_postfix(r["expr"])
        assert res.found and res.size == len(ref), (r, res)
        assert oracle.check(res.postfix, inst.inputs, inst.outputs, 32)
        assert S.format_postfix(res.postfix, "vfb") == res.expr


@pytest.mark.parametrize("bits", [32, 64])
def test_vfb_correct_dedup_vs_oracle(oracle, bits):
    for seed in range(10):
        inst = make_instance(3 + seed % 6, 1 + seed % 3, (16, 32, 64)[seed % 3], 2000 + seed,
                             word_bits=bits)
        res = S.vfb_solve(inst, 8)
        o = oracle.vfb(inst.inputs, inst.outputs, 8, bits)
        assert res.found == o["found"]
        if o["found"]:
            assert res.size == o["size"] and res.op == o["op"]
            assert oracle.check(res.postfix, inst.inputs, inst.outputs, bits)
            # rows per size are deterministic: same vector sets as the oracle
            for L in range(1, res.size):
                assert res.rows_per_size[L] == o["rows_per_size"][L], (L, res, o)


def test_vfb_minimal_size_equals_plain_search(oracle):
    for seed in range(6):
        inst = make_instance(8, 2, 32, 3000 + seed, word_bits=64)
        v = S.vfb_solve(inst, 9)
        p = S.solve(inst, 10, complete=True)
        assert v.found == p.found
        if v.found:
            assert v.size == p.size


def test_vfb_reference_dedup_vs_oracle_emulation(oracle):
    for seed in range(6):
        inst = make_instance(6, 2, 16, 4000 + seed, word_bits=32)
        res = S.vfb_solve(inst, 8, reference_dedup=True)
        o = oracle.vfb(inst.inputs, inst.outputs, 8, 32, ref_inverted=True)
        assert res.found == o["found"]
        if o["found"]:
            assert res.size == o["size"] and res.op == o["op"]
        for L in range(1, (res.size or 8)):
            assert res.rows_per_size[L] == o["rows_per_size"][L]


def test_vfb_cache_full_is_not_found():
    inst = make_instance(12, 3, 32, 7, word_bits=64, unsat=True)
    res = S.vfb_solve(inst, 12, cache_rows=5000)
    assert res.status == S.CACHE_FULL and not res.found and res.expr == "Not found !"


def test_vfb_variable_target_found_at_size_one():
    inst = make_instance(1, 3, 16, 11, word_bits=64)
    res = S.vfb_solve(inst, 4)
    assert res.found and res.size == 1 and res.op == 8


def test_vfb_cli_dropin(tmp_path, oracle, golden):
    exe = ROOT / "simba_b200" / "bin" / "vfb"
    for r in golden["results"]["vfb"][:8]:
        d = golden["instances"][r["idx"]]
        p = tmp_path / f"inst_{r['idx']}.json"
        p.write_text(json.dumps(d))
        out = subprocess.run([str(exe), "--reference-dedup", str(p), str(r["max_len"])],
                             capture_output=True, text=True, timeout=120)
        assert out.returncode == 0
        path, expr, secs = out.stdout.strip().rsplit(",", 2)
        float(secs)
        assert path == str(p)
        if r["expr"] not in ("Not found !", ""):
            assert len(infix_to_postfix(expr)) == len(infix_to_postfix(r["expr"]))
        else:
            assert expr == "Not found !"


@pytest.mark.parametrize("fp_bits", [10, 16])
def test_vfb_exact_dedup_under_forced_fingerprint_collisions(oracle, monkeypatch, fp_bits):
    """With only `fp_bits` bits of the 64-bit fingerprint kept, thousands of
    distinct vectors share a fingerprint; the exact dedup compares stored
    rows element by element, so the rows per size (distinct vectors) still
    equal the oracle's exact vector sets, unsatisfiable targets included."""
    monkeypatch.setenv("SIMBA_VFB_FP_BITS", str(fp_bits))
    for seed, bits in ((0, 64), (1, 32), (2, 64)):
        inst = make_instance(7, 2, 32, 4000 + seed, word_bits=bits, unsat=seed == 2)
        res = S.vfb_solve(inst, 7)
        o = oracle.vfb(inst.inputs, inst.outputs, 7, bits)
        assert res.found == o["found"]
        last = res.size if res.found else 7
        for L in range(1, last):
            assert res.rows_per_size[L] == o["rows_per_size"][L], (fp_bits, seed, L, res, o)
        if o["found"]:
            assert res.size == o["size"] and res.op == o["op"]
            assert oracle.check(res.postfix, inst.inputs, inst.outputs, bits)
