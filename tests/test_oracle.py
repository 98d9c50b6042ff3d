"""The CPU oracle, pinned against the reference's own outputs (no GPU needed).

Pins:
  * ref_instances_u32.json: formulas and uint32 outputs produced by the
    reference's scripts/generate.py + scripts/sample.py;
  * ref_results_u32.json: answers printed by the reference executables
    (simba/src/nocache.cu, vfb/src/full-cache.cu rebuilt for sm_100a) on
    those instances;
  * the rank-space sizes the reference's count table implies.
"""
import numpy as np
import pytest

from simba_b200.instances import (Instance, eval_postfix, infix_to_postfix, make_instance,
                                  postfix_to_infix)

OPS = "~&|^#+-*"


def test_count_table_recurrence(oracle):
    t = oracle.count_table(8, 2)
    assert list(t[1]) == [0] * 8 + [2]
    assert list(t[2]) == [2, 0, 0, 0, 2, 0, 0, 0, 4]
    assert list(t[3]) == [4] * 8 + [32]
    assert [int(t[s][8]) for s in range(2, 8)] == [4, 32, 120, 784, 4144, 28768]


def test_count_table_overflow_detected(oracle):
    with pytest.raises(OverflowError):
        oracle.count_table(22, 6)


@pytest.mark.parametrize("k,size", [(1, 5), (2, 6), (3, 5)])
def test_unrank_is_a_bijection(oracle, k, size):
    t = oracle.count_table(size, k)
    n = int(t[size][8])
    seen = {oracle.unrank(r, size, t) for r in range(n)}
    assert len(seen) == n
    for p in seen:  # every string is a well-formed tree of `size` nodes
        depth = 0
        for c in p:
            if c in "~#":
                assert depth >= 1
            elif c in OPS:
                depth -= 1
            else:
                depth += 1
        assert depth == 1


def test_unrank_block_structure(oracle):
    """Ranks are op-major in the order ~ & | ^ neg + - *; commutative splits
    have left size <= right size (simba/src/nocache.cu:53-79, 137-144)."""
    k, s = 2, 6
    t = oracle.count_table(s, k)
    off = 0
    for op in range(8):
        n = int(t[s][op])
        for r in (off, off + n - 1):
            assert oracle.unrank(r, s, t)[-1] == OPS[op]
        off += n


def test_golden_formulas_evaluate(oracle, golden):
    for d in golden["instances"]:
        inst = Instance.from_json(d)
        p = infix_to_postfix(d["original_formula"])
        assert postfix_to_infix(p) == d["original_formula"]
        assert oracle.check(p, inst.inputs, inst.outputs, 32)
        ev = eval_postfix(p, inst.inputs.astype(np.uint32), 32).astype(np.uint64)
        assert (ev == inst.outputs).all()


def test_oracle_matches_reference_simba(oracle, golden):
    """Same size and same root-operator block as the reference executable;
    identical string whenever the reference's block has a single match."""
    same_string = 0
    for r in golden["results"]["simba"]:
        d = golden["instances"][r["idx"]]
        inst = Instance.from_json(d)
        o = oracle.search(inst.inputs, inst.outputs, r["max_len"], 32)
        if r["expr"] == "Not found !":
            assert not o["found"]
            continue
        p = infix_to_postfix(r["expr"])
        assert oracle.check(p, inst.inputs, inst.outputs, 32)
        assert o["found"] and len(p) == o["size"]
        assert OPS.index(p[-1]) == o["op"]
        if p == o["postfix"]:
            same_string += 1
        else:
            # a multi-match block: the reference returns a racy winner, the
            # oracle the minimum rank; both must be matches of that block
            t = oracle.count_table(o["size"], inst.num_variables)
            lo = int(sum(int(x) for x in t[o["size"]][: o["op"]]))
            hi = lo + int(t[o["size"]][o["op"]])
            e, mr, nh = oracle.scan_range(inst.inputs, inst.outputs, o["size"], lo, hi, 32)
            assert mr == o["rank"]
    assert same_string >= 100


def test_oracle_matches_reference_vfb(oracle, golden):
    """The reference VFB (with its uniqueness test as written) is emulated
    exactly: found / not found and size agree on every golden instance."""
    for r in golden["results"]["vfb"]:
        d = golden["instances"][r["idx"]]
        inst = Instance.from_json(d)
        o = oracle.vfb(inst.inputs, inst.outputs, r["max_len"], 32, ref_inverted=True)
        if r["expr"] in ("Not found !", ""):
            assert not o["found"]
            continue
        p = infix_to_postfix(r["expr"])
        assert oracle.check(p, inst.inputs, inst.outputs, 32)
        assert o["found"] and o["size"] == len(p)


def test_vfb_correct_dedup_is_minimal(oracle):
    """With the documented dedup (keep first occurrence) VFB finds the same
    minimal size as the exhaustive plain search."""
    for seed in range(6):
        inst = make_instance(7, 2, 16, seed, word_bits=64)
        v = oracle.vfb(inst.inputs, inst.outputs, 8, 64)
        s = oracle.search(inst.inputs, inst.outputs, 9, 64, include_edges=True)
        assert v["found"] == s["found"]
        if s["found"]:
            assert v["size"] == s["size"]
            assert oracle.check(v["postfix"], inst.inputs, inst.outputs, 64)


def test_reference_vfb_inverted_dedup_differs():
    """Documented finding: the reference's `insert(...) > 0` keeps repeated
    vectors; on the size-9 two-variable instance it answers one size later."""
    from oracle import oracle as O
    inst = make_instance(9, 2, 32, 0, word_bits=64)
    a = O.vfb(inst.inputs, inst.outputs, 12, 64, ref_inverted=False)
    b = O.vfb(inst.inputs, inst.outputs, 12, 64, ref_inverted=True)
    assert a["size"] == 5 and b["size"] == 6


def test_fingerprint32_properties(oracle):
    v = np.arange(16, dtype=np.uint32)
    f = oracle.fingerprint32(v)
    assert f == oracle.fingerprint32(v.copy())
    v2 = v.copy()
    v2[3] ^= 1
    assert f != oracle.fingerprint32(v2)


def test_u64_wraparound(oracle):
    row = np.array([2 ** 63 + 5, 2 ** 64 - 1], dtype=np.uint64)
    assert oracle.eval1("01+", row, 64) == (2 ** 63 + 5 + 2 ** 64 - 1) % 2 ** 64
    assert oracle.eval1("01*", row, 64) == ((2 ** 63 + 5) * (2 ** 64 - 1)) % 2 ** 64
    assert oracle.eval1("0#", row, 64) == (2 ** 64 - (2 ** 63 + 5)) % 2 ** 64
    assert oracle.eval1("01*", row, 32) == ((5) * (2 ** 32 - 1)) % 2 ** 32


def test_scan_range_counts(oracle):
    inst = make_instance(9, 2, 32, 3, word_bits=64, unsat=True)
    e, mr, nh = oracle.scan_range(inst.inputs, inst.outputs, 6, 0, 5000, 64)
    assert e == 5000 and nh == 0 and mr == 2 ** 64 - 1


def _rtid_brute(oracle, inst, size, op, bits, reference_map):
    """Smallest thread position t of block (size, op) whose rank matches."""
    t = oracle.count_table(size, inst.num_variables)
    off = int(sum(int(x) for x in t[size][:op]))
    N = int(t[size][op])
    c = oracle.rtid_multiplier(N)
    T = (N + 1023) // 1024 * 1024 if reference_map else N
    for x in range(T):
        r = off + ((x * 2246822507) % (1 << 64)) % N if reference_map else off + (x * c) % N
        if oracle.check(oracle.unrank(r, size, t), inst.inputs, inst.outputs, bits):
            return r
    return None


@pytest.mark.parametrize("reference_map", [False, True])
def test_rtid_order_brute_force(oracle, reference_map):
    """RTid order: the first operator block with a match (the same block as
    the rank order when every rank is visited) and, inside it, the match of
    the smallest thread position, checked by a plain loop."""
    for seed in range(8):
        inst = make_instance(6 + seed % 3, 1 + seed % 3, 16, 700 + seed, word_bits=64)
        a = oracle.search(inst.inputs, inst.outputs, 10, 64)
        b = oracle.search_rtid(inst.inputs, inst.outputs, 10, 64, reference_map=reference_map)
        assert a["found"] == b["found"]
        if not a["found"]:
            continue
        assert (a["size"], a["op"], a["candidates"]) == (b["size"], b["op"], b["candidates"])
        assert oracle.check(b["postfix"], inst.inputs, inst.outputs, 64)
        assert b["rank"] == _rtid_brute(oracle, inst, b["size"], b["op"], 64, reference_map)


def test_rtid_multiplier_is_coprime(oracle):
    import math
    C = 2246822507
    assert oracle.rtid_multiplier(1000) == C
    for n in (15809, 142123 * 7, 15809 * 142123, 2 * 15809 * 3):
        c = oracle.rtid_multiplier(n)
        assert c > C and math.gcd(c, n) == 1
        assert all(math.gcd(x, n) != 1 for x in range(C, c))
    # the reference's map on such a block visits only multiples of the gcd
    n = 15809 * 4
    assert len({(x * C) % n for x in range((n + 1023) // 1024 * 1024)}) == 4


def test_oracle_rtid_matches_reference_rtid(oracle):
    """The reference's simba_rtid executable on the golden instances: same
    size and operator block; the returned expression is a match."""
    import json
    from pathlib import Path
    g = Path(__file__).resolve().parent / "golden"
    f = g / "ref_results_rtid_u32.json"
    if not f.exists():
        pytest.skip("reference RTid results not generated")
    insts = json.loads((g / "ref_instances_u32.json").read_text())
    same = 0
    for r in json.loads(f.read_text())["simba_rtid"]:
        inst = Instance.from_json(insts[r["idx"]])
        o = oracle.search_rtid(inst.inputs, inst.outputs, r["max_len"], 32, reference_map=True)
        if r["expr"] == "Not found !":
            assert not o["found"]
            continue
        p = infix_to_postfix(r["expr"])
        assert oracle.check(p, inst.inputs, inst.outputs, 32)
        assert o["found"] and len(p) == o["size"] and OPS.index(p[-1]) == o["op"]
        same += p == o["postfix"]
    assert same >= 100


def test_oracle_matches_widened_reference_u64(oracle):
    """The reference widened to 64-bit words (oracle/build_ref.sh,
    simba_nocache_u64) on the 64-bit golden instances: its expression
    verifies under the oracle's uint64 arithmetic and lies in the oracle's
    size and operator block (random set, sizes 3-10); for the planted
    bench-shape answers (sizes 11-13, too large for a CPU sweep) the
    reference's expression verifies and has at most the planted size."""
    import json
    from pathlib import Path
    g = Path(__file__).resolve().parent / "golden"
    f = g / "ref_results_u64.json"
    if not f.exists():
        pytest.skip("widened reference results not generated")
    insts = json.loads((g / "ref_instances_u64.json").read_text())
    same = 0
    for r in json.loads(f.read_text())["simba_u64"]:
        d = insts[r["idx"]]
        inst = Instance.from_json(d)
        assert inst.word_bits == 64
        if r["expr"] == "Not found !":
            assert d["set"] == "random"
            o = oracle.search(inst.inputs, inst.outputs, r["max_len"], 64)
            assert not o["found"]
            continue
        p = infix_to_postfix(r["expr"])
        assert oracle.check(p, inst.inputs, inst.outputs, 64)
        if d["set"] == "bench_shape":
            assert len(p) <= d["gen_size"]
            continue
        o = oracle.search(inst.inputs, inst.outputs, r["max_len"], 64)
        assert o["found"] and (len(p), OPS.index(p[-1])) == (o["size"], o["op"])
        same += p == o["postfix"]
    assert same >= 30


def test_ext_grammar_oracle_bijection_and_semantics(oracle):
    """Extended grammar oracle: unranking is a bijection of each size (every
    rank gives a distinct postfix that parses back to a well-formed tree);
    shifts by the word width or more give 0; division and modulo by zero
    give the dividend per sample."""
    t = oracle.ext_count_table(6, 3)
    assert [int(t[s][12]) for s in range(1, 5)] == [3, 6, 102, 474]
    for s in range(2, 6):
        seen = {oracle.ext_unrank(r, s, t) for r in range(int(t[s][12]))}
        assert len(seen) == int(t[s][12])
    ev = oracle.ext_eval1
    assert ev("01<", [5, 3], 64) == 40 and ev("01<", [5, 64], 64) == 0
    assert ev("01<", [5, 31], 32) == (5 << 31) & 0xFFFFFFFF and ev("01<", [5, 32], 32) == 0
    assert ev("01>", [2 ** 63, 63], 64) == 1 and ev("01>", [7, 70], 64) == 0
    assert ev("01/", [7, 0], 64) == 7 and ev("01%", [7, 0], 64) == 7
    assert ev("01/", [7, 2], 64) == 3 and ev("01%", [7, 2], 64) == 1


def test_ext_vfb_oracle_whole_vector_division_rule(oracle):
    """VFB composes whole vectors: a divisor vector with one zero element makes
    v0 / v1 equal to v0 on every sample, so with that target VFB finds v0 at
    size 1 while the target v0 / v1 evaluated per sample differs."""
    import numpy as np
    ins = np.array([[9, 0, 1], [8, 3, 1], [7, 2, 1]], dtype=np.uint64)
    per_sample = np.array([oracle.ext_eval1("01/", r, 64) for r in ins], dtype=np.uint64)
    assert list(per_sample) == [9, 2, 3]
    o = oracle.ext_vfb(ins, per_sample, 4, 64)
    # v0 / v1 as a whole vector is v0 (a zero divisor), so it is not the target
    assert not (o["found"] and o["postfix"] == "01/")
    p = oracle.ext_search(ins, per_sample, 4, 64)
    assert p["found"] and p["size"] == 3 and p["postfix"] == "01/"
