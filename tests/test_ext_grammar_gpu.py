"""Extended grammar (~ & | ^ << >> neg + - * / %) on the GPU, through the C ABI.

The reference declares these operators and leaves the four new ones switched
off (vfb/src/full-cache.cu:166-179,460-472; simba/src/mba.cuh:71-131 has no
caller), so no reference output exists: parity is against the oracle's
restatement of the declared semantics (oracle.c, extended grammar section).

Plain search: the answer's size, operator block, minimum rank, postfix and
per-size candidate counts equal the oracle's; the expression reproduces the
target per sample.  VFB: found / not found, size, operator and rows per size
equal the oracle's whole-vector search.
"""
import numpy as np
import pytest

import simba_b200 as S
from simba_b200.instances import Instance, SplitMix64

pytestmark = pytest.mark.gpu


def planted(postfix, n_vars, n_samples, seed, bits, oracle, small=False):
    """Instance whose outputs are `postfix` (extended grammar) evaluated on
    seeded samples; `small` draws small words so that shifts and divisions
    by small amounts (and zero divisors) actually occur."""
    rng = SplitMix64(seed)
    mask = (1 << bits) - 1
    ins = np.zeros((n_samples, n_vars + 1), dtype=np.uint64)
    for i in range(n_samples):
        for j in range(n_vars):
            x = rng.next()
            ins[i, j] = (x % 9) if small else (x & mask)
        ins[i, n_vars] = 1
    outs = np.array([oracle.ext_eval1(postfix, ins[i], bits) for i in range(n_samples)],
                    dtype=np.uint64)
    return Instance(n_vars + 1, ins, outs, bits, None, True)


CASES = [("01<", 2, 16, 1, 64, False), ("01>2+", 2, 16, 2, 32, False),
         ("01/", 2, 16, 3, 64, True), ("01%0^", 2, 16, 4, 64, True),
         ("02<1-", 2, 32, 5, 32, False), ("10%2/", 2, 16, 6, 64, True),
         ("01*2>", 2, 16, 7, 64, False)]


@pytest.mark.parametrize("postfix,nv,ns,seed,bits,small", CASES)
def test_ext_plain_search_matches_oracle(oracle, postfix, nv, ns, seed, bits, small):
    inst = planted(postfix, nv, ns, seed, bits, oracle, small)
    r = S.solve(inst, 7, extended=True)
    o = oracle.ext_search(inst.inputs, inst.outputs, 7, bits)
    assert r.found == o["found"]
    assert (r.size, r.op, r.rank, r.postfix) == (o["size"], o["op"], o["rank"], o["postfix"])
    assert r.candidates == o["candidates"]
    assert list(r.per_size[:8]) == list(o["per_size"][:8])
    assert oracle.ext_check(r.postfix, inst.inputs, inst.outputs, bits)


def test_ext_plain_search_unsat_counts(oracle):
    rng = SplitMix64(99)
    ins = np.array([[rng.next(), 1] for _ in range(16)], dtype=np.uint64)
    outs = np.array([rng.next() for _ in range(16)], dtype=np.uint64)
    inst = Instance(2, ins, outs, 64, None, True)
    r = S.solve(inst, 7, extended=True)
    t = oracle.ext_count_table(6, 2)
    assert r.status == S.NOT_FOUND
    assert r.candidates == int(sum(int(t[s][12]) for s in range(2, 7)))
    assert r.evaluated == r.candidates


@pytest.mark.parametrize("postfix,nv,ns,seed,bits,small", CASES)
def test_ext_vfb_matches_oracle(oracle, postfix, nv, ns, seed, bits, small):
    inst = planted(postfix, nv, ns, seed, bits, oracle, small)
    r = S.vfb_solve(inst, 6, extended=True)
    o = oracle.ext_vfb(inst.inputs, inst.outputs, 6, bits)
    assert r.found == o["found"]
    last = r.size if r.found else 6
    for L in range(1, last):
        assert r.rows_per_size[L] == o["rows_per_size"][L], (L, r, o)
    if o["found"]:
        assert r.size == o["size"] and r.op == o["op"]
        assert r.candidates == o["candidates"]


def test_ext_formatting():
    assert S.format_postfix("01<", extended=True) == "(v0 << v1)"
    assert S.format_postfix("01/2%", "vfb", extended=True) == "((v0)/(v1))%(v2)"
