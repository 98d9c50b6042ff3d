"""Generate the 64-bit golden instances (tests/golden/ref_instances_u64.json).

Two sets, both seeded (SplitMix64) and written in the reference's JSON schema
with ``"size": 64`` values:

* ``bench_shape``: the benchmarked shape -- 3 variables + the constant 1
  (4 terminals), 64 uint64 samples -- with a planted answer ``v0 OP R`` of
  size 11, 12 and 13, R a random expression of size - 2.  With the default
  value tables (sizes <= 10 for 4 terminals in 64-bit words), a root of
  ``+ - *`` over an R without ``&`` / ``|`` lies on spines the engine
  matches by its hash join, and a root of ``&`` / ``|`` on spines it matches
  by nested compares.  The rank of ``v0 OP R`` inside its operator block
  is the rank of R (left operand size 1, variable 0, comes first), which
  keeps the oracle's scan of the block up to the answer within seconds.
* ``random``: targets of the reference generator's distribution, sizes
  3..10, 1..4 variables + 1, 16/32/64 samples.

The answers of the reference's own executable widened to 64-bit words
(``oracle/_ref/simba_nocache_u64``, built by oracle/build_ref.sh) on these
instances are recorded by ``run_reference.py <out> --u64`` on a GPU host
(tests/golden/ref_results_u64.json).

Usage: python tests/golden/make_golden_u64.py
"""
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import numpy as np  # noqa: E402

from simba_b200.instances import (OP_CHARS, SplitMix64, eval_postfix,  # noqa: E402
                                  make_instance, planted_instance)

BENCH_CASES = [(11, "+", True), (11, "&", False), (12, "*", True), (12, "|", False),
               (13, "-", True), (13, "&", False)]


def subtrees(postfix: str):
    """(start, end) of every subtree of a postfix string."""
    st, out = [], []
    for i, c in enumerate(postfix):
        if c not in OP_CHARS:
            st.append(i)
        elif c in "~#":
            pass
        else:
            st.pop()
        out.append((st[-1], i + 1))
    return out


def degenerate(postfix: str, inputs: np.ndarray) -> bool:
    """True when a subtree collapses on the samples: it is constant, or the
    CPU oracle finds an expression of a smaller size (up to 10) with the
    same values, so the planted expression has a shorter equivalent."""
    from oracle import oracle as O
    for a, b in sorted(subtrees(postfix), key=lambda ab: ab[1] - ab[0]):
        if b - a < 2:
            continue
        v = eval_postfix(postfix[a:b], inputs, 64)
        if len(set(v.tolist())) == 1:
            return True
        if O.search(inputs, v, min(b - a - 1, 10), 64, include_edges=True)["found"]:
            return True
    return False


def binary_tree(size: int, rng: SplitMix64, binary) -> str:
    """Random expression of ``size`` nodes over 4 terminals, binary
    operators only except one unary operator when ``size`` is even (random
    trees with many unary nodes mostly collapse to smaller ones)."""
    if size == 1:
        return chr(ord("0") + rng.below(4))
    if size == 2 or (size % 2 == 0 and rng.below(3) == 0):
        return binary_tree(size - 1, rng, binary) + "~#"[rng.below(2)]
    left = 1 + 2 * rng.below((size - 1) // 2)  # odd left size
    if size % 2 == 0 and rng.below(2):
        left = size - 1 - left  # the even side (with the unary node) on the left
    return (binary_tree(left, rng, binary) + binary_tree(size - 1 - left, rng, binary)
            + binary[rng.below(len(binary))])


def bench_shape():
    """Planted answers; seeds whose expression collapses (checked on its
    subtrees by the oracle) are skipped, so the answers keep their planted
    size unless an equivalent of size 11-12 exists."""
    out = []
    for i, (size, root, join) in enumerate(BENCH_CASES):
        binary = ("-", "+", "*", "^") if join else ("-", "+", "*", "&", "|", "^")
        seed = 7000 + 100 * i
        while True:
            rng = SplitMix64(seed ^ 0x5EED)
            r = binary_tree(size - 2, rng, binary)
            inst = planted_instance("0" + r + root, 3, 64, seed, word_bits=64)
            if not degenerate(inst.formula, inst.inputs):
                break
            seed += 1
            if seed > 7000 + 100 * i + 60:
                raise RuntimeError("no planted expression without a shorter equivalent")
        d = inst.to_json()
        d.update({"set": "bench_shape", "gen_size": size, "max_len": size + 1,
                  "join": join})
        out.append(d)
    return out


def random_set():
    out = []
    for i in range(40):
        size = 3 + i % 8
        nv = 1 + i % 4
        ns = (16, 32, 64)[i % 3]
        inst = make_instance(size, nv, ns, 8000 + i, word_bits=64)
        d = inst.to_json()
        d.update({"set": "random", "gen_size": size, "max_len": size + 1})
        out.append(d)
    return out


def main():
    insts = bench_shape() + random_set()
    (HERE / "ref_instances_u64.json").write_text(json.dumps(insts))
    print(f"wrote {len(insts)} instances")


if __name__ == "__main__":
    main()
