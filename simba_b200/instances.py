"""MBA learning instances: the reference's JSON schema, plus a seeded generator.

Schema (read by the reference at simba/src/instance.cpp:7-27 and
vfb/src/utils.h:15-44)::

    {"num_variables": k, "num_examples": S,
     "examples": [{"inputs": [{"value": u, "size": 32}, ...k],
                   "output": [{"value": u, "size": 32}]}, ...S]}

Inputs are stored sample-major (``inputs[i * k + j]`` is variable ``j`` on
sample ``i``), exactly as the reference lays them out.  ``"size"`` is 32 for
the reference's uint32 words; this package also accepts 64, which selects
exact uint64 arithmetic.

The constant terminal ``1`` is represented the way the reference can run it
unchanged: as one extra variable whose value is 1 on every sample
(``const_one=True`` appends it as the last variable).

The random-formula distribution follows the reference generator
(scripts/generate.py:21-49): size 1 is a uniform terminal; size 2 is a
uniform unary op; size >= 3 draws uniformly among 2 unary and 6 binary ops,
and a binary node's left size is uniform in [1, size - 2].  Random numbers
come from SplitMix64 (Steele, Lea, Flood 2014) so that C and Python agree.
"""
from __future__ import annotations

import json
from dataclasses import dataclass, field
from pathlib import Path
from typing import Iterable, List, Optional, Sequence

import numpy as np

M64 = (1 << 64) - 1

# Operator order of the rank space (simba/src/globals.cuh:13-15):
# index 0..7 = '~' '&' '|' '^' '#'(unary minus) '+' '-' '*'
OP_CHARS = "~&|^#+-*"
UNARY = {"~", "#"}
BINARY = {"&", "|", "^", "+", "-", "*"}


class SplitMix64:
    """SplitMix64 generator (public-domain algorithm by Steele, Lea and Flood)."""

    def __init__(self, seed: int) -> None:
        self.state = seed & M64

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & M64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        return z ^ (z >> 31)

    def below(self, n: int) -> int:
        """Uniform integer in [0, n) by rejection (no modulo bias)."""
        if n <= 0:
            raise ValueError("n must be positive")
        limit = (1 << 64) - ((1 << 64) % n)
        while True:
            x = self.next()
            if x < limit:
                return x % n


def random_postfix(size: int, n_terms: int, rng: SplitMix64,
                   binary: Sequence[str] = ("-", "+", "*", "&", "|", "^")) -> str:
    """Random expression of exactly ``size`` nodes, as a postfix string.

    Terminals are written ``'0' + t`` and operators with the reference's
    characters, which is the encoding of ``numberToFormula``
    (simba/src/nocache.cu:44-45,60).  ``binary`` restricts the binary
    operators drawn (default: all six, the generator's distribution).
    """
    if size < 1:
        raise ValueError("size must be >= 1")
    if size == 1:
        return chr(ord("0") + rng.below(n_terms))
    unary = ["#", "~"]
    allowed = unary + (list(binary) if size >= 3 else [])
    op = allowed[rng.below(len(allowed))]
    if op in UNARY:
        return random_postfix(size - 1, n_terms, rng, binary) + op
    left = 1 + rng.below(size - 2)
    right = size - 1 - left
    return (random_postfix(left, n_terms, rng, binary)
            + random_postfix(right, n_terms, rng, binary) + op)


def eval_postfix(postfix: str, inputs: np.ndarray, word_bits: int) -> np.ndarray:
    """Evaluate a postfix expression on every sample at once (numpy).

    ``inputs`` has shape (S, k); arithmetic wraps modulo 2**word_bits.
    """
    dt = np.uint64 if word_bits == 64 else np.uint32
    x = np.asarray(inputs, dtype=dt)
    stack: List[np.ndarray] = []
    with np.errstate(over="ignore"):
        for c in postfix:
            if c not in OP_CHARS:
                stack.append(x[:, ord(c) - ord("0")].copy())
            elif c == "~":
                stack[-1] = ~stack[-1]
            elif c == "#":
                stack[-1] = (dt(0) - stack[-1]).astype(dt)
            else:
                r = stack.pop()
                l = stack.pop()
                if c == "&":
                    stack.append(l & r)
                elif c == "|":
                    stack.append(l | r)
                elif c == "^":
                    stack.append(l ^ r)
                elif c == "+":
                    stack.append((l + r).astype(dt))
                elif c == "-":
                    stack.append((l - r).astype(dt))
                elif c == "*":
                    stack.append((l * r).astype(dt))
                else:
                    raise ValueError(f"bad token {c!r}")
    if len(stack) != 1:
        raise ValueError("malformed postfix")
    return stack[0]


def postfix_to_infix(postfix: str, style: str = "simba",
                     names: Optional[Sequence[str]] = None) -> str:
    """Render a postfix string in the reference's output syntax.

    ``style="simba"`` follows MBAToString (simba/src/nocache.cu:162-195):
    ``v3``, ``(~v0)``, ``(-v0)``, ``(L op R)``.  ``style="vfb"`` follows the
    VFB printer (vfb/src/full-cache.cu:483-509): ``~(x)``, ``-(x)``,
    ``(L)op(R)``.
    """
    st: List[str] = []
    for c in postfix:
        if c in OP_CHARS:
            if c in UNARY:
                a = st.pop()
                sym = "-" if c == "#" else "~"
                st.append(f"({sym}{a})" if style == "simba" else f"{sym}({a})")
            else:
                r = st.pop()
                l = st.pop()
                st.append(f"({l} {c} {r})" if style == "simba" else f"({l}){c}({r})")
        else:
            t = ord(c) - ord("0")
            st.append(names[t] if names else f"v{t}")
    if len(st) != 1:
        raise ValueError("malformed postfix")
    return st[0]


def infix_to_postfix(expr: str) -> str:
    """Parse an expression printed by the reference tools back to postfix.

    Accepts the SIMBA printer's syntax ``(v0 + (~v1))`` / ``(-v0)``
    (simba/src/nocache.cu:162-195, also what scripts/generate.py:38-49
    writes) and the VFB printer's ``(v0)+(~(v1))`` / ``-(v0)``
    (vfb/src/full-cache.cu:483-509).  Variables ``vN`` become ``chr(48+N)``.
    """
    s = expr.replace(" ", "")
    pos = 0

    def peek() -> str:
        return s[pos] if pos < len(s) else ""

    def take(c: str) -> None:
        nonlocal pos
        if peek() != c:
            raise ValueError(f"expected {c!r} at {pos} in {expr!r}")
        pos += 1

    def term() -> str:
        nonlocal pos
        c = peek()
        if c == "v":
            pos += 1
            j = pos
            while pos < len(s) and s[pos].isdigit():
                pos += 1
            return chr(ord("0") + int(s[j:pos]))
        if c in ("~", "-"):
            pos += 1
            return term() + ("~" if c == "~" else "#")
        if c == "(":
            pos += 1
            e = full()
            take(")")
            return e
        raise ValueError(f"unexpected {c!r} at {pos} in {expr!r}")

    def full() -> str:
        nonlocal pos
        left = term()
        c = peek()
        if c in BINARY:
            pos += 1
            right = term()
            return left + right + c
        return left

    out = full()
    if pos != len(s):
        raise ValueError(f"trailing input at {pos} in {expr!r}")
    return out


@dataclass
class Instance:
    """One MBA learning instance (sample-major inputs, one output per sample)."""

    num_variables: int
    inputs: np.ndarray          # shape (S, k), uint64 container
    outputs: np.ndarray         # shape (S,),   uint64 container
    word_bits: int = 64
    formula: Optional[str] = None   # postfix of the generating expression
    const_one: bool = False         # last variable is the constant 1
    meta: dict = field(default_factory=dict)
    unit_log2: int = 0              # batch work-unit size (set by the autotuner)

    @property
    def num_examples(self) -> int:
        return int(self.outputs.shape[0])

    def to_json(self) -> dict:
        size = self.word_bits
        d = {
            "num_variables": int(self.num_variables),
            "num_examples": int(self.num_examples),
            "examples": [
                {"inputs": [{"value": int(v), "size": size} for v in row],
                 "output": [{"value": int(o), "size": size}]}
                for row, o in zip(self.inputs.tolist(), self.outputs.tolist())
            ],
        }
        if self.formula is not None:
            d["original_formula"] = postfix_to_infix(self.formula)
            d["original_postfix"] = self.formula
        if self.const_one:
            d["const_one"] = True
        return d

    def write(self, path: Path | str) -> None:
        Path(path).write_text(json.dumps(self.to_json()))

    @staticmethod
    def from_json(d: dict) -> "Instance":
        k = int(d["num_variables"])
        exs = d["examples"]
        s = int(d.get("num_examples", len(exs)))
        bits = 32
        for ex in exs[:1]:
            for v in ex["inputs"] + ex["output"]:
                if int(v.get("size", 32)) == 64:
                    bits = 64
        ins = np.zeros((s, k), dtype=np.uint64)
        outs = np.zeros((s,), dtype=np.uint64)
        mask = M64 if bits == 64 else 0xFFFFFFFF
        for i, ex in enumerate(exs[:s]):
            outs[i] = int(ex["output"][0]["value"]) & mask
            for j, v in enumerate(ex["inputs"][:k]):
                ins[i, j] = int(v["value"]) & mask
        return Instance(k, ins, outs, bits, d.get("original_postfix"),
                        bool(d.get("const_one", False)))

    @staticmethod
    def read(path: Path | str) -> "Instance":
        return Instance.from_json(json.loads(Path(path).read_text()))


def make_instance(size: int, n_vars: int, n_samples: int, seed: int,
                  word_bits: int = 64, const_one: bool = True,
                  unsat: bool = False) -> Instance:
    """Seeded synthetic instance: a random target of ``size`` nodes.

    The target is drawn over ``n_vars`` variables (+ the constant 1 when
    ``const_one``), sampled on ``n_samples`` uniform random words.  With
    ``unsat=True`` the outputs are replaced by independent random words, so
    (with overwhelming probability) no small expression matches and a search
    sweeps every size completely.
    """
    rng = SplitMix64(seed)
    n_terms = n_vars + (1 if const_one else 0)
    formula = random_postfix(size, n_terms, rng)
    mask = M64 if word_bits == 64 else 0xFFFFFFFF
    ins = np.zeros((n_samples, n_terms), dtype=np.uint64)
    for i in range(n_samples):
        for j in range(n_vars):
            ins[i, j] = rng.next() & mask
        if const_one:
            ins[i, n_vars] = 1
    outs = eval_postfix(formula, ins if word_bits == 64 else ins.astype(np.uint32),
                        word_bits).astype(np.uint64)
    if unsat:
        outs = np.array([rng.next() & mask for _ in range(n_samples)], dtype=np.uint64)
    return Instance(n_terms, ins, outs, word_bits, None if unsat else formula,
                    const_one, {"size": size, "seed": seed, "unsat": unsat})


def planted_instance(postfix: str, n_vars: int, n_samples: int, seed: int,
                     word_bits: int = 64, const_one: bool = True) -> Instance:
    """Instance whose outputs are the given expression evaluated on seeded
    uniform random samples (SplitMix64(seed)), ``n_vars`` variables plus the
    constant 1 when ``const_one``.  The expression is the planted answer: a
    search finds it or an equivalent expression of at most its size."""
    rng = SplitMix64(seed)
    n_terms = n_vars + (1 if const_one else 0)
    mask = M64 if word_bits == 64 else 0xFFFFFFFF
    ins = np.zeros((n_samples, n_terms), dtype=np.uint64)
    for i in range(n_samples):
        for j in range(n_vars):
            ins[i, j] = rng.next() & mask
        if const_one:
            ins[i, n_vars] = 1
    outs = eval_postfix(postfix, ins if word_bits == 64 else ins.astype(np.uint32),
                        word_bits).astype(np.uint64)
    return Instance(n_terms, ins, outs, word_bits, postfix, const_one,
                    {"size": len(postfix), "seed": seed, "planted": True})


def iter_batch(n: int, seed0: int, sizes: Sequence[int], vars_: Sequence[int],
               samples: Sequence[int], word_bits: int = 64,
               const_one: bool = True) -> Iterable[Instance]:
    """Instances ``seed0 .. seed0+n-1`` with size / vars / samples drawn
    uniformly from the given choices (the batched configurations)."""
    for i in range(n):
        r = SplitMix64(0xB47C4 ^ (seed0 + i))
        size = sizes[r.below(len(sizes))]
        nv = vars_[r.below(len(vars_))]
        ns = samples[r.below(len(samples))]
        yield make_instance(size, nv, ns, seed0 + i, word_bits, const_one)
