"""Instance exporters for cross-tool comparison.

* Xyntia trace JSON, as the reference's scripts/convert_to_xyntia.py writes
  it (:7-69): the first example is the "initial" trace and the rest are
  numbered "sampling" traces; input i sits at location "mem<i>", output j at
  EAX, EBX, ECX, EDX (then "out<j>"); sizes and values are Python hex
  strings, values masked to their size.
* SyGuS-IF v2 text for the problem the reference's cvc5/main.py builds
  through the cvc5 API (:16-78): one bit-vector sort of the instance's word
  width, the grammar {and, or, xor, not, add, sub, mul, neg} over the
  variables, and one constraint per example.  Any SyGuS solver reads it
  (`cvc5 --lang=sygus2 file.sl`); cvc5 itself is not part of this package.

    python -m simba_b200.export xyntia IN OUT   # file -> file, or folder -> folder
    python -m simba_b200.export sygus  IN OUT
"""
from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

_REGS = ["EAX", "EBX", "ECX", "EDX"]


def _pair(inputs, outputs) -> dict:
    res = {"inputs": {}, "outputs": {}}
    for i, v in enumerate(inputs):
        bits = int(v["size"])
        res["inputs"][str(i)] = {"location": f"mem{i}", "size": hex(bits),
                                 "value": hex(int(v["value"]) & ((1 << bits) - 1))}
    for j, v in enumerate(outputs):
        bits = int(v["size"])
        res["outputs"][str(j)] = {"location": _REGS[j] if j < len(_REGS) else f"out{j}",
                                  "size": hex(bits),
                                  "value": hex(int(v["value"]) & ((1 << bits) - 1))}
    return res


def to_xyntia(inst: dict) -> dict:
    """Instance JSON (reference schema) -> Xyntia trace JSON."""
    ex = inst.get("examples") or []
    if not ex:
        raise ValueError("no examples in the instance")
    return {"initial": _pair(ex[0]["inputs"], ex[0]["output"]),
            "sampling": {str(i): _pair(e["inputs"], e["output"]) for i, e in enumerate(ex[1:])}}


def _bv(value: int, bits: int) -> str:
    value &= (1 << bits) - 1
    return "#x" + format(value, "0%dx" % (bits // 4)) if bits % 4 == 0 else \
        "#b" + format(value, "0%db" % bits)


def to_sygus(inst: dict) -> str:
    """Instance JSON (reference schema) -> SyGuS-IF v2 problem text."""
    k = int(inst["num_variables"])
    ex = inst["examples"][: int(inst.get("num_examples", len(inst["examples"])))]
    bits = 32
    for e in ex[:1]:
        for v in e["inputs"] + e["output"]:
            bits = int(v.get("size", bits))
    sort = f"(_ BitVec {bits})"
    vars_ = [f"v{i}" for i in range(k)]
    rules = ["(bvand Start Start)", "(bvor Start Start)", "(bvxor Start Start)", "(bvnot Start)",
             "(bvadd Start Start)", "(bvsub Start Start)", "(bvmul Start Start)", "(bvneg Start)"]
    out = ["(set-logic BV)",
           "(synth-fun f (" + " ".join(f"({v} {sort})" for v in vars_) + f") {sort}",
           f"  ((Start {sort}))",
           f"  ((Start {sort} (" + " ".join(rules + vars_) + "))))"]
    for e in ex:
        args = " ".join(_bv(int(v["value"]), bits) for v in e["inputs"][:k])
        out.append(f"(constraint (= (f {args}) {_bv(int(e['output'][0]['value']), bits)}))")
    out.append("(check-synth)")
    return "\n".join(out) + "\n"


def _convert(kind: str, src: Path, dst: Path) -> int:
    def one(a: Path, b: Path) -> None:
        d = json.loads(a.read_text())
        if kind == "xyntia":
            b.write_text(json.dumps(to_xyntia(d), indent=4))
        else:
            b.write_text(to_sygus(d))
    if src.is_dir():
        dst.mkdir(parents=True, exist_ok=True)
        files = sorted(src.glob("*.json"))
        for f in files:
            one(f, dst / (f.name if kind == "xyntia" else f.stem + ".sl"))
        return len(files)
    one(src, dst)
    return 1


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m simba_b200.export")
    ap.add_argument("format", choices=("xyntia", "sygus"))
    ap.add_argument("input", type=Path, help="instance JSON file or folder")
    ap.add_argument("output", type=Path, help="destination file or folder")
    a = ap.parse_args(argv)
    n = _convert(a.format, a.input, a.output)
    print(f"converted {n} instance(s) to {a.format} in {a.output}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
