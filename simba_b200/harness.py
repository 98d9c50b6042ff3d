"""Experiment harness: the reference's `build_all.sh` + `run_all.sh` loop.

The reference generates formulas of sizes 5-30 over 2-10 variables (10 of
each, seed 42) and samples each on 16 points (build_all.sh:17-20), then runs
every solver on every instance file with a 60 s timeout and max size 20,
appending `file,expr,seconds` lines to a CSV; a run that times out writes no
line (run_all.sh:20-43).

    python -m simba_b200.harness generate --out DIR [--size-range 5 30]
           [--var-range 2 10] [--repeats 10] [--samples 16] [--seed 42] [--bits 32]
    python -m simba_b200.harness run --instances DIR --out res.csv
           [--solver simba|vfb] [--exe PATH] [--mode cli|batch] [--max-len 20] [--timeout 60]
    python -m simba_b200.harness compare --ours a.csv --ref b.csv --instances DIR

`--mode cli` runs the drop-in executables one process per instance under a
timeout, exactly like run_all.sh; `--mode batch` solves every instance in
one batched search (simba only; the timeout is then the budget of the whole
batch, not of each instance) and writes the same lines, `seconds` being the
time to solution from the start of the batch.  Instances searched to
max size without a match get a `Not found !` line in both modes, as the
executables print one.

`--exe` runs another executable with the same command line (the reference's
own `simba` build, for a line-by-line comparison); `compare` reads two such
CSVs and reports, over the instances both solved, whether they agree on
found / not found and on the expression size, and checks every expression
of `--ours` against its instance.

Instances come from the formula distribution of the reference's
scripts/generate.py (random_postfix) over `--var-range` variables, sampled
on uniform random words of `--bits` bits; `num_variables` is the requested
count, not the highest variable the formula happens to use.
"""
from __future__ import annotations

import argparse
import subprocess
import sys
import time
from pathlib import Path
from typing import List

from .instances import Instance, make_instance

PKG = Path(__file__).resolve().parent


def generate(out: Path, size_range=(5, 30), var_range=(2, 10), repeats=10, samples=16,
             seed=42, bits=32) -> List[Path]:
    """Instance files in the reference's schema, sizes x variables x repeats."""
    out.mkdir(parents=True, exist_ok=True)
    paths = []
    i = 0
    for size in range(size_range[0], size_range[1] + 1):
        for nv in range(var_range[0], var_range[1] + 1):
            for _ in range(repeats):
                inst = make_instance(size, nv, samples, seed * 1_000_003 + i, word_bits=bits,
                                     const_one=False)
                p = out / f"mba_{i}_seed={seed}.json"
                inst.write(p)
                paths.append(p)
                i += 1
    return paths


def run_cli(files: List[Path], out_csv: Path, solver: str, max_len: int, timeout: float,
            exe: Path = None) -> int:
    exe = exe or PKG / "bin" / solver
    n = 0
    with out_csv.open("w") as f:
        f.write("instance,formula,time\n")
        for p in files:
            try:
                r = subprocess.run([str(exe), str(p), str(max_len)], capture_output=True,
                                   text=True, timeout=timeout)
            except subprocess.TimeoutExpired:
                continue  # like `timeout 60 ... || true`: no line
            if r.stdout.strip():
                f.write(r.stdout.strip().splitlines()[-1] + "\n")
                n += 1
    return n


def run_batch(files: List[Path], out_csv: Path, max_len: int, timeout: float) -> int:
    import simba_b200 as S
    insts = [Instance.read(p) for p in files]
    groups = {}
    for i, inst in enumerate(insts):  # one batch per word width
        groups.setdefault(inst.word_bits, []).append(i)
    rows = {}
    for bits, idx in groups.items():
        res, _ = S.solve_batch([insts[i] for i in idx], max_len, budget=timeout)
        for i, r in zip(idx, res):
            if r.status in (S.OK, S.NOT_FOUND):
                rows[i] = f"{files[i]},{r.expr},{r.seconds}"
    with out_csv.open("w") as f:
        f.write("instance,formula,time\n")
        for i in sorted(rows):
            f.write(rows[i] + "\n")
    return len(rows)


def read_csv(path: Path) -> dict:
    """instance file -> (expression, seconds) of a run CSV."""
    rows = {}
    for line in path.read_text().splitlines()[1:]:
        if line.count(",") < 2:
            continue
        f, e, t = line.rsplit(",", 2)
        rows[f] = (e, float(t))
    return rows


def compare(ours: Path, ref: Path, word_bits: int = 32) -> dict:
    """Line-by-line comparison of two run CSVs over the instances in both."""
    from .instances import infix_to_postfix, eval_postfix
    import numpy as np
    a, b = read_csv(ours), read_csv(ref)
    common = sorted(set(a) & set(b))
    agree_found = agree_size = verified = 0
    diff = []
    for f in common:
        ea, eb = a[f][0], b[f][0]
        fa, fb = ea != "Not found !", eb != "Not found !"
        agree_found += fa == fb
        if fa and fb:
            pa, pb = infix_to_postfix(ea), infix_to_postfix(eb)
            agree_size += len(pa) == len(pb)
            if len(pa) != len(pb):
                diff.append({"instance": f, "ours": ea, "ref": eb})
        if fa:
            inst = Instance.read(f)
            dt = np.uint64 if inst.word_bits == 64 else np.uint32
            got = eval_postfix(infix_to_postfix(ea), inst.inputs.astype(dt), inst.word_bits)
            verified += bool((got.astype(np.uint64) == inst.outputs).all())
    both_found = sum(1 for f in common if a[f][0] != "Not found !" and b[f][0] != "Not found !")
    ta = sorted(a[f][1] for f in common)
    tb = sorted(b[f][1] for f in common)
    med = lambda xs: xs[len(xs) // 2] if xs else None
    return {"ours_lines": len(a), "ref_lines": len(b), "common": len(common),
            "agree_found": agree_found, "both_found": both_found, "agree_size": agree_size,
            "ours_found_verified": verified,
            "ours_found": sum(1 for f in common if a[f][0] != "Not found !"),
            "only_ours": len(set(a) - set(b)), "only_ref": len(set(b) - set(a)),
            "median_seconds_common": {"ours": med(ta), "ref": med(tb)},
            "size_mismatches": diff[:20]}


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m simba_b200.harness")
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("generate")
    g.add_argument("--out", type=Path, required=True)
    g.add_argument("--size-range", type=int, nargs=2, default=(5, 30))
    g.add_argument("--var-range", type=int, nargs=2, default=(2, 10))
    g.add_argument("--repeats", type=int, default=10)
    g.add_argument("--samples", type=int, default=16)
    g.add_argument("--seed", type=int, default=42)
    g.add_argument("--bits", type=int, default=32, choices=(32, 64))
    r = sub.add_parser("run")
    r.add_argument("--instances", type=Path, required=True)
    r.add_argument("--out", type=Path, required=True)
    r.add_argument("--solver", default="simba", choices=("simba", "vfb"))
    r.add_argument("--mode", default="cli", choices=("cli", "batch"))
    r.add_argument("--max-len", type=int, default=20)
    r.add_argument("--timeout", type=float, default=60.0)
    r.add_argument("--exe", type=Path, default=None,
                   help="another executable with the same command line (e.g. the reference's)")
    c = sub.add_parser("compare")
    c.add_argument("--ours", type=Path, required=True)
    c.add_argument("--ref", type=Path, required=True)
    a = ap.parse_args(argv)
    if a.cmd == "compare":
        import json
        print(json.dumps(compare(a.ours, a.ref), indent=1))
        return 0
    if a.cmd == "generate":
        ps = generate(a.out, tuple(a.size_range), tuple(a.var_range), a.repeats, a.samples,
                      a.seed, a.bits)
        print(f"wrote {len(ps)} instances to {a.out}")
        return 0
    files = sorted(a.instances.glob("*.json"))
    t0 = time.time()
    if a.mode == "batch":
        if a.solver != "simba":
            ap.error("--mode batch supports the simba solver only")
        n = run_batch(files, a.out, a.max_len, a.timeout)
    else:
        n = run_cli(files, a.out, a.solver, a.max_len, a.timeout, a.exe)
    print(f"{n}/{len(files)} lines in {a.out} ({time.time() - t0:.1f} s)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
