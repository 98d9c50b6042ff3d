"""Experiment harness: the reference's `build_all.sh` + `run_all.sh` loop.

The reference generates formulas of sizes 5-30 over 2-10 variables (10 of
each, seed 42) and samples each on 16 points (build_all.sh:17-20), then runs
every solver on every instance file with a 60 s timeout and max size 20,
appending `file,expr,seconds` lines to a CSV; a run that times out writes no
line (run_all.sh:20-43).

    python -m simba_b200.harness generate --out DIR [--size-range 5 30]
           [--var-range 2 10] [--repeats 10] [--samples 16] [--seed 42] [--bits 32]
    python -m simba_b200.harness run --instances DIR --out res.csv
           [--solver simba|vfb] [--mode cli|batch] [--max-len 20] [--timeout 60]

`--mode cli` runs the drop-in executables one process per instance under a
timeout, exactly like run_all.sh; `--mode batch` solves every instance in
one batched search (simba only; the timeout is then the budget of the whole
batch, not of each instance) and writes the same lines, `seconds` being the
time to solution from the start of the batch.  Instances searched to
max size without a match get a `Not found !` line in both modes, as the
executables print one.

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


def run_cli(files: List[Path], out_csv: Path, solver: str, max_len: int, timeout: float) -> int:
    exe = PKG / "bin" / solver
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
    a = ap.parse_args(argv)
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
        n = run_cli(files, a.out, a.solver, a.max_len, a.timeout)
    print(f"{n}/{len(files)} lines in {a.out} ({time.time() - t0:.1f} s)")
    return 0


if __name__ == "__main__":
    sys.exit(main())
