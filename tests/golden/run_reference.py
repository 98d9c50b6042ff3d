"""Run the reference binaries (built by oracle/build_ref.sh) on golden instances.

Needs a GPU: the reference is CUDA-only.  For every instance in
``ref_instances_u32.json`` it runs the reference SIMBA executable
(``oracle/_ref/simba_nocache <file> <maxLen>``, simba/src/nocache.cu:291-342)
and the reference VFB executable (``oracle/_ref/vfb_full_cache``,
vfb/src/full-cache.cu:776-854) and records the CSV line each one prints.
It also times unsatisfiable sweeps, which give the reference's
candidate-evals/s.  Output: one JSON file (path = first argument) that is
committed as ``tests/golden/ref_results_u32.json``; with ``--rtid`` after
the path, the reference's RTid build alone (``oracle/_ref/simba_rtid``),
committed as ``tests/golden/ref_results_rtid_u32.json``; with ``--u64``, the
reference widened to 64-bit words (``oracle/_ref/simba_nocache_u64``) on
``ref_instances_u64.json``, committed as ``tests/golden/ref_results_u64.json``.
"""
import json
import subprocess
import sys
import tempfile
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from simba_b200.instances import make_instance  # noqa: E402

SIMBA = ROOT / "oracle" / "_ref" / "simba_nocache"
SIMBA_RTID = ROOT / "oracle" / "_ref" / "simba_rtid"
SIMBA_U64 = ROOT / "oracle" / "_ref" / "simba_nocache_u64"
VFB = ROOT / "oracle" / "_ref" / "vfb_full_cache"


def run(exe: Path, path: Path, max_len: int, timeout: float) -> dict:
    t0 = time.perf_counter()
    try:
        p = subprocess.run([str(exe), str(path), str(max_len)], capture_output=True,
                           text=True, timeout=timeout)
        wall = time.perf_counter() - t0
        line = p.stdout.strip().splitlines()[-1] if p.stdout.strip() else ""
        parts = line.rsplit(",", 1)
        expr = parts[0].split(",", 1)[1] if "," in parts[0] else ""
        secs = float(parts[1]) if len(parts) == 2 else None
        return {"rc": p.returncode, "line": line, "expr": expr, "seconds": secs,
                "wall": wall, "stderr_tail": p.stderr[-400:]}
    except subprocess.TimeoutExpired:
        return {"rc": None, "timeout": timeout, "wall": time.perf_counter() - t0}


def main_rtid(out_path: str) -> None:
    """The reference's RTid build (simba/src/nocache_rtid.cu) on every golden
    instance; committed as tests/golden/ref_results_rtid_u32.json."""
    insts = json.loads((HERE / "ref_instances_u32.json").read_text())
    res = {"simba_rtid": []}
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        for idx, d in enumerate(insts):
            p = td / f"inst_{idx}.json"
            p.write_text(json.dumps(d))
            ml = d["gen_size"] + 1
            r = run(SIMBA_RTID, p, ml, 60)
            r.update({"idx": idx, "max_len": ml})
            res["simba_rtid"].append(r)
    Path(out_path).write_text(json.dumps(res, indent=1))


def main_u64(out_path: str) -> None:
    """The widened 64-bit reference build on the 64-bit golden instances
    (tests/golden/make_golden_u64.py); committed as
    tests/golden/ref_results_u64.json."""
    insts = json.loads((HERE / "ref_instances_u64.json").read_text())
    res = {"simba_u64": []}
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        for idx, d in enumerate(insts):
            p = td / f"inst_{idx}.json"
            p.write_text(json.dumps(d))
            r = run(SIMBA_U64, p, d["max_len"], 120)
            r.update({"idx": idx, "max_len": d["max_len"], "set": d["set"]})
            res["simba_u64"].append(r)
            print(idx, d["set"], d["max_len"], r.get("expr"), r.get("seconds"), flush=True)
    Path(out_path).write_text(json.dumps(res, indent=1))


def main(out_path: str) -> None:
    insts = json.loads((HERE / "ref_instances_u32.json").read_text())
    res = {"simba": [], "vfb": [], "sweeps": []}
    with tempfile.TemporaryDirectory() as td:
        td = Path(td)
        for idx, d in enumerate(insts):
            p = td / f"inst_{idx}.json"
            p.write_text(json.dumps(d))
            ml = d["gen_size"] + 1
            r = run(SIMBA, p, ml, 60)
            r.update({"idx": idx, "max_len": ml})
            res["simba"].append(r)
            ml_v = d["gen_size"]
            r = run(VFB, p, ml_v, 60)
            r.update({"idx": idx, "max_len": ml_v})
            res["vfb"].append(r)
        # Throughput sweeps: unsatisfiable targets, 3 vars + constant 1.
        for (nv, ns, lens) in ((3, 64, (11, 12, 13, 14)), (2, 32, (12, 13, 14))):
            inst = make_instance(15, nv, ns, 1, word_bits=32, const_one=True, unsat=True)
            p = td / f"sweep_{nv}_{ns}.json"
            inst.write(p)
            for ml in lens:
                r = run(SIMBA, p, ml, 400)
                r.update({"n_vars": nv, "n_terms": nv + 1, "samples": ns, "max_len": ml})
                res["sweeps"].append(r)
                print("sweep", nv, ns, ml, r.get("seconds"), r.get("wall"), flush=True)
    Path(out_path).write_text(json.dumps(res, indent=1))


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[2] == "--rtid":
        main_rtid(sys.argv[1])
    elif len(sys.argv) > 2 and sys.argv[2] == "--u64":
        main_u64(sys.argv[1])
    else:
        main(sys.argv[1])
