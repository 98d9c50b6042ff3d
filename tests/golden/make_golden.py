"""Generate the uint32 golden instances from the reference's own generator.

This script imports the reference's Python generator (scripts/generate.py,
``random_formula`` at :38-49) and sampler (scripts/sample.py,
``sample_formula`` at :50-65, ``MbaExpr`` at :32-40) from a checkout of the
reference, so it only runs where that checkout exists (pass its path as the
first argument).  It writes ``ref_instances_u32.json``: every instance with
the formula string the reference generated and the sampled inputs/outputs
the reference computed with numpy uint32.  Those outputs pin the oracle's
evaluator, and the same instances are fed to the reference binaries
(``run_reference.py``) to pin the search results.

Usage: python tests/golden/make_golden.py /path/to/reference
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main(ref_root: str) -> None:
    sys.path.insert(0, str(Path(ref_root) / "scripts"))
    from generate import Sampler as FormulaSampler, random_formula  # noqa: E402
    from sample import MbaExpr, Sampler as ValueSampler, sample_formula  # noqa: E402

    out = []

    # Set "plain": the paper's distribution (build_all.sh:17,20) at small sizes.
    fs = FormulaSampler(42)
    vs = ValueSampler(42)
    for size in range(3, 11):
        for n_var in (1, 2, 3):
            for rep in range(3):
                f = random_formula(size, n_variables=n_var, sampler=fs)
                d = sample_formula(f, 16, vs)
                d["set"] = "plain"
                d["gen_size"] = size
                out.append(d)

    # Set "const1": the last variable is the constant 1 on every sample.  The
    # formula is drawn over n_var + 1 variables and re-evaluated by the
    # reference's own MbaExpr on the patched inputs.
    fs = FormulaSampler(43)
    rng = np.random.default_rng(43)
    for size in range(3, 10):
        for n_var in (1, 2):
            for rep in range(3):
                f = random_formula(size, n_variables=n_var + 1, sampler=fs)
                expr = MbaExpr(f)
                k = max(expr.n_vars, n_var + 1)
                exs = []
                for _ in range(16):
                    vals = [np.uint32(v) for v in rng.integers(
                        np.iinfo(np.uint32).max, size=k, dtype=np.uint32,
                        endpoint=True)]
                    vals[k - 1] = np.uint32(1)
                    with np.errstate(over="ignore"):
                        o = expr(*vals[: expr.n_vars])
                    exs.append({"inputs": [{"value": int(v), "size": 32} for v in vals],
                                "output": [{"value": int(np.uint32(o)), "size": 32}]})
                out.append({"original_formula": f, "num_variables": k,
                            "num_examples": 16, "examples": exs,
                            "set": "const1", "gen_size": size, "const_one": True})

    (HERE / "ref_instances_u32.json").write_text(json.dumps(out))
    print(f"wrote {len(out)} instances")


if __name__ == "__main__":
    import os
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIMBA_REFERENCE")
    if not ref:
        sys.exit("usage: python " + sys.argv[0] + " <reference checkout> (or SIMBA_REFERENCE)")
    main(ref)
