"""Golden Xyntia traces made by the reference's own converter.

Runs the reference's scripts/convert_to_xyntia.py (plain Python, json only)
on the first three instances of ref_instances_u32.json plus one 64-bit
instance, and writes its outputs to tests/golden/xyntia/.  Needs the
reference checkout (first argument, its root folder); the outputs are
committed so the tests need no reference.
"""
import json
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from simba_b200.instances import make_instance  # noqa: E402


def main(ref_root: str) -> None:
    conv = Path(ref_root) / "scripts" / "convert_to_xyntia.py"
    insts = json.loads((HERE / "ref_instances_u32.json").read_text())[:3]
    insts.append(make_instance(6, 3, 8, 77, word_bits=64).to_json())
    out = HERE / "xyntia"
    with tempfile.TemporaryDirectory() as td:
        src, dst = Path(td) / "in", Path(td) / "out"
        src.mkdir()
        for i, d in enumerate(insts):
            (src / f"inst_{i}.json").write_text(json.dumps(d))
        subprocess.run([sys.executable, str(conv), str(src), str(dst)], check=True,
                       capture_output=True)
        out.mkdir(exist_ok=True)
        for i in range(len(insts)):
            shutil.copy(src / f"inst_{i}.json", out / f"inst_{i}.json")
            shutil.copy(dst / f"inst_{i}.json", out / f"inst_{i}.xyntia.json")


if __name__ == "__main__":
    import os
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SIMBA_REFERENCE")
    if not ref:
        sys.exit("usage: python " + sys.argv[0] + " <reference checkout> (or SIMBA_REFERENCE)")
    main(ref)
