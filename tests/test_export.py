"""Exporters: Xyntia traces byte-identical to the reference converter's
output (golden files made by it), SyGuS-IF text of the cvc5 problem."""
import json
import subprocess
import sys
from pathlib import Path

from simba_b200 import export as E
from simba_b200.instances import make_instance

GOLD = Path(__file__).resolve().parent / "golden" / "xyntia"
ROOT = Path(__file__).resolve().parent.parent


def test_xyntia_matches_reference_converter():
    files = sorted(GOLD.glob("inst_?.json"))
    assert len(files) == 4
    for f in files:
        want = (GOLD / (f.stem + ".xyntia.json")).read_text()
        got = json.dumps(E.to_xyntia(json.loads(f.read_text())), indent=4)
        assert got == want, f


def test_xyntia_folder_cli(tmp_path):
    src = tmp_path / "in"
    src.mkdir()
    for f in sorted(GOLD.glob("inst_?.json")):
        (src / f.name).write_text(f.read_text())
    r = subprocess.run([sys.executable, "-m", "simba_b200.export", "xyntia", str(src),
                        str(tmp_path / "out")], capture_output=True, text=True, cwd=ROOT, timeout=120)
    assert r.returncode == 0, r.stderr
    for f in sorted(GOLD.glob("inst_?.json")):
        assert (tmp_path / "out" / f.name).read_text() == (GOLD / (f.stem + ".xyntia.json")).read_text()


def test_sygus_problem_text():
    inst = make_instance(5, 2, 4, 3, word_bits=32, const_one=False).to_json()
    txt = E.to_sygus(inst)
    lines = txt.strip().split("\n")
    assert lines[0] == "(set-logic BV)"
    assert lines[1] == "(synth-fun f ((v0 (_ BitVec 32)) (v1 (_ BitVec 32))) (_ BitVec 32)"
    assert "(bvmul Start Start)" in lines[3] and lines[3].endswith("v0 v1))))")
    cons = [l for l in lines if l.startswith("(constraint")]
    assert len(cons) == 4 and lines[-1] == "(check-synth)"
    ex = inst["examples"][0]
    a = " ".join("#x%08x" % v["value"] for v in ex["inputs"])
    assert cons[0] == "(constraint (= (f %s) #x%08x))" % (a, ex["output"][0]["value"])
    # balanced parentheses
    assert txt.count("(") == txt.count(")")
    # 64-bit instances use 16 hex digits
    i64 = make_instance(4, 1, 2, 5, word_bits=64).to_json()
    assert "(_ BitVec 64)" in E.to_sygus(i64) and "#x" + "%016x" % i64["examples"][1]["output"][0]["value"] in E.to_sygus(i64)
