"""Experiment harness (generate + run loop of the reference's scripts)."""
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from simba_b200 import harness as H
from simba_b200.instances import Instance, eval_postfix, infix_to_postfix

ROOT = Path(__file__).resolve().parent.parent


def test_generate_grid_and_schema(tmp_path):
    ps = H.generate(tmp_path, size_range=(5, 7), var_range=(2, 3), repeats=2, samples=16,
                    seed=42, bits=32)
    assert len(ps) == 3 * 2 * 2 and len(set(ps)) == len(ps)
    for p in ps:
        inst = Instance.read(p)
        assert inst.word_bits == 32 and inst.num_examples == 16
        assert 5 <= len(inst.formula) <= 7
        assert (eval_postfix(inst.formula, inst.inputs.astype(np.uint32), 32)
                .astype(np.uint64) == inst.outputs).all()
    # deterministic in the seed
    again = H.generate(tmp_path / "b", size_range=(5, 7), var_range=(2, 3), repeats=2,
                       samples=16, seed=42, bits=32)
    assert [p.read_text() for p in ps] == [p.read_text() for p in again]


def test_cli_entry_generate(tmp_path):
    r = subprocess.run([sys.executable, "-m", "simba_b200.harness", "generate", "--out",
                        str(tmp_path), "--size-range", "5", "5", "--var-range", "2", "2",
                        "--repeats", "3"], capture_output=True, text=True, cwd=ROOT,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert len(list(tmp_path.glob("*.json"))) == 3


@pytest.mark.gpu
def test_run_cli_and_batch_agree(tmp_path, oracle):
    ps = H.generate(tmp_path / "inst", size_range=(5, 8), var_range=(2, 3), repeats=3,
                    samples=16, seed=7, bits=32)
    a, b = tmp_path / "cli.csv", tmp_path / "batch.csv"
    na = H.run_cli(ps, a, "simba", 9, 120)
    nb = H.run_batch(ps, b, 9, 120)
    assert na == nb == len(ps)
    la = a.read_text().splitlines()
    lb = b.read_text().splitlines()
    assert la[0] == lb[0] == "instance,formula,time"
    for x, y in zip(la[1:], lb[1:]):
        fa, ea, _ = x.rsplit(",", 2)
        fb, eb, _ = y.rsplit(",", 2)
        assert fa == fb
        assert (ea == "Not found !") == (eb == "Not found !")
        if ea != "Not found !":
            inst = Instance.read(fa)
            pa, pb = infix_to_postfix(ea), infix_to_postfix(eb)
            assert len(pa) == len(pb)
            assert oracle.check(pb, inst.inputs, inst.outputs, 32)


def test_compare_csvs(tmp_path):
    """compare: agreement on found / not found and on expression size over the
    instances both runs hold, and our expressions checked on their instances."""
    ps = H.generate(tmp_path / "inst", size_range=(5, 5), var_range=(2, 2), repeats=3,
                    samples=16, seed=3, bits=32)
    insts = [Instance.read(p) for p in ps]
    from simba_b200.instances import postfix_to_infix
    a, b = tmp_path / "a.csv", tmp_path / "b.csv"
    rows_a = [f"{p},{postfix_to_infix(i.formula)},0.1" for p, i in zip(ps, insts)]
    rows_b = [f"{ps[0]},{postfix_to_infix(insts[0].formula)},0.5", f"{ps[1]},Not found !,0.5"]
    a.write_text("instance,formula,time\n" + "\n".join(rows_a) + "\n")
    b.write_text("instance,formula,time\n" + "\n".join(rows_b) + "\n")
    r = H.compare(a, b)
    assert r["common"] == 2 and r["agree_found"] == 1 and r["both_found"] == 1
    assert r["agree_size"] == 1 and r["ours_found_verified"] == 2 and r["only_ours"] == 1
