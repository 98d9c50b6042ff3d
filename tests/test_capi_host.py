"""C ABI of libsimba_b200.so: exports and host-only entry points (no GPU)."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import simba_b200 as S
from simba_b200.instances import make_instance

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"\b([a-z_][a-z0-9_]*)\s*\(", text):
            name = m.group(1)
            if name.startswith(("simba_", "vfb_")):
                names.add(name)
    return sorted(names)


def test_library_loads_and_exports_every_declared_symbol():
    L = S.lib()
    names = declared_functions()
    assert "simba_solve" in names and len(names) >= 10
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_count_table_matches_oracle(oracle):
    for k in (1, 2, 4, 6):
        a = S.count_table(14, k)
        b = oracle.count_table(14, k)
        assert (a == b).all()


def test_unrank_and_rank_of_roundtrip(oracle):
    for k, s in ((2, 6), (4, 5), (3, 7)):
        t = oracle.count_table(s, k)
        n = int(t[s][8])
        for r in np.linspace(0, n - 1, 200).astype(np.int64):
            p = S.unrank(int(r), s, k)
            assert p == oracle.unrank(int(r), s, t)
            assert S.rank_of(p, k) == r


def test_rank_of_rejects_non_enumerated_split():
    # commutative operator with the larger operand on the left is not in the
    # rank space (simba/src/nocache.cu:137-140)
    with pytest.raises(S.SimbaError):
        S.rank_of("01&0+", 2)  # ((v0 & v1) + v0): left size 3 > right size 1


def test_format_styles():
    assert S.format_postfix("01~+") == "(v0 + (~v1))"
    assert S.format_postfix("01~+", "vfb") == "(v0)+(~(v1))"
    assert S.format_postfix("0#") == "(-v0)"
    assert S.format_postfix("0#", "vfb") == "-(v0)"


def test_instance_loader_u32_and_u64(tmp_path):
    for bits in (32, 64):
        inst = make_instance(7, 3, 16, 5, word_bits=bits)
        p = tmp_path / f"i{bits}.json"
        inst.write(p)
        got = S.load_instance(p)
        assert got.word_bits == bits
        assert (got.inputs == inst.inputs).all() and (got.outputs == inst.outputs).all()


def test_instance_loader_masks_to_32_bits(tmp_path):
    # the reference reads values with get<uint32_t>: only the low 32 bits
    p = tmp_path / "wide.json"
    p.write_text('{"num_variables":1,"num_examples":1,"examples":[{"inputs":[{"value":'
                 '4294967301,"size":32}],"output":[{"value":5,"size":32}]}]}')
    got = S.load_instance(p)
    assert got.word_bits == 32 and int(got.inputs[0, 0]) == 5


def test_instance_loader_errors(tmp_path):
    with pytest.raises(S.SimbaError):
        S.load_instance(tmp_path / "missing.json")
    bad = tmp_path / "bad.json"
    bad.write_text('{"num_variables": 2, "num_examples": 1, "examples": [')
    with pytest.raises(S.SimbaError):
        S.load_instance(bad)


def test_solve_rejects_bad_limits():
    inst = make_instance(5, 2, 8, 1)
    with pytest.raises(S.SimbaError):
        S.solve(inst, 40)  # size limit 32 (simba/src/nocache.cu:200-203)
    big = make_instance(3, 2, 8, 1)
    big.num_variables = 17
    big.inputs = np.zeros((8, 17), dtype=np.uint64)
    with pytest.raises(S.SimbaError):
        S.solve(big, 5)


def test_rtid_option_is_rejected_where_unsupported():
    """RTid order is a single-instance option: batch, sessions, the static
    entry point and guided / naive searches refuse it before any GPU work."""
    import numpy as np
    import simba_b200 as S
    from simba_b200.instances import make_instance
    inst = make_instance(5, 2, 16, 1, word_bits=64)
    prior = np.ones(64, dtype=np.float32)
    for call in (lambda: S.solve_batch([inst], 8, rtid=True),
                 lambda: S.solve_noalloc(inst, 8, rtid=True),
                 lambda: S.Session(inst, rtid=True),
                 lambda: S.solve(inst, 8, rtid=True, naive=True),
                 lambda: S.solve(inst, 8, rtid=True, class_prior=prior)):
        with pytest.raises(S.SimbaError, match="rank_order|RTid"):
            call()


def test_noalloc_rejects_options_it_does_not_run():
    """The allocation-free entry point runs the plain spine search only: a
    guided prior or the one-thread-per-rank engine is refused before any GPU
    work instead of being silently dropped."""
    import numpy as np
    import simba_b200 as S
    from simba_b200.instances import make_instance
    inst = make_instance(5, 2, 16, 1, word_bits=64)
    prior = np.ones(64, dtype=np.float32)
    for call in (lambda: S.solve_noalloc(inst, 8, naive=True),
                 lambda: S.solve_noalloc(inst, 8, class_prior=prior)):
        with pytest.raises(S.SimbaError, match="plain spine search only"):
            call()
