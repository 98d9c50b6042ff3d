"""Learned proposal, CPU side: the numpy reference against finite
differences, the shape-class labels, and the features definition."""
import numpy as np
import pytest

from oracle import mlp_ref as R
import simba_b200 as S
from simba_b200.guided import shape_class
from simba_b200.instances import make_instance


def test_reference_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    dims = (12, 8, 8, 5)
    n = 12 * 8 + 8 + 8 * 8 + 8 + 8 * 5 + 5
    w = rng.normal(0, 0.5, n).astype(np.float32)
    X = rng.choice([-1.0, 1.0], size=(6, 12)).astype(np.float32)
    y = rng.integers(0, 5, 6)
    loss, g, _ = R.forward_backward(w, X, y, dims, round_bf16=False)
    eps = 1e-3
    for i in rng.choice(n, 25, replace=False):
        wp, wm = w.astype(np.float64).copy(), w.astype(np.float64).copy()
        wp[i] += eps
        wm[i] -= eps
        lp = R.forward_backward(wp.astype(np.float32), X, y, dims, round_bf16=False)[0]
        lm = R.forward_backward(wm.astype(np.float32), X, y, dims, round_bf16=False)[0]
        num = (lp - lm) / (2 * eps)
        assert abs(num - g[i]) < 2e-3 + 2e-2 * abs(num), (i, num, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0], dtype=np.float32)
    b = R.bf16(x)
    assert b[0] == 1.0 and b[4] == 0.0
    assert b[1] == 1.0          # halfway rounds to even
    assert abs(b[3] + 3.140625) < 1e-6


@pytest.mark.parametrize("postfix,cls", [
    ("01+", 5 * 8 + 1), ("0~", 0 * 8 + 1), ("0~#", 4 * 8 + 2), ("01~&", 1 * 8 + 1),
    ("0~1-", 6 * 8 + 2), ("012++3*", 7 * 8 + 5), ("0", 0),
])
def test_shape_class_labels(postfix, cls):
    assert shape_class(postfix) == cls


def test_features_definition():
    inst = make_instance(7, 2, 16, 3, word_bits=64)
    f = R.features(inst.inputs, inst.outputs)
    assert f.shape == (8192,)
    y0 = int(inst.outputs[0])
    assert all(f[j] == (1.0 if (y0 >> j) & 1 else -1.0) for j in range(64))
    x00 = int(inst.inputs[0, 0])
    assert all(f[64 + b] == (1.0 if ((y0 ^ x00) >> b) & 1 else -1.0) for b in range(16))
    assert (f[64 + 48:128] == 0).all()  # 3 terminals: variable 3 does not exist
    # 16 samples repeated cyclically over the 64 feature slots
    assert (f[:128] == f[16 * 128:17 * 128]).all()
