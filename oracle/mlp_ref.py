"""numpy reference of the learned proposal -- TEST INFRASTRUCTURE ONLY.

Restates, in plain numpy, what simba_b200's MLP kernels compute (features,
forward pass, softmax cross-entropy, backward pass), including the BF16
rounding the GPU applies to GEMM operands (weights, activations, output
gradients), with FP32 (here FP64) accumulation.  The GPU gradients are
checked against it; the reference itself is checked against finite
differences on a small network (tests/test_mlp_cpu.py).

The reference project has no learned component; this has no reference
counterpart.
"""
from __future__ import annotations

import numpy as np

FEAT, HID, CLS = 8192, 512, 64
SAMPLES, PER_SAMPLE = 64, 128


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def features(inputs: np.ndarray, outputs: np.ndarray) -> np.ndarray:
    """8192 features of one instance (inputs S x k, outputs S; uint64)."""
    S, k = inputs.shape
    out = np.zeros(FEAT, dtype=np.float32)
    for f in range(FEAT):
        smp = (f // PER_SAMPLE) % S
        j = f % PER_SAMPLE
        y = int(outputs[smp])
        if j < 64:
            out[f] = 1.0 if (y >> j) & 1 else -1.0
        else:
            var, bit = (j - 64) // 16, (j - 64) % 16
            if var < k:
                x = int(inputs[smp, var])
                out[f] = 1.0 if ((y ^ x) >> bit) & 1 else -1.0
    return out


def split(params: np.ndarray, dims=(FEAT, HID, HID, CLS)):
    d0, d1, d2, d3 = dims
    sizes = [d0 * d1, d1, d1 * d2, d2, d2 * d3, d3]
    parts, o = [], 0
    for n in sizes:
        parts.append(params[o:o + n])
        o += n
    W1, b1, W2, b2, W3, b3 = parts
    return W1.reshape(d0, d1), b1, W2.reshape(d1, d2), b2, W3.reshape(d2, d3), b3


def forward_backward(params: np.ndarray, X: np.ndarray, labels: np.ndarray,
                     dims=(FEAT, HID, HID, CLS), round_bf16: bool = True):
    """Mean cross-entropy and its gradient (flattened like the parameters)."""
    r = bf16 if round_bf16 else (lambda a: np.asarray(a, dtype=np.float32))
    W1, b1, W2, b2, W3, b3 = split(np.asarray(params, dtype=np.float32), dims)
    W1b, W2b, W3b = (r(w).astype(np.float64) for w in (W1, W2, W3))
    Xd = np.asarray(X, dtype=np.float64)
    B = X.shape[0]
    Z1 = Xd @ W1b + b1
    H1 = r(np.maximum(Z1, 0).astype(np.float32)).astype(np.float64)
    Z2 = H1 @ W2b + b2
    H2 = r(np.maximum(Z2, 0).astype(np.float32)).astype(np.float64)
    Z3 = H2 @ W3b + b3
    Z = Z3 - Z3.max(axis=1, keepdims=True)
    P = np.exp(Z)
    P /= P.sum(axis=1, keepdims=True)
    loss = float(-np.log(np.maximum(P[np.arange(B), labels], 1e-30)).mean())
    onehot = np.zeros_like(P)
    onehot[np.arange(B), labels] = 1.0
    dZ3 = r(((P - onehot) / B).astype(np.float32)).astype(np.float64)
    gW3 = H2.T @ dZ3
    gb3 = dZ3.sum(axis=0)
    dH2 = dZ3 @ W3b.T
    dZ2 = r((dH2 * (Z2 > 0)).astype(np.float32)).astype(np.float64)
    gW2 = H1.T @ dZ2
    gb2 = dZ2.sum(axis=0)
    dH1 = dZ2 @ W2b.T
    dZ1 = r((dH1 * (Z1 > 0)).astype(np.float32)).astype(np.float64)
    gW1 = Xd.T @ dZ1
    gb1 = dZ1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g, P
