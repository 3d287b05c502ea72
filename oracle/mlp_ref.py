"""ORACLE -- test infrastructure only, never part of the product.

CPU restatement of the library's learned window planner (a three-layer relu perceptron
with BF16 weights, FP32 biases, FP32 arithmetic) for checking the CUDA forward and
backward kernels.  No reference counterpart: the reference chooses filter degree and
subspace size by hand.  Only ``tests/`` import this module.

Parameter packing (as in the C ABI): W1 (hid x in, row-major), b1, W2 (hid x hid), b2,
W3 (out x hid), b3.  Loss: (1/B) sum_{b,o} w[b,o] (y[b,o] - t[b,o])^2.

With ``bf16=True`` the weight matrices are rounded to BF16 (round to nearest, ties to
even) before use, as the GPU does; the arithmetic is FP64, so GPU results differ only by
FP32 rounding.  With ``bf16=False`` the whole network is smooth FP64, which
:func:`finite_difference_grad` uses to pin :func:`loss_and_grad`.
"""
from __future__ import annotations

import numpy as np


def bf16_round(x: np.ndarray) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even); returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    lsb = (b >> np.uint64(16)) & np.uint64(1)
    r = ((b + np.uint64(0x7FFF) + lsb) & np.uint64(0xFFFF0000)).astype(np.uint32)
    return r.view(np.float32).reshape(np.shape(x))


def sizes(in_dim: int, hid: int, out: int) -> int:
    return hid * in_dim + hid + hid * hid + hid + out * hid + out


def unpack(p: np.ndarray, in_dim: int, hid: int, out: int):
    o = 0
    def take(count, shape):
        nonlocal o
        a = p[o:o + count].reshape(shape)
        o += count
        return a
    W1 = take(hid * in_dim, (hid, in_dim)); b1 = take(hid, (hid,))
    W2 = take(hid * hid, (hid, hid)); b2 = take(hid, (hid,))
    W3 = take(out * hid, (out, hid)); b3 = take(out, (out,))
    return W1, b1, W2, b2, W3, b3


def forward(p, X, in_dim, hid, out, bf16=True):
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, dtype=np.float32), in_dim, hid, out)
    if bf16:
        W1, W2, W3 = bf16_round(W1), bf16_round(W2), bf16_round(W3)
    W1, W2, W3 = (W.astype(np.float64) for W in (W1, W2, W3))
    b1, b2, b3 = (b.astype(np.float64) for b in (b1, b2, b3))
    X = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    y = h2 @ W3.T + b3
    return h1, h2, y, (W1, W2, W3)


def loss_and_grad(p, X, T, w, in_dim, hid, out, bf16=True):
    """Loss and gradient of the packed parameters (gradients flow through the BF16
    weights as if the rounding were the identity, as in the GPU's mixed-precision
    training)."""
    X = np.asarray(X, dtype=np.float64)
    B = X.shape[0]
    h1, h2, y, (W1, W2, W3) = forward(p, X, in_dim, hid, out, bf16)
    wt = np.ones_like(y) if w is None else np.asarray(w, dtype=np.float64)
    r = y - np.asarray(T, dtype=np.float64)
    loss = float(np.sum(wt * r * r) / B)
    dy = 2.0 * wt * r / B
    gW3 = dy.T @ h2; gb3 = dy.sum(axis=0)
    d2 = (dy @ W3) * (h2 > 0)
    gW2 = d2.T @ h1; gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1 = d1.T @ X; gb1 = d1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def finite_difference_grad(p, X, T, w, in_dim, hid, out, idx, h=1e-6):
    """Central differences of the FP64 loss at the parameter indices ``idx``."""
    p = np.asarray(p, dtype=np.float64)
    g = np.empty(len(idx))
    for j, i in enumerate(idx):
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        g[j] = (_loss64(pp, X, T, w, in_dim, hid, out) - _loss64(pm, X, T, w, in_dim, hid, out)) / (2 * h)
    return g


def _loss64(p, X, T, w, in_dim, hid, out):
    W1, b1, W2, b2, W3, b3 = unpack(p, in_dim, hid, out)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    y = h2 @ W3.T + b3
    wt = np.ones_like(y) if w is None else np.asarray(w, dtype=np.float64)
    return float(np.sum(wt * (y - T) ** 2) / X.shape[0])


def loss_and_grad64(p, X, T, w, in_dim, hid, out):
    """The FP64 network's analytic gradient (no BF16 rounding), for the FD pin."""
    X = np.asarray(X, dtype=np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, dtype=np.float64), in_dim, hid, out)
    B = X.shape[0]
    h1 = np.maximum(X @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    y = h2 @ W3.T + b3
    wt = np.ones_like(y) if w is None else np.asarray(w, dtype=np.float64)
    r = y - T
    dy = 2.0 * wt * r / B
    gW3 = dy.T @ h2; gb3 = dy.sum(axis=0)
    d2 = (dy @ W3) * (h2 > 0)
    gW2 = d2.T @ h1; gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1 = d1.T @ X; gb1 = d1.sum(axis=0)
    return float(np.sum(wt * r * r) / B), np.concatenate(
        [gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
