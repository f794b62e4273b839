"""Test infrastructure (oracle only): numpy restatement of the order-selection
network of defmm_b200/csrc/mlp.cu, in float64, to check the CUDA forward,
backward, Adam and BF16 inference kernels.

Only tests/ may import this module, and only as the checker.

Network: x (12) -> relu(W1 x + b1) (64) -> relu(W2 h1 + b2) (64) -> W3 h2 + b3
(6 logits).  Parameters are one flat array, W1 (64 x 12, row-major), b1, W2
(64 x 64), b2, W3 (6 x 64), b3.  Loss: sum_i w_i (-log softmax(z_i)[y_i]) /
sum_i w_i.
"""
from __future__ import annotations

import numpy as np

NIN, NH, NOUT = 12, 64, 6
SHAPES = [("W1", (NH, NIN)), ("b1", (NH,)), ("W2", (NH, NH)), ("b2", (NH,)), ("W3", (NOUT, NH)), ("b3", (NOUT,))]
NPARAM = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(p[o:o + k], dtype=np.float64).reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], dtype=np.float64).ravel() for name, _ in SHAPES])


def forward(p, X):
    w = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    h1 = np.maximum(X @ w["W1"].T + w["b1"], 0.0)
    h2 = np.maximum(h1 @ w["W2"].T + w["b2"], 0.0)
    z = h2 @ w["W3"].T + w["b3"]
    return h1, h2, z


def loss_and_grad(p, X, y, wts=None):
    """Weighted softmax cross-entropy and its gradient (flat, like p)."""
    w = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    n = X.shape[0]
    wts = np.ones(n) if wts is None else np.asarray(wts, dtype=np.float64)
    ws = wts / wts.sum()
    h1, h2, z = forward(p, X)
    zm = z - z.max(axis=1, keepdims=True)
    e = np.exp(zm)
    sm = e / e.sum(axis=1, keepdims=True)
    loss = float(np.sum(ws * (np.log(e.sum(axis=1)) - zm[np.arange(n), y])))
    g3 = sm.copy()
    g3[np.arange(n), y] -= 1.0
    g3 *= ws[:, None]
    d = {"W3": g3.T @ h2, "b3": g3.sum(axis=0)}
    d2 = (g3 @ w["W3"]) * (h2 > 0)
    d["W2"] = d2.T @ h1
    d["b2"] = d2.sum(axis=0)
    d1 = (d2 @ w["W2"]) * (h1 > 0)
    d["W1"] = d1.T @ X
    d["b1"] = d1.sum(axis=0)
    return loss, pack(d)


def adam(p, g, m, v, step, lr, wd=0.0, b1=0.9, b2=0.999, eps=1e-8):
    """Adam with decoupled weight decay: p -= lr (mhat / (sqrt(vhat) + eps) + wd p)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * (mh / (np.sqrt(vh) + eps) + wd * p), m, v


def bf16_round(a):
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.asarray(a, dtype=np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)
