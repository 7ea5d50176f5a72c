"""Test infrastructure only: float64 numpy restatement of the learned tuner's
network (huffman_coding_gap_arrays_b200/csrc/mlp.cu), used as the checker of
its CUDA forward, gradient and Adam kernels.  Nothing in the product imports
this file.

Network: x[9] -> 32 ReLU -> 32 ReLU -> y[2]; parameters flat as
W1[32][9] b1[32] W2[32][32] b2[32] W3[2][32] b3[2];
loss = scale * sum over samples and non-NaN targets of (y - t)^2 / 2.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 10, 32, 2
SHAPES = [("W1", (HID, IN)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (OUT, HID)),
          ("b3", (OUT,))]
PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    p = np.asarray(p, np.float64)
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = p[o:o + k].reshape(shape)
        o += k
    return out


def pack(d):
    return np.concatenate([np.asarray(d[name], np.float64).reshape(-1) for name, _ in SHAPES])


def forward(p, X):
    w = unpack(p)
    X = np.asarray(X, np.float64)
    a1 = X @ w["W1"].T + w["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(a2, 0)
    y = h2 @ w["W3"].T + w["b3"]
    return y, (X, a1, h1, a2, h2)


def loss_grad(p, X, T, scale):
    w = unpack(p)
    y, (X, a1, h1, a2, h2) = forward(p, X)
    T = np.asarray(T, np.float64)
    valid = ~np.isnan(T)
    d = np.where(valid, y - np.where(valid, T, 0), 0.0)
    loss = 0.5 * scale * float((d * d).sum())
    gy = d * scale
    g = {"W3": gy.T @ h2, "b3": gy.sum(0)}
    gh2 = (gy @ w["W3"]) * (a2 > 0)
    g["W2"] = gh2.T @ h1
    g["b2"] = gh2.sum(0)
    gh1 = (gh2 @ w["W2"]) * (a1 > 0)
    g["W1"] = gh1.T @ X
    g["b1"] = gh1.sum(0)
    return loss, pack(g)


def adam(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    g = g + wd * p  # L2 term
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
