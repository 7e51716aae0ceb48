"""FP64 reference of the learned far-field correction's network (test
infrastructure only: the checker for the GPU training and inference
kernels).

Same parameter layout and the same rounding points as the GPU training
kernels: inputs, weights and the two hidden activations are rounded to
bfloat16 (round to nearest even); sums, biases and the loss are exact FP64
here.  Backward passes through the roundings unchanged (straight-through).

Layout of the 1442 parameters: W1[32][9], b1[32], W2[32][32], b2[32],
W3[2][32], b3[2].  A row is 12 floats: 9 features, 2 targets, weight.
"""
from __future__ import annotations

import numpy as np

OFF = {"W1": (0, (32, 9)), "b1": (288, (32,)), "W2": (320, (32, 32)),
       "b2": (1344, (32,)), "W3": (1376, (2, 32)), "b3": (1440, (2,))}
N_PARAMS = 1442


def bf16(x, enabled=True):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    x = np.asarray(x, np.float32)
    if not enabled:
        return x.astype(np.float64)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(P):
    P = np.asarray(P, np.float64)
    return {k: P[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in OFF.items()}


def silu(z):
    return z / (1.0 + np.exp(-z))


def forward(P, X, rounding=True):
    p = unpack(np.asarray(P, np.float32))
    W1, W2, W3 = (bf16(p[k], rounding) for k in ("W1", "W2", "W3"))
    x = bf16(X, rounding)
    z1 = x @ W1.T + p["b1"]
    h1 = bf16(silu(z1), rounding)
    z2 = h1 @ W2.T + p["b2"]
    h2 = bf16(silu(z2), rounding)
    y = h2 @ W3.T + p["b3"]
    return y, (x, z1, h1, z2, h2, W1, W2, W3)


def loss_and_grad(P, rows, rounding=True):
    rows = np.asarray(rows, np.float64)
    X, T, w = rows[:, :9], rows[:, 9:11], rows[:, 11:12]
    n = len(rows)
    y, (x, z1, h1, z2, h2, W1, W2, W3) = forward(P, X, rounding)
    e = y - T
    loss = float((w * e * e).sum() / n)
    dy = 2.0 * w * e / n
    sig2 = 1.0 / (1.0 + np.exp(-z2))
    sig1 = 1.0 / (1.0 + np.exp(-z1))
    dz2 = (dy @ W3) * sig2 * (1.0 + z2 * (1.0 - sig2))
    dz1 = (dz2 @ W2) * sig1 * (1.0 + z1 * (1.0 - sig1))
    g = np.zeros(N_PARAMS)
    g[0:288] = (dz1.T @ x).ravel()
    g[288:320] = dz1.sum(0)
    g[320:1344] = (dz2.T @ h1).ravel()
    g[1344:1376] = dz2.sum(0)
    g[1376:1440] = (dy.T @ h2).ravel()
    g[1440:1442] = dy.sum(0)
    return loss, g
