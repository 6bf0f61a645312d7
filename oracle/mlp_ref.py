"""ORACLE -- test infrastructure, not part of the product.

Double-precision numpy restatement of the engine's sizing MLP
(n_features -> 64 -> 64 -> 64 -> n_outputs, ReLU; loss 0.5*mean((y-t)^2) over
samples and outputs) used to check the GPU forward/backward kernels.  The
parameter layout matches include/bespoke_gpu.h: W1[F][64] b1 W2[64][64] b2
W3[64][64] b3 W4[64][O] b4, row-major, activations computed as x @ W + b.
"""
from __future__ import annotations

import numpy as np

H = 64


def unpack(p: np.ndarray, F: int, O: int):
    p = np.asarray(p, dtype=np.float64)
    shapes = [(F, H), (H,), (H, H), (H,), (H, H), (H,), (H, O), (O,)]
    out, i = [], 0
    for s in shapes:
        k = int(np.prod(s))
        out.append(p[i:i + k].reshape(s))
        i += k
    assert i == p.size
    return out


def forward(p, x, F, O):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p, F, O)
    x = np.asarray(x, dtype=np.float64)
    a1 = np.maximum(x @ W1 + b1, 0)
    a2 = np.maximum(a1 @ W2 + b2, 0)
    a3 = np.maximum(a2 @ W3 + b3, 0)
    return a3 @ W4 + b4, (x, a1, a2, a3)


def loss_and_grad(p, x, t, F, O):
    W1, b1, W2, b2, W3, b3, W4, b4 = unpack(p, F, O)
    y, (x, a1, a2, a3) = forward(p, x, F, O)
    t = np.asarray(t, dtype=np.float64)
    n = x.shape[0]
    e = y - t
    loss = 0.5 * np.sum(e * e) / (n * O)
    dy = e / (n * O)
    gW4 = a3.T @ dy
    gb4 = dy.sum(0)
    d3 = (dy @ W4.T) * (a3 > 0)
    gW3 = a2.T @ d3
    gb3 = d3.sum(0)
    d2 = (d3 @ W3.T) * (a2 > 0)
    gW2 = a1.T @ d2
    gb2 = d2.sum(0)
    d1 = (d2 @ W2.T) * (a1 > 0)
    gW1 = x.T @ d1
    gb1 = d1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3, gW4, gb4)])
    return loss, g


def loss_only(p, x, t, F, O):
    y, _ = forward(p, x, F, O)
    e = y - np.asarray(t, dtype=np.float64)
    return 0.5 * np.sum(e * e) / (x.shape[0] * O)
