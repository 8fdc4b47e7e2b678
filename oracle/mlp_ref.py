"""CPU restatement (float64 numpy) of the selector network -- TEST
INFRASTRUCTURE ONLY, used to check the library's MLP kernels.

The network has no reference counterpart (the reference has no learned
components); this restates its mathematics: in -> H -> H -> out with ReLU,
parameters packed as W1[H][in], b1[H], W2[H][H], b2[H], W3[out][H], b3[out],
loss mean((y - t)^2) over every output of the batch.
"""
from __future__ import annotations

import numpy as np


def unpack(p: np.ndarray, i: int, h: int, o: int):
    p = np.asarray(p, np.float64)
    sizes = [h * i, h, h * h, h, o * h, o]
    parts = np.split(p, np.cumsum(sizes)[:-1])
    W1, b1, W2, b2, W3, b3 = parts
    return W1.reshape(h, i), b1, W2.reshape(h, h), b2, W3.reshape(o, h), b3


def forward(p, x, i, h, o):
    W1, b1, W2, b2, W3, b3 = unpack(p, i, h, o)
    a1 = np.maximum(x @ W1.T + b1, 0.0)
    a2 = np.maximum(a1 @ W2.T + b2, 0.0)
    return a2 @ W3.T + b3, (a1, a2)


def loss_and_grad(p, x, t, i, h, o):
    x = np.asarray(x, np.float64)
    t = np.asarray(t, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(p, i, h, o)
    y, (a1, a2) = forward(p, x, i, h, o)
    n = y.size
    loss = float(((y - t) ** 2).sum() / n)
    dy = 2.0 * (y - t) / n
    gW3 = dy.T @ a2
    gb3 = dy.sum(0)
    da2 = (dy @ W3) * (a2 > 0)
    gW2 = da2.T @ a1
    gb2 = da2.sum(0)
    da1 = (da2 @ W2) * (a1 > 0)
    gW1 = da1.T @ x
    gb1 = da1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g
