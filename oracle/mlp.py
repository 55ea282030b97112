"""CPU restatement of the warm-start network (test infrastructure only).

The same function as the kernels of ``ccq_b200/csrc/mlp.cu``:
y = w3 . tanh(W2 tanh(W1 x + b1) + b2) + b3, parameters packed as
W1[H][F] | b1[H] | W2[H][H] | b2[H] | w3[H] | b3, loss (1/N) sum (y - t)^2.
Forward and backward in float64 numpy; only ``tests/`` use this module.
"""
from __future__ import annotations

import numpy as np

H = 32


def unpack(p, F):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + H * F].reshape(H, F); o += H * F
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(p, X):
    X = np.asarray(X, dtype=np.float64)
    W1, b1, W2, b2, w3, b3 = unpack(p, X.shape[1])
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ w3 + b3


def loss_and_grad(p, X, T):
    X = np.asarray(X, dtype=np.float64)
    T = np.asarray(T, dtype=np.float64)
    N, F = X.shape
    W1, b1, W2, b2, w3, b3 = unpack(p, F)
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    y = h2 @ w3 + b3
    r = y - T
    loss = float(np.mean(r * r))
    g = 2.0 * r / N
    gb3 = g.sum()
    gw3 = h2.T @ g
    g2 = np.outer(g, w3) * (1.0 - h2 * h2)
    gb2 = g2.sum(axis=0)
    gW2 = g2.T @ h1
    g1 = (g2 @ W2) * (1.0 - h1 * h1)
    gb1 = g1.sum(axis=0)
    gW1 = g1.T @ X
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
