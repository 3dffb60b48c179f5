"""Test infrastructure only: float64 numpy restatement of the cost model's
network (in -> 64 -> 64 -> 1, ReLU, mean squared error), used to check the
gradients of libgat's hand-written CUDA kernels (gat_mlp_gradient)."""
from __future__ import annotations

import numpy as np

H = 64


def unpack(p: np.ndarray, n_in: int):
    p = np.asarray(p, np.float64)
    i = 0
    W1 = p[i:i + n_in * H].reshape(n_in, H); i += n_in * H
    b1 = p[i:i + H]; i += H
    W2 = p[i:i + H * H].reshape(H, H); i += H * H
    b2 = p[i:i + H]; i += H
    w3 = p[i:i + H]; i += H
    b3 = p[i]
    return W1, b1, W2, b2, w3, b3


def forward(p, X, n_in):
    W1, b1, W2, b2, w3, b3 = unpack(p, n_in)
    X = np.asarray(X, np.float64)
    h1 = np.maximum(X @ W1 + b1, 0)
    h2 = np.maximum(h1 @ W2 + b2, 0)
    return h2 @ w3 + b3, h1, h2


def loss_and_grad(p, X, T, n_in):
    W1, b1, W2, b2, w3, b3 = unpack(p, n_in)
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    y, h1, h2 = forward(p, X, n_in)
    n = len(X)
    loss = float(np.mean((y - T) ** 2))
    dy = 2 * (y - T) / n
    gw3 = h2.T @ dy
    gb3 = dy.sum()
    d2 = dy[:, None] * w3[None, :] * (h2 > 0)
    gW2 = h1.T @ d2
    gb2 = d2.sum(0)
    d1 = (d2 @ W2.T) * (h1 > 0)
    gW1 = X.T @ d1
    gb1 = d1.sum(0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
