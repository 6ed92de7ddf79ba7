"""Float64 restatement of the learned warm start's network, forward and backward.

TEST INFRASTRUCTURE ONLY (the checker for the GPU's tensor-core kernels):
imported by tests/ alone.

Network: y = w3 . gelu(W2 gelu(W1 x + b1) + b2) + b3, GELU in its erf form,
loss = mean over the batch of (y - target)^2.  Parameters in the canonical
order of include/pbf.h: W1[64][12], b1[64], W2[64][64], b2[64], w3[64], b3.
"""
from __future__ import annotations

import math

import numpy as np

N_IN, N_H = 12, 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_H * N_IN
OFF_W2 = OFF_B1 + N_H
OFF_B2 = OFF_W2 + N_H * N_H
OFF_W3 = OFF_B2 + N_H
OFF_B3 = OFF_W3 + N_H
N_PARAMS = OFF_B3 + 1

_erf = np.vectorize(math.erf)


def unpack(p: np.ndarray):
    p = np.asarray(p, np.float64)
    return (p[OFF_W1:OFF_B1].reshape(N_H, N_IN), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(N_H, N_H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + _erf(x / math.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)


def forward(p, x):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    x = np.asarray(x, np.float64)
    z1 = x @ W1.T + b1
    h1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    y = h2 @ w3 + b3
    return y, (x, z1, h1, z2, h2)


def loss_and_grad(p, x, t):
    """Mean squared error and its gradient with respect to p (canonical order)."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    y, (x, z1, h1, z2, h2) = forward(p, x)
    t = np.asarray(t, np.float64)
    B = x.shape[0]
    e = y - t
    loss = float(np.mean(e * e))
    dy = 2.0 * e / B
    g = np.zeros(N_PARAMS)
    g[OFF_W3:OFF_B3] = h2.T @ dy
    g[OFF_B3] = dy.sum()
    dz2 = (dy[:, None] * w3[None, :]) * gelu_grad(z2)
    g[OFF_W2:OFF_B2] = (dz2.T @ h1).ravel()
    g[OFF_B2:OFF_W3] = dz2.sum(axis=0)
    dz1 = (dz2 @ W2) * gelu_grad(z1)
    g[OFF_W1:OFF_B1] = (dz1.T @ x).ravel()
    g[OFF_B1:OFF_W2] = dz1.sum(axis=0)
    return loss, g
