"""CPU restatement of the cost model's network in float64 (TEST
INFRASTRUCTURE: the checker of the GPU forward, backward and training kernels
of ultraprecise_b200/csrc/up_costmodel.cu; imported by tests only).

Network: x (16) -> z1 = x W1 + b1 -> a1 = silu(z1) (64) -> z2 = a1 W2 + b2 ->
a2 = silu(z2) (64) -> out = a2 . W3 + b3; loss = mean (out - y)^2.  The
parameter vector is W1[16][64], b1[64], W2[64][64], b2[64], W3[64], b3, the
layout of include/ultraprecise_costmodel.h.  Gradients are the analytic
backward pass (chain rule), written independently of the kernel.
"""
from __future__ import annotations

import numpy as np

F, H = 16, 64


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + F * H].reshape(F, H); o += F * H
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, W3, b3


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    z1 = X @ W1 + b1
    a1 = z1 * _sig(z1)
    z2 = a1 @ W2 + b2
    a2 = z2 * _sig(z2)
    return a2 @ W3 + b3, (X, z1, a1, z2, a2)


def loss_and_grads(p, X, y):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    out, (X, z1, a1, z2, a2) = forward(p, X)
    y = np.asarray(y, dtype=np.float64)
    n = len(y)
    e = out - y
    loss = float(np.mean(e * e))
    dout = 2.0 * e / n

    def dsilu(z):
        s = _sig(z)
        return s * (1.0 + z * (1.0 - s))

    gW3 = a2.T @ dout
    gb3 = dout.sum()
    dz2 = np.outer(dout, W3) * dsilu(z2)
    gW2 = a1.T @ dz2
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2 @ W2.T) * dsilu(z1)
    gW1 = X.T @ dz1
    gb1 = dz1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return loss, g
