"""CPU checker for the learned warm start's MLP (test infrastructure only).

The network has no counterpart in the reference.  This is a float64 numpy
restatement of what the tensor-core kernels compute, with the same BF16
rounding points: the feature rows, the weights, the hidden activations H1, H2
and the back-propagated dZ are rounded to BF16 where the kernels store them as
MMA operands; everything else (pre-activations, the output layer, dL/dw4,
dL/db4) stays in high precision.  Parameter layout: W1[64][64], b1[64],
W2[64][64], b2[64], W3[64][64], b3[64], w4[64], b4.
"""
from __future__ import annotations

import numpy as np

F = 64
NPARAM = 3 * F * F + 3 * F + F + 1


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even) and return as float64."""
    a32 = np.asarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = []
    for shape in ((F, F), (F,), (F, F), (F,), (F, F), (F,), (F,), (1,)):
        size = int(np.prod(shape))
        out.append(p[o:o + size].reshape(shape))
        o += size
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X):
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p)
    X = bf16(X)
    z1 = X @ bf16(W1).T + b1
    h1 = bf16(silu(z1))
    z2 = h1 @ bf16(W2).T + b2
    h2 = bf16(silu(z2))
    z3 = h2 @ bf16(W3).T + b3
    y = silu(z3) @ w4 + b4[0]
    return y, (X, z1, h1, z2, h2, z3)


def loss_grad(p, X, t):
    """mean((y - t)^2) and its gradient with respect to the parameter vector."""
    W1, b1, W2, b2, W3, b3, w4, b4 = unpack(p)
    y, (Xb, z1, h1, z2, h2, z3) = forward(p, X)
    n = len(t)
    r = y - t
    dy = 2.0 * r / n
    g = []
    dz3 = bf16(dy[:, None] * w4[None, :] * dsilu(z3))
    dW3, db3 = dz3.T @ h2, dz3.sum(0)
    dh2 = dz3 @ bf16(W3)
    dz2 = bf16(dh2 * dsilu(z2))
    dW2, db2 = dz2.T @ h1, dz2.sum(0)
    dh1 = dz2 @ bf16(W2)
    dz1 = bf16(dh1 * dsilu(z1))
    dW1, db1 = dz1.T @ Xb, dz1.sum(0)
    dw4 = silu(z3).T @ dy
    db4 = np.array([dy.sum()])
    for a in (dW1, db1, dW2, db2, dW3, db3, dw4, db4):
        g.append(np.ravel(a))
    return float(np.mean(r * r)), np.concatenate(g)


def init_params(rng: np.random.Generator, n_in: int = 54) -> np.ndarray:
    """Scaled uniform initialisation; input columns beyond n_in are zero."""
    W1 = rng.uniform(-1, 1, (F, F)) * np.sqrt(3.0 / n_in)
    W1[:, n_in:] = 0.0
    W2 = rng.uniform(-1, 1, (F, F)) * np.sqrt(3.0 / F)
    W3 = rng.uniform(-1, 1, (F, F)) * np.sqrt(3.0 / F)
    w4 = rng.uniform(-1, 1, F) * np.sqrt(3.0 / F)
    parts = [W1, np.zeros(F), W2, np.zeros(F), W3, np.zeros(F), w4, np.zeros(1)]
    return np.concatenate([np.ravel(a) for a in parts]).astype(np.float32)
