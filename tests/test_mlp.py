"""Tensor-core MLP of the learned warm start against its float64 numpy checker
(oracle/mlp_ref.py, same BF16 rounding points).  Tolerances: the kernels
accumulate in FP32 in tensor memory in a different order, and a BF16 rounding
of a hidden activation can land on the other side of a tie, so outputs agree to
2e-3 and gradients to 1e-2 of their largest magnitude."""
from __future__ import annotations

import numpy as np
import pytest

import mlp_ref


def test_bf16_rounding_of_the_checker():
    x = np.array([1.0, 1.0 + 2.0**-8, 1.0 + 3 * 2.0**-9, -2.5, 3.0e38], dtype=np.float32)
    r = mlp_ref.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2.0**-7 and r[3] == -2.5


def _data(n, seed=0):
    rng = np.random.default_rng(seed)
    X = np.zeros((n, 64), np.float32)
    X[:, :54] = rng.standard_normal((n, 54)).astype(np.float32)
    p = mlp_ref.init_params(rng)
    p[mlp_ref.NPARAM - 65:mlp_ref.NPARAM - 1] *= 4.0
    t = np.tanh(X[:, :54] @ rng.standard_normal(54) / 8).astype(np.float32)
    return X, p, t


def _dev(X, t):
    import torch

    Xd = torch.from_numpy(X).to("cuda").to(torch.bfloat16).contiguous()
    td = torch.from_numpy(t).to("cuda")
    return Xd, td


@pytest.mark.gpu
def test_forward_matches_checker():
    from diffusionimex_b200.warmstart import MLP

    X, p, _ = _data(1000)
    m = MLP()
    m.set_params(p)
    Xd, _ = _dev(X, np.zeros(len(X), np.float32))
    y = m.forward(Xd).cpu().numpy()
    yr, _ = mlp_ref.forward(p, X)
    assert np.abs(y - yr).max() <= 2e-3 * np.abs(yr).max()
    m.close()


@pytest.mark.gpu
def test_gradient_matches_checker():
    from diffusionimex_b200.warmstart import MLP

    X, p, t = _data(3000, seed=1)
    m = MLP()
    m.set_params(p)
    Xd, td = _dev(X, t)
    loss, g = m.train_step(Xd, td, 0.0, want_grad=True)
    lr, gr = mlp_ref.loss_grad(p, X, t)
    assert loss == pytest.approx(lr, rel=2e-3)
    # each parameter block separately (W1, b1, W2, b2, W3, b3, w4, b4)
    o = 0
    for size in (4096, 64, 4096, 64, 4096, 64, 64, 1):
        a, b = g[o:o + size], gr[o:o + size]
        assert np.abs(a - b).max() <= 1e-2 * np.abs(b).max() + 1e-9, o
        o += size
    m.close()


@pytest.mark.gpu
def test_training_reduces_the_loss():
    from diffusionimex_b200.warmstart import MLP

    X, p, t = _data(20000, seed=2)
    m = MLP()
    m.set_params(p)
    Xd, td = _dev(X, t)
    first = m.train_step(Xd, td, 0.0)
    for _ in range(300):
        m.train_step(Xd, td, 2e-3)
    last = m.train_step(Xd, td, 0.0)
    assert last < 0.1 * first
    m.close()
