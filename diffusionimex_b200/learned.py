"""Learned warm start: data, training and evaluation (no counterpart in the reference).

The plain solver starts each stage's implicit-pressure Newton from the previous
stage's pressure.  Here a small MLP (tensor-core kernels of libspb6g) predicts the
stage's pressure change from the 3x3 stencil of (rho, rho u, rho v, alpha1, E*,
P_prev); the solver evaluates the residual at the predicted pressure and starts
Newton from it only when its residual norm is below the plain guess's.  Newton and
BiCGStab keep their tolerances, so the converged pressure is the plain solve's to
the solver tolerance.

    python -m diffusionimex_b200.learned --out warmstart.npz            # train
    python -m diffusionimex_b200.learned --eval warmstart.npz --n 2048  # plain vs learned

Training data are (feature row, (P_converged - P_start) / (tau scale)) pairs that the
plain GPU solver writes while it runs (`Solver.set_dump`); features are centred
and scaled per field with statistics from a short pilot run.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import cases
from .solver import Solver
from .warmstart import MLP

FIELDS = ("rho", "rho_u", "rho_v", "alpha1", "E", "P")
IDENTITY = [0.0] * 6 + [1.0] * 6 + [1.0] * 6 + [1.0]


def _torch():
    import torch

    return torch


def pilot_norm(case: dict, warmup: int = 3, stages: int = 4, device: int = 0) -> list[float]:
    """Per-field mean / std of the centre values, std of the neighbour differences and the std
    of the stage pressure rate (P_converged - P_start) / tau, from `stages` stages after
    `warmup` steps of a plain run."""
    torch = _torch()
    n = case["nx"] * case["ny"]
    s = Solver(case, device=device)
    s.set_feature_norm(IDENTITY)
    if warmup > 0:
        s.advance(warmup)
    X = torch.empty((n * stages, 64), dtype=torch.bfloat16, device=f"cuda:{device}")
    T = torch.empty(n * stages, dtype=torch.float32, device=f"cuda:{device}")
    s.set_dump(X, T)
    while s.dump_count() < n * stages:
        s.step()
    k = s.dump_count()
    s.close()
    F = X[:k, :54].float().view(k, 6, 9)
    mean = F[:, :, 0].mean(0)
    std = F[:, :, 0].std(0)
    dstd = F[:, :, 1:].std(dim=(0, 2))
    tscale = T[:k].std()
    fl = lambda v, lo: [max(float(a), lo * (abs(float(m)) + 1e-30)) for a, m in zip(v, mean)]
    norm = [float(m) for m in mean] + fl(std, 1e-6) + fl(dstd, 1e-9) + [max(float(tscale), 1e-30)]
    return norm


def dump_pairs(plan, norm, device: int = 0):
    """plan: list of (case, warmup_steps, stages); returns feature rows and targets on the device."""
    torch = _torch()
    Xs, Ts = [], []
    for case, warmup, stages in plan:
        n = case["nx"] * case["ny"]
        s = Solver(case, device=device)
        s.set_feature_norm(norm)
        if warmup > 0:  # advance(0) would run to t_end
            s.advance(warmup)
        X = torch.empty((n * stages, 64), dtype=torch.bfloat16, device=f"cuda:{device}")
        T = torch.empty(n * stages, dtype=torch.float32, device=f"cuda:{device}")
        s.set_dump(X, T)
        while s.dump_count() < n * stages:
            s.step()
        k = s.dump_count()
        s.close()
        Xs.append(X[:k])
        Ts.append(T[:k])
    return torch.cat(Xs), torch.cat(Ts)


def _init_params(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    F = 64
    W1 = rng.uniform(-1, 1, (F, F)) * np.sqrt(3.0 / 54)
    W1[:, 54:] = 0.0
    W2 = rng.uniform(-1, 1, (F, F)) * np.sqrt(3.0 / F)
    W3 = rng.uniform(-1, 1, (F, F)) * np.sqrt(3.0 / F)
    w4 = rng.uniform(-1, 1, F) * np.sqrt(3.0 / F) * 0.1
    parts = [W1, np.zeros(F), W2, np.zeros(F), W3, np.zeros(F), w4, np.zeros(1)]
    return np.concatenate([np.ravel(a) for a in parts]).astype(np.float32)


def train_mlp(X, T, steps: int = 3000, batch: int = 1 << 20, lr: float = 1e-3, seed: int = 0, device: int = 0,
              params=None, log_every: int = 0):
    """Adam on mean squared error over random mini-batches (rows gathered on the device).
    Returns the trained network and the loss history [(step, batch loss)]."""
    torch = _torch()
    m = MLP(device)
    m.set_params(params if params is not None else _init_params(seed))
    g = torch.Generator(device=f"cuda:{device}")
    g.manual_seed(seed)
    N = X.shape[0]
    hist = []
    for it in range(steps):
        idx = torch.randint(0, N, (min(batch, N),), device=X.device, generator=g)
        xb, tb = X.index_select(0, idx).contiguous(), T.index_select(0, idx).contiguous()
        # cosine decay to 1/20 of the initial rate
        rate = lr * (0.05 + 0.95 * 0.5 * (1 + np.cos(np.pi * it / max(steps - 1, 1))))
        loss = m.train_step(xb, tb, float(rate))
        if log_every and (it % log_every == 0 or it == steps - 1):
            hist.append((it, loss))
    return m, hist


def run_case(case: dict, steps: int, warmup: int, mlp=None, norm=None, device: int = 0) -> dict:
    """Advance `warmup` untimed steps, then `steps` timed ones; counts and device time."""
    torch = _torch()
    s = Solver(case, device=device)
    if mlp is not None:
        s.set_feature_norm(norm)
        s.set_warmstart(mlp)
    if warmup > 0:  # advance(0) would run to t_end
        s.advance(warmup)
    a = s.stats()
    torch.cuda.synchronize()
    s.region_begin()
    s.advance(steps)
    ms = s.region_end()
    b = s.stats()
    P, pref = s.pressure()
    s.close()
    d = {k: b[k] - a[k] for k in ("steps", "stages", "newton_it", "bicg_it", "rejects", "learned")}
    d.update(ms=ms, ms_per_step=ms / max(d["steps"], 1), bicg_per_step=d["bicg_it"] / max(d["steps"], 1),
             newton_per_stage=d["newton_it"] / max(d["stages"], 1), t=b["t"])
    return d, P + pref


def compare(case: dict, mlp, norm, steps: int, warmup: int = 0, device: int = 0) -> dict:
    plain, Pp = run_case(case, steps, warmup, device=device)
    learned, Pl = run_case(case, steps, warmup, mlp=mlp, norm=norm, device=device)
    l1 = float(np.abs(Pl - Pp).mean() / np.abs(Pp).mean())
    return {"plain": plain, "learned": learned, "L1_rel_p": l1,
            "bicg_ratio": plain["bicg_per_step"] / max(learned["bicg_per_step"], 1e-30),
            "time_ratio": plain["ms_per_step"] / max(learned["ms_per_step"], 1e-30)}


def save(path: str, mlp, norm):
    np.savez(path, params=mlp.params(), norm=np.asarray(norm, dtype=np.float64))


def load(path: str, device: int = 0):
    z = np.load(path)
    m = MLP(device)
    m.set_params(z["params"])
    return m, [float(v) for v in z["norm"]]


def default_plan(n: int):
    """Training runs: the 8-bubble water field (seeds 1, 2) and low-Mach bubble fields (seeds 1-3),
    none of them the evaluation case (low-Mach, seed 0)."""
    return [(cases.lowmach_bubbles(n, seed=s), 0, 30) for s in (1, 2, 3)] + \
           [(cases.bubble_field(min(n, 1024), seed=s, nbub=8), 0, 20) for s in (1, 2)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--eval", default=None)
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--train-steps", type=int, default=3000)
    args = ap.parse_args()
    if args.out:
        t0 = time.time()
        norm = pilot_norm(cases.lowmach_bubbles(args.n, seed=1))
        X, T = dump_pairs(default_plan(args.n), norm)
        t1 = time.time()
        m, hist = train_mlp(X, T, steps=args.train_steps, log_every=max(args.train_steps // 10, 1))
        t2 = time.time()
        save(args.out, m, norm)
        print(json.dumps({"pairs": int(X.shape[0]), "dump_s": t1 - t0, "train_s": t2 - t1, "loss": hist}))
    if args.eval:
        m, norm = load(args.eval)
        r = compare(cases.lowmach_bubbles(args.n, seed=0), m, norm, steps=args.steps)
        print(json.dumps(r))


if __name__ == "__main__":
    main()
