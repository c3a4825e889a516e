"""Learned warm start: data, training and evaluation (no counterpart in the reference).

The plain solver starts each stage's implicit-pressure Newton from the previous
stage's pressure.  Here a small MLP (tensor-core kernels of libspb6g) predicts the
stage's pressure P_start + dts (R + sigma y) from the 3x3 stencils of
(rho, rho u, rho v, alpha1, E*, P_prev, R / sigma) and the last rate change
(R - R2) / sigma, R the pressure rate of the last converged stage, sigma its RMS
over the cells and dts the stage's time span: y = 0 is the linear extrapolation
of the pressure, and the network learns the departure from it in units of sigma,
so the target is scale-free across fields, regimes and the start-up ramp.  The
solver starts Newton from the guess of smallest residual max-norm among the plain
guess, the extrapolation, the second-order extrapolation, the network's guess and
(warm-start mode bit 8, on by default) the combination of their steps that
minimises the residual's 2-norm with the residual taken linear in P -- the
network's output is one direction of that combination; when the network's guess
is not the start, its step seeds the first BiCGStab iterate, and the last Newton
correction the stage's later ones (in a least-squares combination with the plain
start, never with a larger initial residual).  Newton and BiCGStab keep their
tolerances, a warm-started stage always takes one Newton step, and the converged
pressure is the plain solve's to the solver tolerance.

At the low-Mach operating point Newton converges linearly (a constant
contraction of about 0.4-0.6 per iteration with full steps), so every factor
the starting residual drops saves iterations, each of them a whole BiCGStab
solve.

    python -m diffusionimex_b200.learned --out warmstart.npz --n 2048          # dump, train, save
    python -m diffusionimex_b200.learned --eval warmstart.npz --n 2048         # plain vs learned

Training data are (feature row, (R' - R) / sigma) pairs that the plain GPU
solver writes while it runs (`Solver.set_dump`); features are centred and
scaled per field with statistics from a short pilot run.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import cases
from .solver import Solver
from .warmstart import MLP

FIELDS = ("rho", "rho_u", "rho_v", "alpha1", "E", "P", "R")
NF = len(FIELDS)
NSTENCIL = 9 * NF  # 63 stencil columns; the 64th is the last rate change of the cell
NFEAT = 64
IDENTITY = [0.0] * NF + [1.0] * NF + [1.0] * NF + [1.0]
# the trained network shipped with the package (low-Mach bubble fields, material CFL 0.8)
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_lowmach.npz")


def _torch():
    import torch

    return torch


def _run_dump(s: Solver, n: int, steps: int, every: int, device: int, first: int = 0):
    """Advance `steps` steps; the stages of every `every`-th step from step `first` on are dumped.
    Returns the feature rows and targets on the device."""
    torch = _torch()
    # capacity: two stages per dumped step (LSDIRK2), and room for stages a halving repeats
    ndump = sum(1 for k in range(steps) if k >= first and (k - first) % every == every - 1)
    cap = n * (3 * ndump + 2)
    X = torch.empty((cap, 64), dtype=torch.bfloat16, device=f"cuda:{device}")
    T = torch.empty(cap, dtype=torch.float32, device=f"cuda:{device}")
    off = 0
    for k in range(steps):
        dump = k >= first and (k - first) % every == every - 1
        if dump:
            s.set_dump(X[off:], T[off:])
        s.step()
        if dump:
            off += s.dump_count()
            s.set_dump(None)
    X, T = X[:off].clone(), T[:off].clone()  # release the unused capacity
    return X, T


def rough_norm(case: dict) -> list[float]:
    """A first normalisation from the initial state alone (per-field mean and spread of rho, rho u,
    rho v, alpha1, E and their x-differences; fixed scales for P - P_REF and R / sigma), enough to
    keep the pilot's feature rows inside the feature kernel's clamp."""
    U = np.asarray(case["U"], dtype=np.float64).reshape(case["ny"], case["nx"], 8)
    fields = [U[..., 1] + U[..., 2], U[..., 3], U[..., 4], U[..., 0], U[..., 7]]
    mean = [float(f.mean()) for f in fields] + [0.0, 0.0]
    std = [max(float(f.std()), 1e-3 * abs(float(f.mean())), 1e-30) for f in fields] + [1e5, 1.0]
    dstd = [max(float(np.abs(np.diff(f, axis=1)).mean()) if case["nx"] > 1 else 0.0, 1e-3 * sd, 1e-30)
            for f, sd in zip(fields, std)] + [1e4, 1.0]
    return mean + std + dstd + [1.0]


def pilot_norm(case: dict, steps: int = 8, device: int = 0) -> list[float]:
    """Per-field mean / std of the centre values, std of the neighbour differences and the std
    of the target, from the stages of the last step of a plain run of `steps` steps: the rows are
    written with the rough normalisation of the initial state and mapped back before the
    statistics are taken."""
    torch = _torch()
    n = case["nx"] * case["ny"]
    rough = rough_norm(case)
    s = Solver(case, device=device)
    s.set_feature_norm(rough)
    X, T = _run_dump(s, n, steps, steps, device)
    s.close()
    k = X.shape[0]
    F = X[:, :NSTENCIL].float().view(k, NF, 9).double()
    m0 = torch.tensor(rough[:NF], dtype=torch.float64, device=F.device)
    s0 = torch.tensor(rough[NF:2 * NF], dtype=torch.float64, device=F.device)
    d0 = torch.tensor(rough[2 * NF:3 * NF], dtype=torch.float64, device=F.device)
    centre = F[:, :, 0] * s0 + m0
    diffs = F[:, :, 1:] * d0[None, :, None]
    mean = centre.mean(0)
    std = centre.std(0)
    dstd = diffs.std(dim=(0, 2))
    tscale = T.std()
    fl = lambda v, lo: [max(float(a), lo * (abs(float(m)) + 1e-30), 1e-30) for a, m in zip(v, mean)]
    return [float(m) for m in mean] + fl(std, 1e-6) + fl(dstd, 1e-9) + [max(float(tscale), 1e-30)]


def dump_pairs(plan, norm, device: int = 0):
    """plan: list of (case, steps, every): a plain run of `steps` steps from t = 0 that dumps the
    stages of every `every`-th step.  Returns feature rows and targets on the device."""
    torch = _torch()
    Xs, Ts = [], []
    for case, steps, every in plan:
        n = case["nx"] * case["ny"]
        s = Solver(case, device=device)
        s.set_feature_norm(norm)
        X, T = _run_dump(s, n, steps, every, device)
        s.close()
        Xs.append(X)
        Ts.append(T)
    if len(Xs) == 1:
        return Xs[0], Ts[0]
    X, T = torch.cat(Xs), torch.cat(Ts)
    del Xs, Ts
    return X, T


def _init_params(seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    F = 64
    W1 = rng.uniform(-1, 1, (F, F)) * np.sqrt(3.0 / NFEAT)
    W2 = rng.uniform(-1, 1, (F, F)) * np.sqrt(3.0 / F)
    W3 = rng.uniform(-1, 1, (F, F)) * np.sqrt(3.0 / F)
    w4 = rng.uniform(-1, 1, F) * np.sqrt(3.0 / F) * 0.1
    parts = [W1, np.zeros(F), W2, np.zeros(F), W3, np.zeros(F), w4, np.zeros(1)]
    return np.concatenate([np.ravel(a) for a in parts]).astype(np.float32)


def zero_network(device: int = 0) -> MLP:
    """The network with every parameter 0: y = 0, so the learned guess is the linear extrapolation
    P_start + dts R alone (the ablation of the trained network: the solver tries the extrapolation
    on its own as well, so with this network every stage gets exactly the extrapolation)."""
    m = MLP(device)
    m.set_params(np.zeros(m.nparam, np.float32))
    return m


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


def run_case(case: dict, steps: int, warmup: int, mlp=None, norm=None, device: int = 0, mode: int = 15,
             smooth: int = 0) -> tuple:
    """Advance `warmup` untimed steps, then `steps` timed ones; counts and device time."""
    torch = _torch()
    s = Solver(case, device=device)
    if mlp is not None:
        s.set_feature_norm(norm)
        s.set_warmstart(mlp, mode, smooth)
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
    d = {k: b[k] - a[k] for k in ("steps", "stages", "newton_it", "bicg_it", "rejects", "learned", "learned_x0",
                                  "extrapolated", "extrapolated2", "combined", "refined")}
    d.update(ms=ms, ms_per_step=ms / max(d["steps"], 1), bicg_per_step=d["bicg_it"] / max(d["steps"], 1),
             newton_per_stage=d["newton_it"] / max(d["stages"], 1), t=b["t"])
    return d, P + pref


def l1_rel(a, b) -> float:
    """Relative L1 difference: mean |a - b| / mean |b|."""
    return float(np.abs(a - b).mean() / max(np.abs(b).mean(), 1e-300))


def compare(case: dict, mlp, norm, steps: int, warmup: int = 0, device: int = 0, extrapolation: bool = True) -> dict:
    """Plain guess against the trained network (and, with `extrapolation`, against the zero network:
    the extrapolation alone) over the same steps; counts, times and L1(p) against the plain run."""
    plain, Pp = run_case(case, steps, warmup, device=device)
    learned, Pl = run_case(case, steps, warmup, mlp=mlp, norm=norm, device=device)
    out = {"plain": plain, "learned": learned, "L1_rel_p": l1_rel(Pl, Pp),
           "bicg_ratio": plain["bicg_per_step"] / max(learned["bicg_per_step"], 1e-30),
           "newton_ratio": plain["newton_per_stage"] / max(learned["newton_per_stage"], 1e-30),
           "time_ratio": plain["ms_per_step"] / max(learned["ms_per_step"], 1e-30),
           "same_steps": plain["steps"] == learned["steps"] and abs(plain["t"] - learned["t"]) <= 1e-12 * plain["t"]}
    if extrapolation:
        z = zero_network(device)
        ex, Pe = run_case(case, steps, warmup, mlp=z, norm=norm, device=device)
        z.close()
        out["extrapolation"] = ex
        out["extrapolation_L1_rel_p"] = l1_rel(Pe, Pp)
    return out


def save(path: str, mlp, norm, meta: dict | None = None):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, params=mlp.params(), norm=np.asarray(norm, dtype=np.float64),
             meta=np.asarray(json.dumps(meta or {})))


def load(path: str = DEFAULT_WEIGHTS, device: int = 0):
    z = np.load(path)
    norm = [float(v) for v in z["norm"]]
    if len(norm) != 3 * NF + 1:
        raise ValueError(f"{path}: feature normalisation of {len(norm)} values, expected {3 * NF + 1}")
    m = MLP(device)
    m.set_params(z["params"])
    return m, norm


def default_plan(n: int, steps: int = 40, every: int = 3):
    """Training runs, none of them the evaluation case (the low-Mach field of seed 0): the low-Mach
    bubble field of seeds 1 and 2 at n x n, material CFL 0.8 (the stages of every `every`-th step
    of the first `steps`), and the 8-bubble water field at rest (seed 1) at min(n, 1024)^2."""
    return [(cases.lowmach_bubbles(n, seed=s), steps, every) for s in (1, 2)] + \
           [(cases.bubble_field(min(n, 1024), seed=1, nbub=8), 30, 2)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--eval", default=None)
    ap.add_argument("--n", type=int, default=1024)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--dump-steps", type=int, default=40)
    ap.add_argument("--every", type=int, default=3)
    ap.add_argument("--train-steps", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=1e-3)
    args = ap.parse_args()
    if args.out:
        torch = _torch()
        t0 = time.time()
        norm = pilot_norm(cases.lowmach_bubbles(args.n, seed=1))
        X, T = dump_pairs(default_plan(args.n, args.dump_steps, args.every), norm)
        torch.cuda.synchronize()
        t1 = time.time()
        m, hist = train_mlp(X, T, steps=args.train_steps, lr=args.lr, log_every=max(args.train_steps // 10, 1))
        t2 = time.time()
        meta = {"pairs": int(X.shape[0]), "dump_s": t1 - t0, "train_s": t2 - t1, "loss": hist, "n": args.n,
                "plan": f"low-Mach seeds 1, 2 at {args.n}^2, {args.dump_steps} steps, every {args.every}th step; "
                        f"8-bubble field seed 1 at {min(args.n, 1024)}^2, 30 steps, every 2nd step",
                "train_steps": args.train_steps, "lr": args.lr, "batch": 1 << 20}
        save(args.out, m, norm, meta)
        print(json.dumps(meta))
        del X, T
        torch.cuda.empty_cache()
    if args.eval:
        m, norm = load(args.eval)
        r = compare(cases.lowmach_bubbles(args.n, seed=0), m, norm, steps=args.steps, warmup=args.warmup)
        print(json.dumps(r))


if __name__ == "__main__":
    main()
