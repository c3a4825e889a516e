#!/usr/bin/env python
"""Benchmark of the SPB6 IMEX stage loop on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workload (default, lowmach2048): the learned form's configuration -- low-Mach
water (p 1e5 Pa, a seeded divergence-free velocity field of amplitude 15 m/s)
with 16 seeded air bubbles on a 2048 x 2048 periodic grid, FP64, material CFL
0.8, Newton tol 1e-10, BiCGStab tol 1e-10 -- run with the learned Newton start
(the trained network shipped in diffusionimex_b200/data/) and, over the same
window, with the plain guess and with the extrapolation alone.  A "step" is one
time step of the solver (explicit predictor + implicit pressure Newton with
BiCGStab per stage, step-size control, acceptance).  Each run takes W untimed
steps from t = 0 and times the next K steps on the device (CUDA events on the
solver's stream, max over ranks).  The working set (~4 GB) is far larger than L2.

metric: cell-updates/s = interior cells x accepted steps / device time (the
learned run), with BiCGStab iterations per step and Newton iterations per stage
of both guesses, their ratios and L1(p) between the runs.

Multi-GPU: the measured path solves one grid on one GPU, so N > 1 runs N independent
replicas ("scaling": "weak"); value is the total over ranks.

--impl reference times the reference's own CPU solver (oracle/_ref, compiled from
its sources) on the same workload on all host cores; rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# Algorithmic FP64 bytes per interior cell (each distinct array element read or
# written once) of the kernel groups the solver times; 2D values.
ALG_BYTES = {
    # fused explicit kernel: reads U^n (8; + 8 per earlier stage H, counted as the stage-1 case here),
    # writes X* 8, alpha2* 1, face velocities 2, limiter factors 2, face donors 16
    "explicit": (8 + 8 + 2 + 2 + 16 + 1 + 8) * 8 + 4 * 8,
    "jacobian": (9 + 5 + 2 + 10 + 2 + 1 + 1 + 1 + 1 + 7) * 8,  # X*,a2s | Qe vol | phi | faces | v* | qph | kw | P | G | sc | A,A1,dinv
    "residual": (9 + 5 + 2 + 10 + 2 + 2 + 1 + 1 + 1) * 8,       # ... + P, G, sc
    # per BiCGStab iteration: pass 1 reads r, p, v, D^-1, 5 diagonals, r0 and writes p, q; pass 2 reads
    # r, q, A1, D^-1, 5 diagonals and writes v, s, t; pass 3 reads D^-1, p, s, t, x, r0 and writes x, r
    "linear": (12 + 12 + 8) * 8,
}


# Algorithmic bytes (compulsory FP64 traffic): the BiCGStab iteration per row (2 x 40 B of
# matrix rows, 24 vector streams x 8 B) and the fused flux kernel per cell, stage 1 / later stages
# (2D: 64 n_in + 8 (8 + 5); 1D: 64 n_in + 8 (8 + 3))
BICG_BYTES_PER_ROW_ITER = 272
FLUX_BYTES = {True: (168, 232), False: (152, 216)}

# DRAM read + write per unit from ncu (dram__bytes_read.sum + dram__bytes_write.sum) of one launch
# on this workload: k_bicg_solve moved 1.93 GB for 11 iterations of 1,048,576 rows
# (profiles/k_bicg_solve_bubbles1024.md).
DRAM_BYTES = {"linear": 1.934e9 / (11 * 1048576)}
# The same from the --set full captures on the low-Mach field 2048^2 (profiles/k_bicg_solve_lowmach2048.md,
# profiles/k_flux_lowmach2048.md): the BiCGStab solve moved 39.09 GB in 36 iterations of 4,194,304 rows,
# the fused flux kernel 1.412 GB for 4,194,304 cells.
DRAM_BYTES_BY_WORKLOAD = {
    "lowmach2048": {"linear": 39.091e9 / (36 * 4194304), "explicit": 1.412e9 / 4194304},
    "bubbles1024": {"linear": 1.934e9 / (11 * 1048576)},
}
KERNEL_OF = {"linear": "k_bicg_solve (BiCGStab solve, one launch per Newton iteration)",
             "jacobian": "k_jac_entries", "residual": "k_residual", "explicit": "k_flux"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="lowmach2048",
                   help="lowmach2048 (default: learned vs plain guess), lowmach2048-plain, bubbles1024, bubbles2048, bubbles256, tube1000, lowmach2048, shock2048x1024, "
                        "bubbles2048-mixed, shock2048x1024-mixed (precision form), riemann512 (batched form), "
                        "undex361x200 (Mie-Grueneisen phases), bubbles1024-relax (p-pT relaxation), "
                        "<2D workload>-rus0 (grid-wide Rusanov speed), <workload>-jreuse (modified Newton), "
                        "bubblecomp200 (chemical relaxation, "
                        "case 72), dodecane2000-rates (finite relaxation rates, case 3), "
                        "mlp (learned warm-start network)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def make_workload(name: str):
    from diffusionimex_b200 import cases

    if name == "bubbles1024":
        c = cases.bubble_field(1024, seed=0, nbub=8)
    elif name == "bubbles2048":
        c = cases.bubble_field(2048, seed=0, nbub=8)
    elif name == "bubbles256":
        c = cases.bubble_field(256, seed=0, nbub=8)
    elif name == "tube1000":
        c = cases.water_air_tube(1000)
    elif name == "lowmach2048":  # the learned form's configuration: learned vs plain Newton start
        c = cases.lowmach_bubbles(2048, seed=0)
        c["learned"] = True
        c["metric"] = "cell-updates/s & BiCGStab iters/step, learned vs plain guess, equal tol, 1 B200"
        c["workload"] = ("low-Mach water with 16 air bubbles 2D periodic, 2048x2048 cells, material CFL 0.8, "
                         "Newton tol 1e-10, BiCGStab tol 1e-10; learned Newton start vs the plain guess")
    elif name == "lowmach2048-plain":
        c = cases.lowmach_bubbles(2048, seed=0)
    elif name == "shock2048x1024":
        c = cases.shock_bubble(2048, 1024)
    elif name.endswith("-jreuse"):  # the same workload with the modified Newton (jreuse = 1)
        c = make_workload(name[:-len("-jreuse")])
        c["jreuse"] = 1
        c["workload"] = c.get("workload", name) + ", modified Newton (jreuse 1)"
    elif name.endswith("-rus0"):  # the same workload with the grid-wide Rusanov speed (rus_local = 0)
        c = make_workload(name[:-len("-rus0")])
        c["rus_local"] = 0
        c["workload"] = c.get("workload", name) + ", grid-wide Rusanov speed (rus 0)"
    elif name in ("bubbles2048-mixed", "shock2048x1024-mixed"):
        c = make_workload(name[:-len("-mixed")])
        c["precision"] = 1
        c["workload"] = c.get("workload", name) + " (precision form)"
    elif name == "undex361x200":
        c = cases.underwater_explosion(361, 200)
    elif name == "bubblecomp200":  # the reference's case 72 at its own 200 x 200 grid
        c = cases.bubble_compression(200, 200)
    elif name == "dodecane2000-rates":  # the reference's case 3 at its own 2000 cells, finite rates
        c = cases.reference_case(3)
        c.update(relax=2, mu_rate=1e-2, theta_rate=1e5, nu_rate=1e3)
        c["workload"] = ("dodecane liquid-vapour shock tube 1D, 2000 cells, relax 2 with finite rates "
                         "mu 1e-2, theta 1e5, nu 1e3")
    elif name == "bubbles1024-relax":
        c = cases.bubble_field(1024, seed=0, nbub=8)
        c.update(relax=1, eps_i=1e-4)
        c["workload"] += ", p-pT relaxation in the interface zone (relax 1, eps_I 1e-4)"
    elif name == "riemann512":
        return {"batch": cases.riemann_batch(count=512, seed=0), "workload": "512 1D Riemann problems, 256-4096 cells"}
    elif name == "mlp":
        return {"mlp": True, "rows": 1 << 21,
                "workload": "learned warm-start network: training passes (forward, backward, Adam) over 2,097,152 "
                            "feature rows of 64 BF16 (54 used), 54-64-64-64-1 SiLU"}
    else:
        raise SystemExit(f"unknown workload {name}")
    return c


def run_reference_batch(args, case, rank: int):
    """The reference solver on a sample of the batch: one grid per host core, single-threaded,
    all at once; value = sum of cells x timed steps / the slowest grid's timed wall time."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from concurrent.futures import ThreadPoolExecutor

    import refio

    cores = os.cpu_count() or 1
    sample = case["batch"][:cores]
    run = (lambda c: refio.run_ref(c, mode=refio.MODE_STEPS, nsteps=args.warmup + args.steps, threads=1,
                                   warmup=args.warmup, budget_s=150.0)) if refio.ref_available() else \
          (lambda c: refio.run_port(c, mode=refio.MODE_STEPS, nsteps=args.warmup + args.steps, warmup=args.warmup,
                                    budget_s=150.0))
    with ThreadPoolExecutor(cores) as ex:
        rs = list(ex.map(run, sample))
    wall = max(r["wall_s"] for r in rs)
    upd = sum(int(r["timed_steps"]) * c["nx"] for r, c in zip(rs, sample))
    value = upd / wall
    kind = "reference" if refio.ref_available() else "port"
    line = {"impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": case["workload"], "instances": len(sample), "seed": 0},
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": kind,
                             "sample": f"first {len(sample)} grids of the batch, one per core, steps "
                                       f"{args.warmup + 1}..{args.warmup + args.steps}"},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_batch(args, case, rank: int, world: int, local_rank: int, dist):
    """Batched form: every grid advances `steps` steps in one replay of the persistent launches (one
    per block size, concurrent; after `warmup` untimed steps in another); value = sum of cells x
    accepted steps / device time."""
    import torch

    from diffusionimex_b200 import BatchSolver

    cs = case["batch"]
    b = BatchSolver(cs, device=local_rank)
    if args.warmup:
        b.advance(args.warmup)
    threads, tile, _ = b.autotune(5)  # from the warmed-up state, restored after every trial
    s0 = [b.instance(i).stats() for i in range(len(cs))]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = ClockSampler(local_rank)
    clk.start()
    ms = b.advance(args.steps)
    clocks = clk.stop()
    s1 = [b.instance(i).stats() for i in range(len(cs))]
    upd = sum((q["steps"] - p["steps"]) * c["nx"] for p, q, c in zip(s0, s1, cs))
    ms_max = max_over_ranks(ms, dist, f"cuda:{local_rank}")
    value = upd * world / (ms_max / 1e3)
    # end to end: the states go host -> device before the launch and come back after it
    e2e = None
    if not args.no_e2e:
        host = [b.instance(i).state() for i in range(len(cs))]
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        import time as _t
        w0 = _t.perf_counter()
        for i in range(len(cs)):
            b.instance(i).upload(host[i])
        ms2 = b.advance(1)
        for i in range(len(cs)):
            host[i] = b.instance(i).state()
        wall = max_over_ranks((_t.perf_counter() - w0) * 1e3, dist, f"cuda:{local_rank}")
        cells = sum(c["nx"] for c in cs)
        e2e = {"value": cells * world / (wall / 1e3), "unit": "cell-updates/s", "h2d_bytes_per_step": 64 * cells,
               "d2h_bytes_per_step": 64 * cells, "steps": 1, "device_ms": ms2}
    if rank == 0:
        cells = sum(c["nx"] for c in cs)
        line = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / max(args.steps, 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": case["workload"], "instances": len(cs), "cells": cells, "seed": 0,
                           "launch": {"threads_largest_grid": threads, "flux_tile": tile}},
                "rejects": sum(q["rejects"] - p["rejects"] for p, q in zip(s0, s1)),
                "newton_iters": sum(q["newton_it"] - p["newton_it"] for p, q in zip(s0, s1)),
                "gpu_launches": b.launches(), "clocks": clocks, "e2e": e2e}
        print(json.dumps(line))
    b.close()


# Learned warm-start network, per feature row of one training pass: tensor-core FLOPs (forward
# 3 x 2*64*64, input gradients 2 x 2*64*64, weight and bias gradients 3 x 2*65*64), special-function
# operations (exp2 and reciprocal of the logistic function, 64 per layer and three layers; the
# backward pass reuses the derivatives the forward epilogues keep) and HBM bytes (the BF16 row
# and the FP32 target).
MLP_FLOP_PER_ROW = 3 * 2 * 64 * 64 + 2 * 2 * 64 * 64 + 3 * 2 * 65 * 64
MLP_SFU_PER_ROW = 3 * 64 * 2
MLP_BYTES_PER_ROW = 64 * 2 + 4
SFU_PER_CLOCK_PER_SM = 16  # nominal special-function results per clock per SM


def mlp_cpu_baseline(rows: int = 1 << 16) -> dict:
    """The float64 numpy checker's training pass (oracle/mlp_ref.py) on a sample of rows."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import mlp_ref

    rng = np.random.default_rng(0)
    X = np.zeros((rows, 64), np.float32)
    X[:, :54] = rng.standard_normal((rows, 54))
    p = mlp_ref.init_params(rng)
    t = np.zeros(rows, np.float32)
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        mlp_ref.loss_grad(p, X, t)
    wall = time.perf_counter() - t0
    return {"value": rows * reps / wall, "unit": "rows/s", "cores": os.cpu_count() or 1, "kind": "port",
            "sample": f"{reps} training passes of the float64 numpy checker over {rows} rows ({wall:.1f} s; "
                      "numpy may use every host core)"}


def run_mlp(args, case, rank: int, world: int, local_rank: int, dist):
    """Training passes of the warm-start network over a fixed synthetic batch: value = rows x
    passes / device time (CUDA events on the launching stream, max over ranks)."""
    import torch

    from diffusionimex_b200 import learned
    from diffusionimex_b200.warmstart import MLP

    n = case["rows"]
    dev = f"cuda:{local_rank}"
    torch.cuda.set_device(local_rank)
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    X = torch.zeros((n, 64), dtype=torch.bfloat16, device=dev)
    X[:, :54] = torch.randn((n, 54), generator=g, device=dev).to(torch.bfloat16)
    T = torch.tanh(X[:, :54].float() @ torch.randn(54, generator=g, device=dev) / 8).contiguous()
    m = MLP(local_rank)
    m.set_params(learned._init_params(0))
    st = torch.cuda.current_stream()
    lr = 1e-3
    for _ in range(args.warmup):
        m.train_async(X, T, lr, st)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(local_rank)
    clk.start()
    e0.record(st)
    for _ in range(args.steps):
        m.train_async(X, T, lr, st)
    e1.record(st)
    e1.synchronize()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    loss = m.last_loss(st) / n
    ms_max = max_over_ranks(ms, dist, dev)
    value = n * args.steps * world / (ms_max / 1e3)
    # inference passes over the same rows
    y = torch.empty(n, dtype=torch.float32, device=dev)
    for _ in range(3):
        m.forward(X, y, stream=st)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    f0.record(st)
    for _ in range(args.steps):
        m.forward(X, y, stream=st)
    f1.record(st)
    f1.synchronize()
    fms = f0.elapsed_time(f1) / args.steps
    # end to end: the batch goes host -> device every pass, the loss comes back
    e2e = None
    if not args.no_e2e:
        Xh = X.cpu().pin_memory()
        Th = T.cpu().pin_memory()
        ke = max(1, min(args.steps, 5))
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0.record(st)
        for _ in range(ke):
            X.copy_(Xh, non_blocking=True)
            T.copy_(Th, non_blocking=True)
            m.train_async(X, T, lr, st)
            m.last_loss(st)
        e1.record(st)
        e1.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1), dist, dev)
        e2e = {"value": n * ke * world / (ems / 1e3), "unit": "rows/s", "h2d_bytes_per_step": n * MLP_BYTES_PER_ROW,
               "d2h_bytes_per_step": 4, "steps": ke}
    peak = None
    try:
        with open(MEASURED_PEAKS) as f:
            pk = json.load(f)
        peak, peak_kind = float(pk["bf16_tflops"]), "measured (burst)"
    except (OSError, KeyError, ValueError):
        peak, peak_kind = 1590.0, "fallback"
    per_pass_s = ms / args.steps / 1e3
    tflops = MLP_FLOP_PER_ROW * n / per_pass_s / 1e12
    smhz = clocks.get("sm_mhz") or 1965.0
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    sfu_peak = SFU_PER_CLOCK_PER_SM * sms * smhz * 1e6
    sfu = MLP_SFU_PER_ROW * n / per_pass_s
    roof = {"bound": "tensor", "kernel": "k_mlp_grad (+ k_mlp_adam, timed together)", "achieved": tflops, "peak": peak,
            "unit": "TFLOP/s", "frac": tflops / peak, "traffic": None, "peak_source": peak_kind,
            "flop_per_row": MLP_FLOP_PER_ROW,
            "special_function": {"ops_per_row": MLP_SFU_PER_ROW, "achieved_per_s": sfu, "nominal_peak_per_s": sfu_peak,
                                 "frac": sfu / sfu_peak},
            "hbm": {"bytes_per_row": MLP_BYTES_PER_ROW, "achieved_GBs": MLP_BYTES_PER_ROW * n / per_pass_s / 1e9}}
    if rank == 0:
        line = {"metric": "rows/s", "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
                "config": {"workload": case["workload"], "rows": n, "seed": 0, "lr": lr,
                           "l2": "inputs (276 MB) larger than L2"},
                "loss": loss, "inference": {"rows_per_s": n / (fms / 1e3), "us_per_pass": fms * 1e3},
                "roofline": roof, "gpu_launches": 2 * args.steps, "clocks": clocks, "e2e": e2e}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = mlp_cpu_baseline()
        print(json.dumps(line))
    m.close()


def workload_config(c: dict, name: str) -> dict:
    return {"workload": c.get("workload", name), "nx": c["nx"], "ny": c["ny"], "fp": "fp64",
            "newton_tol": c["newton_tol"], "bicg_tol": c["bicg_tol"], "cfl": c["cfl"], "seed": c.get("seed", 0),
            "relax": c.get("relax", 0), "rus_local": c.get("rus_local", 1), "jreuse": c.get("jreuse", 0),
            **{k: c[k] for k in ("mu_rate", "theta_rate", "nu_rate") if k in c},
            "l2": "working set > L2 (no flush needed)"}


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu, self.proc, self.lines = gpu, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def cpu_baseline(case: dict, steps: int = 2) -> dict:
    """The reference CPU solver (oracle/_ref when present, else the C restatement) on the first
    `steps` steps of the same workload, all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refio

    cores = os.cpu_count() or 1
    n = case["nx"] * case["ny"]
    if refio.ref_available():
        r = refio.run_ref(case, mode=refio.MODE_STEPS, nsteps=steps, threads=cores)
        kind = "reference"
    else:
        r = refio.run_port(case, mode=refio.MODE_STEPS, nsteps=steps)
        kind, cores = "port", 1
    return {"value": n * r["timed_steps"] / r["wall_s"], "unit": "cell-updates/s", "cores": cores, "kind": kind,
            "sample": f"first {r['timed_steps']} time steps from t=0 of the same workload "
                      f"({r['newton_it']} Newton iterations), {r['wall_s']:.1f} s"}


def max_over_ranks(ms: float, dist, device) -> float:
    """Slowest rank's time: every rank contributes its own device-timed milliseconds (one
    all-reduce, the same collective on every rank)."""
    if not dist:
        return ms
    import torch

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(cells: int, steps: int, world: int, ms_max: float) -> float:
    """Whole-job cell-updates/s of N independent replicas timed by the slowest rank."""
    return cells * steps * world / (ms_max / 1e3)


def dist_init(world: int, local_rank: int):
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    from datetime import timedelta
    dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local_rank))
    return dist


def run_reference(args, case, rank: int):
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refio

    cores = os.cpu_count() or 1
    n = case["nx"] * case["ny"]
    budget = 150.0
    if refio.ref_available():
        r = refio.run_ref(case, mode=refio.MODE_STEPS, nsteps=args.warmup + args.steps, threads=cores,
                          warmup=args.warmup, budget_s=budget)
        kind = "reference"
    else:
        r = refio.run_port(case, mode=refio.MODE_STEPS, nsteps=args.warmup + args.steps, warmup=args.warmup,
                           budget_s=budget)
        kind, cores = "port", 1
    k = max(int(r["timed_steps"]), 1)
    value = n * k / r["wall_s"]
    sample = (f"steps {args.warmup + 1}..{args.warmup + k} from t=0 after {args.warmup} untimed steps"
              + (" (stopped at the time budget)" if k < args.steps else ""))
    line = {
        "impl": "reference", "metric": case.get("metric", "cell-updates/s"), "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus,
        "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * r["wall_s"] / k, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(case, args.workload),
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "newton_it": r["newton_it"], "stages": r["stages"], "bicg_it": r["bicg_it"],
        "bicg_iters_per_step": (r["bicg_it"] / max(int(r["steps"]), 1)) if r["bicg_it"] else None,
        "guess": "plain (the reference always starts Newton from the previous stage's pressure)",
    }
    print(json.dumps(line))


def timed_window(case: dict, args, local_rank: int, dist, mlp=None, norm=None, zero: bool = False):
    """W untimed steps from t = 0, then K steps timed on the device (CUDA events on the solver's
    stream, bracketed by a barrier and a device synchronisation); counts, kernel groups, launches,
    clocks and the final pressure of the window."""
    import torch

    from diffusionimex_b200 import Solver

    s = Solver(case, device=local_rank)
    if mlp is not None:
        s.set_feature_norm(norm)
        s.set_warmstart(mlp)
    if args.warmup > 0:
        s.advance(args.warmup)
    st0 = s.stats()
    l0 = s.kernel_launches()
    s.timing(True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local_rank)
    clk.start()
    s.region_begin()
    s.advance(args.steps)
    ms = s.region_end()
    clocks = clk.stop()
    torch.cuda.synchronize()
    st1 = s.stats()
    out = {"ms": ms, "launches": s.kernel_launches() - l0, "groups": s.timing(), "clocks": clocks,
           "d": {k: st1[k] - st0[k] for k in ("steps", "rejects", "stages", "newton_it", "bicg_it", "learned",
                                              "learned_x0", "extrapolated", "extrapolated2", "combined", "refined")}}
    s.timing(False)
    if case.get("learned"):
        P, pref = s.pressure()
        out["p"] = P + pref
    s.close()
    return out


def counts(r: dict) -> dict:
    d = r["d"]
    return {"ms_per_step": r["ms"] / max(d["steps"], 1), "bicg_iters_per_step": d["bicg_it"] / max(d["steps"], 1),
            "newton_iters_per_stage": d["newton_it"] / max(d["stages"], 1), **d}


def rooflines(r: dict, n: int, two_d: bool, workload: str = "") -> dict:
    """Algorithmic-byte rooflines (the compulsory bytes per unit above) of the BiCGStab solve, the fused
    flux kernel and the whole step, from the window's CUDA-event group times and counts."""
    peak, peak_kind = peaks()
    g, d = r["groups"], r["d"]
    dram = DRAM_BYTES_BY_WORKLOAD.get(workload, {})
    out = {}
    if g.get("linear", (0, 0))[1] > 0 and d["bicg_it"] > 0:
        units = d["bicg_it"] * n
        ach = BICG_BYTES_PER_ROW_ITER * units / (g["linear"][0] / 1e3) / 1e9
        out["bicg"] = {"bound": "hbm", "kernel": KERNEL_OF["linear"], "achieved": ach, "peak": peak, "unit": "GB/s",
                       "frac": ach / peak,
                       "traffic": dram["linear"] * units / g["linear"][1] if "linear" in dram else None,
                       "peak_source": peak_kind,
                       "alg_bytes_per_unit": BICG_BYTES_PER_ROW_ITER, "unit_of_work": "row x BiCGStab iteration",
                       "alg_bytes_per_launch": BICG_BYTES_PER_ROW_ITER * units / g["linear"][1]}
    if g.get("explicit", (0, 0))[1] > 0:
        # stage 1 reads U^n only (168 B / cell); a later stage also its earlier derivatives (232 B); the
        # later stages are the stages beyond one per attempt
        later = max(d["stages"] - d["steps"] - d["rejects"], 0)
        first = g["explicit"][1] - later
        b1, b2 = FLUX_BYTES[two_d]
        alg = (first * b1 + later * b2) * n
        ach = alg / (g["explicit"][0] / 1e3) / 1e9
        out["flux"] = {"bound": "hbm", "kernel": KERNEL_OF["explicit"], "achieved": ach, "peak": peak, "unit": "GB/s",
                       "frac": ach / peak, "traffic": dram["explicit"] * n if "explicit" in dram else None,
                       "peak_source": peak_kind,
                       "alg_bytes_per_cell": [b1, b2], "alg_bytes_per_launch": alg / g["explicit"][1]}
    # whole step: every group's algorithmic bytes over the whole window's device time
    tot = 0.0
    for k, (gms, gcnt) in g.items():
        if k == "linear":
            tot += BICG_BYTES_PER_ROW_ITER * d["bicg_it"] * n
        elif k == "explicit" and "flux" in out:
            tot += out["flux"]["alg_bytes_per_launch"] * gcnt
        elif k in ALG_BYTES:
            tot += ALG_BYTES[k] * gcnt * n
    ach = tot / (r["ms"] / 1e3) / 1e9
    out["step"] = {"bound": "hbm", "kernel": "whole step (B_step)", "achieved": ach, "peak": peak, "unit": "GB/s",
                   "frac": ach / peak, "traffic": None, "peak_source": peak_kind, "alg_bytes_per_step": tot / max(d["steps"], 1)}
    return out


def e2e_run(case: dict, args, local_rank: int, dist, mlp=None, norm=None, ref_counts=None) -> dict:
    """The same window through the public API with host buffers: a solver replays the W untimed
    steps, then every timed step uploads the state from pinned host memory, steps and downloads
    the state (SoA); timed with CUDA events on the solver's stream."""
    import torch

    from diffusionimex_b200 import Solver

    n = case["nx"] * case["ny"]
    s = Solver(case, device=local_rank)
    if mlp is not None:
        s.set_feature_norm(norm)
        s.set_warmstart(mlp)
    if args.warmup > 0:
        s.advance(args.warmup)
    host = torch.empty(8 * n, dtype=torch.float64, pin_memory=True)
    ptr = host.data_ptr()
    s.download_soa(ptr)
    st0 = s.stats()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    s.region_begin()
    for _ in range(args.steps):
        s.upload_soa(ptr)
        s.step()
        s.download_soa(ptr)
    ems = max_over_ranks(s.region_end(), dist, f"cuda:{local_rank}")
    st1 = s.stats()
    s.close()
    same = None
    if ref_counts is not None:
        same = all(st1[k] - st0[k] == ref_counts[k] for k in ("steps", "rejects", "newton_it", "bicg_it"))
    steps = st1["steps"] - st0["steps"]
    return {"value": n * steps * (int(os.environ.get("WORLD_SIZE", "1"))) / (ems / 1e3), "unit": "cell-updates/s",
            "h2d_bytes_per_step": 64 * n, "d2h_bytes_per_step": 64 * n, "steps": steps,
            "ms_per_step": ems / max(steps, 1), "same_work_as_timed_run": same,
            "path": "Solver.upload_soa / step / download_soa every step (spb6g_upload_state, spb6g_step, "
                    "spb6g_download_state), pinned host buffer"}


def run_ours(args, case, rank: int, world: int, local_rank: int, dist):
    n = case["nx"] * case["ny"]
    two_d = case["ny"] > 1
    mlp = norm = zero = None
    if case.get("learned"):
        from diffusionimex_b200 import learned

        if not os.path.exists(learned.DEFAULT_WEIGHTS):
            raise SystemExit(f"trained warm-start network missing: {learned.DEFAULT_WEIGHTS}")
        mlp, norm = learned.load(learned.DEFAULT_WEIGHTS, device=local_rank)
        zero = learned.zero_network(local_rank)
    main_r = timed_window(case, args, local_rank, dist, mlp, norm)
    ms_max = max_over_ranks(main_r["ms"], dist, f"cuda:{local_rank}")
    d = main_r["d"]
    value = job_value(n, d["steps"], world, ms_max)
    extra = {}
    if case.get("learned"):
        from diffusionimex_b200 import learned

        plain_r = timed_window(case, args, local_rank, dist)
        ext_r = timed_window(case, args, local_rank, dist, zero, norm)
        pc, lc, ec = counts(plain_r), counts(main_r), counts(ext_r)
        extra = {
            "learned": lc, "plain": pc, "extrapolation_only": ec,
            "plain_value": job_value(n, plain_r["d"]["steps"], world,
                                     max_over_ranks(plain_r["ms"], dist, f"cuda:{local_rank}")),
            "bicg_ratio_plain_over_learned": pc["bicg_iters_per_step"] / max(lc["bicg_iters_per_step"], 1e-30),
            "newton_ratio_plain_over_learned": pc["newton_iters_per_stage"] / max(lc["newton_iters_per_stage"], 1e-30),
            "wall_ratio_plain_over_learned": pc["ms_per_step"] / max(lc["ms_per_step"], 1e-30),
            "L1_rel_p_learned_vs_plain": learned.l1_rel(main_r["p"], plain_r["p"]),
            "L1_rel_p_extrapolation_vs_plain": learned.l1_rel(ext_r["p"], plain_r["p"]),
            "same_steps": plain_r["d"]["steps"] == d["steps"] and plain_r["d"]["rejects"] == d["rejects"],
            "network": os.path.relpath(learned.DEFAULT_WEIGHTS, ROOT),
            "warmstart_mode": 15,  # the library default: candidate starts, their combination, first iterates
        }
    e2e = None if args.no_e2e else e2e_run(case, args, local_rank, dist, mlp, norm,
                                           {k: d[k] for k in ("steps", "rejects", "newton_it", "bicg_it")})
    roofs = rooflines(main_r, n, two_d, args.workload)
    groups = main_r["groups"]
    shares = {g: {"ms": round(v[0], 3), "launch_groups": int(v[1]), "share": round(v[0] / main_r["ms"], 4)}
              for g, v in groups.items()}
    if rank == 0:
        line = {
            "metric": case.get("metric", "cell-updates/s"), "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": d["steps"], "warmup": args.warmup, "ms_per_step": ms_max / max(d["steps"], 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(case, args.workload),
            "bicg_iters_per_step": d["bicg_it"] / max(d["steps"], 1),
            "newton_iters_per_stage": d["newton_it"] / max(d["stages"], 1),
            "stages": d["stages"], "rejects": d["rejects"], **extra,
            "roofline": roofs.get("bicg", roofs["step"]), "roofline_flux": roofs.get("flux"),
            "roofline_step": roofs["step"], "kernel_groups": shares,
            "timed_groups_ms": round(sum(v[0] for v in groups.values()), 3),
            "gpu_launches": main_r["launches"], "clocks": main_r["clocks"], "e2e": e2e,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(case)
        print(json.dumps(line))
    for m in (mlp, zero):
        if m is not None:
            m.close()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    case = make_workload(args.workload)
    if args.impl == "reference":
        if "mlp" in case:
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned warm start: "
                                  "its Newton always starts from the previous stage's pressure"}))
            return
        if "batch" in case:
            run_reference_batch(args, case, rank)
            return
        run_reference(args, case, rank)
        return
    dist = dist_init(world, local_rank)
    try:
        if "mlp" in case:
            run_mlp(args, case, rank, world, local_rank, dist)
        elif "batch" in case:
            run_batch(args, case, rank, world, local_rank, dist)
        else:
            run_ours(args, case, rank, world, local_rank, dist)
    finally:
        if dist:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
