#!/usr/bin/env python
"""Benchmark of the SPB6 IMEX stage loop on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

Workload (default): water at rest with 8 seeded air bubbles on a 1024 x 1024
grid, FP64, transmissive, material CFL 0.5, Newton tol 1e-10, BiCGStab tol
1e-12 -- the plain-method 2D configuration.  A "step" is one time step of the
solver (explicit predictor + implicit pressure Newton with BiCGStab per stage,
step-size control, acceptance).  The run takes W untimed steps from t = 0 and
times the next K steps on the device (CUDA events on the solver's stream,
max over ranks).  The working set (~1 GB) is far larger than L2.

metric: cell-updates/s = interior cells x accepted steps / device time.

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


# DRAM read + write per unit from ncu (dram__bytes_read.sum + dram__bytes_write.sum) of one launch
# on this workload: k_bicg_solve moved 1.93 GB for 11 iterations of 1,048,576 rows
# (profiles/k_bicg_solve_bubbles1024.md).
DRAM_BYTES = {"linear": 1.934e9 / (11 * 1048576)}
KERNEL_OF = {"linear": "k_bicg_solve (BiCGStab solve, one launch per Newton iteration)",
             "jacobian": "k_jac_entries", "residual": "k_residual", "explicit": "k_flux"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="bubbles1024",
                   help="bubbles1024 (default), bubbles2048, bubbles256, tube1000, lowmach2048, shock2048x1024, "
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
    elif name == "lowmach2048":
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
    """Batched form: every grid advances `steps` steps in one persistent launch (after `warmup`
    untimed steps in another); value = sum of cells x accepted steps / device time."""
    import torch

    from diffusionimex_b200 import BatchSolver

    cs = case["batch"]
    b = BatchSolver(cs, device=local_rank)
    threads, tile, _ = b.autotune(2)
    if args.warmup:
        b.advance(args.warmup)
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
                           "launch": {"threads_per_grid": threads, "flux_tile": tile}},
                "rejects": sum(q["rejects"] - p["rejects"] for p, q in zip(s0, s1)),
                "newton_iters": sum(q["newton_it"] - p["newton_it"] for p, q in zip(s0, s1)),
                "gpu_launches": 1, "clocks": clocks, "e2e": e2e}
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
        "impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": args.gpus,
        "steps": k, "warmup": args.warmup, "ms_per_step": 1e3 * r["wall_s"] / k, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(case, args.workload),
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "newton_it": r["newton_it"], "stages": r["stages"],
    }
    print(json.dumps(line))


def run_ours(args, case, rank: int, world: int, local_rank: int, dist):
    import numpy as np
    import torch

    from diffusionimex_b200 import Solver

    n = case["nx"] * case["ny"]
    s = Solver(case, device=local_rank)
    s.advance(args.warmup)
    # the restart point of the timed window: the end-to-end run below replays its first steps
    rp = s.restart_point() if not args.no_e2e else None
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
    launches = s.kernel_launches() - l0
    groups = s.timing()
    s.timing(False)
    ms_max = max_over_ranks(ms, dist, f"cuda:{local_rank}")
    if dist:
        dist.barrier()
    steps_done = st1["steps"] - st0["steps"]
    value = job_value(n, steps_done, world, ms_max)

    # end to end through the public API: the state goes host -> device before every step and
    # comes back after it (pinned host buffer, SoA layout).  The run replays the timed window's
    # K steps from its restart point, so it does the same work as the device-timed run (checked
    # on the step, rejection, Newton and BiCGStab counts) and the two differ by the copies.
    e2e = None
    if not args.no_e2e:
        host = torch.empty(8 * n, dtype=torch.float64, pin_memory=True)
        ptr = host.data_ptr()
        s.restore(rp)
        s.download_soa(ptr)
        st_e0 = s.stats()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        s.region_begin()
        for _ in range(args.steps):
            s.upload_soa(ptr)
            s.step()
            s.download_soa(ptr)
        ems = max_over_ranks(s.region_end(), dist, f"cuda:{local_rank}")
        st_e1 = s.stats()
        keys = ("steps", "rejects", "newton_it", "bicg_it")
        same = all(st_e1[k] - st_e0[k] == st1[k] - st0[k] for k in keys)
        e2e = {"value": job_value(n, args.steps, world, ems), "unit": "cell-updates/s",
               "h2d_bytes_per_step": 64 * n, "d2h_bytes_per_step": 64 * n, "steps": args.steps,
               "steps_replayed": "the timed window's steps, from its restart point", "ms_per_step": ems / args.steps,
               "same_work_as_timed_run": same}

    # roofline of the dominant kernel group
    peak, peak_kind = peaks()
    newton_its = st1["newton_it"] - st0["newton_it"]
    bicg_its = st1["bicg_it"] - st0["bicg_it"]
    stages = st1["stages"] - st0["stages"]
    # the HBM roofline is the BiCGStab solve's (the dominant memory-bound kernel); the FD Jacobian,
    # the residuals and the shock budget are FP64-arithmetic / latency bound (their shares are
    # in kernel_groups; profiles/ has their FP64-pipe figures)
    dom = "linear" if "linear" in groups and groups["linear"][1] > 0 else \
        max((g for g in groups if g in ALG_BYTES), key=lambda g: groups[g][0])
    gms, gcnt = groups[dom]
    if dom == "linear":
        units = bicg_its * n
    else:
        units = gcnt * n
    achieved = ALG_BYTES[dom] * units / (gms / 1e3) / 1e9
    # DRAM bytes per launch: the ncu-measured bytes per unit, scaled to this run's average launch
    traffic = DRAM_BYTES[dom] * units / max(gcnt, 1) if dom in DRAM_BYTES and args.workload == "bubbles1024" else None
    roof = {"bound": "hbm", "kernel": KERNEL_OF[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
            "alg_bytes_per_cell": ALG_BYTES[dom],
            "alg_bytes_per_launch": ALG_BYTES[dom] * units / max(gcnt, 1)}
    total_ms = sum(v[0] for v in groups.values())
    shares = {g: {"ms": round(v[0], 3), "launch_groups": int(v[1]), "share": round(v[0] / ms, 4)} for g, v in groups.items()}

    if rank == 0:
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world, "steps": steps_done,
            "warmup": args.warmup, "ms_per_step": ms_max / max(steps_done, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(case, args.workload),
            "bicg_iters_per_step": bicg_its / max(steps_done, 1),
            "newton_iters_per_stage": newton_its / max(stages, 1),
            "stages": stages, "rejects": st1["rejects"] - st0["rejects"],
            "roofline": roof, "kernel_groups": shares, "timed_groups_ms": round(total_ms, 3),
            "gpu_launches": launches, "clocks": clocks, "e2e": e2e,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(case)
        print(json.dumps(line))
    s.close()


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
