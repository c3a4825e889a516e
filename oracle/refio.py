"""Test infrastructure: read/write the oracle case and result records (oracle/spb6_case.h)
and run the two CPU oracles

* ``run_ref``   -- oracle/_ref/spb6_ref, the reference solver compiled from its own sources;
* ``run_port``  -- oracle/_build/libspb6_oracle.so, the C restatement (spb6_oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "_ref", "spb6_ref")
REF_BIN_ULP = os.path.join(HERE, "_ref", "spb6_ref_ulp")  # log / exp / pow one ulp up (ulp_libm.c)
PORT_LIB = os.path.join(HERE, "_build", "libspb6_oracle.so")
MAGIC = 0x36425053
MODE_STEPS, MODE_TEND, MODE_STAGE, MODE_SAT = 0, 1, 2, 3

CASE_DT = np.dtype([
    ("magic", "<u4"), ("version", "<i4"), ("nx", "<i4"), ("ny", "<i4"), ("bc", "<i4", 4),
    ("rk", "<i4"), ("ramp", "<i4"), ("rus_local", "<i4"), ("limiter", "<i4"), ("acdt", "<i4"),
    ("newton_iter", "<i4"), ("bicg_iter", "<i4"), ("share_mode", "<i4"), ("mode", "<i4"), ("nsteps", "<i4"),
    ("threads", "<i4"), ("order", "<i4"),
    ("x0", "<f8"), ("x1", "<f8"), ("y0", "<f8"), ("y1", "<f8"), ("bcu", "<f8", 4), ("bcp", "<f8", 4),
    ("g", "<f8", 2), ("pinf", "<f8", 2), ("q", "<f8", 2), ("qp", "<f8", 2), ("cv", "<f8", 2), ("b", "<f8", 2),
    ("cfl", "<f8"), ("cfl_ac", "<f8"), ("dtfix", "<f8"), ("newton_tol", "<f8"), ("bicg_tol", "<f8"), ("tend", "<f8"),
    ("budget_s", "<f8"), ("warmup", "<i4"), ("inject_qph", "<i4"),
    ("kind", "<i4", 2), ("mg_G", "<f8", 2), ("mg_rr", "<f8", 2), ("mg_c1", "<f8", 2), ("mg_c2", "<f8", 2),
    ("mg_e1", "<f8", 2), ("mg_e2", "<f8", 2), ("mg_e0", "<f8", 2), ("relax", "<i4"), ("jreuse", "<i4"),
    ("eps_i", "<f8"),
    ("mu_rate", "<f8"), ("theta_rate", "<f8"), ("nu_rate", "<f8"), ("nu_cr", "<f8"), ("nu_pc", "<f8"),
    ("relax_form", "<i4"), ("unify", "<i4"), ("unify_proj", "<i4"), ("nu_law", "<i4"),
])
# relaxation-rate settings of a case and their defaults (the reference's, physics :34-46)
RATE_DEFAULTS = {"mu_rate": float("inf"), "theta_rate": -1.0, "nu_rate": -1.0, "nu_cr": 1.0, "nu_pc": 22.064e6,
                 "relax_form": 0, "unify": 0, "unify_proj": 1, "nu_law": 0}
MG_KEYS = ("G", "rr", "c1", "c2", "e1", "e2", "e0")
RESULT_DT = np.dtype([
    ("magic", "<u4"), ("status", "<i4"), ("nx", "<i4"), ("ny", "<i4"),
    ("steps", "<i8"), ("rejects", "<i8"), ("rk1", "<i8"), ("stages", "<i8"), ("newton_it", "<i8"),
    ("floor_count", "<i8"), ("bicg_it", "<i8"), ("timed_steps", "<i8"),
    ("t", "<f8"), ("dt", "<f8"), ("maxres", "<f8"), ("p_ref", "<f8"), ("wall_s", "<f8"), ("dM", "<f8", 3),
])


def case_record(cfg: dict, mode: int = MODE_STEPS, nsteps: int = 1, threads: int = 0, warmup: int = 0,
                budget_s: float = 0.0) -> np.ndarray:
    r = np.zeros((), CASE_DT)
    r["magic"], r["version"] = MAGIC, 4
    for k in ("nx", "ny", "rk", "ramp", "rus_local", "limiter", "acdt", "newton_iter", "bicg_iter", "share_mode"):
        r[k] = int(cfg[k])
    r["bc"] = cfg["bc"]
    r["mode"], r["nsteps"], r["threads"] = mode, nsteps, threads
    r["warmup"], r["budget_s"] = warmup, budget_s
    for k in ("x0", "x1", "y0", "y1", "cfl", "cfl_ac", "dtfix", "newton_tol", "bicg_tol", "tend"):
        r[k] = float(cfg[k])
    r["bcu"], r["bcp"] = cfg["bcu"], cfg["bcp"]
    for f in ("g", "pinf", "q", "qp", "cv", "b"):
        r[f] = [cfg["phases"][0][f], cfg["phases"][1][f]]
    r["kind"] = [int(cfg["phases"][k].get("kind", 0)) for k in range(2)]
    for f in MG_KEYS:
        r["mg_" + f] = [float(cfg["phases"][k].get(f, 0.0)) for k in range(2)]
    r["relax"] = int(cfg.get("relax", 0))
    r["jreuse"] = int(cfg.get("jreuse", 0))
    r["order"] = int(cfg.get("order", 2))
    r["eps_i"] = float(cfg.get("eps_i", 1e-4))
    for k, v in RATE_DEFAULTS.items():
        r[k] = type(v)(cfg.get(k, v))
    return r


def parse_result(buf: bytes, nx: int, ny: int, mode: int) -> dict:
    res = np.frombuffer(buf[:RESULT_DT.itemsize], RESULT_DT)[0]
    arr = np.frombuffer(buf[RESULT_DT.itemsize:], "<f8")
    n = nx * ny
    out = {k: res[k].item() if res[k].ndim == 0 else np.array(res[k]) for k in RESULT_DT.names}
    o = 0
    out["U"] = arr[o:o + n * 8].reshape(ny, nx, 8).copy(); o += n * 8
    out["P"] = arr[o:o + n].reshape(ny, nx).copy() if arr.size >= o + n else None; o += n
    if mode == MODE_SAT:  # n, pcrit, vcrit, pmin, ln p[n], Tsat[n]
        out["sat"] = arr[o:].copy()
        return out
    if mode == MODE_STAGE and arr.size > o:
        out["Xs"] = arr[o:o + n * 8].reshape(ny, nx, 8).copy(); o += n * 8
        out["a2s"] = arr[o:o + n].reshape(ny, nx).copy(); o += n
        out["ube_x"] = arr[o:o + (nx + 1) * ny].reshape(ny, nx + 1).copy(); o += (nx + 1) * ny
        out["ube_y"] = arr[o:o + nx * (ny + 1)].reshape(ny + 1, nx).copy(); o += nx * (ny + 1)
        out["phi_x"] = arr[o:o + n].reshape(ny, nx).copy(); o += n
        out["phi_y"] = arr[o:o + n].reshape(ny, nx).copy(); o += n
        if arr.size >= o + 4 * (nx + 1) * ny + 4 * nx * (ny + 1) + 3 * n:  # stage data (C restatement only)
            for k in ("fx_ubs", "fx_kp", "fx_wl", "fx_pv"):
                out[k] = arr[o:o + (nx + 1) * ny].reshape(ny, nx + 1).copy(); o += (nx + 1) * ny
            for k in ("fy_ubs", "fy_kp", "fy_wl", "fy_pv"):
                out[k] = arr[o:o + nx * (ny + 1)].reshape(ny + 1, nx).copy(); o += nx * (ny + 1)
            for k in ("kw", "qph0", "qph1"):
                out[k] = arr[o:o + n].reshape(ny, nx).copy(); o += n
    return out


def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def run_ref(cfg: dict, mode: int = MODE_STEPS, nsteps: int = 1, threads: int = 0, timeout: float = 3600,
            warmup: int = 0, budget_s: float = 0.0, variant: str | None = None) -> dict:
    """Run the reference solver (compiled from its sources) on cfg['U'].  With `warmup`, the first
    steps are excluded from wall_s; with `budget_s`, stepping stops once the timed steps used it.
    variant "ulp" / "ulpdown": the reference with its log / exp / pow results one ulp up / down."""
    U = np.ascontiguousarray(cfg["U"], dtype="<f8")
    with tempfile.TemporaryDirectory() as d:
        ci, co = os.path.join(d, "case.bin"), os.path.join(d, "out.bin")
        with open(ci, "wb") as f:
            f.write(case_record(cfg, mode, nsteps, threads, warmup, budget_s).tobytes())
            f.write(U.tobytes())
        env = dict(os.environ)
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        if variant == "ulpdown":
            env["SPB6_ULP_DOWN"] = "1"
        subprocess.run([REF_BIN_ULP if variant in ("ulp", "ulpdown") else REF_BIN, ci, co], check=True,
                       timeout=timeout, env=env)
        with open(co, "rb") as f:
            return parse_result(f.read(), cfg["nx"], cfg["ny"], mode)


def run_ref_main(args: list[str], nx: int, ny: int = 1, timeout: float = 3600) -> dict:
    """Run the reference's own main() (key=value arguments) and return its final state."""
    with tempfile.TemporaryDirectory() as d:
        co = os.path.join(d, "out.bin")
        subprocess.run([REF_BIN, "--main", co, *args], check=True, timeout=timeout,
                       stdout=subprocess.DEVNULL)
        with open(co, "rb") as f:
            return parse_result(f.read(), nx, ny, MODE_STEPS)


def run_ref_main_files(args: list[str], out_name: str = "run.dat", timeout: float = 3600, nx: int = 0,
                       ny: int = 1) -> dict:
    """Run the reference's own main() with out=<tmp>/<out_name> and the given key=value
    arguments; returns {"files": {name: bytes} of every file it wrote, "stdout": text} and,
    with nx given, "U": the state of the last profile it wrote."""
    with tempfile.TemporaryDirectory() as d:
        co = os.path.join(d, "result.bin")
        r = subprocess.run([REF_BIN, "--main-files", co, f"out={os.path.join(d, out_name)}", *args], check=True,
                           timeout=timeout, stdout=subprocess.PIPE, text=True)
        files = {}
        for name in sorted(os.listdir(d)):
            if name != "result.bin":
                with open(os.path.join(d, name), "rb") as f:
                    files[name] = f.read()
        out = {"files": files, "stdout": r.stdout}
        if nx:
            with open(co, "rb") as f:
                out["U"] = parse_result(f.read(), nx, ny, MODE_STEPS)["U"]
        return out


_port = {}
VARIANTS = {None: "libspb6_oracle.so", "ulp": "libspb6_oracle_ulp.so", "fd": "libspb6_oracle_fd.so"}


def _port_lib(variant=None):
    if variant not in _port:
        path = os.path.join(HERE, "_build", VARIANTS[variant])
        if not os.path.exists(path):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, stdout=subprocess.DEVNULL)
        lib = ctypes.CDLL(path)
        lib.spb6_oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
        lib.spb6_oracle_run.restype = ctypes.c_int
        _port[variant] = lib
    return _port[variant]


def run_port(cfg: dict, mode: int = MODE_STEPS, nsteps: int = 1, threads: int = 1, warmup: int = 0,
             budget_s: float = 0.0, variant: str | None = None, qph: np.ndarray | None = None) -> dict:
    """Run the C restatement on cfg['U'] (same record format as run_ref).

    variant: None, "ulp" (shock-shooting exp/log/pow one ulp up) or "fd" (FD Jacobian step
    1.01e-7) -- the round-off perturbations that define the reference's own noise level.
    qph: stage mode only -- (2, ny, nx) shock budget Q_1, Q_2 used instead of the computed one."""
    lib = _port_lib(variant)
    rec = case_record(cfg, mode, nsteps, threads, warmup, budget_s)
    U = np.ascontiguousarray(cfg["U"], dtype="<f8")
    if qph is not None:
        rec["inject_qph"] = 1
        U = np.concatenate([U.ravel(), np.ascontiguousarray(qph, dtype="<f8").ravel()])
    nx, ny = cfg["nx"], cfg["ny"]
    n = nx * ny
    cap = RESULT_DT.itemsize + 8 * (n * 8 + n + n * 8 + n + (nx + 1) * ny + nx * (ny + 1) + 2 * n
                                    + 4 * (nx + 1) * ny + 4 * nx * (ny + 1) + 3 * n)
    out = np.zeros(cap, np.uint8)
    size = lib.spb6_oracle_run(rec.ctypes.data, U.ctypes.data, out.ctypes.data, cap)
    if size <= 0:
        raise RuntimeError(f"oracle port rejected the case ({size})")
    return parse_result(out[:size].tobytes(), nx, ny, mode)
