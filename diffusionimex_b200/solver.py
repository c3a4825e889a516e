"""Python host layer over the C ABI (include/spb6g.h).

Mirrors the reference driver's interface (src/SPB6_PC_IMEX_omp.cpp): a solver
object holds what main() keeps in globals and local grids; ``caldt``,
``step``, ``advance`` and the stage-level ``stage_dump`` correspond to caldt
(:502), one iteration of the time loop (:1316-1384), the loop itself, and
TVDReconstruction + Update + PressureSubsystem (:369, :264, :908).
Failures are reported as the reference does (a step that cannot be completed
after 30 halvings, a time-step underflow) by raising ``SolverError`` with the
library's status code.

The CUDA library must exist (``python -m diffusionimex_b200.build``); there is
no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from .build import LIB

NV = 8

STATUS = {
    0: "ok", 1: "inadmissible state", 2: "Newton failed", 3: "BiCGStab failed", 4: "step failed after 30 halvings",
    5: "time step underflow", 6: "CUDA error", 7: "bad argument", 8: "unsupported configuration", 9: "no CUDA device",
    10: "grid larger than the allocation-free entry point's fixed scratch",
}


class SolverError(RuntimeError):
    def __init__(self, status: int, where: str):
        super().__init__(f"{where}: {STATUS.get(status, status)} (status {status})")
        self.status = status


class Config(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32),
        ("x0", ctypes.c_double), ("x1", ctypes.c_double), ("y0", ctypes.c_double), ("y1", ctypes.c_double),
        ("bc", ctypes.c_int32 * 4), ("bcu", ctypes.c_double * 4), ("bcp", ctypes.c_double * 4),
        ("gamma", ctypes.c_double * 2), ("pinf", ctypes.c_double * 2), ("q", ctypes.c_double * 2),
        ("qp", ctypes.c_double * 2), ("cv", ctypes.c_double * 2), ("b", ctypes.c_double * 2),
        ("rk", ctypes.c_int32), ("cfl", ctypes.c_double), ("cfl_ac", ctypes.c_double), ("ramp", ctypes.c_int32),
        ("dtfix", ctypes.c_double), ("rus_local", ctypes.c_int32), ("limiter", ctypes.c_int32), ("acdt", ctypes.c_int32),
        ("newton_tol", ctypes.c_double), ("newton_iter", ctypes.c_int32), ("bicg_tol", ctypes.c_double),
        ("bicg_iter", ctypes.c_int32), ("share_mode", ctypes.c_int32), ("tend", ctypes.c_double),
        ("device", ctypes.c_int32), ("precision", ctypes.c_int32), ("kind", ctypes.c_int32 * 2),
        ("relax", ctypes.c_int32), ("jreuse", ctypes.c_int32), ("order", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 1),
        ("mg_G", ctypes.c_double * 2), ("mg_rr", ctypes.c_double * 2), ("mg_c1", ctypes.c_double * 2),
        ("mg_c2", ctypes.c_double * 2), ("mg_e1", ctypes.c_double * 2), ("mg_e2", ctypes.c_double * 2),
        ("mg_e0", ctypes.c_double * 2), ("eps_i", ctypes.c_double),
        ("mu_rate", ctypes.c_double), ("theta_rate", ctypes.c_double), ("nu_rate", ctypes.c_double),
        ("nu_cr", ctypes.c_double), ("nu_pc", ctypes.c_double), ("relax_form", ctypes.c_int32),
        ("unify", ctypes.c_int32), ("unify_proj", ctypes.c_int32), ("nu_law", ctypes.c_int32),
    ]
RATE_KEYS = ("mu_rate", "theta_rate", "nu_rate", "nu_cr", "nu_pc", "relax_form", "unify", "unify_proj", "nu_law")


class Stats(ctypes.Structure):
    _fields_ = [
        ("steps", ctypes.c_int64), ("rejects", ctypes.c_int64), ("rk1", ctypes.c_int64), ("stages", ctypes.c_int64),
        ("newton_it", ctypes.c_int64), ("floor_count", ctypes.c_int64), ("bicg_it", ctypes.c_int64),
        ("learned", ctypes.c_int64), ("t", ctypes.c_double), ("dt", ctypes.c_double), ("maxres", ctypes.c_double),
        ("p_ref", ctypes.c_double), ("tmax", ctypes.c_double * 2), ("learned_x0", ctypes.c_int64),
        ("extrapolated", ctypes.c_int64), ("extrapolated2", ctypes.c_int64), ("combined", ctypes.c_int64),
        ("refined", ctypes.c_int64),
    ]


class Output(ctypes.Structure):
    _fields_ = [
        ("out_file", ctypes.c_char_p), ("snaps", ctypes.c_void_p), ("nsnap", ctypes.c_int32), ("probe", ctypes.c_int32),
        ("probe_x", ctypes.c_double), ("probe_y", ctypes.c_double), ("prec", ctypes.c_int32),
    ]


_lib = None


def library() -> ctypes.CDLL:
    """Load libspb6g.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        raise RuntimeError(f"CUDA library missing: {LIB}; run `python -m diffusionimex_b200.build`")
    lib = ctypes.CDLL(LIB)
    P, I, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    sig = {
        "spb6g_default_config": (None, [P]),
        "spb6g_create": (I, [P, P]),
        "spb6g_destroy": (I, [P]),
        "spb6g_upload_state": (I, [P, P, I]),
        "spb6g_download_state": (I, [P, P, I]),
        "spb6g_init_pressure": (I, [P]),
        "spb6g_set_pressure": (I, [P, P, D]),
        "spb6g_get_pressure": (I, [P, P, P]),
        "spb6g_caldt": (I, [P, I, P]),
        "spb6g_step": (I, [P]),
        "spb6g_advance": (I, [P, I]),
        "spb6g_stage_dump": (I, [P, D, P, P, P, P, P, P]),
        "spb6g_get_stats": (I, [P, P]),
        "spb6g_set_output": (I, [P, P]),
        "spb6g_write_profile": (I, [P, ctypes.c_char_p, I]),
        "spb6g_format_profile": (I, [P, P, ctypes.c_char_p, I]),
        "spb6g_conserved_totals": (I, [P, P]),
        "spb6g_stats_line": (I, [P, I, D, ctypes.c_char_p, ctypes.c_size_t]),
        "spb6g_set_time": (I, [P, D, D, I]),
        "spb6g_get_time": (I, [P, P, P, P]),
        "spb6g_timing_enable": (I, [P, I]),
        "spb6g_timing_get": (I, [P, P, P, I, P]),
        "spb6g_timing_name": (ctypes.c_char_p, [I]),
        "spb6g_status_string": (ctypes.c_char_p, [I]),
        "spb6g_region_begin": (I, [P]),
        "spb6g_region_end": (I, [P, P]),
        "spb6g_kernel_launches": (ctypes.c_int64, [P]),
        "spb6g_stage_data": (I, [P, P, P, P, P]),
        "spb6g_stage": (I, [P, I, P, P, D, P]),
        "spb6g_stage_accept": (I, [P, D]),
        "spb6g_caldt_noalloc": (I, [P, P, I, P, P]),
        "spb6g_saturation_table": (I, [P, P, I, P]),
        "spb6g_batch_create": (I, [P, I, P]),
        "spb6g_batch_destroy": (None, [P]),
        "spb6g_batch_instance": (P, [P, I]),
        "spb6g_batch_status": (I, [P, I]),
        "spb6g_batch_set_shape": (I, [P, I, I]),
        "spb6g_batch_advance": (I, [P, I, P]),
        "spb6g_batch_autotune": (I, [P, I, P, P, P]),
        "spb6g_batch_launches": (I, [P]),
        "spb6g_batch_block_sizes": (I, [P, I, I, ctypes.c_int64, P, P]),
        "spb6g_set_feature_norm": (I, [P, P]),
        "spb6g_set_warmstart": (I, [P, P]),
        "spb6g_set_warmstart_mode": (I, [P, I]),
        "spb6g_set_warmstart_smoothing": (I, [P, I]),
        "spb6g_set_dump": (I, [P, P, P, ctypes.c_int64]),
        "spb6g_dump_count": (I, [P, P]),
        "spb6g_mlp_create": (I, [I, P]),
        "spb6g_mlp_destroy": (None, [P]),
        "spb6g_mlp_param_count": (I, []),
        "spb6g_mlp_set_params": (I, [P, P]),
        "spb6g_mlp_get_params": (I, [P, P]),
        "spb6g_mlp_forward": (I, [P, P, I, P, P]),
        "spb6g_mlp_train_step": (I, [P, P, P, I, ctypes.c_float, P, P]),
        "spb6g_mlp_train_async": (I, [P, P, P, I, ctypes.c_float, P]),
        "spb6g_mlp_last_loss": (I, [P, P, P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype, f.argtypes = res, args
    _lib = lib
    return lib


def make_config(case: dict, device: int = 0) -> Config:
    c = Config()
    library().spb6g_default_config(ctypes.byref(c))
    for k in ("nx", "ny", "rk", "ramp", "rus_local", "limiter", "acdt", "newton_iter", "bicg_iter", "share_mode"):
        setattr(c, k, int(case[k]))
    for k in ("x0", "x1", "y0", "y1", "cfl", "cfl_ac", "dtfix", "newton_tol", "bicg_tol", "tend"):
        setattr(c, k, float(case[k]))
    for q in range(4):
        c.bc[q] = int(case["bc"][q])
        c.bcu[q] = float(case["bcu"][q])
        c.bcp[q] = float(case["bcp"][q])
    for k in range(2):
        ph = case["phases"][k]
        c.gamma[k], c.pinf[k], c.q[k], c.qp[k], c.cv[k], c.b[k] = ph["g"], ph["pinf"], ph["q"], ph["qp"], ph["cv"], ph["b"]
        c.kind[k] = int(ph.get("kind", 0))
        for f in ("G", "rr", "c1", "c2", "e1", "e2", "e0"):
            getattr(c, "mg_" + f)[k] = float(ph.get(f, 0.0))
    c.device = device
    c.precision = int(case.get("precision", 0))
    c.relax = int(case.get("relax", 0))
    c.jreuse = int(case.get("jreuse", 0))
    c.order = int(case.get("order", 2))
    c.eps_i = float(case.get("eps_i", 1e-4))
    for k in RATE_KEYS:  # absent keys keep spb6g_default_config's values
        if k in case:
            setattr(c, k, type(getattr(c, k))(case[k]))
    return c


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def saturation_table(case: dict) -> dict:
    """The saturation line of the case's two phases as chemical relaxation uses it (host only):
    n points ln p, Tsat(p), the critical pressure and volume and the lowest tabulated pressure
    (build_sat, src/spb6_physics_omp.h:127-153)."""
    lib = library()
    cfg = make_config(case)
    n = ctypes.c_int()
    rc = lib.spb6g_saturation_table(ctypes.byref(cfg), None, 0, ctypes.byref(n))
    if rc != 0:
        raise SolverError(rc, "spb6g_saturation_table")
    buf = np.empty(n.value, dtype=np.float64)
    rc = lib.spb6g_saturation_table(ctypes.byref(cfg), _ptr(buf), n.value, ctypes.byref(n))
    if rc != 0:
        raise SolverError(rc, "spb6g_saturation_table")
    k = int(buf[0])
    return {"raw": buf, "n": k, "pcrit": buf[1], "vcrit": buf[2], "pmin": buf[3], "lp": buf[4:4 + k],
            "T": buf[4 + k:4 + 2 * k]}


def format_profile(case: dict, U: np.ndarray, path: str, prec: int = 16):
    """The reference's 17-column profile of a host state U (ny, nx, 8) on the case's grid (host code)."""
    lib = library()
    cfg = make_config(case, 0)
    U = np.ascontiguousarray(U, dtype=np.float64)
    rc = lib.spb6g_format_profile(ctypes.byref(cfg), _ptr(U), path.encode(), int(prec))
    if rc != 0:
        raise SolverError(rc, "spb6g_format_profile")


def run_main(case: dict, out_file: str, snaps=(), probe=None, prec: int = 16, device: int = 0) -> str:
    """The output sequence of the reference's main() (src/SPB6_PC_IMEX_omp.cpp:1305-1427) on one
    case: probe line at t = 0, steps to t_end with snapshots and probe lines, final profile;
    returns its end-of-run line (wall time of the time loop)."""
    import time

    s = Solver(case, device=device)
    try:
        s.set_output(out_file, snaps=snaps, probe=probe, prec=prec)
        t0 = time.perf_counter()
        s.advance(0)
        return s.stats_line(int(case.get("case", 0)), time.perf_counter() - t0)
    finally:
        s.close()


class Solver:
    """One grid on one GPU: state, pressure unknown, time and statistics."""

    def __init__(self, case: dict, device: int = 0, init_pressure: bool = True):
        self.lib = library()
        self.case = case
        self.nx, self.ny = int(case["nx"]), int(case["ny"])
        self.cfg = make_config(case, device)
        h = ctypes.c_void_p()
        self._check(self.lib.spb6g_create(ctypes.byref(self.cfg), ctypes.byref(h)), "spb6g_create")
        self.h = h
        if "U" in case:
            self.upload(case["U"])
            if init_pressure:
                self.init_pressure()

    def _check(self, rc: int, where: str):
        if rc != 0:
            raise SolverError(rc, where)

    def close(self):
        if getattr(self, "h", None) and not getattr(self, "_borrowed", False):
            self.lib.spb6g_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # state ------------------------------------------------------------------------------
    def upload(self, U: np.ndarray):
        U = np.ascontiguousarray(U, dtype=np.float64).reshape(self.ny, self.nx, NV)
        self._check(self.lib.spb6g_upload_state(self.h, _ptr(U), 0), "spb6g_upload_state")

    def state(self) -> np.ndarray:
        U = np.empty((self.ny, self.nx, NV))
        self._check(self.lib.spb6g_download_state(self.h, _ptr(U), 0), "spb6g_download_state")
        return U

    def init_pressure(self):
        self._check(self.lib.spb6g_init_pressure(self.h), "spb6g_init_pressure")

    def pressure(self):
        P = np.empty((self.ny, self.nx))
        pref = ctypes.c_double()
        self._check(self.lib.spb6g_get_pressure(self.h, _ptr(P), ctypes.byref(pref)), "spb6g_get_pressure")
        return P, pref.value

    def set_pressure(self, P: np.ndarray, p_ref: float):
        P = np.ascontiguousarray(P, dtype=np.float64)
        self._check(self.lib.spb6g_set_pressure(self.h, _ptr(P), float(p_ref)), "spb6g_set_pressure")

    def time_state(self) -> tuple[float, float, bool]:
        """(t, dtprev, startup): with the state and the pressure, a restart point."""
        t, dtp, su = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._check(self.lib.spb6g_get_time(self.h, ctypes.byref(t), ctypes.byref(dtp), ctypes.byref(su)), "get_time")
        return t.value, dtp.value, bool(su.value)

    def set_time(self, t: float, dtprev: float, startup: bool):
        self._check(self.lib.spb6g_set_time(self.h, float(t), float(dtprev), int(startup)), "set_time")

    def restart_point(self) -> dict:
        """Everything the next step depends on (state, pressure unknown, time-loop state)."""
        P, pref = self.pressure()
        return {"U": self.state(), "P": P, "p_ref": pref, "time": self.time_state()}

    def restore(self, rp: dict):
        self.upload(rp["U"])
        self.set_pressure(rp["P"], rp["p_ref"])
        self.set_time(*rp["time"])

    # reference driver entry points --------------------------------------------------------
    def caldt(self, acoustic: bool = False) -> float:
        out = ctypes.c_double()
        self._check(self.lib.spb6g_caldt(self.h, int(acoustic), ctypes.byref(out)), "caldt")
        return out.value

    def step(self):
        self._check(self.lib.spb6g_step(self.h), "step")

    def advance(self, nsteps: int = 0):
        """nsteps > 0: that many steps (or until t_end); 0: run to t_end."""
        self._check(self.lib.spb6g_advance(self.h, int(nsteps)), "advance")

    def stage_dump(self, dt: float) -> dict:
        nx, ny = self.nx, self.ny
        out = dict(Xs=np.empty((ny, nx, NV)), a2s=np.empty((ny, nx)), ube_x=np.empty((ny, nx + 1)),
                   ube_y=np.empty((ny + 1, nx)), phi_x=np.empty((ny, nx)), phi_y=np.empty((ny, nx)))
        self._check(self.lib.spb6g_stage_dump(self.h, float(dt), *(_ptr(out[k]) for k in
                                                                  ("Xs", "a2s", "ube_x", "ube_y", "phi_x", "phi_y"))),
                    "stage_dump")
        return out

    def stage(self, rks: int, Ae_row, Ai_row, dt: float) -> int:
        """Stage rks of the current attempt (spb6g_stage: TVDReconstruction + Update +
        PressureSubsystem with Qe, Qs combined from Ae_row, Ai_row and adt = Ai_row[rks] dt).
        Returns 0 when the stage converged, else the failure status (1 inadmissible, 2 Newton,
        3 BiCGStab), after which the caller halves dt and starts again at rks = 0, as main()
        does (:1366-1376); bad arguments and CUDA errors raise."""
        ae = np.ascontiguousarray(list(Ae_row[:rks]) + [0.0], dtype=np.float64)
        ai = np.ascontiguousarray(list(Ai_row[:rks + 1]), dtype=np.float64)
        rc = self.lib.spb6g_stage(self.h, int(rks), _ptr(ae), _ptr(ai), float(dt), None)
        if rc not in (0, 1, 2, 3):
            raise SolverError(rc, "spb6g_stage")
        return rc

    def stage_accept(self, dt: float):
        """Accept the attempt: the state and the pressure of its last stage become U^n and P (:1374)."""
        self._check(self.lib.spb6g_stage_accept(self.h, float(dt)), "spb6g_stage_accept")

    def stage_data(self) -> dict:
        """Face coefficients, residual scale and shock budget of the last stage."""
        nx, ny, n = self.nx, self.ny, self.nx * self.ny
        fx = np.empty((4, ny, nx + 1))
        fy = np.empty((4, ny + 1, nx))
        kw = np.empty((ny, nx))
        qph = np.empty((2, ny, nx))
        self._check(self.lib.spb6g_stage_data(self.h, _ptr(fx), _ptr(fy), _ptr(kw), _ptr(qph)), "stage_data")
        out = {f"fx_{k}": fx[q] for q, k in enumerate(("ubs", "kp", "wl", "pv"))}
        out.update({f"fy_{k}": fy[q] for q, k in enumerate(("ubs", "kp", "wl", "pv"))})
        out.update(kw=kw, qph0=qph[0], qph1=qph[1])
        return out

    def stats(self) -> dict:
        s = Stats()
        self._check(self.lib.spb6g_get_stats(self.h, ctypes.byref(s)), "spb6g_get_stats")
        out = {}
        for k, _ in Stats._fields_:
            v = getattr(s, k)
            out[k] = list(v) if isinstance(v, ctypes.Array) else v
        return out

    # ---- output of the reference's main() (profile, snapshots, probe, stats line)
    def set_output(self, out_file: str | None, snaps=(), probe=None, prec: int = 16):
        """Files main() writes: the final profile `out_file` (at t_end or when a step fails),
        `<out>_s<k>.dat` at the snapshot times (the step size lands on them) and, with
        probe=(x, y), `<out>.probe` with one line before the first step and one per step."""
        if not out_file:
            self._check(self.lib.spb6g_set_output(self.h, None), "set_output")
            return
        self._snaps = np.ascontiguousarray(snaps, dtype=np.float64)
        o = Output(out_file.encode(), self._snaps.ctypes.data if len(self._snaps) else None, len(self._snaps),
                   1 if probe is not None else 0, float(probe[0]) if probe is not None else 0.0,
                   float(probe[1]) if probe is not None else 0.0, int(prec))
        self._check(self.lib.spb6g_set_output(self.h, ctypes.byref(o)), "set_output")

    def write_profile(self, path: str, prec: int = 16):
        self._check(self.lib.spb6g_write_profile(self.h, path.encode(), int(prec)), "write_profile")

    def conserved_totals(self):
        M = np.empty(3)
        self._check(self.lib.spb6g_conserved_totals(self.h, _ptr(M)), "conserved_totals")
        return M

    def stats_line(self, case_id: int, wall_s: float = 0.0) -> str:
        buf = ctypes.create_string_buffer(1024)
        self._check(self.lib.spb6g_stats_line(self.h, int(case_id), float(wall_s), buf, len(buf)), "stats_line")
        return buf.value.decode()

    def region_begin(self):
        self._check(self.lib.spb6g_region_begin(self.h), "region_begin")

    def region_end(self) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.spb6g_region_end(self.h, ctypes.byref(ms)), "region_end")
        return ms.value

    # ---- learned warm start (no counterpart in the reference)
    NORM_LEN = 22

    def set_feature_norm(self, norm):
        """22 values: mean[7], std[7] of the centre values, std[7] of the neighbour differences of
        (rho, rho u, rho v, alpha1, E*, P - P_REF, R), R the last converged stage's pressure rate,
        then the target scale.  Setting it starts the tracking of R."""
        if len(norm) != self.NORM_LEN:
            raise ValueError(f"feature normalisation has {self.NORM_LEN} values, got {len(norm)}")
        a = (ctypes.c_double * self.NORM_LEN)(*[float(v) for v in norm])
        self._check(self.lib.spb6g_set_feature_norm(self.h, a), "spb6g_set_feature_norm")

    def set_warmstart(self, mlp, mode: int = 15, smooth: int = 0):
        """mode bits -- 1: learned Newton start (the guess of smallest residual among the plain guess,
        the extrapolation and the network's); 2: learned first BiCGStab iterate; 4: the last Newton
        correction as the first iterate's candidate of the stage's later solves.  smooth: radius of
        the box average of the network's output (0: none)."""
        self._warm = mlp
        self._check(self.lib.spb6g_set_warmstart(self.h, mlp.handle if mlp is not None else None), "spb6g_set_warmstart")
        if mlp is not None:
            self._check(self.lib.spb6g_set_warmstart_mode(self.h, int(mode)), "spb6g_set_warmstart_mode")
            self._check(self.lib.spb6g_set_warmstart_smoothing(self.h, int(smooth)), "spb6g_set_warmstart_smoothing")

    def set_dump(self, X=None, t=None):
        """X: (cap, 64) torch.bfloat16, t: (cap,) torch.float32 on the device, or None to stop."""
        self._dump = (X, t)
        if X is None:
            self._check(self.lib.spb6g_set_dump(self.h, None, None, 0), "spb6g_set_dump")
            return
        assert X.shape[0] == t.shape[0] and X.shape[1] == 64
        self._check(self.lib.spb6g_set_dump(self.h, X.data_ptr(), t.data_ptr(), X.shape[0]), "spb6g_set_dump")

    def dump_count(self) -> int:
        v = ctypes.c_int64()
        self._check(self.lib.spb6g_dump_count(self.h, ctypes.byref(v)), "spb6g_dump_count")
        return v.value

    def kernel_launches(self) -> int:
        return int(self.lib.spb6g_kernel_launches(self.h))

    def upload_soa(self, ptr: int):
        """Upload from a host buffer (pointer) in k-major SoA layout (8 x ny x nx doubles)."""
        self._check(self.lib.spb6g_upload_state(self.h, ctypes.c_void_p(ptr), 1), "spb6g_upload_state")

    def download_soa(self, ptr: int):
        self._check(self.lib.spb6g_download_state(self.h, ctypes.c_void_p(ptr), 1), "spb6g_download_state")

    def timing(self, enable: bool | None = None) -> dict:
        if enable is not None:
            self._check(self.lib.spb6g_timing_enable(self.h, int(enable)), "timing")
            return {}
        ms = (ctypes.c_double * 16)()
        cnt = (ctypes.c_int64 * 16)()
        ng = ctypes.c_int()
        self._check(self.lib.spb6g_timing_get(self.h, ms, cnt, 16, ctypes.byref(ng)), "timing")
        return {self.lib.spb6g_timing_name(g).decode(): (ms[g], cnt[g]) for g in range(ng.value)}


def batch_block_sizes(cells, threads: int, slots: int = 0):
    """Block size of each grid of a batch (spb6g_batch_block_sizes; host only): threads in proportion
    to its cells, a multiple of 32 from 32 to `threads`, with the fewest cells per thread for which
    the blocks' threads fit in `slots` (0: no limit).  Returns (block sizes, cells per thread)."""
    lib = library()
    c = np.ascontiguousarray(cells, dtype=np.int64)
    out = np.zeros(len(c), dtype=np.int32)
    per = ctypes.c_int64()
    rc = lib.spb6g_batch_block_sizes(_ptr(c), int(len(c)), int(threads), int(slots), _ptr(out), ctypes.byref(per))
    if rc != 0:
        raise SolverError(rc, "spb6g_batch_block_sizes")
    return out, per.value


class BatchSolver:
    """Independent 1D grids advanced together: one persistent launch (a captured CUDA graph),
    one thread block per grid.  `instance(i)` is an ordinary Solver view of grid i."""

    def __init__(self, case_list, device: int = 0, init_pressure: bool = True):
        self.lib = library()
        self.cases = list(case_list)
        cfgs = (Config * len(self.cases))(*[make_config(c, device) for c in self.cases])
        h = ctypes.c_void_p()
        rc = self.lib.spb6g_batch_create(cfgs, len(self.cases), ctypes.byref(h))
        if rc != 0:
            raise SolverError(rc, "spb6g_batch_create")
        self.h = h
        self._inst = []
        for i, c in enumerate(self.cases):
            v = Solver.__new__(Solver)
            v.lib, v.case, v.nx, v.ny = self.lib, c, int(c["nx"]), int(c["ny"])
            v.cfg, v._borrowed = cfgs[i], True
            v.h = ctypes.c_void_p(self.lib.spb6g_batch_instance(h, i))
            if "U" in c:
                v.upload(c["U"])
                if init_pressure:
                    v.init_pressure()
            self._inst.append(v)

    def __len__(self):
        return len(self._inst)

    def instance(self, i: int) -> Solver:
        return self._inst[i]

    def set_shape(self, threads: int, tile: int):
        self._check(self.lib.spb6g_batch_set_shape(self.h, threads, tile), "spb6g_batch_set_shape")

    def advance(self, nsteps: int) -> float:
        """nsteps steps of every grid; returns the launch's device time in ms."""
        ms = ctypes.c_float()
        self._check(self.lib.spb6g_batch_advance(self.h, int(nsteps), ctypes.byref(ms)), "spb6g_batch_advance")
        return ms.value

    def autotune(self, nsteps: int = 2):
        t, w, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        self._check(self.lib.spb6g_batch_autotune(self.h, int(nsteps), ctypes.byref(t), ctypes.byref(w), ctypes.byref(ms)),
                    "spb6g_batch_autotune")
        return t.value, w.value, ms.value

    def status(self, i: int) -> int:
        return self.lib.spb6g_batch_status(self.h, i)

    def launches(self) -> int:
        """Kernel launches of one advance under the current shape (one per block size)."""
        return self.lib.spb6g_batch_launches(self.h)

    def close(self):
        if getattr(self, "h", None):
            for v in self._inst:
                v.h = None
            self.lib.spb6g_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _check(rc, where):
        if rc != 0:
            raise SolverError(rc, where)
