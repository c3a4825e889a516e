"""Shared helpers for the parity tests: golden fixtures and field comparisons."""
from __future__ import annotations

import json
import os

import numpy as np

from diffusionimex_b200 import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELDS = ["alpha1", "m1", "m2", "rho_u", "rho_v", "eps1", "eps2", "E"]


def load_golden(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
    out = {k: z[k] for k in z.files if k != "meta"}
    out["meta"] = json.loads(str(z["meta"]))
    return out


def golden_case(name: str) -> tuple[dict, str, int]:
    """The case, mode and step count a fixture was made with (same builders as make_golden.py)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    c, mode, nsteps = mg.build_case(name)
    return c, mode, nsteps


def fieldwise_maxrel(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """max |a - b| / max |b| per conservative variable (field-max-normalised)."""
    a = a.reshape(-1, 8)
    b = b.reshape(-1, 8)
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return np.abs(a - b).max(axis=0) / scale


def fieldwise_l1(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """mean |a - b| / max |b| per conservative variable."""
    a = a.reshape(-1, 8)
    b = b.reshape(-1, 8)
    scale = np.maximum(np.abs(b).max(axis=0), 1e-300)
    return np.abs(a - b).mean(axis=0) / scale


def mixture_pressure(case: dict, U: np.ndarray) -> np.ndarray:
    """alpha1 p1 + alpha2 p2 of the reference profile writer (cell_diag, physics :1161-1172)."""
    ph = case["phases"]
    U = U.reshape(-1, 8)
    a1 = U[:, 0]
    p = []
    for k, (a, m, e) in enumerate(((a1, U[:, 1], U[:, 5]), (1 - a1, U[:, 2], U[:, 6]))):
        h = ph[k]
        p.append((e - m * h["q"]) * (h["g"] - 1.0) / (a - m * h["b"]) - h["g"] * h["pinf"])
    return a1 * p[0] + (1 - a1) * p[1]


__all__ = ["cases", "load_golden", "golden_case", "fieldwise_maxrel", "fieldwise_l1", "mixture_pressure", "FIELDS"]
