"""Test infrastructure: exact Riemann solutions, the secondary check of the solver.

Two solvers (numpy / scipy, no GPU); the tests compare whole GPU runs of Riemann problems
with them in the relative L1 density error the reference publishes (Eq. (51) of Schropff,
Petitpas & Daniel 2026, tests/plot_schropff.py:69-72 of the reference):

* ``stiffened_gas`` -- the Euler equations for two stiffened gases separated by a contact:
  the classical exact Riemann solver (Toro, "Riemann Solvers and Numerical Methods for Fluid
  Dynamics", ch. 4) with every pressure shifted by the gas's pi; the reference solves the
  same problem in tests/exact_sg.py:4-22.
* ``mixture`` -- the mechanical-equilibrium (5-equation, Kapila) model of a two-phase mixture
  whose mass fractions are uniform on each side: across a shock every phase follows its own
  Hugoniot at the common pressure (the shock relations of Saurel, Petitpas & Berry 2009,
  (II.5)), across a rarefaction every phase is isentropic and the mixture's sound speed is
  Wood's; NASG phases enter through their covolume b, whose excess volume v - b follows the
  stiffened-gas relations (the reference: tests/exact5.py:7-43).
"""
from __future__ import annotations

import numpy as np
from scipy.integrate import quad
from scipy.optimize import brentq


# ---------------------------------------------------------------------------- two stiffened gases
def stiffened_gas(left, right, x0: float, t: float, x):
    """left / right: (rho, u, p, gamma, pinf).  Returns rho(x), u(x), p(x) at time t, and p*, u*."""
    x = np.asarray(x, dtype=np.float64)

    def wave(p, rho, pk, g, pi):
        """Velocity change across the wave from state k to pressure p (positive for a shock)."""
        P, Pk = p + pi, pk + pi
        if p > pk:
            a = 2.0 / ((g + 1.0) * rho)
            b = (g - 1.0) / (g + 1.0) * Pk
            return (p - pk) * np.sqrt(a / (P + b))
        ck = np.sqrt(g * Pk / rho)
        return 2.0 * ck / (g - 1.0) * ((P / Pk) ** ((g - 1.0) / (2.0 * g)) - 1.0)

    rl, ul, pl, gl, pil = left
    rr, ur, pr, gr, pir = right
    F = lambda p: wave(p, rl, pl, gl, pil) + wave(p, rr, pr, gr, pir) + (ur - ul)
    lo = max(-pil, -pir)
    lo = lo + 1e-9 * max(abs(lo), 1.0)
    ps = brentq(F, lo, 10.0 * max(pl, pr) + 10.0 * max(pil, pir), xtol=1e-12, rtol=1e-15)
    us = 0.5 * (ul + ur) + 0.5 * (wave(ps, rr, pr, gr, pir) - wave(ps, rl, pl, gl, pil))
    xi = (x - x0) / t

    def one_side(rho, u, pk, g, pi, s):
        """Sample the side s (-1 left, +1 right) of the contact."""
        Pk, P = pk + pi, ps + pi
        ck = np.sqrt(g * Pk / rho)
        if ps > pk:  # shock
            rs = rho * ((P / Pk + (g - 1.0) / (g + 1.0)) / ((g - 1.0) / (g + 1.0) * P / Pk + 1.0))
            S = u + s * ck * np.sqrt((g + 1.0) / (2.0 * g) * P / Pk + (g - 1.0) / (2.0 * g))
            ahead = s * (xi - S) > 0
            return np.where(ahead, rho, rs), np.where(ahead, u, us), np.where(ahead, pk, ps)
        rs = rho * (P / Pk) ** (1.0 / g)
        cs = ck * (P / Pk) ** ((g - 1.0) / (2.0 * g))
        head, tail = u + s * ck, us + s * cs
        ahead, behind = s * (xi - head) > 0, s * (xi - tail) < 0
        # inside the fan: the characteristic through the origin, xi = u - s c
        cf = np.maximum(2.0 / (g + 1.0) * (ck - s * (g - 1.0) / 2.0 * (u - xi)), 1e-300)
        uf = 2.0 / (g + 1.0) * (-s * ck + (g - 1.0) / 2.0 * u + xi)
        rf = rho * (cf / ck) ** (2.0 / (g - 1.0))
        pf = Pk * (cf / ck) ** (2.0 * g / (g - 1.0)) - pi
        return (np.where(ahead, rho, np.where(behind, rs, rf)), np.where(ahead, u, np.where(behind, us, uf)),
                np.where(ahead, pk, np.where(behind, ps, pf)))

    L = one_side(rl, ul, pl, gl, pil, -1.0)
    R = one_side(rr, ur, pr, gr, pir, 1.0)
    m = xi < us
    return np.where(m, L[0], R[0]), np.where(m, L[1], R[1]), np.where(m, L[2], R[2]), ps, us


# ---------------------------------------------------------------------------- two-phase mixture
class MixtureState:
    """One side of the Riemann problem: phase volume fractions a_k and densities r_k, velocity u,
    pressure p, and the phases' gamma_k, pi_k, covolume b_k.  The mass fractions Y_k are fixed."""

    def __init__(self, a, r, u, p, gamma, pinf, b=(0.0, 0.0)):
        self.a = np.asarray(a, dtype=np.float64)
        self.r = np.asarray(r, dtype=np.float64)
        self.u, self.p = float(u), float(p)
        self.g = np.asarray(gamma, dtype=np.float64)
        self.pi = np.asarray(pinf, dtype=np.float64)
        self.b = np.asarray(b, dtype=np.float64)
        self.rho = float((self.a * self.r).sum())
        self.Y = self.a * self.r / self.rho
        self.w0 = 1.0 / self.r - self.b  # excess specific volumes v_k - b_k

    def phase_volumes(self, p, shock: bool):
        """v_k(p): along each phase's Hugoniot (shock) or isentrope from the state."""
        P, P0 = p + self.pi, self.p + self.pi
        g = self.g
        if shock:
            w = self.w0 * ((g - 1.0) * P + (g + 1.0) * P0) / ((g + 1.0) * P + (g - 1.0) * P0)
        else:
            w = self.w0 * (P0 / P) ** (1.0 / g)
        return self.b + w

    def volume(self, p, shock: bool) -> float:
        return float((self.Y * self.phase_volumes(p, shock)).sum())

    def impedance(self, p) -> float:
        """rho c along the isentrope (Wood's sound speed): (rho c)^-2 = -dv/dp = sum Y_k w_k / (gamma_k P_k)."""
        w = self.phase_volumes(p, False) - self.b
        return 1.0 / np.sqrt(float((self.Y * w / (self.g * (p + self.pi))).sum()))

    def wave(self, p) -> float:
        """Velocity change across the wave to pressure p, positive for compression: the mass flux
        of the shock (sqrt((p - p0)(v0 - v))), or minus the Riemann invariant's integral of
        dp / (rho c) over the rarefaction (in ln p: the pressures may span decades)."""
        if p > self.p:
            return np.sqrt((p - self.p) * (1.0 / self.rho - self.volume(p, True)))
        val, _ = quad(lambda z: np.exp(z) / self.impedance(np.exp(z)), np.log(p), np.log(self.p), epsabs=0.0,
                      epsrel=1e-11, limit=400)
        return -val


def mixture(L: MixtureState, R: MixtureState, x0: float, t: float, x, fan_points: int = 2000):
    """Exact solution at time t on the points x.  Returns a dict of p, u, rho, a1 (phase 1 volume
    fraction), r1, r2, and p*, u*.  A vacuum between two rarefactions is not handled."""
    x = np.asarray(x, dtype=np.float64)
    F = lambda p: L.wave(p) + R.wave(p) + (R.u - L.u)
    lo = max(float(-L.pi.min()), float(-R.pi.min()), 0.0)
    lo = lo + 1e-10 + 1e-9 * lo
    if F(lo) > 0:
        raise ValueError("the rarefactions do not meet (vacuum): not handled")
    ps = brentq(F, lo, 10.0 * max(L.p, R.p) + 10.0 * float(max(L.pi.max(), R.pi.max())), xtol=1e-9, rtol=1e-15)
    us = 0.5 * (L.u + R.u) + 0.5 * (R.wave(ps) - L.wave(ps))
    xi = (x - x0) / t
    out = {k: np.zeros_like(x) for k in ("p", "u", "rho", "a1", "r1", "r2")}

    def put(mask, S, p, u, shock):
        vk = S.phase_volumes(p, shock) if p != S.p else 1.0 / S.r
        v = float((S.Y * vk).sum())
        out["p"][mask] = p
        out["u"][mask] = u
        out["rho"][mask] = 1.0 / v
        out["a1"][mask] = S.Y[0] * vk[0] / v
        out["r1"][mask] = 1.0 / vk[0]
        out["r2"][mask] = 1.0 / vk[1]

    for S, s in ((L, -1.0), (R, 1.0)):
        side = (xi < us) if s < 0 else (xi >= us)
        if ps > S.p:  # shock: its speed from the mass flux m, W = u + s m v0
            W = S.u + s * np.sqrt((ps - S.p) / (1.0 / S.rho - S.volume(ps, True))) / S.rho
            put(side & (s * (xi - W) > 0), S, S.p, S.u, False)
            put(side & (s * (xi - W) <= 0), S, ps, us, True)
            continue
        head = S.u + s * S.impedance(S.p) / S.rho
        tail = us + s * S.impedance(ps) * S.volume(ps, False)
        put(side & (s * (xi - head) > 0), S, S.p, S.u, False)
        put(side & (s * (xi - tail) <= 0), S, ps, us, False)
        fan = side & (s * (xi - head) <= 0) & (s * (xi - tail) > 0)
        if fan.any():
            # the fan's characteristics xi = u(p) + s c(p), tabulated over p and inverted
            P = np.geomspace(S.p, ps, fan_points)
            U = np.array([S.u + s * S.wave(q) for q in P])
            C = np.array([S.impedance(q) * S.volume(q, False) for q in P])
            X = U + s * C
            o = np.argsort(X)
            pf = np.interp(xi[fan], X[o], P[o])
            uf = np.interp(xi[fan], X[o], U[o])
            for k, (q, uq) in zip(np.flatnonzero(fan), zip(pf, uf)):
                m = np.zeros_like(fan)
                m[k] = True
                put(m, S, q, uq, False)
    return out, ps, us


def relative_l1_rho(rho_num, rho_exact, rho_exact0) -> float:
    """Relative L1 density error, Eq. (51) of Schropff et al. (2026): sum |rho - rho_exact(t)| dx over
    sum |rho_exact(0)| dx on a uniform grid (the reference's tests/plot_schropff.py:71-72)."""
    return float(np.abs(np.asarray(rho_num) - rho_exact).sum() / np.abs(rho_exact0).sum())
