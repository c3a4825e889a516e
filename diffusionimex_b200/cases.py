"""Initial data for the SPB 6+1-equation two-phase solver.

Every case is a dict of solver settings (the fields of ``spb6g_config`` in
``include/spb6g.h``) plus the initial conservative state ``U`` as a float64
array of shape (ny, nx, 8) in the reference variable order
alpha1, m1, m2, rho*u, rho*v, eps1, eps2, E (src/spb6_physics_omp.h:27-28).

Two families:

* reference cases (``reference_case``): a few of the reference's own
  ``test_setup``/``test_state`` entries (src/spb6_physics_omp.h:1017-1157),
  restated with the same arithmetic so the states are bitwise identical to the
  reference's ``u_initialization`` for SUBCELL = 1;
* seeded synthetic workloads (``water_air_tube``, ``bubble_field``,
  ``shock_bubble``, ``riemann_batch``, ``lowmach_bubbles``) used by the bench
  and the parity tests.  They are generated from ``numpy.random.default_rng``
  with a recorded seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

NUM_VARS = 8
IA1, IM1, IM2, IMU, IMV, IE1, IE2, IEN = range(8)
BC_TRANS, BC_WALL, BC_PERIODIC, BC_PRES = 0, 1, 2, 3

WATER_SG = dict(g=4.4, pinf=6e8, q=0.0, qp=0.0, cv=1000.0, b=0.0)
AIR_SG = dict(g=1.4, pinf=0.0, q=0.0, qp=0.0, cv=1000.0, b=0.0)
# Mie-Grueneisen phases of the reference's cases 60, 61, 73 (src/spb6_physics_omp.h:1047-1070):
# kind 1 Cochran-Chan, kind 2 JWL; fields besides G, rr, c1, c2, e1, e2, e0 as Phase{} leaves them
NITROMETHANE_CC = dict(g=2.19, pinf=0.0, q=0.0, qp=0.0, cv=0.0, b=0.0, kind=1, G=1.19, rr=1134.0, c1=0.819181e9,
                       c2=1.50835e9, e1=4.52969, e2=1.42144, e0=0.0)
DETONATION_JWL = dict(g=1.25, pinf=0.0, q=0.0, qp=0.0, cv=0.0, b=0.0, kind=2, G=0.25, rr=1840.0, c1=854.5e9, c2=20.5e9,
                      e1=4.6, e2=1.35, e0=0.0)
WATER_NASG = dict(g=1.187, pinf=7028e5, q=-1177788.0, qp=0.0, cv=3610.0, b=6.61e-4)
# Liquid / vapour pairs of the reference's phase-transition cases (test_setup, physics :1019-1064;
# set_SG(k, g, pi, q, qp, cv)): water SG (P-S 2014), dodecane SG (P-S 2014), water NASG (Pelanti
# 2022 8.2.1), dodecane NASG (Pelanti 8.2.2), water NASG 350-550 K (Pelanti 8.2.4, Bartak)
WATER_LIQ_SG = dict(g=2.35, pinf=1e9, q=-1167e3, qp=0.0, cv=1816.0, b=0.0)
WATER_VAP_SG = dict(g=1.43, pinf=0.0, q=2030e3, qp=-23.4e3, cv=1040.0, b=0.0)
DODECANE_LIQ_SG = dict(g=2.35, pinf=4e8, q=-775.269e3, qp=0.0, cv=1077.7, b=0.0)
DODECANE_VAP_SG = dict(g=1.025, pinf=0.0, q=-237.547e3, qp=-24.4e3, cv=1956.45, b=0.0)
WATER_LIQ_NASG = dict(WATER_NASG)
WATER_VAP_NASG = dict(g=1.467, pinf=0.0, q=2077616.0, qp=14317.0, cv=955.0, b=0.0)
DODECANE_LIQ_NASG = dict(g=1.206, pinf=1681e5, q=-996054.0, qp=0.0, cv=2532.0, b=7.51e-4)
DODECANE_VAP_NASG = dict(g=1.021, pinf=0.0, q=-384592.0, qp=-4301.0, cv=2274.0, b=0.0)
WATER_LIQ_BARTAK = dict(g=1.387, pinf=8899e5, q=-1244191.0, qp=0.0, cv=3202.0, b=4.78e-4)
WATER_VAP_BARTAK = dict(g=1.954, pinf=0.0, q=2287484.0, qp=6417.0, cv=462.0, b=0.0)


def v_pT(ph: dict, p, T):
    """Specific volume of a SG / NASG phase at (p, T) (v_pT, physics :80)."""
    return (ph["g"] - 1.0) * ph["cv"] * T / (p + ph["pinf"]) + ph["b"]


def rho_pT(ph: dict, p, T):
    """rho_pT (physics :1015)."""
    return 1.0 / v_pT(ph, p, T)


def default_settings() -> dict:
    """Solver settings with the reference's defaults (src/SPB6_PC_IMEX_omp.cpp:55-95)."""
    return dict(
        nx=100, ny=1, x0=0.0, x1=1.0, y0=0.0, y1=1.0,
        bc=[BC_TRANS] * 4, bcu=[0.0] * 4, bcp=[0.0] * 4,
        phases=[dict(WATER_SG), dict(AIR_SG)],
        rk=2, cfl=0.2, cfl_ac=0.4, ramp=1, dtfix=0.0, rus_local=1, limiter=1,
        acdt=0, newton_tol=1e-13, newton_iter=60, bicg_tol=1e-13, bicg_iter=4000,
        share_mode=0, tend=1.0,
    )


def mg_ref(ph: dict, r: float):
    """Mie-Grueneisen reference curves pr, pr', er at density r (src/spb6_physics_omp.h:60-69),
    with the C library's pow / exp as the reference calls them."""
    if ph["kind"] == 1:
        x = r / ph["rr"]
        t1, t2 = ph["c1"] * math.pow(x, ph["e1"]), ph["c2"] * math.pow(x, ph["e2"])
        return t1 - t2, (ph["e1"] * t1 - ph["e2"] * t2) / r, (t1 / (ph["e1"] - 1.0) - t2 / (ph["e2"] - 1.0)) / r
    t1, t2 = ph["c1"] * math.exp(-ph["e1"] * ph["rr"] / r), ph["c2"] * math.exp(-ph["e2"] * ph["rr"] / r)
    return (t1 + t2, (ph["e1"] * t1 + ph["e2"] * t2) * ph["rr"] / (r * r),
            t1 / (ph["e1"] * ph["rr"]) + t2 / (ph["e2"] * ph["rr"]) - ph["e0"])


def eps_amp(ph: dict, a, m, p):
    """Phase internal energy per unit volume, src/spb6_physics_omp.h:71-73: SG/NASG, or
    Mie-Grueneisen m er(m/a) + a (p - pr(m/a)) / G (cell by cell, scalar libm)."""
    if ph.get("kind", 0):
        a, m, p = np.broadcast_arrays(np.asarray(a, np.float64), np.asarray(m, np.float64), np.asarray(p, np.float64))
        out = np.empty(a.shape)
        for i in np.ndindex(a.shape):
            pr, _, er = mg_ref(ph, float(m[i]) / float(a[i]))
            out[i] = float(m[i]) * er + float(a[i]) * (float(p[i]) - pr) / ph["G"]
        return out
    return (p + ph["g"] * ph["pinf"]) * (a - m * ph["b"]) / (ph["g"] - 1.0) + m * ph["q"]


def prim2cell(phases, a1, r1, r2, u, v, p1, p2):
    """Primitive -> conservative, src/spb6_physics_omp.h:904-909 (vectorised, same op order)."""
    a1 = np.asarray(a1, dtype=np.float64)
    a2 = 1 - a1
    m1 = a1 * r1
    m2 = a2 * r2
    rho = m1 + m2
    out = np.empty(np.broadcast(a1, r1, r2, u, v, p1, p2).shape + (NUM_VARS,))
    out[..., IA1] = a1
    out[..., IM1] = m1
    out[..., IM2] = m2
    out[..., IMU] = rho * u
    out[..., IMV] = rho * v
    out[..., IE1] = eps_amp(phases[0], a1, m1, p1)
    out[..., IE2] = eps_amp(phases[1], a2, m2, p2)
    out[..., IEN] = out[..., IE1] + out[..., IE2] + 0.5 * rho * (u * u + v * v)
    return out


def cell_centres(cfg: dict):
    nx, ny = cfg["nx"], cfg["ny"]
    dx = (cfg["x1"] - cfg["x0"]) / nx
    dy = (cfg["y1"] - cfg["y0"]) / ny
    x = cfg["x0"] + (np.arange(nx) + 0.5) * dx
    y = cfg["y0"] + (np.arange(ny) + 0.5) * dy
    return x, y, dx, dy


# --------------------------------------------------------------------------------------------
# Reference cases (test_setup / test_state, src/spb6_physics_omp.h:1017-1157)
# --------------------------------------------------------------------------------------------
def reference_case(case: int, nx: int | None = None, ny: int | None = None) -> dict:
    """A subset of the reference's 1D cases: 4 (interface advection), 5 (SPB 4.3.1 water-air),
    12 and 13 (SPB 5.1 / 5.2 epoxy-spinel mixture; 13 takes the grid-wide Rusanov speed,
    rus_local = 0), the liquid-vapour cases of phase transition -- 1, 2 (P-S 2014 5.1 water
    cavitation tube, +-2 and +-500 m/s), 3 (P-S 5.2 dodecane shock tube, SG), 30 (Pelanti 2022
    8.2.1 water cavitation, NASG), 31 (Pelanti 8.2.2 dodecane, NASG), 32 (Pelanti 8.2.4 Bartak
    depressurisation: pressure outlet left, wall right, relax 2), 40, 41 (uniform non-equilibrium
    states, periodic) -- 80-88 (Schropff 2026 Riemann problems), and the Mie-Grueneisen shock tubes
    60 (SPB 4.2 nitromethane, Cochran-Chan) and 61 (Pelanti 8.1.1, JWL detonation gas against NASG
    water); 0 (SPB 4.4 water cavitation), 6 (SPB 4.3.2 water-air at 1 TPa), 20 and 21 (smooth
    gas and smooth water advection).  The relaxation level is the case's own (32: 2; the others 0);
    set "relax" to run one with thermal or chemical relaxation.  The 2D cases 56-58 and 70-73 come
    from their builders (nx, ny their grid, each builder's own by default)."""
    builders_2d = {56: lambda a, b: vortex_bb(a), 57: lambda a, b: taylor_green(a), 58: lambda a, b: taylor_green(a, True),
                   70: he_bubble, 71: richtmyer_meshkov, 72: bubble_compression, 73: underwater_explosion}
    if case in builders_2d:
        defaults = {56: (40, 40), 57: (50, 50), 58: (50, 50), 70: (600, 160), 71: (300, 100), 72: (200, 200),
                    73: (361, 200)}[case]
        return builders_2d[case](nx or defaults[0], ny or defaults[1])
    c = default_settings()
    air, water = dict(AIR_SG), dict(WATER_SG)
    if case == 4:
        c.update(phases=[water, air], tend=2.79e-3, nx=200)
    elif case == 5:
        c.update(phases=[water, air], tend=240e-6, nx=1000)
    elif case in (80, 82, 83, 84):
        c.update(phases=[dict(air), dict(air)], nx=1000,
                 tend={80: 0.5, 82: 0.14, 83: 2.5e-6, 84: 0.15}[case])
    elif case in (81, 85):
        c.update(phases=[dict(water), dict(water)], nx=1000, tend=1e-4 if case == 81 else 0.15e-3)
    elif case in (86, 87):
        c.update(phases=[water, air], nx=1000, tend=0.25 if case == 86 else 241e-6)
    elif case == 88:
        c.update(phases=[dict(WATER_SG, g=2.43, pinf=5.3e9), dict(AIR_SG, g=1.62, pinf=141e9)], nx=1000, tend=30e-6)
    elif case in (1, 2):  # physics :1021-1023
        c.update(phases=[dict(WATER_LIQ_SG), dict(WATER_VAP_SG)], nx=5000, tend=3.2e-3 if case == 1 else 0.58e-3)
    elif case in (3, 31):  # :1024-1025, :1036
        pair = (DODECANE_LIQ_SG, DODECANE_VAP_SG) if case == 3 else (DODECANE_LIQ_NASG, DODECANE_VAP_NASG)
        c.update(phases=[dict(pair[0]), dict(pair[1])], nx=2000, tend=473e-6)
        if case == 3:
            c["cfl"] = 0.05
    elif case == 30:  # :1035
        c.update(phases=[dict(WATER_LIQ_NASG), dict(WATER_VAP_NASG)], nx=5000, tend=3e-3)
    elif case == 32:  # :1037-1039
        c.update(phases=[dict(WATER_LIQ_BARTAK), dict(WATER_VAP_BARTAK)], x0=0.0, x1=1.7, tend=17.5e-3, nx=1000,
                 relax=2, bc=[BC_PRES, BC_WALL, BC_TRANS, BC_TRANS], bcp=[1e5, 0.0, 0.0, 0.0])
    elif case in (40, 41):  # :1040
        c.update(phases=[dict(WATER_LIQ_SG), dict(WATER_VAP_SG)], tend=1e-4, bc=[BC_PERIODIC, BC_PERIODIC, BC_TRANS, BC_TRANS])
    elif case in (0, 6):  # :1019, :1028
        c.update(phases=[dict(WATER_SG), dict(AIR_SG)], nx=1000, tend=1.85e-3 if case == 0 else 8.3e-6)
    elif case in (20, 21):  # :1033-1034
        c.update(phases=[dict(AIR_SG), dict(AIR_SG)] if case == 20 else [dict(WATER_SG), dict(AIR_SG)],
                 tend=5e-4 if case == 20 else 1e-4)
    elif case in (12, 13):  # test_setup physics :1029-1032
        c.update(phases=[dict(WATER_SG, g=2.43, pinf=5.3e9), dict(AIR_SG, g=1.62, pinf=141e9)], nx=500,
                 tend=80e-6 if case == 12 else 34e-6)
        if case == 12:
            c["cfl"] = 0.05
        else:
            c["rus_local"] = 0
    elif case == 60:  # SPB 4.2 nitromethane shock tube, Cochran-Chan for both phases
        c.update(phases=[dict(NITROMETHANE_CC), dict(NITROMETHANE_CC)], nx=500, tend=67e-6)
    elif case == 61:  # Pelanti 8.1.1 detonation gas (JWL) - water (NASG) shock tube on [-10, 10] m
        c.update(phases=[dict(DETONATION_JWL), dict(WATER_NASG)], nx=500, tend=0.9e-3, x0=-10.0, x1=10.0)
    else:
        raise ValueError(f"reference case {case} is not restated here")
    if nx is not None:
        c["nx"] = nx
    c["case"] = case
    x, _, _, _ = cell_centres(c)
    ph = c["phases"]
    if case == 4:
        L = x < 0.5
        U = prim2cell(ph, np.where(L, 1 - 1e-8, 1e-8), 1000.0, 10.0, 100.0, 0.0, 1e5, 1e5)
    elif case == 5:
        L = x < 0.75
        pl = np.where(L, 1e9, 1e5)
        U = prim2cell(ph, np.where(L, 1 - 1e-6, 1e-6), 1000.0, 1.0, 0.0, 0.0, pl, pl)
    elif case in (80, 81, 82, 83, 84, 85):
        xi, rL, uL, pL, rR, uR, pR = {
            80: (0.25, 1000, 1, 1e5, 0.01, 1, 1e5),
            81: (0.5, 1000, 0, 1e8, 1000, 15, 0.98e8),
            82: (0.5, 0.445, 0.698, 3.528, 0.5, 0, 0.571),
            83: (0.5, 1, 0, 1e10, 0.125, 0, 0.1),
            84: (0.5, 1, -1, 0.4, 1, 1, 0.4),
            85: (0.5, 1000, 0, 1e6, 1000, 0, 1e5),
        }[case]
        L = x < xi
        r = np.where(L, float(rL), float(rR))
        u = np.where(L, float(uL), float(uR))
        p = np.where(L, float(pL), float(pR))
        U = prim2cell(ph, np.full_like(x, 1 - 1e-8), r, r, u, 0.0, p, p)
    elif case in (86, 87):
        adv = case == 86
        L = x < (0.25 if adv else 0.7)
        p = np.full_like(x, 1e5) if adv else np.where(L, 1e9, 1e5)
        U = prim2cell(ph, np.where(L, 1 - 1e-7, 1e-7), 1000.0, 0.01 if adv else 50.0, 1.0 if adv else 0.0, 0.0, p, p)
    elif case == 0:  # test_state :1089
        u = np.where(x < 0.5, -100.0, 100.0)
        U = prim2cell(ph, np.full_like(x, 1 - 1e-2), 1000.0, 1.0, u, 0.0, 1e5, 1e5)
    elif case == 6:  # :1132-1134
        L = x < 0.6
        p = np.where(L, 1e12, 1e5)
        U = prim2cell(ph, np.where(L, 1 - 1e-6, 1e-6), 1000.0, 10.0, 0.0, 0.0, p, p)
    elif case in (20, 21):  # :1157-1159, exp and sin of the C library point by point
        gs = np.array([math.exp(-(xv - 0.5) * (xv - 0.5) / 0.01) for xv in x])
        a1 = 0.5 + 0.2 * np.array([math.sin(2 * math.pi * xv) for xv in x])
        p = 1e5 * (1 + 0.2 * gs)
        U = prim2cell(ph, a1, 2.0 if case == 20 else 1000.0, 1.0, 50.0 * gs, 0.0, p, p)
    elif case in (1, 2, 30):  # test_state :1090-1092, :1141
        T0 = 353.0 if case == 30 else 354.728
        U0 = 500.0 if case == 2 else 2.0
        u = np.where(x < 0.5, -U0, U0)
        U = prim2cell(ph, np.full_like(x, 1 - 1e-2), rho_pT(ph[0], 1e5, T0), rho_pT(ph[1], 1e5, T0), u, 0.0, 1e5, 1e5)
    elif case in (3, 31):  # :1095
        L = x < 0.75
        p = np.where(L, 1e8, 1e5)
        U = prim2cell(ph, np.where(L, 1 - 1e-8, 1e-8), 500.0, 2.0, 0.0, 0.0, p, p)
    elif case == 32:  # :1093-1094
        p, T = 12.5e6, 563.15
        U = prim2cell(ph, np.full_like(x, 1 - 1e-3), rho_pT(ph[0], p, T), rho_pT(ph[1], p, T), 0.0, 0.0, p, p)
    elif case == 40:  # :1143
        T1, T2, p1, p2 = 350.0, 380.0, 1.2e5, 0.8e5
        U = prim2cell(ph, np.full_like(x, 1 - 0.2), rho_pT(ph[0], p1, T1), rho_pT(ph[1], p2, T2), 0.0, 0.0, p1, p2)
    elif case == 41:  # :1142
        T0, p0 = 380.0, 0.8e5
        U = prim2cell(ph, np.full_like(x, 1 - 0.2), rho_pT(ph[0], p0, T0), rho_pT(ph[1], p0, T0), 0.0, 0.0, p0, p0)
    elif case in (12, 13, 88):
        p = np.where(x < 0.6, 2e11 if case == 13 else 1e10, 1e5)
        U = prim2cell(ph, np.full_like(x, 0.5954), 1185.0, 3622.0, 0.0, 0.0, p, p)
    elif case == 60:
        L = x < 0.5
        p = np.where(L, 20e9, 0.2e6)
        U = prim2cell(ph, np.where(L, 1 - 1e-8, 1e-8), 1134.0, 1200.0, 0.0, 0.0, p, p)
    else:  # 61
        L = x < 0.0
        p = np.where(L, 4.6406e10, 1e5)
        U = prim2cell(ph, np.where(L, 1 - 1e-8, 1e-8), 2000.0, 1044.0, 0.0, 0.0, p, p)
    c["U"] = U.reshape(1, c["nx"], NUM_VARS)
    return c


# --------------------------------------------------------------------------------------------
# Synthetic workloads
# --------------------------------------------------------------------------------------------
def water_air_tube(nx: int = 1000) -> dict:
    """1D water-air shock tube: water SG (4.4, 6e8) | air (1.4, 0) on [0, 1] m, interface 0.7,
    alpha_w 1-1e-6 | 1e-6, rho_w 1000, rho_a 50, p 1e9 | 1e5, u = 0; transmissive; material
    CFL 0.5; Newton tol 1e-10, BiCGStab tol 1e-12; t_end 240 us."""
    c = default_settings()
    c.update(nx=nx, ny=1, phases=[dict(WATER_SG), dict(AIR_SG)], cfl=0.5, newton_tol=1e-10,
             bicg_tol=1e-12, tend=240e-6)
    x, _, _, _ = cell_centres(c)
    L = x < 0.7
    p = np.where(L, 1e9, 1e5)
    c["U"] = prim2cell(c["phases"], np.where(L, 1 - 1e-6, 1e-6), 1000.0, 50.0, 0.0, 0.0, p, p).reshape(1, nx, 8)
    c["workload"] = f"water-air shock tube 1D, {nx} cells"
    return c


def _place_bubbles(rng, n, rmin, rmax, dx, lo=0.0, hi=1.0, ylo=0.0, yhi=1.0, tries=100000):
    """Rejection-sample n non-overlapping discs: radius U[rmin, rmax], centre uniform in
    [R, 1-R]^2, |c_i - c_j| > R_i + R_j + 4 dx."""
    out = []
    for _ in range(tries):
        if len(out) == n:
            break
        R = rng.uniform(rmin, rmax)
        cx = rng.uniform(lo + R, hi - R)
        cy = rng.uniform(ylo + R, yhi - R)
        if all(math.hypot(cx - qx, cy - qy) > R + qR + 4 * dx for qx, qy, qR in out):
            out.append((cx, cy, R))
    if len(out) < n:
        raise RuntimeError("could not place the requested bubbles")
    return out


def _bubble_blend(x, y, bubbles, dx):
    """f = 1/2 (1 + tanh((r - R)/(2 dx))), 0 inside a bubble and 1 in the liquid; the nearest
    bubble (minimum of f over the non-overlapping bubbles) decides."""
    X, Y = np.meshgrid(x, y)
    f = np.ones_like(X)
    for cx, cy, R in bubbles:
        r = np.hypot(X - cx, Y - cy)
        f = np.minimum(f, 0.5 * (1.0 + np.tanh((r - R) / (2.0 * dx))))
    return f


def bubble_field(n: int = 1024, seed: int = 0, nbub: int = 8, steps: int = 200) -> dict:
    """Water at rest (SG 4.4/6e8, rho 1000, p 1e7) with `nbub` air bubbles (alpha_w 1e-6,
    rho_a 1, p 1e5) on an n x n grid over [0, 1]^2; radii U[0.03, 0.08]; tanh profile over
    2 cells; transmissive; material CFL 0.5; Newton tol 1e-10, BiCGStab tol 1e-12."""
    c = default_settings()
    c.update(nx=n, ny=n, phases=[dict(WATER_SG), dict(AIR_SG)], cfl=0.5, newton_tol=1e-10,
             bicg_tol=1e-12, tend=1.0)
    x, y, dx, _ = cell_centres(c)
    rng = np.random.default_rng(seed)
    bubbles = _place_bubbles(rng, nbub, 0.03, 0.08, dx)
    f = _bubble_blend(x, y, bubbles, dx)
    a1 = 1e-6 + (1 - 1e-6 - 1e-6) * f
    p = 1e5 + (1e7 - 1e5) * f
    c["U"] = prim2cell(c["phases"], a1, 1000.0, 1.0, 0.0, 0.0, p, p)
    c["seed"], c["bubbles"], c["steps"] = seed, bubbles, steps
    c["workload"] = f"water with {nbub} air bubbles 2D, {n}x{n} cells"
    return c


def shock_bubble(nx: int = 2048, ny: int = 1024) -> dict:
    """Mach-1.5 planar shock in air (1.4, 0; 1.29 kg/m3, 101325 Pa) moving left onto a light-gas
    bubble (1.67, 0; rho 0.167, R 0.1 at (0.35, 0.5)) on [0, 2] x [0, 1] m; post-shock state from
    the ideal-gas Rankine-Hugoniot relations as in the reference's case 70
    (src/spb6_physics_omp.h:1098-1104); shock front at x = 0.5."""
    c = default_settings()
    c.update(nx=nx, ny=ny, x0=0.0, x1=2.0, y0=0.0, y1=1.0,
             phases=[dict(AIR_SG), dict(AIR_SG, g=1.67)], tend=1.0)
    x, y, dx, _ = cell_centres(c)
    g, Ms, p0, r0 = 1.4, 1.5, 101325.0, 1.29
    c0 = math.sqrt(g * p0 / r0)
    p1 = p0 * (1 + 2 * g / (g + 1) * (Ms * Ms - 1))
    r1 = r0 * (g + 1) * Ms * Ms / ((g - 1) * Ms * Ms + 2)
    u1 = -Ms * c0 * (1 - r0 / r1)
    X, Y = np.meshgrid(x, y)
    inside = (X - 0.35) ** 2 + (Y - 0.5) ** 2 < 0.1 * 0.1
    post = X > 0.5
    a1 = np.where(post, 1 - 1e-6, np.where(inside, 1e-6, 1 - 1e-6))
    r_air = np.where(post, r1, r0)
    u = np.where(post, u1, 0.0)
    p = np.where(post, p1, p0)
    c["U"] = prim2cell(c["phases"], a1, r_air, 0.167, u, 0.0, p, p)
    c["workload"] = f"Mach-1.5 shock on a light-gas bubble 2D, {nx}x{ny} cells"
    return c


def lowmach_bubbles(n: int = 2048, seed: int = 0, nbub: int = 16, amp: float = 15.0) -> dict:
    """Low-Mach water field (p 1e5, rho 1000) with a seeded divergence-free velocity of max
    amplitude `amp` m/s from a stream function of Fourier modes 1 <= |k| <= 4, differenced at
    cell centres (discrete divergence zero, as the reference's wellprep,
    src/SPB6_PC_IMEX_omp.cpp:1260-1272), and `nbub` air bubbles (rho 1, p 1e5, radii
    U[0.01, 0.04]); periodic; material CFL 0.8; Newton tol 1e-10, BiCGStab tol 1e-10."""
    c = default_settings()
    c.update(nx=n, ny=n, bc=[BC_PERIODIC] * 4, phases=[dict(WATER_SG), dict(AIR_SG)], cfl=0.8,
             newton_tol=1e-10, bicg_tol=1e-10, tend=1.0)
    x, y, dx, dy = cell_centres(c)
    rng = np.random.default_rng(seed)
    modes = [(kx, ky) for kx in range(-4, 5) for ky in range(-4, 5) if 1 <= math.hypot(kx, ky) <= 4]
    coef = rng.normal(size=(len(modes), 2))

    def psi(X, Y):
        s = np.zeros_like(X)
        for (kx, ky), (a, b) in zip(modes, coef):
            ph = 2 * math.pi * (kx * X + ky * Y)
            s += a * np.sin(ph) + b * np.cos(ph)
        return s
    X, Y = np.meshgrid(x, y)
    u = (psi(X, Y + dy) - psi(X, Y - dy)) / (2 * dy)
    v = -(psi(X + dx, Y) - psi(X - dx, Y)) / (2 * dx)
    scale = amp / max(np.abs(u).max(), np.abs(v).max())
    u, v = u * scale, v * scale
    bubbles = _place_bubbles(rng, nbub, 0.01, 0.04, dx)
    f = _bubble_blend(x, y, bubbles, dx)
    a1 = 1e-6 + (1 - 1e-6 - 1e-6) * f
    c["U"] = prim2cell(c["phases"], a1, 1000.0, 1.0, u, v, 1e5, 1e5)
    c["seed"], c["bubbles"] = seed, bubbles
    c["workload"] = f"low-Mach water with {nbub} bubbles 2D periodic, {n}x{n} cells"
    return c


NASG_LIQ = dict(g=2.35, pinf=4e8, q=0.0, qp=0.0, cv=1000.0, b=7.5e-4)
NASG_VAP = dict(g=1.025, pinf=0.0, q=0.0, qp=0.0, cv=1000.0, b=0.0)


def riemann_batch(count: int = 512, seed: int = 0, nmin: int = 256, nmax: int = 4096, steps: int = 200):
    """`count` independent 1D two-phase Riemann problems: cells U{nmin..nmax}, p_L log-U[1e6, 1e9],
    p_R log-U[1e4, 1e6], interface U[0.3, 0.7], alpha 1-1e-6 | 1e-6, phase pair water/air SG
    (rho 1000 / 50) or NASG liquid/vapour (rho 500 / 2) with probability 1/2; q = 0,
    c_v = 1000; `steps` steps each."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(nmin, nmax + 1))
        pL = float(np.exp(rng.uniform(np.log(1e6), np.log(1e9))))
        pR = float(np.exp(rng.uniform(np.log(1e4), np.log(1e6))))
        x0 = float(rng.uniform(0.3, 0.7))
        nasg = bool(rng.random() < 0.5)
        c = default_settings()
        ph = [dict(NASG_LIQ), dict(NASG_VAP)] if nasg else [dict(WATER_SG), dict(AIR_SG)]
        rl, rv = (500.0, 2.0) if nasg else (1000.0, 50.0)
        c.update(nx=n, ny=1, phases=ph, cfl=0.5, newton_tol=1e-10, bicg_tol=1e-12, tend=1.0)
        x, _, _, _ = cell_centres(c)
        L = x < x0
        p = np.where(L, pL, pR)
        c["U"] = prim2cell(ph, np.where(L, 1 - 1e-6, 1e-6), rl, rv, 0.0, 0.0, p, p).reshape(1, n, 8)
        c.update(steps=steps, instance=k, nasg=nasg)
        out.append(c)
    return out


def subcell_average(c: dict, state, sub: int = 4) -> np.ndarray:
    """Cell averages of state(x, y) -> conservative values over sub x sub points per cell, summed
    in the reference's order (u_initialization :482-487: a over x outer, b over y inner, each
    term divided by sub^2)."""
    x, y, dx, dy = cell_centres(c)
    X, Y = np.meshgrid(x, y)
    U = np.zeros((c["ny"], c["nx"], NUM_VARS))
    for a in range(sub):
        for b in range(sub):
            U = U + state(X + ((a + 0.5) / sub - 0.5) * dx, Y + ((b + 0.5) / sub - 0.5) * dy) / (sub * sub)
    return U


_exp, _pow = np.vectorize(math.exp), np.vectorize(math.pow)
_sin, _cos = np.vectorize(math.sin), np.vectorize(math.cos)  # the C library's, point by point


def vortex_bb(n: int = 40, p0: float = 1.0) -> dict:
    """The reference's case 56 (Battisti-Boscheri 4.1, physics :1041-1043, :1148-1155): a Hu-Shu
    isentropic vortex (eps 5) in two ideal gases (gamma 1.35 and 1.4) at one density and pressure,
    alpha2 a passive smooth bump, translated by (2, 2) across the periodic [-5, 5]^2 (t_end 5 is one
    period, so the exact solution is the initial state); background pressure p0 (p0=); 4 x 4 sub-cell
    averages."""
    c = default_settings()
    c.update(nx=n, ny=n, x0=-5.0, x1=5.0, y0=-5.0, y1=5.0, tend=5.0,
             phases=[dict(AIR_SG, g=1.35), dict(AIR_SG)], bc=[BC_PERIODIC] * 4, case=56)
    ph = c["phases"]
    g, eps = 1.4, 5.0

    def state(x, y):
        r2 = x * x + y * y
        du = eps / (2 * math.pi) * _exp(0.5 * (1 - r2))
        dT = -(g - 1) * eps * eps / (8 * g * math.pi * math.pi) * _exp(1 - r2)
        T = p0 + dT
        rho = _pow(T / p0, 1.0 / (g - 1))
        p = rho * T
        a2 = 0.5 + 0.25 * _exp(0.5 * (1 - r2))
        return prim2cell(ph, 1 - a2, rho, rho, 2.0 - du * y, 2.0 + du * x, p, p)

    c["U"] = subcell_average(c, state)
    c["workload"] = f"two-phase isentropic vortex 2D, {n}x{n} cells, p0 {p0}"
    return c


def taylor_green(n: int = 50, two_phase: bool = False, p0: float = 1.0) -> dict:
    """The reference's cases 57 / 58 (Battisti-Boscheri 4.4, physics :1044-1046, :1144-1147): the
    low-Mach Taylor-Green vortex u = sin x cos y, v = -cos x sin y, p = p0 + (cos 2x + cos 2y) / 4
    in two ideal gases of gamma 1.4 and density 1 on the periodic [0, 2 pi]^2 to t = 0.2; alpha2 0.5
    (57) or 0.5 + 0.1 (cos 2x + cos 2y) (58); 4 x 4 sub-cell averages."""
    c = default_settings()
    c.update(nx=n, ny=n, x0=0.0, x1=2 * math.pi, y0=0.0, y1=2 * math.pi, tend=0.2,
             phases=[dict(AIR_SG), dict(AIR_SG)], bc=[BC_PERIODIC] * 4, case=58 if two_phase else 57)
    ph = c["phases"]

    def state(x, y):
        p = p0 + 0.25 * (_cos(2 * x) + _cos(2 * y))
        a2 = 0.5 + 0.1 * (_cos(2 * x) + _cos(2 * y)) if two_phase else np.full_like(x, 0.5)
        return prim2cell(ph, 1 - a2, 1.0, 1.0, _sin(x) * _cos(y), -_cos(x) * _sin(y), p, p)

    c["U"] = subcell_average(c, state)
    c["workload"] = f"Taylor-Green vortex 2D, {n}x{n} cells, {'two phases' if two_phase else 'one phase'}"
    return c


def he_bubble(nx: int = 600, ny: int = 160) -> dict:
    """The reference's case 70 (SPB 2009 4.6, physics :1055-1056, :1099-1104): a Mach-1.5 shock in
    air (ideal-gas Rankine-Hugoniot post-shock state for x > 0.221 m, moving left) reaching a
    helium bubble (radius 0.02 m at (0.2, 0.04) m) on [0, 0.3] x [0, 0.08] m; transmissive in x,
    walls in y; 4 x 4 sub-cell averages."""
    c = default_settings()
    c.update(nx=nx, ny=ny, x0=0.0, x1=0.3, y0=0.0, y1=0.08, tend=600e-6,
             phases=[dict(AIR_SG), dict(AIR_SG, g=1.67)], bc=[BC_TRANS, BC_TRANS, BC_WALL, BC_WALL], case=70)
    ph = c["phases"]
    g, Ms, p0, r0 = 1.4, 1.5, 101325.0, 1.29
    c0 = math.sqrt(g * p0 / r0)
    p1 = p0 * (1 + 2 * g / (g + 1) * (Ms * Ms - 1))
    r1 = r0 * (g + 1) * Ms * Ms / ((g - 1) * Ms * Ms + 2)
    u1 = -Ms * c0 * (1 - r0 / r1)

    def state(x, y):
        inside = (x - 0.2) * (x - 0.2) + (y - 0.04) * (y - 0.04) < 0.02 * 0.02
        post = x > 0.221
        a1 = np.where(post, 1 - 1e-6, np.where(inside, 1e-6, 1 - 1e-6))
        r = np.where(post, r1, r0)
        u = np.where(post, u1, 0.0)
        p = np.where(post, p1, p0)
        return prim2cell(ph, a1, r, 0.167, u, 0.0, p, p)

    c["U"] = subcell_average(c, state)
    c["workload"] = f"shock on a helium bubble 2D, {nx}x{ny} cells"
    return c


def richtmyer_meshkov(nx: int = 300, ny: int = 100) -> dict:
    """The reference's case 71 (SPB 2009 4.7, physics :1057-1060, :1105-1107): water left of the arc
    x = 1.2 + sqrt(0.36 - (y - 0.5)^2) against gas (gamma 1.8), everything at -200 m/s and 1 atm,
    on [0, 3] x [0, 1] m; a wall on the left (the flow hits it), transmissive on the right, walls
    in y; the grid-wide Rusanov speed; 4 x 4 sub-cell averages."""
    c = default_settings()
    c.update(nx=nx, ny=ny, x0=0.0, x1=3.0, y0=0.0, y1=1.0, tend=8.6e-3, rus_local=0,
             phases=[dict(WATER_SG), dict(AIR_SG, g=1.8)], bc=[BC_WALL, BC_TRANS, BC_WALL, BC_WALL], case=71)
    ph = c["phases"]

    def state(x, y):
        d = y - 0.5
        xi = 1.2 + np.sqrt(np.maximum(0.0, 0.36 - d * d))
        W = x < xi
        return prim2cell(ph, np.where(W, 1 - 1e-6, 1e-6), 1000.0, 100.0, -200.0, 0.0, 101325.0, 101325.0)

    c["U"] = subcell_average(c, state)
    c["workload"] = f"cavitating Richtmyer-Meshkov 2D, {nx}x{ny} cells"
    return c


def bubble_compression(nx: int = 200, ny: int = 200) -> dict:
    """The reference's case 72 (P-S 2014 5.4, src/spb6_physics_omp.h:1062-1064, :1115-1117): a
    dodecane vapour bubble (radius 0.2 m, centred) in liquid dodecane at 1e5 Pa and 600 K on the
    unit square, walls all round, the left wall a piston at 100 m/s; p-pT-pTg relaxation
    (relax 2), the grid-wide Rusanov speed (rus_local 0).  Cell values are the reference's
    averages over 4 x 4 sub-points (u_initialization :482-487, summed in its order)."""
    c = default_settings()
    c.update(nx=nx, ny=ny, tend=1.2e-3, phases=[dict(DODECANE_LIQ_SG), dict(DODECANE_VAP_SG)],
             bc=[BC_WALL] * 4, bcu=[100.0, 0.0, 0.0, 0.0], relax=2, rus_local=0, case=72)
    ph = c["phases"]
    r1, r2 = rho_pT(ph[0], 1e5, 600.0), rho_pT(ph[1], 1e5, 600.0)

    def state(x, y):
        inside = (x - 0.5) * (x - 0.5) + (y - 0.5) * (y - 0.5) < 0.04
        return prim2cell(ph, np.where(inside, 1e-6, 1 - 1e-6), r1, r2, 0.0, 0.0, 1e5, 1e5)

    c["U"] = subcell_average(c, state)
    c["workload"] = f"piston-compressed dodecane vapour bubble 2D, {nx}x{ny} cells, relax 2"
    return c


def underwater_explosion(nx: int = 361, ny: int = 200) -> dict:
    """The reference's case 73 geometry (Pelanti 8.1.2, src/spb6_physics_omp.h:1067-1069, :1112-1113):
    a JWL detonation-gas bubble (radius 0.05 m, centre (0, -0.32) m, 4.6406e10 Pa) in NASG water at
    1e5 Pa on [-1.35, 1.35] x [-1.5, 0] m, a wall at y = 0, transmissive elsewhere; 4 x 4 sub-cell
    averages as the reference's u_initialization."""
    c = default_settings()
    c.update(nx=nx, ny=ny, x0=-1.35, x1=1.35, y0=-1.5, y1=0.0, tend=0.4e-3,
             phases=[dict(DETONATION_JWL), dict(WATER_NASG)], bc=[BC_TRANS, BC_TRANS, BC_TRANS, BC_WALL], case=73)
    ph = c["phases"]

    def state(x, y):
        inside = x * x + (y + 0.32) * (y + 0.32) < 0.05 * 0.05
        p = np.where(inside, 4.6406e10, 1e5)
        return prim2cell(ph, np.where(inside, 1 - 1e-6, 1e-6), 2000.0, 1044.0, 0.0, 0.0, p, p)

    c["U"] = subcell_average(c, state)
    c["workload"] = f"underwater explosion (JWL gas bubble in NASG water) 2D, {nx}x{ny} cells"
    return c
