"""Secondary check against exact Riemann solutions (oracle/exact_riemann.py).

The reference measures its Riemann-problem runs against exact solutions of the
mechanical-equilibrium model (tests/exact5.py, tests/exact_sg.py of the reference) in the
relative L1 density error of Eq. (51) of Schropff et al. (2026), and publishes the errors
of its cases 80-88 (data/Schropff2026_Riemann_problems/L1_table.md).  Here:

  * (CPU) the two exact solvers agree with each other in the single-phase limit, and the
    mixture solver reproduces the published table from the reference's own archived runs
    (tests/golden/ref_schropff_profiles.npz) -- this pins the exact solutions;
  * (GPU) the GPU runs of cases 80-88 have the compiled reference's errors and the published
    ones (where the reference's archived run is that of its current code); the 1000-cell
    water-air tube (interface 0.7, alpha 1 - 1e-6 | 1e-6, t_end 240 us) and a NASG liquid-
    vapour instance of the 512 batched Riemann problems are compared with the exact solution,
    the latter beside the C restatement of the reference on the same instance.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

import exact_riemann as er
from diffusionimex_b200 import cases
from helpers import GOLDEN, mixture_pressure

SCHROPFF = (80, 81, 82, 83, 84, 85, 86, 87, 88)


def riemann_sides(c: dict):
    """The two constant states of a 1D Riemann problem from its initial cells (first and last cell)
    and the face between them: MixtureState left / right and the interface x0."""
    U = np.asarray(c["U"], dtype=np.float64).reshape(-1, 8)
    ph = c["phases"]
    p = mixture_pressure(c, U)
    n = U.shape[0]
    dx = (c["x1"] - c["x0"]) / n
    diff = np.flatnonzero(np.any(np.abs(U - U[0]) > 1e-12 * np.abs(U[0]).max(axis=0, initial=0) + 1e-300, axis=1))
    x0 = c["x0"] + diff[0] * dx
    sides = []
    for k in (0, n - 1):
        a1 = U[k, 0]
        r1, r2 = U[k, 1] / a1, U[k, 2] / (1.0 - a1)
        sides.append(er.MixtureState([a1, 1.0 - a1], [r1, r2], U[k, 3] / (U[k, 1] + U[k, 2]), p[k],
                                     [ph[0]["g"], ph[1]["g"]], [ph[0]["pinf"], ph[1]["pinf"]],
                                     [ph[0]["b"], ph[1]["b"]]))
    return sides[0], sides[1], x0


def exact_rho(c: dict, n: int, t: float):
    """Exact density at the centres of n cells at time t, and at t = 0 (the denominator of Eq. (51))."""
    L, R, x0 = riemann_sides(c)
    x = c["x0"] + (np.arange(n) + 0.5) * (c["x1"] - c["x0"]) / n
    o, _, _ = er.mixture(L, R, x0, t, x, fan_points=1500)
    return o, np.where(x < x0, L.rho, R.rho)


def test_exact_solvers_agree_in_the_single_phase_limit():
    """Two identical phases make the mixture solver a stiffened-gas solver: both agree on a water
    shock tube with a rarefaction and on the Lax tube."""
    x = np.linspace(0.0, 1.0, 801)
    for l, r, t in (((1000.0, 0.0, 1e8), (1000.0, 15.0, 0.98e8), 1e-4), ((0.445, 0.698, 3.528), (0.5, 0.0, 0.571), 0.14)):
        g, pi = (4.4, 6e8) if l[0] == 1000.0 else (1.4, 0.0)
        L = er.MixtureState([1 - 1e-8, 1e-8], [l[0], l[0]], l[1], l[2], [g, g], [pi, pi])
        R = er.MixtureState([1 - 1e-8, 1e-8], [r[0], r[0]], r[1], r[2], [g, g], [pi, pi])
        o, ps, us = er.mixture(L, R, 0.5, t, x)
        rho, u, p, ps2, us2 = er.stiffened_gas((*l, g, pi), (*r, g, pi), 0.5, t, x)
        assert abs(ps - ps2) <= 1e-9 * ps and abs(us - us2) <= 1e-9 * max(abs(us), 1.0)
        assert np.abs(o["rho"] - rho).max() <= 1e-8 * rho.max()
        assert np.abs(o["u"] - u).max() <= 1e-8 * max(np.abs(u).max(), 1.0)


def test_exact_solution_reproduces_the_published_errors():
    """The reference's archived runs of its cases 80-88 measured against the mixture solver give the
    relative L1 density errors the reference publishes for them, to their printed digits."""
    z = np.load(os.path.join(GOLDEN, "ref_schropff_profiles.npz"))
    for key in sorted(k for k in z.files if k.startswith("pub_")):
        case, n = (int(v) for v in key[len("pub_c"):].split("_"))
        c = cases.reference_case(case, n)
        o, rho0 = exact_rho(c, n, c["tend"])
        e = er.relative_l1_rho(z[f"rho_c{case}_{n}"], o["rho"], rho0)
        assert abs(e - float(z[key])) <= 5e-4 * float(z[key]) + 5e-8, (key, e, float(z[key]))


def _gpu_run(c: dict, nsteps: int = 0):
    from diffusionimex_b200 import Solver

    s = Solver(c)
    s.advance(nsteps)
    st = s.stats()
    U = s.state().reshape(-1, 8)
    s.close()
    return U, st


# The reference's archived runs of these cases at 200 cells predate its current code: the compiled
# reference gives 4.744e-2 (case 82) and 3.158e-2 (case 83) against the published 5.073e-2 and 3.117e-2
# (its densities differ from the archived ones by 3.5 % and 4.5 % of the maximum), and so does the GPU.
STALE_ARCHIVE = {(82, 200), (83, 200)}


@pytest.mark.gpu
@pytest.mark.parametrize("case,n", [(c, 200) for c in SCHROPFF] + [(87, 1000)])
def test_gpu_runs_reproduce_the_published_errors(case, n):
    """Each GPU run, to t_end, has the relative L1 density error of the compiled reference on the same
    case and resolution, to 1 % (the two runs differ in L1 by about 1e-6 of the field maximum, far below
    the discretisation error measured here), and that is the error the reference publishes, to 1 %,
    except where its archived run predates its current code."""
    import refio

    z = np.load(os.path.join(GOLDEN, "ref_schropff_profiles.npz"))
    c = cases.reference_case(case, n)
    U, st = _gpu_run(c)
    assert abs(st["t"] - c["tend"]) <= 1e-12 * c["tend"]
    o, rho0 = exact_rho(c, n, c["tend"])
    e = er.relative_l1_rho(U[:, 1] + U[:, 2], o["rho"], rho0)
    Ur = refio.run_ref(c, mode=refio.MODE_TEND, threads=os.cpu_count() or 1)["U"].reshape(-1, 8)
    e_ref = er.relative_l1_rho(Ur[:, 1] + Ur[:, 2], o["rho"], rho0)
    pub = float(z[f"pub_c{case}_{n}"])
    print(f"case {case}, {n} cells: L1(rho) GPU {e:.4e}, compiled reference {e_ref:.4e}, published {pub:.4e}")
    assert abs(e - e_ref) <= 0.01 * e_ref, (e, e_ref)
    if (case, n) not in STALE_ARCHIVE:
        assert abs(e - pub) <= 0.01 * pub, (e, pub)


def _l1_fields(U, o, c):
    rho = U[:, 1] + U[:, 2]
    u = U[:, 3] / rho
    p = mixture_pressure(c, U)
    return {"rho": float(np.abs(rho - o["rho"]).mean() / np.abs(o["rho"]).mean()),
            "u": float(np.abs(u - o["u"]).mean() / max(np.abs(o["u"]).max(), 1e-300)),
            "p": float(np.abs(p - o["p"]).mean() / np.abs(o["p"]).max())}


@pytest.mark.gpu
def test_water_air_tube_against_the_exact_solution():
    """The 1000-cell water-air tube to 240 us: the relative L1 density error is that of the reference's
    own water-air tube at the same resolution (case 87, alpha 1e-7 and 241 us: 3.53e-3) within 20 %,
    and velocity and pressure are close to the exact ones in L1 (relative to their maxima)."""
    c = cases.water_air_tube(1000)
    U, st = _gpu_run(c)
    o, rho0 = exact_rho(c, 1000, st["t"])
    e = er.relative_l1_rho(U[:, 1] + U[:, 2], o["rho"], rho0)
    f = _l1_fields(U, o, c)
    print(f"water-air tube 1000 cells: L1(rho) Eq. (51) {e:.3e}; L1 rho / mean {f['rho']:.3e}, u / max {f['u']:.3e}, "
          f"p / max {f['p']:.3e}")
    assert e <= 1.2 * 3.531e-3, e
    assert f["u"] <= 2e-2 and f["p"] <= 2e-2, f


@pytest.mark.gpu
def test_nasg_instance_against_the_exact_solution():
    """The first NASG liquid-vapour problem of the batched workload (covolume 7.5e-4 m^3/kg), 200 steps:
    against the exact solution at its final time the GPU run's relative L1 density error is the C
    restatement of the reference's (run here on the same instance) to 1 %."""
    import refio

    c = next(b for b in cases.riemann_batch(count=512, seed=0) if b["nasg"])
    U, st = _gpu_run(c, 200)
    r = refio.run_port(c, mode=refio.MODE_STEPS, nsteps=200)
    assert r["steps"] == st["steps"] and abs(r["t"] - st["t"]) <= 1e-12 * st["t"]
    n = c["nx"]
    o, rho0 = exact_rho(c, n, st["t"])
    e_gpu = er.relative_l1_rho(U[:, 1] + U[:, 2], o["rho"], rho0)
    Ur = r["U"].reshape(-1, 8)
    e_ref = er.relative_l1_rho(Ur[:, 1] + Ur[:, 2], o["rho"], rho0)
    print(f"NASG instance {c['instance']} ({n} cells, t {st['t']:.3e}): L1(rho) GPU {e_gpu:.4e}, reference {e_ref:.4e}")
    assert abs(e_gpu - e_ref) <= 0.01 * e_ref and e_gpu <= 0.05, (e_gpu, e_ref)
