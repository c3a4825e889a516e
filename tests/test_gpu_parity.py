"""GPU parity tests: the sm_100a path through the C ABI against the reference's
own outputs (golden fixtures) and the C restatement.

Tolerances (field-max-normalised, per conservative variable):
  * explicit predictor (reconstruction + Rusanov update): no reductions are
    involved, so X*, alpha2*, face velocities and limiters must agree to 1e-15;
  * one stage / one step: 1e-12 (the one-step bar for FP64 parity).  In 1D the linear
    solve is the same sequential Thomas sweep as the reference and the result is
    typically bit-identical; in 2D BiCGStab's dot products are summed in a
    different (deterministic, tree) order, so the converged pressure differs at
    the solver-tolerance level;
  * runs of many steps: mean |diff| / max <= 1e-6 (the reference's own serial-vs-
    OpenMP variants differ by 1e-6 on case 87 N200, tests/test_oracle.py).

The shock dissipation budget of strong-shock cells comes from an adaptive RK45
profile shooting whose step control calls pow / exp / log; CUDA's libm and glibc
differ by an ulp on some arguments, which moves the shooting result at its own
tolerance (1e-8..1e-10) and, in ill-conditioned cells, the per-phase split much
more.  The reference is equally sensitive: a one-ulp change of those calls in the
C restatement (oracle variant "ulp") changes the same cells by the same amounts.
Cases with strong shocks are therefore held to the reference's own acceptance
rule (docs/code/openmp_optimisation.md:81-82): the GPU may differ from the
reference by no more than 10x the reference's change under a round-off
perturbation (one-ulp libm, FD step 1e-7 -> 1.01e-7), and stages are checked
exactly with the GPU's budget injected into the oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

import refio
from helpers import FIELDS, fieldwise_l1, fieldwise_maxrel, golden_case, load_golden
from diffusionimex_b200 import Solver, SolverError, cases

pytestmark = pytest.mark.gpu


def run_gpu(case, mode, nsteps):
    s = Solver(case)
    if mode == "stage":
        out = s.stage_dump(case["dtfix"])
    elif mode == "steps":
        s.advance(nsteps)
        out = {}
    else:
        s.advance(0)
        out = {}
    out["U"] = s.state()
    out["P"], out["p_ref"] = s.pressure()
    out["stats"] = s.stats()
    s.close()
    return out


def report(a, b):
    return {f: f"{v:.2e}" for f, v in zip(FIELDS, fieldwise_maxrel(a, b))}


@pytest.mark.parametrize("name", ["tube_N200_stage", "bubble48_stage", "lowmach_order1_32_stage"])
def test_stage_explicit_and_implicit(name):
    g = load_golden(name)
    c, mode, _ = golden_case(name)
    r = run_gpu(c, mode, 0)
    for k in ("a2s", "ube_x", "ube_y", "phi_x", "phi_y"):
        scale = max(np.abs(g[k]).max(), 1e-300)
        assert np.abs(r[k] - g[k]).max() / scale <= 1e-15, k
    assert fieldwise_maxrel(r["Xs"], g["Xs"]).max() <= 1e-15, report(r["Xs"], g["Xs"])
    assert fieldwise_maxrel(r["U"], g["U"]).max() <= 1e-12, report(r["U"], g["U"])
    pscale = np.abs(g["P"]).max() + abs(g["meta"]["p_ref"])
    assert np.abs(r["P"] - g["P"]).max() / pscale <= 1e-12


@pytest.mark.parametrize("name", ["tube_N1000_1step", "bubble48_4steps"])
def test_first_steps_match_reference(name):
    g = load_golden(name)
    c, mode, nsteps = golden_case(name)
    r = run_gpu(c, mode, nsteps)
    assert r["stats"]["steps"] == g["meta"]["steps"]
    assert fieldwise_maxrel(r["U"], g["U"]).max() <= 1e-12, report(r["U"], g["U"])


def noise_level(c, mode, nsteps, U_ref):
    """Per-field change of the reference under round-off perturbations (one-ulp libm in the shock
    shooting; FD Jacobian step 1.01e-7), field-max-normalised."""
    m = {"steps": refio.MODE_STEPS, "tend": refio.MODE_TEND, "stage": refio.MODE_STAGE}[mode]
    lv = [fieldwise_maxrel(refio.run_port(c, mode=m, nsteps=nsteps, variant=v)["U"], U_ref) for v in ("ulp", "fd")]
    return np.maximum(lv[0], lv[1])


@pytest.mark.parametrize("name", ["lowmach32_3steps", "shock64x32_3steps", "bubble48_4steps", "tube_N1000_1step"])
def test_first_steps_within_reference_noise(name):
    g = load_golden(name)
    c, mode, nsteps = golden_case(name)
    r = run_gpu(c, mode, nsteps)
    assert r["stats"]["steps"] == g["meta"]["steps"]
    d = fieldwise_maxrel(r["U"], g["U"])
    noise = noise_level(c, mode, nsteps, g["U"])
    assert np.all(d <= np.maximum(10 * noise, 1e-12)), {"gpu": report(r["U"], g["U"]), "noise": noise.tolist()}


def test_1d_tube_one_step_bitwise():
    """1D water-air tube (1000 cells), first step: Thomas path, bit-identical to the reference."""
    g = load_golden("tube_N1000_1step")
    c, mode, nsteps = golden_case("tube_N1000_1step")
    r = run_gpu(c, mode, nsteps)
    assert r["stats"]["newton_it"] == g["meta"]["newton_it"]
    assert np.array_equal(r["U"], g["U"]), report(r["U"], g["U"])


@pytest.mark.parametrize("name", ["case87_N200_tend", "case5_N100_tend", "tube_N1000_tend", "nasg256_20steps",
                                  "tube_walls_N200_20steps", "tube_piston_N200_20steps", "tube_outlet_N200_20steps",
                                  "tube_periodic_N200_10steps", "bubble_walls32_3steps", "bubble_outlet32_3steps",
                                  "case83_N200_10steps", "case13_N200_20steps", "lowmach_rus0_32_3steps",
                                  "tube_order1_N200_20steps", "bubble_order1_32_3steps", "hebubble75x20_3steps",
                                  "rm60x20_3steps", "vortex24_3steps", "taylorgreen24_3steps"])
def test_runs_match_reference_in_l1(name):
    """Whole runs in L1: within 1e-6 of the field maximum, or within 10x the reference's own L1
    change under round-off perturbations (one-ulp libm, FD step 1.01e-7) where that is larger --
    case 87 to t_end moves by 1e-6 in rho u under either perturbation."""
    g = load_golden(name)
    c, mode, nsteps = golden_case(name)
    r = run_gpu(c, mode, nsteps)
    assert r["stats"]["steps"] == g["meta"]["steps"]
    d = fieldwise_l1(r["U"], g["U"])
    if d.max() > 1e-6:
        m = {"steps": refio.MODE_STEPS, "tend": refio.MODE_TEND}[mode]
        noise = np.maximum(*[fieldwise_l1(refio.run_port(c, mode=m, nsteps=nsteps, variant=v)["U"], g["U"])
                             for v in ("ulp", "fd")])
        assert np.all(d <= np.maximum(10 * noise, 1e-6)), {"gpu": report(r["U"], g["U"]), "noise": noise.tolist()}


def test_deterministic_repeat():
    c, mode, nsteps = golden_case("bubble48_4steps")
    a = run_gpu(c, mode, nsteps)
    b = run_gpu(c, mode, nsteps)
    assert np.array_equal(a["U"], b["U"]) and np.array_equal(a["P"], b["P"])


def test_against_c_restatement_odd_sizes():
    """Ragged grids (odd, non-square, thin) against the C restatement, 2 steps."""
    for nx, ny in ((17, 5), (33, 7), (5, 31)):
        c = cases.bubble_field(nx, seed=2, nbub=1)
        # rebuild on a non-square grid with the same recipe
        c = dict(c)
        c.update(nx=nx, ny=ny, newton_tol=1e-13, bicg_tol=1e-13)
        x, y, dx, _ = cases.cell_centres(c)
        X, Y = np.meshgrid(x, y)
        f = 0.5 * (1 + np.tanh((np.hypot(X - 0.5, Y - 0.5) - 0.3) / (2 * dx)))
        a1 = 1e-6 + (1 - 2e-6) * f
        p = 1e5 + (1e7 - 1e5) * f
        c["U"] = cases.prim2cell(c["phases"], a1, 1000.0, 1.0, 0.0, 0.0, p, p)
        o = refio.run_port(c, mode=refio.MODE_STEPS, nsteps=2)
        r = run_gpu(c, "steps", 2)
        assert r["stats"]["steps"] == o["steps"]
        assert fieldwise_maxrel(r["U"], o["U"]).max() <= 1e-11, (nx, ny, report(r["U"], o["U"]))


def test_periodic_conservation_at_scale():
    """Periodic low-Mach field at 256^2: mass and energy are conserved to round-off."""
    c = cases.lowmach_bubbles(256, seed=0, nbub=4)
    s = Solver(c)
    U0 = s.state().reshape(-1, 8)
    s.advance(3)
    U1 = s.state().reshape(-1, 8)
    for k in (1, 2, 7):
        assert abs(U1[:, k].sum() - U0[:, k].sum()) / abs(U0[:, k].sum()) < 1e-12
    assert s.stats()["bicg_it"] > 0


def test_inadmissible_state_fails_like_reference():
    """A negative phase mass makes every attempt fail (Update's rho check), so the step ends
    in the reference's FAILED state after 30 halvings (main :1375-1378)."""
    c = cases.water_air_tube(64)
    U = c["U"].copy()
    U[0, 10, 1] = -1.0
    U[0, 10, 2] = -1.0
    c["U"] = U
    s = Solver(c, init_pressure=False)
    s.set_pressure(np.zeros((1, 64)), 1e5)
    with pytest.raises(SolverError) as e:
        s.step()
    assert e.value.status == 4
    assert s.stats()["rejects"] == 30


STAGE_KEYS = ["Xs", "a2s", "ube_x", "ube_y", "phi_x", "phi_y", "fx_ubs", "fx_kp", "fx_wl", "fx_pv",
              "fy_ubs", "fy_kp", "fy_wl", "fy_pv", "kw"]


@pytest.mark.parametrize("name", ["lowmach32_stage", "shock64x32_stage", "bubble48_stage", "lowmach_rus0_32_stage"])
def test_stage_data_matches_restatement(name):
    """Every array one stage produces -- explicit predictor, face coefficients of the implicit
    face velocity/pressure, residual scale, shock budget -- against the C restatement, then the
    stage's final state against the reference fixture."""
    c, mode, _ = golden_case(name)
    o = refio.run_port(c, mode=refio.MODE_STAGE)
    s = Solver(c)
    r = s.stage_dump(c["dtfix"])
    r.update(s.stage_data())
    U = s.state()
    s.close()
    bad = {}
    for k in STAGE_KEYS:
        a, b = np.asarray(r[k]), np.asarray(o[k])
        scale = max(np.abs(b).max(), 1e-300)
        d = np.abs(a - b).max() / scale
        if not d <= 1e-14:
            idx = np.unravel_index(np.argmax(np.abs(a - b)), a.shape)
            bad[k] = f"{d:.2e} at {idx}: gpu {a[idx]!r} oracle {b[idx]!r}"
    assert not bad, bad
    # shock budget: total Q per cell to the shooting tolerance; the per-phase split within 10x the
    # reference's own one-ulp-libm change
    ou = refio.run_port(c, mode=refio.MODE_STAGE, variant="ulp")
    tot_g, tot_o = r["qph0"] + r["qph1"], o["qph0"] + o["qph1"]
    assert np.abs(tot_g - tot_o).max() <= 1e-8 * max(np.abs(tot_o).max(), 1e-300)
    for k in ("qph0", "qph1"):
        scale = max(np.abs(o[k]).max(), 1e-300)
        assert np.abs(r[k] - o[k]).max() / scale <= max(10 * np.abs(ou[k] - o[k]).max() / scale, 1e-14), k
    # the implicit solve with the GPU's budget injected into the oracle: same state to 1e-12
    oi = refio.run_port(c, mode=refio.MODE_STAGE, qph=np.stack([r["qph0"], r["qph1"]]))
    assert fieldwise_maxrel(U, oi["U"]).max() <= 1e-12, report(U, oi["U"])


@pytest.mark.parametrize("name", ["tube_jreuse_N1000_20steps", "bubble_jreuse48_4steps", "lowmach_jreuse32_3steps"])
def test_modified_newton_matches_reference(name):
    """jreuse = 1 (Newton_Solver :826-830, :887): the kept Jacobian's linear convergence takes the
    reference's own number of Newton iterations (205 against 86 with a fresh Jacobian on the
    tube), and the runs agree in L1 as the plain ones do."""
    g = load_golden(name)
    c, mode, nsteps = golden_case(name)
    r = run_gpu(c, mode, nsteps)
    st = r["stats"]
    assert (st["steps"], st["rejects"], st["newton_it"]) == (g["meta"]["steps"], g["meta"]["rejects"],
                                                            g["meta"]["newton_it"]), (st, g["meta"])
    d = fieldwise_l1(r["U"], g["U"])
    assert np.all(d <= 1e-6), report(r["U"], g["U"])
