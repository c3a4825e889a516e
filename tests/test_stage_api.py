"""The stage-level ABI (spb6g_stage / spb6g_stage_accept): main()'s time loop
(src/SPB6_PC_IMEX_omp.cpp:1316-1384) restated here in Python with its three stage
calls -- TVDReconstruction, Update, PressureSubsystem -- replaced by spb6g_stage, as
a harness that swaps them would do.  Driven stage by stage it must give bitwise the
handle's own loop (spb6g_step), and the reference's run of the same case."""
from __future__ import annotations

import math

import numpy as np
import pytest

from diffusionimex_b200 import Solver, SolverError, cases
from helpers import fieldwise_l1, golden_case, load_golden

pytestmark = pytest.mark.gpu

RAMP_FACTOR = 1.2  # ramp_factor (:76)


def set_tab(rk: int):
    """main()'s set_tab (:1281-1303): the explicit and implicit tableaux."""
    Ae = [[0.0] * 3 for _ in range(3)]
    Ai = [[0.0] * 3 for _ in range(3)]
    if rk == 1:
        Ai[0][0] = 1.0
    elif rk == 2:
        bb = 1.0 - 1.0 / math.sqrt(2.0)
        cc = 1.0 / (2.0 * bb)
        Ae[1][0] = cc
        Ai[0][0] = bb
        Ai[1][0] = 1 - bb
        Ai[1][1] = bb
    elif rk == 3:
        r12, r13, r14 = 0.5, 1.0 / 3.0, 1.0 / 4.0
        Ae[1][0] = Ae[2][0] = Ae[2][1] = r12
        Ai[0][0] = Ai[1][1] = r14
        Ai[2][0] = Ai[2][1] = Ai[2][2] = r13
    return Ae, Ai


def main_loop(s: Solver, c: dict, nsteps: int) -> dict:
    """nsteps iterations of main()'s do-while loop over the stage API (nsteps <= 0: to t_end)."""
    t, dtprev, startup = 0.0, -1.0, True
    tend = c["tend"]
    steps = rejects = 0
    while t < tend * (1 - 1e-12) and (nsteps <= 0 or steps < nsteps):
        ramping = False
        if c.get("dtfix", 0.0) > 0:
            dt = c["dtfix"]
        else:
            dt = c["cfl"] * s.caldt(bool(c.get("acdt", 0)))
            if c.get("ramp", 1):
                if dtprev < 0:
                    dtprev = c["cfl_ac"] * s.caldt(True) / RAMP_FACTOR
                if dt > RAMP_FACTOR * dtprev:
                    dt = RAMP_FACTOR * dtprev
                    ramping = True
            if not math.isfinite(dt):
                dt = c["cfl_ac"] * s.caldt(True)
        dt = min(dt, tend - t)
        assert dt > 1e-12 * tend
        done = False
        for _ in range(30):
            rk = 1 if (c.get("ramp", 1) and ramping and startup) else c["rk"]
            Ae, Ai = set_tab(rk)
            ok = True
            for rks in range(rk):
                ok = s.stage(rks, Ae[rks], Ai[rks], dt) == 0
                if not ok:
                    break
            if ok:
                s.stage_accept(dt)
                done = True
                break
            rejects += 1
            dt *= 0.5
        assert done
        t = t + dt
        dtprev = dt
        steps += 1
        if not ramping:
            startup = False
    return {"steps": steps, "rejects": rejects, "t": t}


@pytest.mark.parametrize("name,builder,nsteps", [
    ("case 87 N200 (1D, Thomas)", lambda: cases.reference_case(87, 200), 30),
    ("bubble field 48^2 (2D, ramp + LSDIRK2)", lambda: cases.bubble_field(48, seed=0, nbub=2), 8),
    ("low-Mach 32^2, SSP2(3,3,2)", lambda: dict(cases.lowmach_bubbles(32, seed=0, nbub=2), rk=3), 4),
])
def test_stage_loop_is_bitwise_the_handle_loop(name, builder, nsteps):
    c = builder()
    a = Solver(c)
    a.advance(nsteps)
    b = Solver(c)
    info = main_loop(b, c, nsteps)
    sa, sb = a.stats(), b.stats()
    assert (sb["steps"], info["rejects"]) == (sa["steps"], sa["rejects"]), (sa, sb, info)
    assert sb["newton_it"] == sa["newton_it"] and sb["bicg_it"] == sa["bicg_it"]
    assert np.array_equal(a.state(), b.state()), name
    Pa, ra = a.pressure()
    Pb, rb = b.pressure()
    assert np.array_equal(Pa, Pb) and ra == rb
    assert a.time_state()[0] == b.time_state()[0] == info["t"]
    a.close()
    b.close()


def test_stage_loop_matches_reference_case87():
    """Case 87 (N = 200) to t_end through the stage API against the reference's run."""
    g = load_golden("case87_N200_tend")
    c, mode, nsteps = golden_case("case87_N200_tend")
    s = Solver(c)
    info = main_loop(s, c, 0)
    assert info["steps"] == g["meta"]["steps"]
    d = fieldwise_l1(s.state(), g["U"])
    s.close()
    # the bar of the handle's own loop on this case: 1e-6 of the field maximum, or 10x the
    # reference's own L1 change under round-off perturbations (one-ulp libm, FD step 1.01e-7)
    if d.max() > 1e-6:
        import refio

        noise = np.maximum(*[fieldwise_l1(refio.run_port(c, mode=refio.MODE_TEND, variant=v)["U"], g["U"])
                             for v in ("ulp", "fd")])
        assert np.all(d <= np.maximum(10 * noise, 1e-6)), (d, noise)


def test_stage_api_refuses_out_of_order_stages():
    c = cases.bubble_field(32, seed=0, nbub=1)
    s = Solver(c)
    Ae, Ai = set_tab(2)
    with pytest.raises(SolverError):  # stage 1 before stage 0 of the attempt
        s.stage(1, Ae[1], Ai[1], 1e-7)
    with pytest.raises(SolverError):  # nothing to accept
        s.stage_accept(1e-7)
    assert s.stage(0, Ae[0], Ai[0], 1e-7) == 0
    assert s.stage(1, Ae[1], Ai[1], 1e-7) == 0
    s.stage_accept(1e-7)
    assert s.stats()["steps"] == 1
    s.close()
