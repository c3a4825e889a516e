"""CPU tests of the oracle: the C restatement (oracle/spb6_oracle.c) against the
reference solver's own outputs (golden fixtures made by the compiled reference),
the reference harness loop against the reference main(), and the oracle against
the reference's archived profiles."""
from __future__ import annotations

import os

import numpy as np
import pytest

import refio
from helpers import golden_case, load_golden, mixture_pressure
from diffusionimex_b200 import cases

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

FIXTURES = ["case87_N200_tend", "case5_N100_tend", "case83_N200_10steps", "tube_N1000_1step", "tube_N200_stage",
            "bubble48_stage", "bubble48_4steps", "lowmach32_3steps", "shock64x32_3steps", "nasg256_20steps",
            # boundary variants: walls, pistons, pressure outlets, 1D periodic (cyclic matrix on BiCGStab)
            "tube_walls_N200_20steps", "tube_piston_N200_20steps", "tube_outlet_N200_20steps",
            "tube_periodic_N200_10steps", "bubble_walls32_3steps", "bubble_outlet32_3steps",
            # grid-wide Rusanov dissipation speed (rus_local = 0)
            "case13_N200_20steps", "lowmach_rus0_32_stage", "lowmach_rus0_32_3steps"]
MODES = {"tend": refio.MODE_TEND, "steps": refio.MODE_STEPS, "stage": refio.MODE_STAGE}


@pytest.mark.parametrize("name", FIXTURES)
def test_port_bitwise_equals_reference(name):
    """The C restatement reproduces the compiled reference bit for bit."""
    g = load_golden(name)
    c, mode, nsteps = golden_case(name)
    assert np.array_equal(c["U"], g["U0"]), "case builder drifted from the fixture"
    r = refio.run_port(c, mode=MODES[mode], nsteps=nsteps)
    assert r["status"] == g["meta"]["status"]
    assert r["steps"] == g["meta"]["steps"] and r["newton_it"] == g["meta"]["newton_it"]
    assert np.array_equal(r["U"], g["U"])
    assert np.array_equal(r["P"], g["P"])
    if mode == "stage":
        for k in ("Xs", "a2s", "ube_x", "ube_y", "phi_x", "phi_y"):
            assert np.array_equal(r[k], g[k]), k


def test_port_long_tube_run():
    """Config 1 (1D water-air tube, 1000 cells, to 240 us) bitwise against the reference."""
    g = load_golden("tube_N1000_tend")
    c, _, _ = golden_case("tube_N1000_tend")
    r = refio.run_port(c, mode=refio.MODE_TEND)
    assert r["steps"] == g["meta"]["steps"] == 243
    assert np.array_equal(r["U"], g["U"])


@pytest.mark.skipif(not refio.ref_available(), reason="needs the compiled reference (oracle/_ref)")
def test_harness_loop_equals_reference_main():
    """The harness's restated time loop equals the reference main() on its own case 87."""
    m = refio.run_ref_main(["case=87", "N=200"], 200)
    r = refio.run_ref(cases.reference_case(87, 200), mode=refio.MODE_TEND)
    assert m["steps"] == r["steps"]
    assert np.array_equal(m["U"], r["U"])


# measured: case 5 N100 p/u/rho mean <= 6e-11, max <= 7e-10; case 87 N200 mean <= 1.3e-6, max <= 1.5e-5
@pytest.mark.parametrize("tag,case,n,tmean,tmax", [("archived_case5_N100", 5, 100, 1e-9, 1e-8),
                                                  ("archived_case87_N200", 87, 200, 1e-5, 1e-4)])
def test_oracle_vs_archived_profiles(golden_dir, tag, case, n, tmean, tmax):
    """The archived profiles come from the serial-root variant (src/SPB6_PC_IMEX.cpp); the OpenMP
    variant reorders root finding, so agreement is at the round-off-amplification level the
    reference documents (case 5: p mean 2.9e-8 / max 2.5e-7 of max|p|)."""
    z = np.load(os.path.join(golden_dir, f"{tag}.npz"))
    c = cases.reference_case(case, n)
    r = refio.run_port(c, mode=refio.MODE_TEND)
    U = r["U"].reshape(-1, 8)
    p = mixture_pressure(c, U)
    rho = U[:, 1] + U[:, 2]
    u = U[:, 3] / rho
    scale_p, scale_u = np.abs(z["p"]).max(), np.abs(z["u"]).max()
    scale_r = np.abs(z["rho"]).max()
    for a, b, s in ((p, z["p"], scale_p), (u, z["u"], scale_u), (rho, z["rho"], scale_r)):
        assert np.abs(a - b).mean() / s < tmean
        assert np.abs(a - b).max() / s < tmax


def test_epoxy_spinel_initial_states_are_the_reference():
    """Cases 12 and 13 (SPB 5.1 / 5.2; case 13 with the grid-wide Rusanov speed) as the
    reference's own u_initialization builds them, where the compiled reference exists."""
    if not refio.ref_available():
        pytest.skip("compiled reference not available")
    for case in (12, 13):
        r = refio.run_ref_main_files([f"case={case}", "N=200", "init=1"], nx=200)
        assert np.array_equal(r["U"], cases.reference_case(case, 200)["U"])
    assert cases.reference_case(13)["rus_local"] == 0 and cases.reference_case(12)["rus_local"] == 1


def test_fixture_builders_keep_their_settings():
    """Every fixture's case builder still produces the settings the fixture was made with (a
    changed tolerance, step size or rate would leave U0 alone but the run different)."""
    import glob
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(GOLDEN_DIR, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    names = [os.path.basename(f)[4:-4] for f in sorted(glob.glob(os.path.join(GOLDEN_DIR, "ref_*.npz")))]
    checked = 0
    for name in names:
        if name not in mg.CASES:
            continue
        meta = load_golden(name)["meta"]
        c, _, _ = mg.build_case(name)
        assert mg.case_settings(c) == meta["config"], name
        checked += 1
    assert checked == len(mg.CASES)


def test_reference_2d_initial_states():
    """Cases 56, 57, 58, 70, 71, 72, 73 as the reference's own u_initialization builds them, 4 x 4
    sub-cell averages included, where the compiled reference exists."""
    if not refio.ref_available():
        pytest.skip("compiled reference not available")
    for case, build, nx, ny in ((56, lambda nx, ny: cases.vortex_bb(nx), 40, 40),
                                (57, lambda nx, ny: cases.taylor_green(nx), 50, 50),
                                (58, lambda nx, ny: cases.taylor_green(nx, True), 50, 50),
                                (70, cases.he_bubble, 60, 16), (71, cases.richtmyer_meshkov, 60, 20),
                                (72, cases.bubble_compression, 32, 32), (73, cases.underwater_explosion, 60, 40)):
        r = refio.run_ref_main_files([f"case={case}", f"N={nx}", f"ny={ny}", "init=1"], nx=nx, ny=ny)
        c = build(nx, ny)
        assert np.array_equal(r["U"].reshape(c["U"].shape), c["U"]), case


def test_reference_1d_initial_states():
    """Every 1D case reference_case restates (0-6, 12, 13, 20, 21, 30-32, 40, 41, 60, 61, 80-88) as
    the reference's own u_initialization builds it, where the compiled reference exists; the 2D
    ids go to their builders."""
    if not refio.ref_available():
        pytest.skip("compiled reference not available")
    for case in (0, 1, 2, 3, 4, 5, 6, 12, 13, 20, 21, 30, 31, 32, 40, 41, 60, 61, 80, 81, 82, 83, 84, 85, 86, 87, 88):
        r = refio.run_ref_main_files([f"case={case}", "N=64", "init=1"], nx=64)
        assert np.array_equal(r["U"], cases.reference_case(case, 64)["U"]), case
    c = cases.reference_case(73, 60, 40)
    assert (c["nx"], c["ny"], c["case"]) == (60, 40, 73)
