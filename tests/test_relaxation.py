"""p-pT relaxation (RELAX_LEVEL 1: instantaneous thermal relaxation in the
interface zone eps_I <= alpha1 <= 1 - eps_I) against the compiled reference.

Fixtures (tests/golden/make_golden.py), run by the reference itself through its
own RelaxationActivation at every attempt: the water-air tube (200 cells, 20
steps; its interface cells enter the zone as it smears, and the projection costs
the reference three halvings) and the 32 x 32 bubble field (tanh interfaces, 735
cells in the zone at t = 0; 3 steps).  The pT closure solves for p in
y = ln(p - p_lo) with exp / log (an ulp apart between glibc and CUDA's libm), so
whole runs are compared in L1 within 1e-6 per conservative variable, with the
same step and rejection counts.

Chemical relaxation (RELAX_LEVEL 2 p-pT-pTg, 3 p-pTg): the reference's
liquid-vapour cases 3 (dodecane shock tube, levels 2 and 3), 1 (water
cavitation tube), 32 (Bartak depressurisation, its own level 2), 41 (uniform
superheated state, periodic) and 72 (piston-compressed vapour bubble, 32 x 32,
grid-wide Rusanov speed), each of which moves vapour mass against its level-1
run.  The saturation table the pTg closure starts from is the reference's, bit
for bit (tests/golden/ref_sat_tables.npz)."""
from __future__ import annotations

import os

import numpy as np
import pytest

from helpers import FIELDS, fieldwise_l1, golden_case, load_golden

RELAX_FIXTURES = ["tube_relax_N200_20steps", "bubble_relax32_3steps",
                  # chemical relaxation
                  "dodecane_relax2_N200_20steps", "dodecane_relax3_N200_20steps", "cavitation_relax2_N200_20steps",
                  "bartak_N200_20steps", "chem0d_N16_10steps", "bubblecomp32_3steps",
                  "dodecane_relax2_N200_2steps", "dodecane_relax3_N200_2steps", "bartak_N200_5steps",
                  "bubblecomp32_1step",
                  # finite rates: mu, theta, nu in both forms, all three at once, unify = 1, the nu law
                  "mu0d_N4_10steps", "mu0d_expo_N4_10steps", "theta0d_N4_10steps", "theta0d_expo_N4_10steps",
                  "nu0d_N4_10steps", "nu0d_expo_N4_10steps", "dodecane_rates_N200_2steps",
                  "dodecane_rates_N200_20steps", "dodecane_unify_N200_2steps", "bartak_nulaw_N200_5steps",
                  "bartak_nulaw_N200_20steps", "bubble_theta32_3steps", "dodecane_unifyproj0_N200_2steps",
                  "dodecane_relax3_nulaw_N200_5steps"]
SAT_FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_sat_tables.npz")


@pytest.mark.parametrize("name", RELAX_FIXTURES)
def test_case_builders_reproduce_the_fixture_states(name):
    c, _, _ = golden_case(name)
    assert (c.get("relax", 0) >= 1 or "mu_rate" in c) and np.array_equal(c["U"], load_golden(name)["U0"])


@pytest.mark.parametrize("case", [1, 3, 30, 31, 32])
def test_saturation_table_is_the_reference_table(case):
    """The host table of the liquid / vapour pair equals the reference's SAT bit for bit: the
    same 1600-point ln p grid, first root, Newton continuation and critical-point bisection."""
    from diffusionimex_b200 import cases
    from diffusionimex_b200.solver import saturation_table

    ref = np.load(SAT_FIX)[f"case{case}"]
    t = saturation_table(dict(cases.reference_case(case, 16), relax=2))
    assert t["n"] > 1000 and np.isfinite(t["pcrit"]) and t["vcrit"] > 0
    assert np.array_equal(t["raw"], ref)


def test_saturation_line_is_the_gibbs_equality():
    """On the table, g_1(p, Tsat) = g_2(p, Tsat) to the Newton tolerance and Tsat rises with p."""
    from diffusionimex_b200 import cases
    from diffusionimex_b200.solver import saturation_table

    c = cases.reference_case(3, 16)
    t = saturation_table(c)
    p, T = np.exp(t["lp"]), t["T"]

    def gibbs(ph):
        s = ph["cv"] * (ph["g"] * np.log(T) - (ph["g"] - 1.0) * np.log(p + ph["pinf"])) + ph["qp"]
        return ph["g"] * ph["cv"] * T + ph["b"] * p + ph["q"] - T * s

    g1, g2 = gibbs(c["phases"][0]), gibbs(c["phases"][1])
    assert np.all(np.abs(g1 - g2) <= 1e-8 * (np.abs(g1) + 1.0))
    assert np.all(np.diff(T) > 0)


def test_relaxation_case_states_are_the_reference_initialisation():
    """Cases 1, 3, 30, 31, 32, 40, 41 and the 32 x 32 case 72 as the reference's own
    u_initialization builds them (sub-cell averages for case 72), where the compiled reference
    exists."""
    import refio
    from diffusionimex_b200 import cases

    if not refio.ref_available():
        pytest.skip("compiled reference not available")
    for case in (1, 3, 30, 31, 32, 40, 41):
        r = refio.run_ref_main_files([f"case={case}", "N=100", "init=1"], nx=100)
        assert np.array_equal(r["U"], cases.reference_case(case, 100)["U"]), case
    r = refio.run_ref_main_files(["case=72", "N=32", "ny=32", "init=1"], nx=32, ny=32)
    c = cases.bubble_compression(32, 32)
    assert np.array_equal(r["U"].reshape(c["U"].shape), c["U"])


def test_c_restatement_rejects_thermal_relaxation():
    import refio

    c, _, _ = golden_case("bubble_relax32_3steps")
    with pytest.raises(Exception):
        refio.run_port(c, mode=refio.MODE_STEPS, nsteps=1)


@pytest.mark.gpu
@pytest.mark.parametrize("name", RELAX_FIXTURES)
def test_relaxation_runs_match_reference(name):
    from diffusionimex_b200 import Solver

    g = load_golden(name)
    c, mode, nsteps = golden_case(name)
    s = Solver(c)
    s.advance(nsteps)
    U, st = s.state(), s.stats()
    s.close()
    assert st["steps"] == g["meta"]["steps"] and st["rejects"] == g["meta"]["rejects"], (st, g["meta"])
    assert np.isfinite(U).all()
    d = fieldwise_l1(U, g["U"])
    # Chemical relaxation decides a cell's closure type by comparing its temperature with Tsat(p),
    # and a pTg cell sits at T = Tsat(p): those decisions are round-off decisions, so the
    # reference's own answer moves under a one-ulp change of its log / exp / pow (the fixture's
    # `noise`, per field the larger of the ulp-up and ulp-down runs).  Bar: 1e-6, or 10x that
    # noise where it is larger; 1e-9 for a run the perturbation leaves within 1e-12 (one that has
    # made no such decision: the closures themselves are then compared).
    bar = np.full(8, 1e-6)
    if "noise" in g:
        bar = np.full(8, 1e-9) if g["noise"].max() < 1e-12 else np.maximum(1e-6, 10 * g["noise"])
    assert np.all(d <= bar), {f: f"{v:.2e} (bar {b:.2e})" for f, v, b in zip(FIELDS, d, bar)}
