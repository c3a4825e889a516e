"""p-pT relaxation (RELAX_LEVEL 1: instantaneous thermal relaxation in the
interface zone eps_I <= alpha1 <= 1 - eps_I) against the compiled reference.

Fixtures (tests/golden/make_golden.py), run by the reference itself through its
own RelaxationActivation at every attempt: the water-air tube (200 cells, 20
steps; its interface cells enter the zone as it smears, and the projection costs
the reference three halvings) and the 32 x 32 bubble field (tanh interfaces, 735
cells in the zone at t = 0; 3 steps).  The pT closure solves for p in
y = ln(p - p_lo) with exp / log (an ulp apart between glibc and CUDA's libm), so
whole runs are compared in L1 within 1e-6 per conservative variable, with the
same step and rejection counts."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import FIELDS, fieldwise_l1, golden_case, load_golden

RELAX_FIXTURES = ["tube_relax_N200_20steps", "bubble_relax32_3steps"]


@pytest.mark.parametrize("name", RELAX_FIXTURES)
def test_case_builders_reproduce_the_fixture_states(name):
    c, _, _ = golden_case(name)
    assert c["relax"] == 1 and np.array_equal(c["U"], load_golden(name)["U0"])


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
    assert np.all(d <= 1e-6), {f: f"{v:.2e}" for f, v in zip(FIELDS, d)}
