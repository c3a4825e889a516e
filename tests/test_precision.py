"""Precision form (no counterpart in the reference): FP32 reconstruction, Rusanov
fluxes and SpMV; FP64 EOS inversion, relaxation Newton, BiCGStab reductions and
residuals.  Its results are compared with the FP64 path on the same runs, on small
grids and on the precision form's own configurations (the 8-bubble field on 2048^2
and the shock-bubble on 2048 x 1024, ten steps after three); the L1 errors of
alpha, p and u (relative to the field mean) are printed and held to the bounds
below."""
from __future__ import annotations

import numpy as np
import pytest

from diffusionimex_b200 import Solver, cases

pytestmark = pytest.mark.gpu


def _run(c, steps, warmup):
    s = Solver(c)
    s.advance(warmup)
    s.advance(steps)
    st = s.stats()
    U = s.state()
    P, pref = s.pressure()
    s.close()
    return U, P + pref, st


def _l1(a, b):
    return float(np.abs(a - b).mean() / max(np.abs(b).mean(), 1e-300))


@pytest.mark.parametrize("name,make,bounds,steps", [
    ("bubbles256", lambda: cases.bubble_field(256, seed=0, nbub=4), (1e-5, 1e-4, 2e-2), 8),
    ("shock256x128", lambda: cases.shock_bubble(256, 128), (1e-5, 1e-4, 1e-3), 8),
    ("tube1000", lambda: cases.water_air_tube(1000), (1e-5, 1e-4, 1e-2), 8),
    # the precision form's own configurations, ten steps after three
    ("bubbles2048", lambda: cases.bubble_field(2048, seed=0, nbub=8), (1e-6, 1e-5, 1e-2), 10),
    ("shock2048x1024", lambda: cases.shock_bubble(2048, 1024), (1e-6, 1e-4, 1e-4), 10),
])
def test_precision_form_against_fp64(name, make, bounds, steps, record_property):
    c64, c32 = make(), make()
    c32["precision"] = 1
    U1, P1, s1 = _run(c64, steps, 3)
    U2, P2, s2 = _run(c32, steps, 3)
    assert s2["steps"] == s1["steps"] and s2["rejects"] == s1["rejects"]
    assert np.isfinite(U2).all() and np.isfinite(P2).all()
    rho1, rho2 = U1[..., 1] + U1[..., 2], U2[..., 1] + U2[..., 2]
    e_alpha, e_p, e_u = _l1(U2[..., 0], U1[..., 0]), _l1(P2, P1), _l1(U2[..., 3] / rho2, U1[..., 3] / rho1)
    record_property("L1_alpha_p_u", [e_alpha, e_p, e_u])
    print(f"precision form {name}: L1 alpha {e_alpha:.2e} p {e_p:.2e} u {e_u:.2e}")
    assert e_alpha < bounds[0] and e_p < bounds[1] and e_u < bounds[2], (e_alpha, e_p, e_u)
    # and it is a different computation (FP32 really runs)
    assert not np.array_equal(U1, U2)
