"""Learned warm start inside the solver (no counterpart in the reference).

The solver evaluates the residual at the network's guess and starts Newton from it
only when its residual norm is below the plain guess's; Newton keeps its
tolerance, so the run must reach the plain run's solution either way.  The last
test trains a network on other seeds of the 8-bubble field and records what it
gains over the plain guess on seed 0 (stages where the learned guess was chosen,
BiCGStab iterations, Newton iterations)."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from diffusionimex_b200 import cases

pytestmark = pytest.mark.gpu

N = 256


def _run(case, steps, warmup, mlp=None, norm=None):
    from diffusionimex_b200 import learned

    return learned.run_case(case, steps, warmup, mlp=mlp, norm=norm)


def test_dump_pairs_and_feature_rows():
    import torch

    from diffusionimex_b200 import learned

    c = cases.bubble_field(N, seed=1, nbub=4)
    norm = learned.pilot_norm(c, warmup=3, stages=2)
    assert len(norm) == 19 and all(np.isfinite(norm)) and norm[18] > 0
    X, T = learned.dump_pairs([(c, 3, 2)], norm)
    assert X.shape == (2 * N * N, 64) and T.shape == (2 * N * N,)
    Xf = X.float()
    assert torch.isfinite(Xf).all() and torch.isfinite(T).all()
    assert (Xf[:, 54:] == 0).all()  # padding columns
    # centre features are standardised with the pilot's statistics
    assert abs(float(Xf[:, 0].mean())) < 1.0 and 0.1 < float(Xf[:, 0].std()) < 10.0


def test_bad_guess_is_never_chosen_and_changes_nothing():
    """A network that predicts a pressure change of 50 target standard deviations everywhere
    has the larger residual every stage, so the plain guess stands everywhere and the run is
    bitwise the plain run."""
    from diffusionimex_b200 import learned
    from diffusionimex_b200.warmstart import MLP

    c = cases.bubble_field(N, seed=0, nbub=4)
    norm = learned.pilot_norm(cases.bubble_field(N, seed=1, nbub=4), warmup=3, stages=2)
    m = MLP()
    p = np.zeros(m.nparam, np.float32)
    p[-1] = 50.0  # output bias: y = 50 for every cell
    m.set_params(p)
    plain, Pp = _run(c, 6, 3)
    warm, Pw = _run(c, 6, 3, mlp=m, norm=norm)
    assert warm["learned"] == 0
    assert np.array_equal(Pp, Pw)
    assert warm["newton_it"] == plain["newton_it"] and warm["bicg_it"] == plain["bicg_it"]
    m.close()


def test_trained_warm_start_reaches_the_plain_solution_and_records_its_gain():
    import torch

    from diffusionimex_b200 import learned

    norm = learned.pilot_norm(cases.bubble_field(N, seed=1, nbub=4), warmup=3, stages=4)
    X, T = learned.dump_pairs([(cases.bubble_field(N, seed=s, nbub=4), 3, 30) for s in (1, 2)], norm)
    m, hist = learned.train_mlp(X, T, steps=400, batch=1 << 18, lr=2e-3, log_every=100)
    assert hist[-1][1] < hist[0][1]
    del X, T
    torch.cuda.empty_cache()
    r = learned.compare(cases.bubble_field(N, seed=0, nbub=4), m, norm, steps=15, warmup=3)
    # same converged pressure to the Newton tolerance (scaled residual 1e-10 allows ~1e-8 relative)
    assert r["L1_rel_p"] < 1e-6
    assert r["learned"]["steps"] == r["plain"]["steps"]
    out = os.environ.get("SPB6G_LEARNED_REPORT")
    if out:
        with open(out, "w") as f:
            json.dump(r, f)
    m.close()
