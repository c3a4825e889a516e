"""Batched form (no counterpart in the reference): independent 1D Riemann problems
(water/air stiffened gas or NASG liquid/vapour, uneven sizes) advanced in one
persistent launch.  Every grid runs the same per-cell arithmetic and the same
Thomas sweep as a single-grid solver, so each grid must match a single-grid run
of its own case bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

from diffusionimex_b200 import BatchSolver, Solver, cases

pytestmark = pytest.mark.gpu


def _single(c, steps):
    s = Solver(c)
    s.advance(steps)
    U, st = s.state(), s.stats()
    P, pref = s.pressure()
    s.close()
    return U, P, pref, st


@pytest.mark.parametrize("threads,tile", [(128, 256), (96, 128), (32, 128)])
def test_batch_matches_single_grid_runs(threads, tile):
    """`threads` is the block size of the largest grid; the others get block sizes in proportion
    to their cells (multiples of 32), one concurrent launch per block size -- here 1 to 4 of them."""
    cs = cases.riemann_batch(count=10, seed=3, nmin=64, nmax=600)
    b = BatchSolver(cs)
    b.set_shape(threads, tile)
    b.advance(6)
    b.advance(4)  # a second launch continues from the first
    assert 1 <= b.launches() <= threads // 32
    for i, c in enumerate(cs):
        assert b.status(i) == 0
        v = b.instance(i)
        U, P, pref, st = _single(c, 10)
        sb = v.stats()
        assert sb["steps"] == st["steps"] == 10
        assert (sb["rejects"], sb["newton_it"], sb["stages"]) == (st["rejects"], st["newton_it"], st["stages"])
        assert np.array_equal(v.state(), U), i
        Pb, prefb = v.pressure()
        assert prefb == pref and np.array_equal(Pb, P), i
    b.close()


def test_autotune_restores_the_state_and_keeps_a_shape():
    cs = cases.riemann_batch(count=6, seed=4, nmin=64, nmax=300)
    b = BatchSolver(cs)
    threads, tile, ms = b.autotune(2)
    assert threads in (64, 96, 128, 256) and tile in (128, 256) and ms > 0
    b.advance(5)
    for i, c in enumerate(cs):
        U, P, _, st = _single(c, 5)
        assert b.instance(i).stats()["steps"] == 5
        assert np.array_equal(b.instance(i).state(), U), i
    b.close()


@pytest.mark.parametrize("which", ["tube1000_30steps", "case87_N200_tend", "nasg_instance_50steps"])
def test_batch_of_one_matches_the_host_loop_to_t_end(which):
    """One grid in the batched kernel against the host-driven loop: state, pressure, counters, time,
    step size, largest residual and the phase-temperature maxima (st_Tmax) bitwise -- also over a
    whole run to t_end, where the kernel stops as spb6g_advance does."""
    if which == "tube1000_30steps":
        c, steps = cases.water_air_tube(1000), 30
    elif which == "case87_N200_tend":
        c, steps = cases.reference_case(87, 200), 0
    else:
        c, steps = next(b for b in cases.riemann_batch(count=512, seed=0) if b["nasg"]), 50
    Uh, Ph, ph, sh = _single(c, steps)
    b = BatchSolver([c])
    b.advance(steps if steps > 0 else 1 << 20)
    assert b.status(0) == 0
    v = b.instance(0)
    sd = v.stats()
    Pd, pd = v.pressure()
    assert np.array_equal(v.state(), Uh) and np.array_equal(Pd, Ph) and pd == ph
    for k in ("steps", "rejects", "rk1", "stages", "newton_it", "floor_count", "t", "dt", "maxres"):
        assert sd[k] == sh[k], (k, sd[k], sh[k])
    assert sd["tmax"] == sh["tmax"]
    b.close()
