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
