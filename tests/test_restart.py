"""Restart points: the state, the pressure unknown and the time-loop state (spb6g_download_state,
spb6g_get_pressure, spb6g_get_time) are everything the next step depends on, so restoring them
replays the following steps bit for bit.  The reference writes no restart file; this is the
restart its time loop (src/SPB6_PC_IMEX_omp.cpp:1316-1384) would need, and the end-to-end bench
replays its timed window from one."""
from __future__ import annotations

import numpy as np
import pytest

from helpers import golden_case


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["bubble48_4steps", "tube_N1000_1step", "bubble_relax32_3steps"])
def test_restart_point_replays_bitwise(name):
    from diffusionimex_b200 import Solver

    c, _, _ = golden_case(name)
    s = Solver(c)
    s.advance(2)
    rp = s.restart_point()
    st0 = s.stats()
    s.advance(3)
    Ua, (Pa, ra), ta, sta = s.state(), s.pressure(), s.time_state(), s.stats()
    s.restore(rp)
    s.advance(3)
    Ub, (Pb, rb), tb, stb = s.state(), s.pressure(), s.time_state(), s.stats()
    s.close()
    assert np.array_equal(Ua, Ub) and np.array_equal(Pa, Pb) and ra == rb and ta == tb
    for k in ("steps", "rejects", "newton_it", "bicg_it"):
        assert sta[k] - st0[k] == stb[k] - sta[k], k
