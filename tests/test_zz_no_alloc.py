"""The allocation-free time-step rate (spb6g_caldt_noalloc).

Some callers cannot let a library allocate device memory: a framework that owns
every device byte through its own arena or pool, a time-critical loop that cannot
afford the device-wide synchronisation cudaMalloc / cudaFree may cause, or a
service whose device footprint must not grow after start-up.  This entry point
takes the state as device pointers the caller owns and keeps its only scratch
in a fixed file-scope device array.  The test feeds it a state held in device
buffers allocated by the test itself (torch) and checks it against the regular
spb6g_caldt of a solver holding the same state, on two calls in a row (the
second call reuses the scratch the first one left behind).
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from diffusionimex_b200 import Solver, cases, library
from diffusionimex_b200.solver import make_config

pytestmark = pytest.mark.gpu


def device_state(U: np.ndarray):
    import torch

    soa = np.ascontiguousarray(np.moveaxis(U, -1, 0)).reshape(8, -1)
    t = torch.from_numpy(soa).to("cuda:0")
    ptrs = (ctypes.c_void_p * 8)(*[t[k].data_ptr() for k in range(8)])
    return t, ptrs


@pytest.mark.parametrize("acoustic", [0, 1])
def test_noalloc_caldt_matches_solver(acoustic):
    lib = library()
    for c in (cases.lowmach_bubbles(96, seed=1, nbub=3), cases.water_air_tube(300)):
        s = Solver(c)
        ref = s.caldt(bool(acoustic))
        s.close()
        keep, ptrs = device_state(c["U"])
        cfg = make_config(c)
        for _ in range(2):
            out = ctypes.c_double(-1.0)
            rc = lib.spb6g_caldt_noalloc(ctypes.byref(cfg), ptrs, acoustic, None, ctypes.byref(out))
            assert rc == 0
            assert out.value == pytest.approx(ref, rel=1e-15, abs=0.0)
        del keep


def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = library()
    c = cases.water_air_tube(64)
    cfg = make_config(c)
    cfg.nx, cfg.ny = 4096, 1025  # one row more than the 4 Mi-cell scratch holds
    keep, ptrs = device_state(c["U"])
    out = ctypes.c_double(0.0)
    assert lib.spb6g_caldt_noalloc(ctypes.byref(cfg), ptrs, 0, None, ctypes.byref(out)) == 10
    del keep


def test_noalloc_checks_the_device_of_its_pointers():
    """The call runs on cfg->device and refuses, before any launch, pointers that are not memory
    of that device (here host memory) and a device ordinal beyond the count; the caller's current
    device is unchanged afterwards."""
    import torch

    lib = library()
    c = cases.water_air_tube(300)
    cfg = make_config(c)
    host = np.ascontiguousarray(np.moveaxis(c["U"], -1, 0)).reshape(8, -1)
    hptrs = (ctypes.c_void_p * 8)(*[host[k].ctypes.data for k in range(8)])
    out = ctypes.c_double(-1.0)
    assert lib.spb6g_caldt_noalloc(ctypes.byref(cfg), hptrs, 0, None, ctypes.byref(out)) == 7  # SPB6G_BAD_ARG
    cfg.device = torch.cuda.device_count()
    keep, ptrs = device_state(c["U"])
    assert lib.spb6g_caldt_noalloc(ctypes.byref(cfg), ptrs, 0, None, ctypes.byref(out)) == 9  # SPB6G_NO_DEVICE
    assert torch.cuda.current_device() == 0
    del keep
