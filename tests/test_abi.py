"""CPU tests of the C ABI: the in-tree library loads without a GPU and exports
every entry point include/spb6g.h declares; a handle cannot be created without
a device, and bad arguments are rejected before any device call."""
from __future__ import annotations

import ctypes
import os
import re

import pytest

from diffusionimex_b200 import build, solver

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "spb6g.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(spb6g_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("spb6g_create", "spb6g_step", "spb6g_caldt", "spb6g_stage_dump", "spb6g_destroy"):
        assert must in names


def test_library_exports_every_declared_symbol():
    if build.needs_build():
        build.build()
    lib = ctypes.CDLL(build.LIB)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_default_config_and_status_strings():
    lib = solver.library()
    c = solver.Config()
    lib.spb6g_default_config(ctypes.byref(c))
    assert c.rk == 2 and c.cfl == 0.2 and c.newton_tol == 1e-13 and c.bicg_iter == 4000
    assert lib.spb6g_status_string(0) == b"ok"
    assert lib.spb6g_status_string(4).startswith(b"step failed")


def test_bad_arguments_rejected_before_device_use():
    lib = solver.library()
    c = solver.Config()
    lib.spb6g_default_config(ctypes.byref(c))
    h = ctypes.c_void_p()
    c.nx = 0
    assert lib.spb6g_create(ctypes.byref(c), ctypes.byref(h)) == 7  # SPB6G_BAD_ARG
    lib.spb6g_default_config(ctypes.byref(c))
    c.bc[0] = 2  # periodic on one side only
    assert lib.spb6g_create(ctypes.byref(c), ctypes.byref(h)) == 7
    lib.spb6g_default_config(ctypes.byref(c))
    c.rus_local = 2
    assert lib.spb6g_create(ctypes.byref(c), ctypes.byref(h)) == 7
    assert lib.spb6g_destroy(None) == 7


def test_batched_form_takes_the_per_face_rusanov_speed_only():
    """The batched kernel has no grid-wide speed pass: rus_local = 0 is refused before any
    device use."""
    lib = solver.library()
    c = solver.Config()
    lib.spb6g_default_config(ctypes.byref(c))
    c.rus_local = 0
    b = ctypes.c_void_p()
    assert lib.spb6g_batch_create(ctypes.byref(c), 1, ctypes.byref(b)) == 8  # SPB6G_UNSUPPORTED
    # nor modified Newton, first order, relaxation, finite or unified rates
    for field, value in (("jreuse", 1), ("order", 1), ("relax", 1), ("mu_rate", 1e-3), ("unify", 1)):
        lib.spb6g_default_config(ctypes.byref(c))
        setattr(c, field, value)
        assert lib.spb6g_batch_create(ctypes.byref(c), 1, ctypes.byref(b)) == 8, field


def test_no_device_reported_on_cpu_host():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = solver.library()
    c = solver.Config()
    lib.spb6g_default_config(ctypes.byref(c))
    h = ctypes.c_void_p()
    assert lib.spb6g_create(ctypes.byref(c), ctypes.byref(h)) == 9  # SPB6G_NO_DEVICE


def test_saturation_table_errors():
    """The host saturation table: the length query, a buffer too small (SPB6G_TOO_LARGE), and a
    Mie-Grueneisen pair, which has no SG / NASG saturation line (SPB6G_UNSUPPORTED)."""
    from diffusionimex_b200 import cases

    lib = solver.library()
    c = solver.make_config(cases.reference_case(3, 16))
    n = ctypes.c_int()
    assert lib.spb6g_saturation_table(ctypes.byref(c), None, 0, ctypes.byref(n)) == 0 and n.value > 4
    buf = (ctypes.c_double * 4)()
    assert lib.spb6g_saturation_table(ctypes.byref(c), buf, 4, ctypes.byref(n)) == 10  # SPB6G_TOO_LARGE
    mg = solver.make_config(cases.reference_case(60, 16))
    assert lib.spb6g_saturation_table(ctypes.byref(mg), None, 0, ctypes.byref(n)) == 8  # SPB6G_UNSUPPORTED
    assert lib.spb6g_saturation_table(None, None, 0, ctypes.byref(n)) == 7  # SPB6G_BAD_ARG


def test_new_settings_validated_before_device_use():
    """Out-of-range order, jreuse, relaxation rates and forms are SPB6G_BAD_ARG, and relaxation or a
    finite mu with a Mie-Grueneisen phase is SPB6G_UNSUPPORTED, before any device is touched."""
    from diffusionimex_b200 import cases

    lib = solver.library()
    h = ctypes.c_void_p()
    base = cases.reference_case(5, 16)
    for bad in (dict(order=3), dict(jreuse=2), dict(relax_form=2), dict(unify=3), dict(unify_proj=2),
                dict(nu_law=2), dict(mu_rate=-1.0), dict(nu_pc=0.0), dict(relax=4), dict(rus_local=2)):
        c = solver.make_config(dict(base, **bad))
        assert lib.spb6g_create(ctypes.byref(c), ctypes.byref(h)) == 7, bad  # SPB6G_BAD_ARG
    mg = cases.reference_case(60, 16)
    for unsup in (dict(relax=1), dict(mu_rate=1e-3)):
        c = solver.make_config(dict(mg, **unsup))
        assert lib.spb6g_create(ctypes.byref(c), ctypes.byref(h)) == 8, unsup  # SPB6G_UNSUPPORTED


def test_noalloc_caldt_arguments_rejected_before_device_use():
    """spb6g_caldt_noalloc checks the domain, the phase kinds and the device ordinal before it
    touches a device: a degenerate domain, a kind outside 0..2 and a negative device are
    SPB6G_BAD_ARG, a Mie-Grueneisen phase SPB6G_UNSUPPORTED (the pointers are never read)."""
    from diffusionimex_b200 import cases

    lib = solver.library()
    ptrs = (ctypes.c_void_p * 8)(*([16] * 8))  # never dereferenced: every case stops before a launch
    out = ctypes.c_double(0.0)
    base = solver.make_config(cases.water_air_tube(64))
    for field, value in (("x1", 0.0), ("y1", 0.0), ("device", -1)):
        c = solver.make_config(cases.water_air_tube(64))
        setattr(c, field, value)
        assert lib.spb6g_caldt_noalloc(ctypes.byref(c), ptrs, 0, None, ctypes.byref(out)) == 7, field
    c = solver.make_config(cases.water_air_tube(64))
    c.kind[0] = 5
    assert lib.spb6g_caldt_noalloc(ctypes.byref(c), ptrs, 0, None, ctypes.byref(out)) == 7
    c.kind[0] = 1
    assert lib.spb6g_caldt_noalloc(ctypes.byref(c), ptrs, 0, None, ctypes.byref(out)) == 8
    assert lib.spb6g_caldt_noalloc(ctypes.byref(base), None, 0, None, ctypes.byref(out)) == 7


def test_noalloc_caldt_without_a_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from diffusionimex_b200 import cases

    lib = solver.library()
    ptrs = (ctypes.c_void_p * 8)(*([16] * 8))
    out = ctypes.c_double(0.0)
    c = solver.make_config(cases.water_air_tube(64))
    assert lib.spb6g_caldt_noalloc(ctypes.byref(c), ptrs, 0, None, ctypes.byref(out)) == 9  # SPB6G_NO_DEVICE
