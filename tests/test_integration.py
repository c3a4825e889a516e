"""INTEGRATION.md's C++ binding, compiled and run.

The blocks of INTEGRATION.md that follow a `<!-- compiled: NAME -->` marker are the code a
maintainer adds to the reference's main().  They are wrapped here into a program whose
reference globals come from tests/integration/reference_side.h, compiled with g++ against
include/spb6g.h and libspb6g.so, and run on the reference's case 87 (N = 200) to t_end:
once with the whole loop on the GPU (spb6g_advance) and once with the reference's own
loop driving spb6g_stage.  Both must give the same state, within the reference's whole-run
bar of its own fixture.  Without a GPU only the compile step is tested."""
from __future__ import annotations

import os
import re
import subprocess

import numpy as np
import pytest

from diffusionimex_b200 import build
from diffusionimex_b200.solver import make_config
from helpers import fieldwise_l1, golden_case, load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DOC = os.path.join(ROOT, "INTEGRATION.md")
HARNESS = os.path.join(ROOT, "tests", "integration")


def blocks() -> dict:
    text = open(DOC).read()
    return {m.group(1): m.group(2) for m in re.finditer(r"<!-- compiled: (\w+) -->\s*```cpp\n(.*?)```", text, re.S)}


def program_source() -> str:
    b = blocks()
    cfg = b["config"].replace('#include "spb6g.h"', "")
    funcs = []
    for name in ("whole_loop", "stage_loop"):
        funcs.append(f"static int binding_{name}(const char* out) {{\n{cfg}\n{b[name]}\n"
                     "    FILE* o = std::fopen(out, \"wb\");\n"
                     "    if (!o) return 3;\n"
                     "    std::fwrite(interior.data(), sizeof(double), interior.size(), o);\n"
                     "    std::fclose(o);\n    return 0;\n}\n")
    return ('#include "reference_side.h"\n#include "spb6g.h"\n\n' + "\n".join(funcs) +
            "int main(int argc, char** argv) {\n"
            "    if (argc != 5 || !load_case(argv[1], argv[2])) return 4;\n"
            "    return std::strcmp(argv[3], \"stage\") == 0 ? binding_stage_loop(argv[4]) : binding_whole_loop(argv[4]);\n"
            "}\n")


def compile_program(tmp) -> str:
    if build.needs_build():
        build.build()
    src = os.path.join(tmp, "binding.cpp")
    exe = os.path.join(tmp, "binding")
    with open(src, "w") as f:
        f.write(program_source())
    libdir = os.path.dirname(build.LIB)
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-Wno-unused-function", "-I", os.path.join(ROOT, "include"),
                        "-I", HARNESS, src, "-o", exe, f"-L{libdir}", "-lspb6g", f"-Wl,-rpath,{libdir}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def write_case(c: dict, tmp) -> tuple[str, str]:
    cfg = make_config(c)
    fmt = lambda *v: " ".join(repr(float(x)) if isinstance(x, float) else str(int(x)) for x in v)
    lines = [
        f"nxCells {cfg.nx}", f"nyCells {cfg.ny}", f"domain {fmt(cfg.x0, cfg.x1, cfg.y0, cfg.y1)}",
        f"BCS {fmt(*cfg.bc)}", f"BCU {fmt(*cfg.bcu)}", f"BCP {fmt(*cfg.bcp)}",
        f"g {fmt(*cfg.gamma)}", f"pi {fmt(*cfg.pinf)}", f"q {fmt(*cfg.q)}", f"qp {fmt(*cfg.qp)}",
        f"cv {fmt(*cfg.cv)}", f"b {fmt(*cfg.b)}", f"kind {fmt(*cfg.kind)}",
        "mg " + " ".join(fmt(cfg.mg_G[p], cfg.mg_rr[p], cfg.mg_c1[p], cfg.mg_c2[p], cfg.mg_e1[p], cfg.mg_e2[p],
                             cfg.mg_e0[p]) for p in range(2)),
        f"RKs {cfg.rk}", f"RAMP {cfg.ramp}", f"RUS_LOCAL {cfg.rus_local}", f"LIMITER {cfg.limiter}",
        f"NewtonIter {cfg.newton_iter}", f"GMRESiter {cfg.bicg_iter}", f"SHARE_MODE {cfg.share_mode}",
        f"SpaceOrder {cfg.order or 2}", f"JREUSE {cfg.jreuse}", f"RELAX_LEVEL {cfg.relax}", f"NU_LAW {cfg.nu_law}",
        f"RELAX_FORM {cfg.relax_form}", f"UNIFY {cfg.unify}", f"UNIFY_PROJ {cfg.unify_proj}",
        f"caltimestep {cfg.acdt}", f"CFL {fmt(cfg.cfl)}", f"CFL_ac {fmt(cfg.cfl_ac)}", f"DTFIX {fmt(cfg.dtfix)}",
        f"NewtonTol {fmt(cfg.newton_tol)}", f"GMREStol {fmt(cfg.bicg_tol)}", f"time_stop {fmt(cfg.tend)}",
        f"EPS_I {fmt(cfg.eps_i)}", f"mu_rate {fmt(cfg.mu_rate)}", f"theta_rate {fmt(cfg.theta_rate)}",
        f"nu_rate {fmt(cfg.nu_rate)}", f"NU_CR {fmt(cfg.nu_cr)}", f"NU_PC {fmt(cfg.nu_pc)}",
    ]
    cp = os.path.join(tmp, "case.txt")
    sp = os.path.join(tmp, "state.bin")
    with open(cp, "w") as f:
        f.write("\n".join(lines) + "\n")
    np.ascontiguousarray(c["U"], dtype=np.float64).tofile(sp)
    return cp, sp


def test_integration_blocks_compile(tmp_path):
    b = blocks()
    assert set(b) >= {"config", "whole_loop", "stage_loop"}
    compile_program(str(tmp_path))


@pytest.mark.gpu
def test_integration_binding_runs_case87(tmp_path):
    exe = compile_program(str(tmp_path))
    g = load_golden("case87_N200_tend")
    c, mode, _ = golden_case("case87_N200_tend")
    cp, sp = write_case(c, str(tmp_path))
    out = {}
    for m in ("whole", "stage"):
        o = os.path.join(str(tmp_path), f"{m}.bin")
        r = subprocess.run([exe, cp, sp, m, o], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, (m, r.returncode, r.stderr[-2000:])
        out[m] = np.fromfile(o, dtype=np.float64).reshape(c["U"].shape)
    # the reference's loop over spb6g_stage does what spb6g_advance does, bit for bit
    assert np.array_equal(out["whole"], out["stage"])
    d = fieldwise_l1(out["stage"], g["U"])
    if d.max() > 1e-6:  # the whole-run bar of tests/test_gpu_parity.py
        import refio

        noise = np.maximum(*[fieldwise_l1(refio.run_port(c, mode=refio.MODE_TEND, variant=v)["U"], g["U"])
                             for v in ("ulp", "fd")])
        assert np.all(d <= np.maximum(10 * noise, 1e-6)), (d, noise)
