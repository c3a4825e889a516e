"""Generate the golden fixtures in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py

Needs oracle/_ref/spb6_ref (built by `make -C oracle ref` from the reference
sources) and the reference tree for the archived profiles.  Each fixture is
the reference solver's output on one small seeded case; the GPU parity tests
compare against these files (and against the C restatement) on machines
where the reference tree does not exist.

Fixtures:
  ref_<name>.npz      U0 (initial state), U, P, p_ref and run counters of the
                      compiled reference on the case built by CASES[name]
  ref_main_profile2d.npz
                      the final profile of the reference main()'s 2D case 70 (30 x 8) and its state
  ref_sat_tables.npz  the reference's saturation tables (SAT after build_sat) of the
                      liquid / vapour pairs in SAT_CASES
  ref_main_outputs.npz
                      the files the reference's own main() writes (profile, snapshot
                      profiles, probe) and its end-of-run line, for the runs in
                      MAIN_RUNS, with the captured final state of each run
  archived_case5_N100.npz, archived_case87_N200.npz
                      columns x, p, u, rho, alpha2 of the reference's archived
                      profiles data/SPB2009_4.3.1_water_air/water_air_N100_t240us.dat
                      and data/Schropff2026_Riemann_problems/c87_200.dat
                      (produced by the serial-root program src/SPB6_PC_IMEX.cpp)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))  # tests/helpers.py

from diffusionimex_b200 import cases  # noqa: E402

REF_TREE = os.environ.get("SPB6_REFERENCE", "/root/reference")  # the reference source tree


def _tube(n):
    return cases.water_air_tube(n)


def _bubble(n, seed=1, nbub=3):
    c = cases.bubble_field(n, seed=seed, nbub=nbub)
    return c


def _lowmach(n):
    return cases.lowmach_bubbles(n, seed=3, nbub=2, amp=15.0)


def _shock(nx, ny):
    return cases.shock_bubble(nx, ny)


def _nasg(n):
    b = cases.riemann_batch(count=8, seed=5, nmin=n, nmax=n)
    return next(c for c in b if c["nasg"])


def _bc(c, bc, bcu=(0.0, 0.0, 0.0, 0.0), bcp=(0.0, 0.0, 0.0, 0.0)):
    """Boundary variant of a case: kinds left, right, bottom, top (cases.BC_*), wall velocities
    (piston) and outlet pressures."""
    c = dict(c)
    c.update(bc=list(bc), bcu=list(bcu), bcp=list(bcp))
    return c


T, W, PER, PRES = cases.BC_TRANS, cases.BC_WALL, cases.BC_PERIODIC, cases.BC_PRES

# name -> (builder, mode, nsteps, overrides)
CASES = {
    "case87_N200_tend": (lambda: cases.reference_case(87, 200), "tend", 0, {}),
    "case5_N100_tend": (lambda: cases.reference_case(5, 100), "tend", 0, {}),
    "case83_N200_10steps": (lambda: cases.reference_case(83, 200), "steps", 10, {}),
    "tube_N1000_1step": (lambda: _tube(1000), "steps", 1, {}),
    "tube_N1000_tend": (lambda: _tube(1000), "tend", 0, {}),
    "tube_N200_stage": (lambda: _tube(200), "stage", 0, {"dtfix": 2e-7}),
    "bubble48_stage": (lambda: _bubble(48), "stage", 0, {"dtfix": 1e-5, "newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "bubble48_4steps": (lambda: _bubble(48), "steps", 4, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "lowmach32_3steps": (lambda: _lowmach(32), "steps", 3, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "lowmach32_stage": (lambda: _lowmach(32), "stage", 0, {"dtfix": 2e-6, "newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "shock64x32_stage": (lambda: _shock(64, 32), "stage", 0, {"dtfix": 5e-6, "newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "shock64x32_3steps": (lambda: _shock(64, 32), "steps", 3, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "nasg256_20steps": (lambda: _nasg(256), "steps", 20, {}),
    # boundary variants (bc_apply physics :982-1013, M_P :709-718, residual_at :728-729)
    "tube_walls_N200_20steps": (lambda: _bc(_tube(200), (W, W, T, T)), "steps", 20, {}),
    "tube_piston_N200_20steps": (lambda: _bc(_tube(200), (W, W, T, T), bcu=(50.0, -20.0, 0, 0)), "steps", 20, {}),
    "tube_outlet_N200_20steps": (lambda: _bc(_tube(200), (T, PRES, T, T), bcp=(0, 2e5, 0, 0)), "steps", 20, {}),
    "tube_periodic_N200_10steps": (lambda: _bc(_tube(200), (PER, PER, T, T)), "steps", 10,
                                   {"bicg_tol": 1e-13}),
    "bubble_walls32_3steps": (lambda: _bc(_bubble(32), (W, W, W, W), bcu=(0, 0, 5.0, 0)), "steps", 3,
                              {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # Mie-Grueneisen phases (physics :51-111, closure_p_mg :585-629, hug_v / K_G :279-301)
    "nm_N200_20steps": (lambda: cases.reference_case(60, 200), "steps", 20, {}),
    "jwl_N200_20steps": (lambda: cases.reference_case(61, 200), "steps", 20, {}),
    "undex120x80_3steps": (lambda: cases.underwater_explosion(120, 80), "steps", 3,
                           {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # p-pT relaxation: instantaneous thermal relaxation in the interface zone (RELAX_LEVEL 1;
    # closure_type_of :870-886, closure_pT :716-726, RelaxationActivation :563-586)
    "tube_relax_N200_20steps": (lambda: dict(_tube(200), relax=1, eps_i=1e-4), "steps", 20, {}),
    "bubble_relax32_3steps": (lambda: dict(_bubble(32), relax=1, eps_i=1e-4), "steps", 3,
                              {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "bubble_outlet32_3steps": (lambda: _bc(_bubble(32), (PRES, PRES, W, W), bcp=(1.2e7, 0.8e7, 0, 0)), "steps", 3,
                               {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # chemical relaxation (RELAX_LEVEL 2 p-pT-pTg, 3 p-pTg; closure_pTg :811-834, Tsat :114-163,
    # closure_type_of :870-886) on the reference's liquid-vapour cases
    "dodecane_relax2_N200_20steps": (lambda: dict(cases.reference_case(3, 200), relax=2), "steps", 20, {}),
    "dodecane_relax3_N200_20steps": (lambda: dict(cases.reference_case(3, 200), relax=3), "steps", 20, {}),
    "cavitation_relax2_N200_20steps": (lambda: dict(cases.reference_case(1, 200), relax=2), "steps", 20, {}),
    "bartak_N200_20steps": (lambda: cases.reference_case(32, 200), "steps", 20, {}),
    "chem0d_N16_10steps": (lambda: dict(cases.reference_case(41, 16), relax=2), "steps", 10,
                           {"bicg_tol": 1e-13, "dtfix": 1e-5}),
    "bubblecomp32_3steps": (lambda: cases.bubble_compression(32, 32), "steps", 3,
                            {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # the same before their first round-off type decision (pTg already active, noise < 1e-12)
    "dodecane_relax2_N200_2steps": (lambda: dict(cases.reference_case(3, 200), relax=2), "steps", 2, {}),
    "dodecane_relax3_N200_2steps": (lambda: dict(cases.reference_case(3, 200), relax=3), "steps", 2, {}),
    "bartak_N200_5steps": (lambda: cases.reference_case(32, 200), "steps", 5, {}),
    "bubblecomp32_1step": (lambda: cases.bubble_compression(32, 32), "steps", 1,
                           {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # finite relaxation rates (closure_mu :636, closure_theta :732, closure_nu :771; relaxform 0
    # backward Euler, 1 exponential; unify = 1; the nu law :174-179)
    "mu0d_N4_10steps": (lambda: dict(cases.reference_case(40, 4), mu_rate=1e-5), "steps", 10,
                        {"bicg_tol": 1e-13, "dtfix": 1e-5}),
    "mu0d_expo_N4_10steps": (lambda: dict(cases.reference_case(40, 4), mu_rate=1e-5, relax_form=1), "steps", 10,
                             {"bicg_tol": 1e-13, "dtfix": 1e-5}),
    "theta0d_N4_10steps": (lambda: dict(cases.reference_case(40, 4), relax=1, theta_rate=1e4), "steps", 10,
                           {"bicg_tol": 1e-13, "dtfix": 1e-5}),
    "theta0d_expo_N4_10steps": (lambda: dict(cases.reference_case(40, 4), relax=1, theta_rate=1e4, relax_form=1),
                                "steps", 10, {"bicg_tol": 1e-13, "dtfix": 1e-5}),
    "nu0d_N4_10steps": (lambda: dict(cases.reference_case(41, 4), relax=2, nu_rate=1e3), "steps", 10,
                        {"bicg_tol": 1e-13, "dtfix": 1e-5}),
    "nu0d_expo_N4_10steps": (lambda: dict(cases.reference_case(41, 4), relax=2, nu_rate=1e3, relax_form=1), "steps",
                             10, {"bicg_tol": 1e-13, "dtfix": 1e-5}),
    "dodecane_rates_N200_2steps": (lambda: dict(cases.reference_case(3, 200), relax=2, mu_rate=1e-3, theta_rate=1e5,
                                                nu_rate=1e3), "steps", 2, {}),
    "dodecane_rates_N200_20steps": (lambda: dict(cases.reference_case(3, 200), relax=2, mu_rate=1e-3, theta_rate=1e5,
                                                 nu_rate=1e3), "steps", 20, {}),
    "dodecane_unify_N200_2steps": (lambda: dict(cases.reference_case(3, 200), relax=2, unify=1), "steps", 2, {}),
    "bartak_nulaw_N200_5steps": (lambda: dict(cases.reference_case(32, 200), nu_law=1), "steps", 5, {}),
    "bartak_nulaw_N200_20steps": (lambda: dict(cases.reference_case(32, 200), nu_law=1), "steps", 20, {}),
    "dodecane_unifyproj0_N200_2steps": (lambda: dict(cases.reference_case(3, 200), relax=2, unify_proj=0), "steps", 2,
                                        {}),
    "dodecane_relax3_nulaw_N200_5steps": (lambda: dict(cases.reference_case(3, 200), relax=3, nu_law=1), "steps", 5,
                                          {}),
    "bubble_theta32_3steps": (lambda: dict(_bubble(32), relax=1, theta_rate=1e3, mu_rate=1e-4), "steps", 3,
                              {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # first order: no reconstruction (order=1, TVDReconstruction :372-375, psi_face :979)
    "tube_order1_N200_20steps": (lambda: dict(_tube(200), order=1), "steps", 20, {}),
    "bubble_order1_32_3steps": (lambda: dict(_bubble(32), order=1), "steps", 3, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "lowmach_order1_32_stage": (lambda: dict(_lowmach(32), order=1), "stage", 0,
                               {"dtfix": 2e-6, "newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # modified Newton (JREUSE :83, Newton_Solver :826-830, :887)
    "tube_jreuse_N1000_20steps": (lambda: dict(_tube(1000), jreuse=1), "steps", 20, {}),
    "bubble_jreuse48_4steps": (lambda: dict(_bubble(48), jreuse=1), "steps", 4, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "lowmach_jreuse32_3steps": (lambda: dict(_lowmach(32), jreuse=1), "steps", 3, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # the reference's own 2D cases 70 (helium bubble) and 71 (cavitating Richtmyer-Meshkov), 4 x 4
    # sub-cell averaged initial states
    "hebubble75x20_3steps": (lambda: cases.he_bubble(75, 20), "steps", 3, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "rm60x20_3steps": (lambda: cases.richtmyer_meshkov(60, 20), "steps", 3, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # cases 56 (two-phase vortex) and 58 (two-phase Taylor-Green), periodic in both directions
    "vortex24_3steps": (lambda: cases.vortex_bb(24), "steps", 3, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "taylorgreen24_3steps": (lambda: cases.taylor_green(24, True), "steps", 3, {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
    # grid-wide Rusanov dissipation speed (RUS_LOCAL = 0; RusanovC_x/y :237-259, Update :266-298)
    "case13_N200_20steps": (lambda: cases.reference_case(13, 200), "steps", 20, {}),
    "lowmach_rus0_32_stage": (lambda: dict(_lowmach(32), rus_local=0), "stage", 0,
                              {"dtfix": 2e-6, "newton_tol": 1e-13, "bicg_tol": 1e-13}),
    "lowmach_rus0_32_3steps": (lambda: dict(_lowmach(32), rus_local=0), "steps", 3,
                               {"newton_tol": 1e-13, "bicg_tol": 1e-13}),
}


# reference main() runs with output: tag -> (case, N, key=value arguments besides case, N, out)
MAIN_RUNS = {
    "case5_N100": (5, 100, ["snap=8e-5,1.6e-4", "probe=0.6,0.5"]),
    "case87_N200": (87, 200, ["snap=1e-4", "probe=0.5,0.5"]),
    "case60_N100": (60, 100, ["snap=3e-5", "probe=0.6,0.5"]),  # Mie-Grueneisen (Cochran-Chan) phases
    "case5_relax_N100": (5, 100, ["relax=1", "snap=1.2e-4", "probe=0.75,0.5"]),  # p-pT relaxation
    "case5_order1_N100": (5, 100, ["order=1", "snap=1.2e-4", "probe=0.75,0.5"]),  # first order
}


def main_outputs():
    """Files and stdout of the reference main() for MAIN_RUNS, one compressed archive."""
    import refio

    out = {}
    for tag, (case, n, args) in MAIN_RUNS.items():
        r = refio.run_ref_main_files([f"case={case}", f"N={n}", *args], out_name="run.dat", nx=n)
        res = refio.run_ref_main_files([f"case={case}", f"N={n}", *args], out_name="run.dat")
        assert r["files"] == res["files"], "the reference main() is not deterministic"
        for name, data in r["files"].items():
            out[f"{tag}/{name}"] = np.frombuffer(data, dtype=np.uint8)
        out[f"{tag}/stdout"] = np.frombuffer(r["stdout"].encode(), dtype=np.uint8)
        out[f"{tag}/args"] = np.frombuffer(json.dumps([case, n, args]).encode(), dtype=np.uint8)
        out[f"{tag}/U"] = r["U"]
        print(tag, {k: len(v) for k, v in r["files"].items()}, r["stdout"].strip()[:80])
    np.savez_compressed(os.path.join(HERE, "ref_main_outputs.npz"), **out)


def main_profile_2d():
    """The final profile the reference's main() writes for its 2D case 70 on 30 x 8 cells (t_end cut
    to 2e-5 s), with the captured state: the 2D layout of write_profile (:1083-1094)."""
    import refio

    args = ["case=70", "N=30", "ny=8", "tend=2e-5"]
    r = refio.run_ref_main_files(args, out_name="run.dat", nx=30, ny=8)
    np.savez_compressed(os.path.join(HERE, "ref_main_profile2d.npz"), profile=np.frombuffer(r["files"]["run.dat"], np.uint8),
                        U=r["U"], args=np.frombuffer(json.dumps(args).encode(), np.uint8))
    print("profile2d", len(r["files"]["run.dat"]), r["stdout"].strip()[:80])


# liquid / vapour pairs whose saturation tables (build_sat, physics :127-153) are pinned
SAT_CASES = (1, 3, 30, 31, 32)


def schropff_profiles():
    """The reference's archived runs of its cases 80-88 (data/Schropff2026_Riemann_problems/c<case>_<N>.dat,
    the density column) and the relative L1 density errors it publishes for them (L1_table.md there),
    to pin the exact Riemann solvers of oracle/exact_riemann.py: they must reproduce the table."""
    import re

    base = "data/Schropff2026_Riemann_problems"
    out = {}
    for f in sorted(os.listdir(os.path.join(REF_TREE, base))):
        m = re.fullmatch(r"c(\d+)_(\d+)\.dat", f)
        if m:
            d = np.loadtxt(os.path.join(REF_TREE, base, f))
            out[f"rho_c{m.group(1)}_{m.group(2)}"] = d[:, 5]
    for line in open(os.path.join(REF_TREE, base, "L1_table.md")):
        m = re.match(r"\|\s*(\d+)\s*\|[^|]*\|\s*(\d+)\s*\|\s*([0-9.eE+-]+)\s*\|", line)
        if m:
            out[f"pub_c{m.group(1)}_{m.group(2)}"] = np.float64(m.group(3))
    np.savez_compressed(os.path.join(HERE, "ref_schropff_profiles.npz"), source=base, **out)
    print("schropff profiles", len(out))


def sat_tables():
    """The reference's own saturation table (its global SAT after build_sat) for the phase pairs of
    SAT_CASES, one archive: n, pcrit, vcrit, pmin, ln p[n], Tsat[n] per case."""
    import refio

    out = {}
    for case in SAT_CASES:
        c = dict(cases.reference_case(case, 16), relax=2)
        out[f"case{case}"] = refio.run_ref(c, mode=refio.MODE_SAT)["sat"]
        print("sat table", case, int(out[f"case{case}"][0]), "points")
    np.savez_compressed(os.path.join(HERE, "ref_sat_tables.npz"), **out)


def case_settings(c: dict) -> dict:
    """The scalar settings and phases of a case (everything but its state), as JSON values."""
    def plain(v):
        if isinstance(v, dict):
            return {k: plain(x) for k, x in v.items()}
        if isinstance(v, (list, tuple)):
            return [plain(x) for x in v]
        if isinstance(v, (np.floating, float)):
            return float(v) if np.isfinite(v) else repr(float(v))
        if isinstance(v, (np.integer, int, bool, str)):
            return v if isinstance(v, (bool, str)) else int(v)
        return None
    return {k: plain(v) for k, v in c.items() if not isinstance(v, np.ndarray) and plain(v) is not None}


def build_case(name):
    fn, mode, nsteps, over = CASES[name]
    c = fn()
    c.update(over)
    return c, mode, nsteps


def main():
    import refio

    if not refio.ref_available():
        raise SystemExit("oracle/_ref/spb6_ref is missing: run `make -C oracle ref` first")
    modes = {"tend": refio.MODE_TEND, "steps": refio.MODE_STEPS, "stage": refio.MODE_STAGE}
    only = sys.argv[1:]
    if only == ["sat"]:
        sat_tables()
        return
    if only == ["schropff"]:
        schropff_profiles()
        return
    if only == ["profile2d"]:
        main_profile_2d()
        return
    for name in (only or CASES):
        c, mode, nsteps = build_case(name)
        r = refio.run_ref(c, mode=modes[mode], nsteps=nsteps)
        meta = {k: r[k] for k in ("status", "steps", "rejects", "rk1", "stages", "newton_it", "floor_count", "t", "dt",
                                  "maxres", "p_ref")}
        meta["config"] = case_settings(c)
        extra = {}
        if mode == "stage":
            extra = {k: r[k] for k in ("Xs", "a2s", "ube_x", "ube_y", "phi_x", "phi_y")}
        if c.get("relax", 0) >= 1 or "mu_rate" in c:  # the reference's own one-ulp libm noise (its type decisions at
            # T = Tsat(p) are round-off decisions): per-field L1 of the ulp-up / ulp-down runs
            from helpers import fieldwise_l1

            extra["noise"] = np.maximum(*[fieldwise_l1(refio.run_ref(c, mode=modes[mode], nsteps=nsteps,
                                                                     variant=v)["U"], r["U"])
                                          for v in ("ulp", "ulpdown")])
        np.savez_compressed(os.path.join(HERE, f"ref_{name}.npz"), U0=c["U"], U=r["U"], P=r["P"],
                            meta=json.dumps(meta), **extra)
        print(name, meta)
    if only:
        return
    main_outputs()
    main_profile_2d()
    sat_tables()
    schropff_profiles()
    for tag, path in (("archived_case5_N100", "data/SPB2009_4.3.1_water_air/water_air_N100_t240us.dat"),
                      ("archived_case87_N200", "data/Schropff2026_Riemann_problems/c87_200.dat")):
        d = np.loadtxt(os.path.join(REF_TREE, path))
        np.savez_compressed(os.path.join(HERE, f"{tag}.npz"), x=d[:, 0], p=d[:, 2], u=d[:, 3], rho=d[:, 5],
                            alpha2=d[:, 6], source=path)
        print(tag, d.shape)


if __name__ == "__main__":
    main()
