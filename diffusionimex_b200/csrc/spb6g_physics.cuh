// Per-cell physics of the SPB 6+1-equation model on the device: stiffened-gas /
// NASG and Mie-Grueneisen (Cochran-Chan, JWL) equations of state, the
// mechanical (p) relaxation closure, the shock dissipation budget and the
// primitive-variable map.
//
// Each function follows the reference line for line in operation order
// (src/spb6_physics_omp.h, cited per function); the library is compiled with
// -fmad=false so that no multiply-add contraction changes the rounding, and
// FP64 division / sqrt are IEEE correctly rounded on the device as on the host.
// std::max / std::min semantics (NaN handling) are kept through SMAX / SMIN.
#pragma once
#include <cmath>
#include <cstdint>

#define SPB6G_DEV __device__ __forceinline__
// SPB6G_MG = 1 compiles the Mie-Grueneisen branches in.  The library builds the kernels twice:
// with SPB6G_MG = 0 they are exactly the stiffened-gas / NASG kernels, and a configuration with a
// Mie-Grueneisen phase runs the second build (namespace spb6g_mg) instead.
#ifndef SPB6G_MG
#define SPB6G_MG 0
#endif
#define SMAX(a, b) ((a) < (b) ? (b) : (a))
#define SMIN(a, b) ((b) < (a) ? (b) : (a))

namespace spb6g {

enum { IA1 = 0, IM1, IM2, IMU, IMV, IE1, IE2, IEN, NV = 8 };
enum { BC_TRANS = 0, BC_WALL = 1, BC_PERIODIC = 2, BC_PRES = 3 };

// A phase: stiffened gas / NASG (kind 0: g, pi, q, qp, cv, b; b = 0 is stiffened gas), or
// Mie-Grueneisen p = G rho (e - er(rho)) + pr(rho) with constant G and er' = pr / rho^2
// (physics :51-56): Cochran-Chan (kind 1) or JWL (kind 2), reference curve parameters rr,
// c1, c2, e1, e2, e0; cv > 0 gives the temperature (e - er) / cv (output only).
struct PhaseD {
    double g, pi, q, qp, cv, b;
    int kind, pad;
    double G, rr, c1, c2, e1, e2, e0;
};

// Phases and scheme switches shared by every kernel (passed by value).
struct Phys {
    PhaseD ph[2];
    int share_mode;  // SHARE_MODE, src/spb6_physics_omp.h:436
    int limiter;     // LIMITER, :969
    int rus_local;   // RUS_LOCAL, src/SPB6_PC_IMEX_omp.cpp:93
    int mg;          // a Mie-Grueneisen phase is present (mg_any, :58)
    int relax;       // RELAX_LEVEL (:39): 0 mechanical relaxation only; in the interface zone 1 p-pT
                     // (instantaneous thermal relaxation), 2 p-pT-pTg and 3 p-pTg (instantaneous
                     // chemical relaxation where a phase is above the saturation temperature)
    int pad;
    double eps_i;    // EPS_I (:40): interface zone eps_I <= alpha1 <= 1 - eps_I
    const double* sat;  // relax >= 2: the saturation table (SatTable :114), packed as n, pcrit, vcrit,
                        // pmin, ln p[n], Tsat[n]
    // relaxation rates (mu_rate, theta_rate, nu_rate :35; INFINITY instantaneous; theta and nu
    // resolved to the level's defaults, nu 0 under the nu law), the nu law's coefficient and
    // pressure (NU_CR, NU_PC :38), RELAX_FORM (:42), UNIFY, UNIFY_PROJ (:45), NU_LAW (:37)
    double mu_rate, theta_rate, nu_rate, nu_cr, nu_pc;
    int relax_form, unify, unify_proj, nu_law;
    int mech;  // the mechanical closure type: CL_P (mu = inf) or CL_MU
    int order; // SpaceOrder (:73): 2 MUSCL, 1 cell values on the faces (no reconstruction)
    int rates; // a finite mu or unify = 1: closure kernels take the extended build even at relax 0
};
// Closure types (ClosureType :228): p, finite mu, pT, finite theta, finite nu, pTg.  CL_PND is
// internal: the p closure without the energy defect (ClIn::nodelta :236), the prediction of the
// p-pTg activation test (:878).
enum { CL_P = 0, CL_MU = 1, CL_PT = 2, CL_THETA = 3, CL_NU = 4, CL_PTG = 5, CL_PND = 6 };

// ------------------------------------------------------------ EOS, src/spb6_physics_omp.h:60-111
// Mie-Grueneisen reference curves pr(rho), pr'(rho), er(rho) (mg_ref :60-69): Cochran-Chan
// pr = c1 x^e1 - c2 x^e2 with x = rho / rr; JWL pr = c1 exp(-e1 rr / rho) + c2 exp(-e2 rr / rho).
// The Mie-Grueneisen routines are kept out of line and take their arguments by value: the
// SG / NASG kernels then carry only a call in a branch they never take, with no pow / exp in
// their register allocation and no kernel parameter copied to local memory.
struct MgRef {
    double pr, dpr, er;
};
static __device__ __noinline__ MgRef mg_curve(int kind, double rr, double c1, double c2, double e1, double e2, double e0,
                                              double r) {
    MgRef o;
    if (kind == 1) {
        const double x = r / rr, t1 = c1 * pow(x, e1), t2 = c2 * pow(x, e2);
        o.pr = t1 - t2;
        o.dpr = (e1 * t1 - e2 * t2) / r;
        o.er = (t1 / (e1 - 1.0) - t2 / (e2 - 1.0)) / r;
    } else {
        const double t1 = c1 * exp(-e1 * rr / r), t2 = c2 * exp(-e2 * rr / r);
        o.pr = t1 + t2;
        o.dpr = (e1 * t1 + e2 * t2) * rr / (r * r);
        o.er = t1 / (e1 * rr) + t2 / (e2 * rr) - e0;
    }
    return o;
}
SPB6G_DEV void mg_ref(const PhaseD& h, double r, double& pr, double& dpr, double& er) {
    const MgRef o = mg_curve(h.kind, h.rr, h.c1, h.c2, h.e1, h.e2, h.e0, r);
    pr = o.pr;
    dpr = o.dpr;
    er = o.er;
}
SPB6G_DEV double eps_amp(const Phys& P, int k, double a, double m, double p) {
    const PhaseD& h = P.ph[k];
    if (SPB6G_MG && h.kind) {
        double pr, dpr, er;
        mg_ref(h, m / a, pr, dpr, er);
        return m * er + a * (p - pr) / h.G;
    }
    return (p + h.g * h.pi) * (a - m * h.b) / (h.g - 1.0) + m * h.q;
}
SPB6G_DEV double p_ame(const Phys& P, int k, double a, double m, double e) {
    const PhaseD& h = P.ph[k];
    if (SPB6G_MG && h.kind) {
        double pr, dpr, er;
        mg_ref(h, m / a, pr, dpr, er);
        return h.G * (e - m * er) / a + pr;
    }
    return (e - m * h.q) * (h.g - 1.0) / (a - m * h.b) - h.g * h.pi;
}
SPB6G_DEV double c2_rp(const Phys& P, int k, double r, double p) {
    const PhaseD& h = P.ph[k];
    if (SPB6G_MG && h.kind) {
        double pr, dpr, er;
        mg_ref(h, r, pr, dpr, er);
        return (h.G + 1.0) * (p - pr) / r + dpr;
    }
    return h.g * (p + h.pi) / (r * (1.0 - r * h.b));
}
SPB6G_DEV double dedp_am(const Phys& P, int k, double a, double m) {
    const PhaseD& h = P.ph[k];
    if (SPB6G_MG && h.kind) return a / h.G;
    return (a - m * h.b) / (h.g - 1.0);
}
SPB6G_DEV double T_amp(const Phys& P, int k, double a, double m, double p) {
    const PhaseD& h = P.ph[k];
    if (SPB6G_MG && h.kind) {
        if (!(h.cv > 0)) return NAN;
        double pr, dpr, er;
        mg_ref(h, m / a, pr, dpr, er);
        return (a * (p - pr) / (h.G * m)) / h.cv;
    }
    return (a / m - h.b) * (p + h.pi) / ((h.g - 1.0) * h.cv);
}
SPB6G_DEV double p_mix(const Phys& P, double a1, double m1, double m2, double rhoe) {
    const double a[2] = {a1, 1.0 - a1}, m[2] = {m1, m2};
    double num = rhoe, den = 0.0;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        if (SPB6G_MG && P.ph[k].kind) {  // (A2.7)
            double pr, dpr, er;
            mg_ref(P.ph[k], m[k] / a[k], pr, dpr, er);
            num -= m[k] * er - a[k] * pr / P.ph[k].G;
        } else {
            num -= m[k] * P.ph[k].q + P.ph[k].g * P.ph[k].pi * dedp_am(P, k, a[k], m[k]);
        }
        den += dedp_am(P, k, a[k], m[k]);
    }
    return num / den;
}
// Admissible phase state (:103-106): NASG p + pi > 0; Mie-Grueneisen c^2 > 0.
SPB6G_DEV bool p_admissible(const Phys& P, int k, double a, double m, double p) {
    if (SPB6G_MG && P.ph[k].kind) return isfinite(p) && c2_rp(P, k, m / a, p) > 0;
    return p + P.ph[k].pi > 0;
}
// Round-off scale of eps_k besides |eps_k| (:108-111): NASG |m q|; MG |m er| + |alpha pr / G|.
SPB6G_DEV double eps_round(const Phys& P, int k, double a, double m) {
    if (SPB6G_MG && P.ph[k].kind) {
        double pr, dpr, er;
        mg_ref(P.ph[k], m / a, pr, dpr, er);
        return fabs(m * er) + fabs(a * pr / P.ph[k].G);
    }
    return fabs(m * P.ph[k].q);
}

// ------------------------------------------------------------ closure, :229-243, :430-548, :842-866
struct ClIn {
    double atr[2], mtr[2], etr[2], s, rhoeC, pguess, Qph[2];
    int type;     // closure type, frozen per step by the activation
    double tau;   // finite rates: the stage's implicit step a_ii dt (0 at activation)
    double Z[2];  // finite mu: the phases' acoustic impedances, frozen per stage (1 otherwise)
    double nu;    // finite nu: the cell's rate under the nu law, < 0 for nu_rate
};
struct ClOut {
    double a[2], e[2], pbar;
    double m[2], Tk[2];  // closures other than p: phase masses (pTg and nu move mass) and temperatures
};

SPB6G_DEV double E_above(const Phys& P, const ClIn& in, int k) {  // :430-433
    if (SPB6G_MG && P.ph[k].kind) {  // thermal energy above the cold curve, eps_k - m_k er
        if (!(in.atr[k] > 0 && in.mtr[k] > 0)) return 0.0;
        double pr, dpr, er;
        mg_ref(P.ph[k], in.mtr[k] / in.atr[k], pr, dpr, er);
        return SMAX(0.0, in.etr[k] - in.mtr[k] * er);
    }
    const double v = in.etr[k] - in.mtr[k] * P.ph[k].q - (in.atr[k] - in.mtr[k] * P.ph[k].b) * P.ph[k].pi;
    return SMAX(0.0, v);
}

// Quantities of the p-closure that do not depend on the trial pressure (:481-489).
struct ClPre {
    double D0, lE[2], A0[2], Qb;
    bool byMass;
};
SPB6G_DEV void closure_pre(const Phys& P, const ClIn& in, ClPre& pr) {
    pr.D0 = (SPB6G_MG && in.type == CL_PND) ? 0.0 : in.rhoeC - in.etr[0] - in.etr[1];
    const double sm = in.mtr[0] + in.mtr[1];
    pr.byMass = P.share_mode == 2;
    double E[2], sE = 0.0;
#pragma unroll
    for (int k = 0; k < 2; k++) { E[k] = E_above(P, in, k); sE += E[k]; }
    if (pr.byMass) {
        for (int k = 0; k < 2; k++) pr.lE[k] = sm > 0 ? in.mtr[k] / sm : 0.5;
    } else if (sE > 0) {
        for (int k = 0; k < 2; k++) pr.lE[k] = E[k] / sE;
    } else {
        for (int k = 0; k < 2; k++) pr.lE[k] = sm > 0 ? in.mtr[k] / sm : 0.5;
    }
    pr.Qb = (pr.byMass || P.share_mode == 1) ? 0.0 : in.Qph[0] + in.Qph[1];
#pragma unroll
    for (int k = 0; k < 2; k++) pr.A0[k] = in.etr[k] - in.mtr[k] * P.ph[k].q;
}
// Segment of the piecewise-affine defect split Lambda_k(delta(p)) (:491-511).
SPB6G_DEV void seg_lambda(const ClIn& in, const ClPre& pr, double p, double lam[2], double ex[2]) {
    ex[0] = ex[1] = 0.0;
    if (pr.byMass) { lam[0] = pr.lE[0]; lam[1] = pr.lE[1]; return; }
    const double delta = pr.D0 + p * in.s;
    if (!(delta > 0.0) || !(pr.Qb > 0.0)) { lam[0] = pr.lE[0]; lam[1] = pr.lE[1]; }
    else if (delta < pr.Qb) { lam[0] = in.Qph[0] / pr.Qb; lam[1] = in.Qph[1] / pr.Qb; }
    else {
        for (int k = 0; k < 2; k++) { lam[k] = pr.lE[k]; ex[k] = in.Qph[k] - pr.Qb * pr.lE[k]; }
    }
}
// Phi(p) = sum_k alpha_k(p) - 1 and its derivative (:502-519).
SPB6G_DEV double PhiD(const Phys& P, const ClIn& in, const ClPre& pr, double p, double& df) {
    double lam[2], ex[2];
    seg_lambda(in, pr, p, lam, ex);
    double f = 0.0;
    df = 0.0;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const PhaseD& h = P.ph[k];
        const double A = pr.A0[k] + lam[k] * pr.D0 + ex[k], B = in.atr[k] + lam[k] * in.s,
                     N = A - (B - in.mtr[k] * h.b) * h.pi;
        f += ((h.g - 1.0) * (A + B * p) + (p + h.g * h.pi) * in.mtr[k] * h.b) / (h.g * (p + h.pi));
        df += -(h.g - 1.0) * N / (h.g * (p + h.pi) * (p + h.pi));
    }
    return f - 1.0;
}
// alpha_k(p) of a Mie-Grueneisen phase (alpha_mg :552-584): the root of
// f(a) = m er(m/a) + a (p - pr)/G + p a - A - B p on the branch where f' = rho c^2 / G > 0;
// the bracket grows from the guess (moved up first if the guess lies where c^2 <= 0), then a
// safeguarded Newton.  Kept out of line: the SG/NASG kernels do not carry its registers.
static __device__ __noinline__ bool alpha_mg(const PhaseD& h, double m, double A, double B, double p, double guess, double& al,
                                      double& dal) {
    auto F = [&](double a, double& df) {
        double pr, dpr, er;
        const double r = m / a;
        mg_ref(h, r, pr, dpr, er);
        df = ((h.G + 1.0) * (p - pr) + r * dpr) / h.G;
        return m * er + a * (p - pr) / h.G + p * a - A - B * p;
    };
    double lo = guess, hi = guess, d;
    double flo = F(lo, d), fhi = flo;
    if (!isfinite(flo)) return false;
    if (!(d > 0)) {
        for (int it = 0; it < 200 && !(d > 0); it++) {
            guess *= 2.0;
            flo = F(guess, d);
            if (!isfinite(flo)) return false;
        }
        if (!(d > 0)) return false;
        lo = hi = guess;
        fhi = flo;
    }
    if (flo < 0) {
        for (int it = 0; it < 200 && fhi < 0; it++) {
            lo = hi; flo = fhi; hi *= 2.0;
            fhi = F(hi, d);
            if (!isfinite(fhi)) return false;
        }
        if (fhi < 0) return false;
    } else {
        for (int it = 0; it < 200 && flo > 0; it++) {
            hi = lo; fhi = flo; lo *= 0.5;
            flo = F(lo, d);
            if (!isfinite(flo)) return false;
            if (d <= 0) {  // past the c^2 = 0 point: bisect [lo, hi] for F <= 0 on the admissible branch
                bool found = false;
                for (int b = 0; b < 200; b++) {
                    const double mid = sqrt(lo * hi);
                    double dm;
                    const double fm = F(mid, dm);
                    if (!isfinite(fm)) return false;
                    if (!(dm > 0)) lo = mid;
                    else if (fm > 0) { hi = mid; fhi = fm; }
                    else { lo = mid; flo = fm; found = true; break; }
                    if (hi - lo <= 1e-15 * hi) break;
                }
                if (!found) return false;
                break;
            }
        }
        if (flo > 0) return false;
    }
    double a = (flo == 0) ? lo : (fhi == 0 ? hi : (guess >= lo && guess <= hi ? guess : sqrt(lo * hi)));
    for (int it = 0; it < 200; it++) {
        double df;
        const double fa = F(a, df);
        if (fa == 0) break;
        if (fa < 0) lo = a; else hi = a;
        double an = (df > 0) ? a - fa / df : -1.0;
        if (an > 0 && fabs(an - a) <= 4e-16 * a) { a = an; break; }
        if (!(an > lo && an < hi)) an = sqrt(lo * hi);
        if (fabs(an - a) <= 4e-16 * a || hi - lo <= 4e-16 * hi) { a = an; break; }
        a = an;
    }
    double df;
    F(a, df);
    if (!(df > 0)) return false;
    al = a;
    dal = -(a / h.G + a - B) / df;
    return true;
}
// The p-closure with a Mie-Grueneisen phase (closure_p_mg :585-629): the defect split's
// segment is taken at the guess; Phi(p) = sum_k alpha_k(p) - 1 with alpha_mg for MG phases and
// the closed form (B6.2) for NASG ones; bracket grown from the guess, then bracketed Newton.
struct ClMg {
    ClOut o;
    int ok;
};
static __device__ __noinline__ ClMg closure_p_mg(const Phys P, const ClIn in) {
    ClMg res;
    res.ok = 0;
    ClOut& o = res.o;
    if (!(in.mtr[0] + in.mtr[1] > 0)) return res;  // p_coef's failure condition
    ClPre pr;
    closure_pre(P, in, pr);
    double lam[2], ex[2], A[2], B[2], N[2];
    seg_lambda(in, pr, in.pguess, lam, ex);
#pragma unroll
    for (int k = 0; k < 2; k++) {
        A[k] = pr.A0[k] + lam[k] * pr.D0 + ex[k];
        B[k] = in.atr[k] + lam[k] * in.s;
        N[k] = A[k] - (B[k] - in.mtr[k] * P.ph[k].b) * P.ph[k].pi;
    }
    double ag[2] = {in.atr[0] / (in.atr[0] + in.atr[1]), in.atr[1] / (in.atr[0] + in.atr[1])};
    auto Phi = [&](double p, double& dPhi, bool upd) -> double {  // NaN: a phase has no solution at this p
        double s = -1.0, an[2];
        dPhi = 0.0;
        for (int k = 0; k < 2; k++) {
            const PhaseD& h = P.ph[k];
            double a, da;
            if (SPB6G_MG && h.kind) {
                if (!alpha_mg(h, in.mtr[k], A[k], B[k], p, ag[k], a, da)) return NAN;
            } else {
                if (!(p + h.pi > 0) || !(N[k] > 0)) return NAN;
                a = ((h.g - 1.0) * (A[k] + B[k] * p) + (p + h.g * h.pi) * in.mtr[k] * h.b) / (h.g * (p + h.pi));
                da = -(h.g - 1.0) * N[k] / (h.g * (p + h.pi) * (p + h.pi));
            }
            an[k] = a;
            s += a;
            dPhi += da;
        }
        if (upd) { ag[0] = an[0]; ag[1] = an[1]; }
        return s;
    };
    double p = in.pguess, d;
    const double f = Phi(p, d, true);
    double scale = 1e-6 * (fabs(p) + 1e5);
    double lo, hi, flo, fhi;
    if (!isfinite(f) || f > 0) {  // p too low: search upwards for Phi < 0
        lo = p; flo = f; hi = p;
        for (int it = 0; it < 300; it++) {
            hi = p + scale;
            fhi = Phi(hi, d, false);
            if (isfinite(fhi) && fhi <= 0) break;
            if (isfinite(fhi)) { lo = hi; flo = fhi; }
            scale *= 2.0;
        }
        if (!(isfinite(fhi) && fhi <= 0)) return res;
    } else {
        hi = p; fhi = f; lo = p;
        for (int it = 0; it < 300; it++) {
            lo = p - scale;
            flo = Phi(lo, d, false);
            if (isfinite(flo) && flo >= 0) break;
            if (!isfinite(flo)) {
                scale *= 0.5;
                if (scale < 1e-300) return res;
                continue;
            }
            hi = lo; fhi = flo; scale *= 2.0;
        }
        if (!(isfinite(flo) && flo >= 0)) return res;
    }
    p = (isfinite(f) && in.pguess >= lo && in.pguess <= hi) ? in.pguess : 0.5 * (lo + hi);
    for (int it = 0; it < 300; it++) {
        double df;
        const double fp = Phi(p, df, true);
        if (fp == 0.0) break;
        if (!isfinite(fp) || fp > 0) lo = p; else hi = p;
        double pn = (isfinite(fp) && df < 0) ? p - fp / df : 0.5 * (lo + hi);
        if (isfinite(fp) && df < 0 && fabs(pn - p) <= 2e-16 * (fabs(p) + fabs(pn))) { p = pn; break; }
        if (!(pn > lo && pn < hi)) pn = 0.5 * (lo + hi);
        if (fabs(pn - p) <= 2e-16 * (fabs(p) + fabs(pn)) || hi - lo <= 4e-16 * (fabs(hi) + fabs(lo))) { p = pn; break; }
        p = pn;
    }
    double df;
    if (!isfinite(Phi(p, df, true))) return res;
    for (int k = 0; k < 2; k++) {
        o.a[k] = ag[k];
        if (!p_admissible(P, k, o.a[k], in.mtr[k], p)) return res;
        o.e[k] = eps_amp(P, k, o.a[k], in.mtr[k], p);
    }
    o.pbar = p;
    res.ok = isfinite(p) ? 1 : 0;
    return res;
}

// ---- instantaneous thermal relaxation (pT closure, B6.3), built with the extended physics
// Brent's bracketed root search (brent :183-205): f(a), f(b) of opposite signs.
template <class Fn>
SPB6G_DEV bool brent(Fn f, double a, double b, double fa, double fb, double tol, double& root) {
    if (!(fa * fb <= 0)) return false;
    if (fa == 0) { root = a; return true; }
    if (fb == 0) { root = b; return true; }
    double c = a, fc = fa, d = b - a, e = d;
    for (int it = 0; it < 200; it++) {
        if (fb * fc > 0) { c = a; fc = fa; d = b - a; e = d; }
        if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
        const double tol1 = 2.0 * 1e-16 * fabs(b) + 0.5 * tol, xm = 0.5 * (c - b);
        if (fabs(xm) <= tol1 || fb == 0) { root = b; return true; }
        if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
            double s = fb / fa, p, q;
            if (a == c) { p = 2 * xm * s; q = 1 - s; }
            else {
                const double qq = fa / fc, r = fb / fc;
                p = s * (2 * xm * qq * (qq - r) - (b - a) * (r - 1));
                q = (qq - 1) * (r - 1) * (s - 1);
            }
            if (p > 0) q = -q;
            p = fabs(p);
            if (2 * p < SMIN(3 * xm * q - fabs(tol1 * q), fabs(e * q))) { e = d; d = p / q; }
            else { d = xm; e = d; }
        } else { d = xm; e = d; }
        a = b; fa = fb;
        b += (fabs(d) > tol1) ? d : (xm > 0 ? tol1 : -tol1);
        fb = f(b);
        if (!isfinite(fb)) return false;
    }
    root = b;
    return true;
}
// Root of f on (plo, inf) through y = ln(p - plo): a sign change bracketed from the guess, then
// Brent (root_above :207-225); f is positive (or undefined) just above plo and negative at inf.
template <class Fn>
SPB6G_DEV bool root_above(Fn f, double plo, double guess, double& root) {
    auto F = [&](double y) { return f(plo + exp(y)); };
    const double y0 = log(SMAX(guess - plo, 1e-6 * (fabs(plo) + 1.0) + 1e-12));
    const double f0 = F(y0);
    if (f0 == 0.0) { root = plo + exp(y0); return true; }
    double ya = y0, yb = y0, fa = f0, fb = f0, st = 0.1;
    if (!isfinite(f0)) {  // upwards to a feasible point
        for (int k = 0; k < 200 && !isfinite(fb); k++) { yb += 1.0; fb = F(yb); }
        if (!isfinite(fb)) return false;
        ya = yb; fa = fb;
    }
    if (fa > 0) {
        for (int k = 0; k < 400 && !(fb < 0); k++) {
            ya = yb; fa = fb; yb += st; st *= 1.6;
            fb = F(yb);
            if (!isfinite(fb)) return false;
        }
    } else {
        for (int k = 0; k < 400 && !(fa > 0); k++) {
            yb = ya; fb = fa; ya -= st; st *= 1.6;
            fa = F(ya);
            if (!isfinite(fa)) {
                ya = yb; fa = fb;
                for (int q = 0; q < 60; q++) {
                    const double ym = ya - st / ldexp(1.0, q + 1), fm = F(ym);
                    if (isfinite(fm) && fm > 0) { ya = ym; fa = fm; break; }
                }
                break;
            }
        }
    }
    if (fa == 0.0) { root = plo + exp(ya); return true; }
    if (fb == 0.0) { root = plo + exp(yb); return true; }
    if (!(fa > 0 && fb < 0)) return false;
    double y;
    if (!brent(F, ya, yb, fa, fb, 1e-15, y)) return false;
    root = plo + exp(y);
    return true;
}
// pT closure (closure_pT :716-726): common p and T with T(p) explicit from the energy and
// sum_k m_k v_k(p, T) = 1 (SG / NASG v_pT, e_pT :80-81).
static __device__ __noinline__ ClMg closure_pT(const Phys P, double m0, double m1, double rhoeC, double pguess) {
    ClMg res;
    res.ok = 0;
    const double m[2] = {m0, m1};
    const double Eth = rhoeC - m[0] * P.ph[0].q - m[1] * P.ph[1].q;
    if (!(Eth > 0)) return res;
    auto Tof = [&](double p) {
        double d = 0;
        for (int k = 0; k < 2; k++) d += m[k] * P.ph[k].cv * (p + P.ph[k].g * P.ph[k].pi) / (p + P.ph[k].pi);
        return Eth / d;
    };
    auto v_pT = [&](int k, double p, double T) { return (P.ph[k].g - 1.0) * P.ph[k].cv * T / (p + P.ph[k].pi) + P.ph[k].b; };
    auto e_pT = [&](int k, double p, double T) { return P.ph[k].cv * T * (p + P.ph[k].g * P.ph[k].pi) / (p + P.ph[k].pi) + P.ph[k].q; };
    auto Phi = [&](double p) {
        const double T = Tof(p);
        return m[0] * v_pT(0, p, T) + m[1] * v_pT(1, p, T) - 1.0;
    };
    double p;
    if (!root_above(Phi, SMAX(-P.ph[0].pi, -P.ph[1].pi), pguess, p)) return res;
    const double T = Tof(p);
    for (int k = 0; k < 2; k++) {
        res.o.a[k] = m[k] * v_pT(k, p, T);
        res.o.e[k] = m[k] * e_pT(k, p, T);
        res.o.m[k] = m[k];
        res.o.Tk[k] = T;
    }
    res.o.pbar = p;
    res.ok = T > 0;
    return res;
}

// ---- instantaneous chemical relaxation (pTg closure, B6.6), built with the extended physics
// Specific volume, energy, entropy and Gibbs function of a SG / NASG phase at (p, T) (:80-83).
SPB6G_DEV double v_pT(const PhaseD& h, double p, double T) { return (h.g - 1.0) * h.cv * T / (p + h.pi) + h.b; }
SPB6G_DEV double e_pT(const PhaseD& h, double p, double T) { return h.cv * T * (p + h.g * h.pi) / (p + h.pi) + h.q; }
SPB6G_DEV double s_pT(const PhaseD& h, double p, double T) {
    return h.cv * (h.g * log(T) - (h.g - 1.0) * log(p + h.pi)) + h.qp;
}
SPB6G_DEV double g_pT(const PhaseD& h, double p, double T) { return h.g * h.cv * T + h.b * p + h.q - T * s_pT(h, p, T); }
// Saturation temperature of pressure p, the root of g_1 - g_2 on the physical branch (Tsat
// :155-163): a first guess interpolated linearly in ln p from the table, then Newton with the
// step held within [T/2, 2T] (sat_newton :116-126); NaN off the table's range (p <= 0 or at or
// above the critical pressure) or where Newton does not converge.
SPB6G_DEV double sat_temperature(const Phys& P, double p) {
    const double* S = P.sat;
    const int n = (int)S[0];
    if (!(p > 0) || !(p < S[1]) || n < 1) return NAN;
    const double* lp = S + 4;
    const double* Tt = lp + n;
    const double l = log(p);
    double T;
    if (l <= lp[0]) T = Tt[0];
    else if (l >= lp[n - 1]) T = Tt[n - 1];
    else {
        const double h = lp[1] - lp[0];
        const int i = SMIN((int)((l - lp[0]) / h), n - 2);
        const double w = (l - lp[i]) / h;
        T = (1 - w) * Tt[i] + w * Tt[i + 1];
    }
    const PhaseD &h0 = P.ph[0], &h1 = P.ph[1];
    for (int it = 0; it < 60; it++) {
        const double f = g_pT(h0, p, T) - g_pT(h1, p, T), d = s_pT(h1, p, T) - s_pT(h0, p, T);
        if (!(d > 0) || !isfinite(f)) return NAN;
        double Tn = T - f / d;
        if (Tn < 0.5 * T) Tn = 0.5 * T;
        if (Tn > 2.0 * T) Tn = 2.0 * T;
        if (fabs(Tn - T) < 1e-14 * T) return Tn;
        T = Tn;
    }
    return fabs(g_pT(h0, p, T) - g_pT(h1, p, T)) < 1e-8 * fabs(g_pT(h0, p, T)) + 1e-8 ? T : NAN;
}
// Temperature of the mixture at pressure p, vapour mass fraction Y and specific energy eC
// (T_from_energy :766-769).
SPB6G_DEV double T_of_energy(const Phys& P, double p, double Y, double eC) {
    const PhaseD &h0 = P.ph[0], &h1 = P.ph[1];
    const double d = (1 - Y) * h0.cv * (p + h0.g * h0.pi) / (p + h0.pi) + Y * h1.cv * (p + h1.g * h1.pi) / (p + h1.pi);
    return (eC - (1 - Y) * h0.q - Y * h1.q) / d;
}
constexpr double Y_MIN = 1e-10;  // YMIN :245: the mass fractions stay within [Y_MIN, 1 - Y_MIN]
// pTg closure (closure_pTg :825-834 with pTg_state :811-824): at pressure p the temperature is
// Tsat(p) and Y follows from the energy, clamped to [Y_MIN, 1 - Y_MIN] (then T from the energy);
// at or above the critical pressure one phase by v against the critical volume; p solves
// rho ((1 - Y) v_1 + Y v_2) = 1 by root_above.
static __device__ __noinline__ ClMg closure_pTg(const Phys P, double m0, double m1, double rhoeC, double pguess) {
    ClMg res;
    res.ok = 0;
    const double rho = m0 + m1, eC = rhoeC / rho;
    auto state = [&](double p, double& Y, double& T) -> bool {
        const double Ts = sat_temperature(P, p);
        if (isfinite(Ts)) {
            const double el = e_pT(P.ph[0], p, Ts), ev = e_pT(P.ph[1], p, Ts);
            Y = (eC - el) / (ev - el);
            if (Y > Y_MIN && Y < 1 - Y_MIN) { T = Ts; return true; }
            Y = SMIN(SMAX(Y, Y_MIN), 1 - Y_MIN);
        } else {
            if (!(p >= P.sat[1])) return false;
            Y = (1.0 / rho < P.sat[2]) ? Y_MIN : 1 - Y_MIN;
        }
        T = T_of_energy(P, p, Y, eC);
        return T > 0;
    };
    auto Phi = [&](double p) {
        double Y, T;
        if (!state(p, Y, T)) return (double)NAN;
        return rho * ((1 - Y) * v_pT(P.ph[0], p, T) + Y * v_pT(P.ph[1], p, T)) - 1.0;
    };
    double p;
    if (!root_above(Phi, SMAX(-P.ph[0].pi, -P.ph[1].pi), pguess, p)) return res;
    double Y, T;
    if (!state(p, Y, T)) return res;
    res.o.m[0] = rho * (1 - Y);
    res.o.m[1] = rho * Y;
    for (int k = 0; k < 2; k++) {
        res.o.a[k] = res.o.m[k] * v_pT(P.ph[k], p, T);
        res.o.e[k] = res.o.m[k] * e_pT(P.ph[k], p, T);
        res.o.Tk[k] = T;
    }
    res.o.pbar = p;
    res.ok = 1;
    return res;
}

// ---- finite relaxation rates (B6.2, B6.4, B6.5), built with the extended physics
// Finite pressure relaxation (closure_mu :636-714): the volume transfer R of phase 1 over the
// stage, with (p1, p2)(R) from the 2 x 2 linear energy system (pressure work at the interface
// pressure weighted by the impedances Z), solves F(R) = R - tau mu (p1 - p2) = 0 (backward
// Euler) between 0 and the sign change of F, bracketed outwards and refined by Brent.  For
// tau mu = inf, or the exponential form (relaxform 1), it first solves p1 = p2 (R_eq, bracketed
// from the acoustic linearisation, not across the system's singularity); the exponential form
// then takes R = R_eq (1 - exp(-tau mu D)) with the secant D = dp(0) / R_eq.
static __device__ __noinline__ ClMg closure_mu(const Phys P, const ClIn in, double mrate) {
    ClMg res;
    res.ok = 0;
    const PhaseD &h0 = P.ph[0], &h1 = P.ph[1];
    const double sa = in.atr[0] + in.atr[1];
    const double om[2] = {in.atr[0] / sa, in.atr[1] / sa};
    const double ak[2] = {in.atr[0] / sa, in.atr[1] / sa};
    ClPre pr;
    closure_pre(P, in, pr);
    const double D0 = pr.D0;
    double lam[2], ex[2];
    seg_lambda(in, pr, in.pguess, lam, ex);
    const double w1 = in.Z[0] + in.Z[1] > 0 ? in.Z[1] / (in.Z[0] + in.Z[1]) : 0.5, w2 = 1.0 - w1;
    const double tm = isinf(mrate) ? INFINITY : in.tau * mrate;
    double det = 0.0;
    auto solve = [&](double R, double& p1, double& p2) -> bool {
        const double a1 = ak[0] + R, a2 = ak[1] - R;
        const double C1 = dedp_am(P, 0, a1, in.mtr[0]) + om[0] * in.s, C2 = dedp_am(P, 1, a2, in.mtr[1]) + om[1] * in.s;
        const double M11 = C1 + R * w1 - lam[0] * in.s * om[0], M12 = R * w2 - lam[0] * in.s * om[1];
        const double M21 = -R * w1 - lam[1] * in.s * om[0], M22 = C2 - R * w2 - lam[1] * in.s * om[1];
        const double r1 = in.etr[0] - in.mtr[0] * h0.q - h0.g * h0.pi * dedp_am(P, 0, a1, in.mtr[0]) + lam[0] * D0 + ex[0];
        const double r2 = in.etr[1] - in.mtr[1] * h1.q - h1.g * h1.pi * dedp_am(P, 1, a2, in.mtr[1]) + lam[1] * D0 + ex[1];
        det = M11 * M22 - M12 * M21;
        if (!(fabs(det) > 0)) return false;
        p1 = (r1 * M22 - M12 * r2) / det;
        p2 = (M11 * r2 - M21 * r1) / det;
        return isfinite(p1) && isfinite(p2);
    };
    double R = 0.0, p1, p2;
    const bool eq = P.relax_form == 1 || isinf(tm);
    if (tm > 0) {
        double det0 = 0.0, r0 = 0.0;  // r0: start of the bracket, inside the admissible volumes for R_eq
        if (eq) {
            const double Rlo = in.mtr[0] * h0.b - ak[0], Rhi = ak[1] - in.mtr[1] * h1.b;
            if (!(Rlo < Rhi)) return res;
            if (!(Rlo < 0.0 && 0.0 < Rhi)) r0 = Rlo >= 0.0 ? Rlo + 1e-9 * (Rhi - Rlo) : Rhi - 1e-9 * (Rhi - Rlo);
        }
        auto Fa = [&](double r, double& f) -> bool {
            double q1, q2;
            if (!solve(r, q1, q2)) return false;
            const double a1 = ak[0] + r, a2 = ak[1] - r;
            if (!(a1 > in.mtr[0] * h0.b && a2 > in.mtr[1] * h1.b)) return false;
            if (eq) {
                if (r != r0 && !(det * det0 > 0)) return false;  // not across the singularity
            } else if (!(q1 + h0.pi > 0 && q2 + h1.pi > 0)) {
                return false;
            }
            f = eq ? q2 - q1 : r - tm * (q1 - q2);
            return isfinite(f);
        };
        double f0;
        if (!Fa(r0, f0)) return res;
        det0 = det;
        if (eq && fabs(f0) <= 1e-13 * (fabs(in.pguess) + h0.g * fabs(h0.pi) + h1.g * fabs(h1.pi))) f0 = 0.0;
        R = r0;
        if (f0 != 0.0) {
            double hi = -f0;
            if (eq) {  // acoustic linearisation, else half the compressed phase's compressible volume
                double q[2], k = 0.0;
                solve(r0, q[0], q[1]);
                for (int j = 0; j < 2; j++) {
                    const double a = ak[j] + (j == 0 ? r0 : -r0), r = in.mtr[j] / a;
                    k += r * c2_rp(P, j, r, q[j]) / a;
                }
                hi = -f0 / k;
                if (!(isfinite(hi) && hi * -f0 > 0))
                    hi = f0 < 0 ? 0.5 * (ak[1] - r0 - in.mtr[1] * h1.b) : -0.5 * (ak[0] + r0 - in.mtr[0] * h0.b);
                hi += r0;
            }
            double lo = r0, flo = f0, fhi = NAN;
            bool ok = false, exact = false;
            for (int it = 0; it < 200; it++) {
                if (Fa(hi, fhi)) {
                    if (eq && fhi == 0.0) { ok = exact = true; break; }
                    if (fhi * flo < 0) { ok = true; break; }
                    lo = hi;
                    flo = fhi;
                    hi = lo + (lo - r0 == 0 ? -f0 : (lo - r0));
                } else {
                    hi = 0.5 * (lo + hi);
                }
            }
            if (!ok) return res;
            auto F = [&](double r) {
                double f;
                return Fa(r, f) ? f : (double)NAN;
            };
            if (exact) R = hi;
            else if (!brent(F, SMIN(lo, hi), SMAX(lo, hi), lo < hi ? flo : fhi, lo < hi ? fhi : flo,
                            1e-16 * (fabs(lo) + fabs(hi)) + 1e-300, R))
                return res;
        }
        if (P.relax_form == 1 && !isinf(tm)) {
            const double D = R != 0.0 && r0 == 0.0 ? -f0 / R : 0.0;
            if (D > 0 && isfinite(D)) R = -R * expm1(-tm * D);
        }
    }
    if (!solve(R, p1, p2)) return res;
    const double pp[2] = {p1, p2};
    for (int k = 0; k < 2; k++) {
        res.o.a[k] = ak[k] + (k == 0 ? R : -R);
        res.o.m[k] = in.mtr[k];
        if (!(res.o.a[k] > res.o.m[k] * P.ph[k].b) || !(pp[k] + P.ph[k].pi > 0)) return res;
        res.o.e[k] = eps_amp(P, k, res.o.a[k], res.o.m[k], pp[k]);
        res.o.Tk[k] = T_amp(P, k, res.o.a[k], res.o.m[k], pp[k]);
    }
    res.o.pbar = res.o.a[0] * p1 + res.o.a[1] * p2;
    res.ok = 1;
    return res;
}

// Finite heat exchange at mu = inf (closure_theta :732-764): at fixed p each phase's temperature is
// linear in the heat dQ moved, so dQ has a closed form -- backward Euler tt (T2 - T1) / (1 + tt S)
// or the exponential (T2 - T1)(1 - exp(-tt S)) / S, tt = tau theta, S = 1/Cp1 + 1/Cp2 -- and p
// solves sum_k alpha_k(p, dQ(p)) = 1 by root_above.
static __device__ __noinline__ ClMg closure_theta(const Phys P, const ClIn in, double th) {
    ClMg res;
    res.ok = 0;
    if (!(in.mtr[0] + in.mtr[1] > 0)) return res;
    ClPre pr;
    closure_pre(P, in, pr);
    double lam[2], ex[2];
    seg_lambda(in, pr, in.pguess, lam, ex);
    double A[2], B[2], N[2];  // p_coef (:452-465)
    for (int k = 0; k < 2; k++) {
        A[k] = in.etr[k] - in.mtr[k] * P.ph[k].q + lam[k] * pr.D0 + ex[k];
        B[k] = in.atr[k] + lam[k] * in.s;
        N[k] = A[k] - (B[k] - in.mtr[k] * P.ph[k].b) * P.ph[k].pi;
    }
    const double tt = isinf(th) ? INFINITY : in.tau * th;
    if (tt > 0 && !isinf(tt))
        for (int k = 0; k < 2; k++)
            if (!(N[k] > 0)) return res;
    const double Cp[2] = {P.ph[0].g * P.ph[0].cv * in.mtr[0], P.ph[1].g * P.ph[1].cv * in.mtr[1]};
    const double S = 1.0 / Cp[0] + 1.0 / Cp[1];
    auto eval = [&](double p, double a[2]) {
        double a0[2], T0[2];
        for (int k = 0; k < 2; k++) {  // alpha_p (:466)
            const PhaseD& h = P.ph[k];
            a0[k] = ((h.g - 1.0) * (A[k] + B[k] * p) + (p + h.g * h.pi) * in.mtr[k] * h.b) / (h.g * (p + h.pi));
            T0[k] = T_amp(P, k, a0[k], in.mtr[k], p);
        }
        double dQ;
        if (P.relax_form == 1) dQ = (T0[1] - T0[0]) * (-expm1(-tt * S)) / S;
        else if (isinf(tt)) dQ = (T0[1] - T0[0]) / S;
        else dQ = tt * (T0[1] - T0[0]) / (1.0 + tt * (1.0 / Cp[0] + 1.0 / Cp[1]));
        a[0] = a0[0] + (P.ph[0].g - 1.0) * dQ / (P.ph[0].g * (p + P.ph[0].pi));
        a[1] = a0[1] - (P.ph[1].g - 1.0) * dQ / (P.ph[1].g * (p + P.ph[1].pi));
    };
    auto Phi = [&](double p) {
        double a[2];
        eval(p, a);
        return a[0] + a[1] - 1.0;
    };
    double p;
    if (!root_above(Phi, SMAX(-P.ph[0].pi, -P.ph[1].pi), in.pguess, p)) return res;
    double a[2];
    eval(p, a);
    for (int k = 0; k < 2; k++) {
        res.o.a[k] = a[k];
        res.o.m[k] = in.mtr[k];
        if (!(res.o.a[k] > res.o.m[k] * P.ph[k].b)) return res;
        res.o.e[k] = eps_amp(P, k, res.o.a[k], res.o.m[k], p);
        res.o.Tk[k] = T_amp(P, k, res.o.a[k], res.o.m[k], p);
    }
    res.o.pbar = p;
    res.ok = 1;
    return res;
}

// Finite mass transfer at mu = theta = inf (closure_nu :771-809): at each trial p the vapour
// fraction Y solves rho Y - m2 + tau nu (g2 - g1)(p, T(p, Y)) = 0 (backward Euler; Brent on the
// admissible interval, clamped to its end where it has no root), or for the exponential form Y =
// Y_eq + (Y0 - Y_eq) exp(-tau nu D / rho) with the secant D through Y_eq and the transported Y0;
// p solves rho ((1 - Y) v1 + Y v2) = 1 by root_above.
static __device__ __noinline__ ClMg closure_nu(const Phys P, const ClIn in, double nr) {
    ClMg res;
    res.ok = 0;
    const double rho = in.mtr[0] + in.mtr[1], eC = in.rhoeC / rho;
    const double tn = isinf(nr) ? INFINITY : in.tau * nr;
    const double Y0 = in.mtr[1] / rho;
    const PhaseD &h0 = P.ph[0], &h1 = P.ph[1];
    auto Yof = [&](double p, double& Y, double& T) -> bool {
        auto G = [&](double y) {
            const double TT = T_of_energy(P, p, y, eC);
            if (!(TT > 0)) return (double)NAN;
            return g_pT(h1, p, TT) - g_pT(h0, p, TT);
        };
        auto Rf = [&](double y) {
            if (P.relax_form == 1 || isinf(tn)) return G(y);
            const double TT = T_of_energy(P, p, y, eC);
            if (!(TT > 0)) return (double)NAN;
            return rho * y - in.mtr[1] + tn * (g_pT(h1, p, TT) - g_pT(h0, p, TT));
        };
        double ya = Y_MIN, yb = 1.0 - Y_MIN;  // T(p, y) > 0 bounds y on the side of the larger q
        const double dq = h1.q - h0.q, yT = dq != 0.0 ? (eC - h0.q) / dq : INFINITY;
        if (dq > 0) yb = SMIN(yb, yT * (1.0 - 1e-12));
        else if (dq < 0) ya = SMAX(ya, yT * (1.0 + 1e-12));
        if (!(ya < yb)) return false;
        if (P.relax_form == 1 && tn == 0.0) {
            Y = SMIN(SMAX(Y0, ya), yb);
            T = T_of_energy(P, p, Y, eC);
            return T > 0;
        }
        const double Ra = Rf(ya), Rb = Rf(yb);
        if (!isfinite(Ra) || !isfinite(Rb)) return false;
        if (Ra >= 0) Y = ya;
        else if (Rb <= 0) Y = yb;
        else if (!brent(Rf, ya, yb, Ra, Rb, 1e-16, Y)) return false;
        if (P.relax_form == 1 && !isinf(tn)) {  // Y is Y_eq(p)
            const double Yeq = Y, Ys = SMIN(SMAX(Y0, ya), yb);
            const double D = Ys != Yeq ? G(Ys) / (Ys - Yeq) : 0.0;
            if (D > 0 && isfinite(D)) {
                Y = SMIN(SMAX(Yeq + (Y0 - Yeq) * exp(-(tn * D) / rho), ya), yb);
            } else if (fabs(Ys - Yeq) <= 1e-14) {
                Y = Yeq;
            } else {  // G not monotone: the backward-Euler root
                auto Rbe = [&](double y) {
                    const double gg = G(y);
                    return isfinite(gg) ? rho * y - in.mtr[1] + tn * gg : (double)NAN;
                };
                const double ra = Rbe(ya), rb = Rbe(yb);
                if (!isfinite(ra) || !isfinite(rb)) return false;
                if (ra >= 0) Y = ya;
                else if (rb <= 0) Y = yb;
                else if (!brent(Rbe, ya, yb, ra, rb, 1e-16, Y)) return false;
            }
        }
        T = T_of_energy(P, p, Y, eC);
        return T > 0;
    };
    auto Phi = [&](double p) {
        double Y, T;
        if (!Yof(p, Y, T)) return (double)NAN;
        return rho * ((1 - Y) * v_pT(h0, p, T) + Y * v_pT(h1, p, T)) - 1.0;
    };
    double p;
    if (!root_above(Phi, SMAX(-h0.pi, -h1.pi), in.pguess, p)) return res;
    double Y, T;
    if (!Yof(p, Y, T)) return res;
    res.o.m[0] = rho * (1 - Y);
    res.o.m[1] = rho * Y;
    for (int k = 0; k < 2; k++) {
        res.o.a[k] = res.o.m[k] * v_pT(P.ph[k], p, T);
        res.o.e[k] = res.o.m[k] * e_pT(P.ph[k], p, T);
        res.o.Tk[k] = T;
    }
    res.o.pbar = p;
    res.ok = 1;
    return res;
}

// Every closure but p for SG / NASG phases (closure :842-866): the instantaneous pT and pTg, the
// finite-rate mu, theta and nu, and under unify = 1 the instantaneous p, pT and pTg as the mu,
// theta and nu closures at rate = inf (closure_rate_inf :836-841).
static __device__ __noinline__ ClMg closure_relaxed(const Phys P, const ClIn in) {
    const bool inst = in.type == CL_P || in.type == CL_PT || in.type == CL_PTG;
    if (P.unify == 1 && inst) {
        if (in.type == CL_P) return closure_mu(P, in, INFINITY);
        if (in.type == CL_PT) return closure_theta(P, in, INFINITY);
        return closure_nu(P, in, INFINITY);
    }
    switch (in.type) {
        case CL_MU: return closure_mu(P, in, P.mu_rate);
        case CL_PT: return closure_pT(P, in.mtr[0], in.mtr[1], in.rhoeC, in.pguess);
        case CL_THETA: return closure_theta(P, in, P.theta_rate);
        case CL_NU: return closure_nu(P, in, in.nu >= 0 ? in.nu : P.nu_rate);
        default: return closure_pTg(P, in.mtr[0], in.mtr[1], in.rhoeC, in.pguess);
    }
}

// Saturation pressure of temperature T, the inverse of Tsat by bisection in ln p over the table's
// range (psat :165-172): 0 below it, INFINITY above.
SPB6G_DEV double sat_pressure(const Phys& P, double T) {
    if ((int)P.sat[0] < 1) return NAN;
    double a = P.sat[3], b = P.sat[1] * (1 - 1e-12);
    const double Ta = sat_temperature(P, a), Tb = sat_temperature(P, b);
    if (!(T > Ta)) return 0.0;
    if (!(T < Tb)) return INFINITY;
    for (int it = 0; it < 80; it++) {
        const double c = sqrt(a * b);
        if (sat_temperature(P, c) < T) a = c;
        else b = c;
        if (b / a - 1 < 1e-14) break;
    }
    return sqrt(a * b);
}
// The mass transfer rate of a cell (nu_law :174-179, Pelanti 2022 (84)): nu_cr alpha_v^0.6
// ((psat(T) - p) / (nu_pc - psat(T)))^1.76 for superheated liquid (p < psat(T)), else 0.
SPB6G_DEV double nu_law(const Phys& P, double p, double T, double av) {
    const double ps = sat_pressure(P, T);
    if (!isfinite(ps) || !(ps > p) || !(ps < P.nu_pc) || !(av > 0)) return 0.0;
    return P.nu_cr * pow(av, 0.6) * pow((ps - p) / (P.nu_pc - ps), 1.76);
}


// Bracketed safeguarded Newton on Phi (closure_p, :472-548), preceded by the
// admissibility checks of closure() (:842-866).  At most 400 iterations.
SPB6G_DEV bool closure(const Phys& P, const ClIn& in, ClOut& o) {
#pragma unroll
    for (int k = 0; k < 2; k++)
        if (!(in.atr[k] > 0) || !(in.mtr[k] > 0) || !isfinite(in.etr[k])) return false;
    if (!isfinite(in.rhoeC) || !isfinite(in.s)) return false;
    if (SPB6G_MG && in.type != CL_PND) {
        if (P.mg && in.type != CL_P) return false;  // Mie-Grueneisen phases relax mechanically only (:846)
        if (!P.mg && (in.type != CL_P || P.unify == 1)) {
            const ClMg r = closure_relaxed(P, in);
            o = r.o;
            return r.ok && isfinite(o.pbar);
        }
    }
    if (SPB6G_MG && P.mg) {
        const ClMg r = closure_p_mg(P, in);
        o = r.o;
        return r.ok && isfinite(o.pbar);
    }
    if (!(in.mtr[0] + in.mtr[1] > 0)) return false;
    const double plo = SMAX(-P.ph[0].pi, -P.ph[1].pi);
    ClPre pr;
    closure_pre(P, in, pr);
    double p = plo + SMAX(in.pguess - plo, 1e-3 * (fabs(plo) + 1.0));
    double lo = plo, hi = INFINITY;
    bool conv = false;
    for (int it = 0; it < 400; it++) {
        double df;
        const double f = PhiD(P, in, pr, p, df);
        if (f == 0.0) { conv = true; break; }
        if (f > 0) lo = p; else hi = p;
        double pn = df < 0 ? p - f / df : NAN;
        if (fabs(pn - p) <= 2e-16 * (fabs(p) + fabs(plo))) { p = pn; conv = true; break; }
        if (!(pn > lo && pn < hi)) {
            if (!isfinite(hi)) pn = plo + 4.0 * (p - plo);
            else if (lo == plo) pn = plo + 0.25 * (hi - plo);
            else pn = (hi - plo > 1e3 * (lo - plo + 1e-300) && lo > plo) ? plo + sqrt((lo - plo) * (hi - plo)) : 0.5 * (lo + hi);
        }
        if (fabs(pn - p) <= 2e-16 * (fabs(p) + fabs(plo)) || (hi < INFINITY && hi - lo <= 4e-16 * (fabs(hi) + fabs(lo)))) {
            p = pn; conv = true; break;
        }
        p = pn;
    }
    if (!conv) return false;
    double lam[2], ex[2];
    seg_lambda(in, pr, p, lam, ex);
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const PhaseD& h = P.ph[k];
        const double A = pr.A0[k] + lam[k] * pr.D0 + ex[k], B = in.atr[k] + lam[k] * in.s;
        o.a[k] = ((h.g - 1.0) * (A + B * p) + (p + h.g * h.pi) * in.mtr[k] * h.b) / (h.g * (p + h.pi));  // alpha_p :465
        if (!(o.a[k] > in.mtr[k] * h.b) || !(p + h.pi > 0)) return false;
        o.e[k] = eps_amp(P, k, o.a[k], in.mtr[k], p);
    }
    o.pbar = p;
    return isfinite(p);
}
// Round-off floor of the closure pressure (SPB6_PC_IMEX_omp.cpp:657-664, via p_coef :453-464).
SPB6G_DEV double closure_roundoff(const Phys& P, const ClIn& in, double p) {
    if (SPB6G_MG && (P.mg || in.type != CL_P)) return 0.0;  // floor of the p-closure without MG phases only (closure_roundoff :657-658)
    if (!(in.mtr[0] + in.mtr[1] > 0)) return 0.0;
    const double D0 = in.rhoeC - in.etr[0] - in.etr[1];
    // defect_split (:438-449) at delta = D0 + p s
    double lam[2], ex[2] = {0.0, 0.0};
    if (P.share_mode == 2) {
        const double sm = in.mtr[0] + in.mtr[1];
        for (int k = 0; k < 2; k++) lam[k] = sm > 0 ? in.mtr[k] / sm : 0.5;
    } else {
        double E[2], sE = 0.0;
        for (int k = 0; k < 2; k++) { E[k] = E_above(P, in, k); sE += E[k]; }
        double lE[2];
        if (sE > 0) for (int k = 0; k < 2; k++) lE[k] = E[k] / sE;
        else { const double sm = in.mtr[0] + in.mtr[1]; for (int k = 0; k < 2; k++) lE[k] = sm > 0 ? in.mtr[k] / sm : 0.5; }
        const double Q = P.share_mode == 1 ? 0.0 : in.Qph[0] + in.Qph[1];
        const double delta = D0 + p * in.s;
        if (!(delta > 0.0) || !(Q > 0.0)) { lam[0] = lE[0]; lam[1] = lE[1]; }
        else if (delta < Q) { lam[0] = in.Qph[0] / Q; lam[1] = in.Qph[1] / Q; }
        else for (int k = 0; k < 2; k++) { lam[k] = lE[k]; ex[k] = in.Qph[k] - Q * lE[k]; }
    }
    double dphi = 0.0, sens = 0.0;
    for (int k = 0; k < 2; k++) {
        const PhaseD& h = P.ph[k];
        const double A = in.etr[k] - in.mtr[k] * h.q + lam[k] * D0 + ex[k], B = in.atr[k] + lam[k] * in.s;
        const double N = A - (B - in.mtr[k] * h.b) * h.pi;
        dphi += -(h.g - 1.0) * N / (h.g * (p + h.pi) * (p + h.pi));
        sens += fabs(lam[k]) * (h.g - 1.0) / (h.g * (p + h.pi));
    }
    const double en = 2.220446049250313e-16 * (fabs(in.rhoeC) + fabs(in.etr[0]) + fabs(in.etr[1]) +
                                              fabs(in.mtr[0] * P.ph[0].q) + fabs(in.mtr[1] * P.ph[1].q));
    return dphi < 0 ? en * sens / -dphi : 0.0;
}

// ------------------------------------------------------------ primitives, :893-913
struct Prim {
    double u, v, rho, cf;
};
SPB6G_DEV bool prim_of(const Phys& P, const double* Q, Prim& w) {
    const double a1 = Q[IA1], a2 = 1 - a1, m1 = Q[IM1], m2 = Q[IM2];
    if (!(a1 > 0 && a2 > 0 && m1 > 0 && m2 > 0)) return false;
    w.rho = m1 + m2;
    const double r1 = m1 / a1, r2 = m2 / a2;
    w.u = Q[IMU] / w.rho;
    w.v = Q[IMV] / w.rho;
    const double p1 = p_ame(P, 0, a1, m1, Q[IE1]), p2 = p_ame(P, 1, a2, m2, Q[IE2]);
    if (!(p_admissible(P, 0, a1, m1, p1) && p_admissible(P, 1, a2, m2, p2))) return false;
    w.cf = sqrt((m1 * c2_rp(P, 0, r1, p1) + m2 * c2_rp(P, 1, r2, p2)) / w.rho);
    return true;
}
SPB6G_DEV double pbar_of(const Phys& P, const double* Q) {
    const double a1 = Q[IA1];
    return a1 * p_ame(P, 0, a1, Q[IM1], Q[IE1]) + (1 - a1) * p_ame(P, 1, 1 - a1, Q[IM2], Q[IE2]);
}

// ------------------------------------------------------------ shock budget, :267-428
template <bool MG = true>
SPB6G_DEV bool eos_ok(const Phys& P, int k, double p, double v) {  // :273-277
    if (!(v > 0) || !isfinite(p)) return false;
    if (MG && SPB6G_MG && P.ph[k].kind) return c2_rp(P, k, 1.0 / v, p) > 0;
    return v > P.ph[k].b && p + P.ph[k].pi > 0;
}
// Mie-Grueneisen Hugoniot from (p0, v0) to p1 (:285-292): bisection on (0, v0].
static __device__ __noinline__ double hug_v_mg(const PhaseD h, double p0, double p1, double v0) {
    auto e_pv = [&](double p, double v) {
        double pr, dpr, er;
        mg_ref(h, 1.0 / v, pr, dpr, er);
        return er + v * (p - pr) / h.G;
    };
    const double e0 = e_pv(p0, v0);
    auto g = [&](double v) { return e_pv(p1, v) - e0 + 0.5 * (p0 + p1) * (v - v0); };
    double hi = v0, lo = v0, gl = g(v0);
    if (!(gl > 0)) return v0;
    for (int it = 0; it < 80 && gl > 0; it++) {
        hi = lo;
        lo *= 0.9;
        gl = g(lo);
        if (!isfinite(gl)) return NAN;
    }
    if (gl > 0) return NAN;
    for (int it = 0; it < 100; it++) {
        const double m = 0.5 * (lo + hi), gm = g(m);
        if (gm > 0) hi = m; else lo = m;
        if (hi - lo <= 1e-14 * v0) break;
    }
    return 0.5 * (lo + hi);
}
SPB6G_DEV double hug_v(const Phys& P, int k, double p0, double p1, double v0) {  // NASG closed form, :279-284
    const PhaseD& h = P.ph[k];
    if (SPB6G_MG && h.kind) return hug_v_mg(h, p0, p1, v0);
    const double x0 = p0 + h.pi, x1 = p1 + h.pi;
    return h.b + (v0 - h.b) * ((h.g - 1.0) * x1 + (h.g + 1.0) * x0) / ((h.g + 1.0) * x1 + (h.g - 1.0) * x0);
}
SPB6G_DEV void K_G(const Phys& P, int k, double p, double v, double& K, double& Gm) {  // :296-301
    K = c2_rp(P, k, 1.0 / v, p) / v;
    if (SPB6G_MG && P.ph[k].kind) {  // MG: dK/dp along the isentrope dv = -v dp / K by a difference
        const double dp = 1e-6 * K, K2 = c2_rp(P, k, 1.0 / (v * (1.0 - dp / K)), p + dp) / (v * (1.0 - dp / K));
        Gm = 0.5 * (1.0 + (K2 - K) / dp);
        return;
    }
    Gm = 0.5 * (P.ph[k].g + 1.0);
    if (P.ph[k].b != 0.0) Gm *= v / (v - P.ph[k].b);
}

// Per-cell constants of the profile ODE: 1/Y_2 and, per phase, 1/(g-1) and g/(g-1); lamY
// holds lambda_k / Y_k for the integration's c.  The right-hand side below is the
// reference's (:304-312) with these reciprocals hoisted: 3 divisions per evaluation
// instead of 13.  The strong-shock branch is round-off sensitive in the reference itself
// (a one-ulp change of its libm calls moves Q by up to 1e-2 in ill-conditioned cells), and
// the hoisting changes the result at that round-off level only.
struct ShockProf {
    double Y[2], vk0[2], v0, p0, j2, vend;
    double iY1, ig1[2], ggm[2], lamY[2];
};
SPB6G_DEV void prof_consts(const Phys& P, ShockProf& S) {
    S.iY1 = 1.0 / S.Y[1];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        S.ig1[k] = 1.0 / (P.ph[k].g - 1.0);
        S.ggm[k] = P.ph[k].g * S.ig1[k];
    }
}
// The right-hand side with a Mie-Grueneisen phase, in the reference's own form (:304-312 with
// eos_ep_ev :268-272).
struct ProfRhs {
    double dy[3];
    int ok;
};
static __device__ __noinline__ ProfRhs prof_rhs_mg(const Phys P, const ShockProf S, double v, double y0, double y1) {
    ProfRhs res;
    res.ok = 0;
    double* dy = res.dy;
    const double p = y0, v1 = y1, v2 = (v - S.Y[0] * v1) / S.Y[1], Pr = S.p0 + S.j2 * (S.v0 - v);
    if (!eos_ok(P, 0, p, v1) || !eos_ok(P, 1, p, v2)) return res;
    const double vk[2] = {v1, v2};
    double num = -1.0, den = 0.0, r[2], ep[2], evp[2];
    for (int k = 0; k < 2; k++) {
        const PhaseD& h = P.ph[k];
        if (SPB6G_MG && h.kind) {
            double pr, dpr, er;
            const double rr = 1.0 / vk[k];
            mg_ref(h, rr, pr, dpr, er);
            ep[k] = vk[k] / h.G;
            evp[k] = (p - pr) * (1.0 + 1.0 / h.G) + rr * dpr / h.G;
        } else {
            ep[k] = (vk[k] - h.b) / (h.g - 1.0);
            evp[k] = h.g * (p + h.pi) / (h.g - 1.0);
        }
        r[k] = S.lamY[k] * (p - Pr);
        num += S.Y[k] * r[k] / evp[k];
        den += S.Y[k] * ep[k] / evp[k];
    }
    dy[0] = num / den;
    dy[1] = (r[0] - ep[0] * dy[0]) / evp[0];
    dy[2] = p - Pr;
    res.ok = isfinite(dy[0]) && isfinite(dy[1]);
    return res;
}
// MG: the strong-shock routine is instantiated twice, and the SG / NASG instantiation makes no
// Mie-Grueneisen call inside its integration loop.
template <bool MG>
SPB6G_DEV bool prof_rhs(const Phys& P, const ShockProf& S, double v, const double* y, double* dy) {  // :304-312
    if constexpr (MG) {
        const ProfRhs r = prof_rhs_mg(P, S, v, y[0], y[1]);
        dy[0] = r.dy[0];
        dy[1] = r.dy[1];
        dy[2] = r.dy[2];
        return r.ok;
    }
    const double p = y[0], v1 = y[1], v2 = (v - S.Y[0] * v1) * S.iY1, Pr = S.p0 + S.j2 * (S.v0 - v);
    if (!eos_ok<false>(P, 0, p, v1) || !eos_ok<false>(P, 1, p, v2)) return false;
    const double vk[2] = {v1, v2}, dp = p - Pr;
    double num = -1.0, den = 0.0, r[2], ep[2], iev[2];
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const PhaseD& h = P.ph[k];
        ep[k] = (vk[k] - h.b) * S.ig1[k];                 // eos_ep_ev :268-272
        iev[k] = 1.0 / ((p + h.pi) * S.ggm[k]);           // 1 / e_{v,p}
        r[k] = S.lamY[k] * dp;
        num += S.Y[k] * r[k] * iev[k];
        den += S.Y[k] * ep[k] * iev[k];
    }
    dy[0] = num / den;
    dy[1] = (r[0] - ep[0] * dy[0]) * iev[0];
    dy[2] = dp;
    return isfinite(dy[0]) && isfinite(dy[1]);
}
// Kapila shock profile integrated with the adaptive Cash-Karp embedded RK4(5)
// pair (Cash & Karp 1990), :313-343.  At most 4000 steps.
template <bool MG>
SPB6G_DEV bool prof_integrate(const Phys& P, ShockProf& S, double c, double& v1end, double& qend) {
    S.lamY[0] = c / S.Y[0];
    S.lamY[1] = (1.0 - c) / S.Y[1];
    const double A[6] = {0, 0.2, 0.3, 0.6, 1.0, 0.875};
    const double B[6][5] = {{0, 0, 0, 0, 0},
                            {0.2, 0, 0, 0, 0},
                            {3.0 / 40, 9.0 / 40, 0, 0, 0},
                            {0.3, -0.9, 1.2, 0, 0},
                            {-11.0 / 54, 2.5, -70.0 / 27, 35.0 / 27, 0},
                            {1631.0 / 55296, 175.0 / 512, 575.0 / 13824, 44275.0 / 110592, 253.0 / 4096}};
    const double C5[6] = {37.0 / 378, 0, 250.0 / 621, 125.0 / 594, 0, 512.0 / 1771};
    const double C4[6] = {2825.0 / 27648, 0, 18575.0 / 48384, 13525.0 / 55296, 277.0 / 14336, 0.25};
    double y[3] = {S.p0, S.vk0[0], 0.0}, v = S.v0;
    const double L = S.vend - S.v0;
    const double isc[3] = {1.0 / (fabs(S.p0) + S.j2 * fabs(L)), 1.0 / S.vk0[0], 1.0 / (S.j2 * L * L + 1e-300)};
    double h = L / 32.0;
    for (int it = 0; it < 4000; it++) {
        const bool last = (L < 0 && v + h <= S.vend) || (L > 0 && v + h >= S.vend);
        if (last) h = S.vend - v;
        double k[6][3], yt[3];
        bool ok = true;
        for (int st = 0; st < 6 && ok; st++) {
            for (int n = 0; n < 3; n++) {
                yt[n] = y[n];
                for (int q = 0; q < st; q++) yt[n] += h * B[st][q] * k[q][n];
            }
            ok = prof_rhs<MG>(P, S, v + A[st] * h, yt, k[st]);
        }
        double err = 0.0, y5[3];
        if (ok)
            for (int n = 0; n < 3; n++) {
                double d5 = 0, d4 = 0;
                for (int st = 0; st < 6; st++) { d5 += C5[st] * k[st][n]; d4 += C4[st] * k[st][n]; }
                y5[n] = y[n] + h * d5;
                err = SMAX(err, fabs(h * (d5 - d4)) * isc[n]);
            }
        if (!ok || !(err <= 1e-8)) {
            h *= ok ? SMAX(0.1, 0.9 * sqrt(sqrt(1e-8 / err))) : 0.25;
            if (fabs(h) < 1e-14 * fabs(L)) return false;
            continue;
        }
        for (int n = 0; n < 3; n++) y[n] = y5[n];
        if (last) { v1end = y[1]; qend = y[2]; return true; }
        v += h;
        h *= SMIN(5.0, 0.9 * pow(1e-8 / SMAX(err, 1e-30), 0.2));
    }
    return false;
}
template <bool MG>
SPB6G_DEV double shoot_F(const Phys& P, ShockProf& S, const double vH[2], const double vpre[2], double t, double& qq) {
    const double c = 1.0 / (1.0 + exp(-t));
    double v1e;
    if (!prof_integrate<MG>(P, S, c, v1e, qq)) return NAN;
    return (v1e - vH[0]) / vpre[0];
}
// Weak-shock analytic share; returns false and sets `strong` when the profile
// shooting (shock_share's Illinois branch) is needed.
SPB6G_DEV bool shock_share_weak(const Phys& P, const double Y[2], const double vpre[2], double p0, double p1,
                                double lam[2], double& q, bool& strong, double K[2], double Gm[2]) {
    strong = false;
    double w[2], sw = 0.0, Kmin = INFINITY;
    for (int k = 0; k < 2; k++) {
        K_G(P, k, p0, vpre[k], K[k], Gm[k]);
        if (!(K[k] > 0)) return false;
        Kmin = SMIN(Kmin, K[k]);
    }
    const double dp = p1 - p0;
    if (dp < 1e-2 * Kmin) {
        q = 0.0;
        for (int k = 0; k < 2; k++) { w[k] = Y[k] * vpre[k] * Gm[k] / (K[k] * K[k]); sw += w[k]; }
        for (int k = 0; k < 2; k++) lam[k] = w[k] / sw;
        q = sw * dp * dp * dp / 6.0;
        return true;
    }
    strong = true;
    return false;
}
// Strong-shock branch of shock_share (:356-392): Illinois false position on logit(c).
template <bool MG>
SPB6G_DEV bool shock_share_strong_t(const Phys& P, const double Y[2], const double vpre[2], double p0, double p1,
                                  const double K[2], const double Gm[2], double lam[2], double& q) {
    const double dp = p1 - p0;
    ShockProf S;
    S.p0 = p0;
    double vH[2];
    for (int k = 0; k < 2; k++) {
        S.Y[k] = Y[k];
        S.vk0[k] = vpre[k];
        vH[k] = hug_v(P, k, p0, p1, vpre[k]);
        if (!isfinite(vH[k])) return false;
    }
    S.v0 = Y[0] * vpre[0] + Y[1] * vpre[1];
    S.vend = Y[0] * vH[0] + Y[1] * vH[1];
    prof_consts(P, S);
    if (!(S.vend < S.v0)) return false;
    S.j2 = dp / (S.v0 - S.vend);
    double t0;
    {
        double ww[2];
        for (int k = 0; k < 2; k++) ww[k] = Y[k] * vpre[k] * Gm[k] / (K[k] * K[k]);
        const double c0 = SMIN(1.0 - 1e-12, SMAX(1e-12, ww[0] / (ww[0] + ww[1])));
        t0 = isfinite(c0) ? log(c0 / (1.0 - c0)) : 0.0;
    }
    double ta = SMAX(-40.0, t0 - 1.0), tb = SMIN(40.0, t0 + 1.0), qa = 0, qb = 0;
    double fa = shoot_F<MG>(P, S, vH, vpre, ta, qa), fb = shoot_F<MG>(P, S, vH, vpre, tb, qb);
    if (!isfinite(fa) || !isfinite(fb)) return false;
    for (double st = 2.0; fa >= 0 && ta > -40.0; st *= 2.0) {
        tb = ta; fb = fa; qb = qa;
        ta = SMAX(-40.0, ta - st);
        fa = shoot_F<MG>(P, S, vH, vpre, ta, qa);
        if (!isfinite(fa)) return false;
    }
    for (double st = 2.0; fb <= 0 && tb < 40.0; st *= 2.0) {
        ta = tb; fa = fb; qa = qb;
        tb = SMIN(40.0, tb + st);
        fb = shoot_F<MG>(P, S, vH, vpre, tb, qb);
        if (!isfinite(fb)) return false;
    }
    double t, qt;
    if (fa >= 0) { t = ta; qt = qa; }
    else if (fb <= 0) { t = tb; qt = qb; }
    else {
        int side = 0;
        t = ta; qt = qa;
        for (int it = 0; it < 100; it++) {
            t = (ta * fb - tb * fa) / (fb - fa);
            if (!(t > ta && t < tb)) t = 0.5 * (ta + tb);
            const double ft = shoot_F<MG>(P, S, vH, vpre, t, qt);
            if (!isfinite(ft)) return false;
            if (fabs(ft) < 1e-10 || tb - ta < 1e-10) break;
            if (ft < 0) { ta = t; fa = ft; if (side == -1) fb *= 0.5; side = -1; }
            else { tb = t; fb = ft; if (side == 1) fa *= 0.5; side = 1; }
        }
    }
    const double c = 1.0 / (1.0 + exp(-t));
    lam[0] = c;
    lam[1] = 1.0 - c;
    q = qt;
    return q > 0;
}
struct ShockShare {
    double lam[2], q;
    int ok;
};
static __device__ __noinline__ ShockShare shock_share_strong_mg(const Phys P, const double Y0, const double Y1, const double v0,
                                                                const double v1, double p0, double p1, double K0, double K1,
                                                                double G0, double G1) {
    ShockShare r;
    const double Y[2] = {Y0, Y1}, vpre[2] = {v0, v1}, K[2] = {K0, K1}, Gm[2] = {G0, G1};
    r.ok = shock_share_strong_t<true>(P, Y, vpre, p0, p1, K, Gm, r.lam, r.q) ? 1 : 0;
    return r;
}
SPB6G_DEV bool shock_share_strong(const Phys& P, const double Y[2], const double vpre[2], double p0, double p1,
                                  const double K[2], const double Gm[2], double lam[2], double& q) {
    if (SPB6G_MG && P.mg) {
        const ShockShare r = shock_share_strong_mg(P, Y[0], Y[1], vpre[0], vpre[1], p0, p1, K[0], K[1], Gm[0], Gm[1]);
        lam[0] = r.lam[0];
        lam[1] = r.lam[1];
        q = r.q;
        return r.ok != 0;
    }
    return shock_share_strong_t<false>(P, Y, vpre, p0, p1, K, Gm, lam, q);
}
// stencil_state (:395-400): {a1, a2, m1, m2, p, u, v}; p = NaN when inadmissible.
SPB6G_DEV void stencil_state(const Phys& P, const double* c, double* st) {
    const double a1 = c[IA1], m1 = c[IM1], m2 = c[IM2], r = m1 + m2;
    st[0] = a1; st[1] = 1.0 - a1; st[2] = m1; st[3] = m2; st[4] = NAN;
    st[5] = r > 0 ? c[IMU] / r : 0.0;
    st[6] = r > 0 ? c[IMV] / r : 0.0;
    if (a1 > 0 && a1 < 1 && m1 > 0 && m2 > 0) {
        const double p = p_mix(P, a1, m1, m2, c[IE1] + c[IE2]);
        if (p_admissible(P, 0, a1, m1, p) && p_admissible(P, 1, 1.0 - a1, m2, p)) st[4] = p;
    }
}

}  // namespace spb6g
