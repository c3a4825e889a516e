// Per-cell physics of the SPB 6+1-equation model on the device: stiffened-gas /
// NASG equations of state, the mechanical (p) relaxation closure, the shock
// dissipation budget and the primitive-variable map.
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
#define SMAX(a, b) ((a) < (b) ? (b) : (a))
#define SMIN(a, b) ((b) < (a) ? (b) : (a))

namespace spb6g {

enum { IA1 = 0, IM1, IM2, IMU, IMV, IE1, IE2, IEN, NV = 8 };
enum { BC_TRANS = 0, BC_WALL = 1, BC_PERIODIC = 2, BC_PRES = 3 };

struct PhaseD {
    double g, pi, q, qp, cv, b;
};

// Phases and scheme switches shared by every kernel (passed by value).
struct Phys {
    PhaseD ph[2];
    int share_mode;  // SHARE_MODE, src/spb6_physics_omp.h:436
    int limiter;     // LIMITER, :969
    int rus_local;   // RUS_LOCAL, src/SPB6_PC_IMEX_omp.cpp:93
    int pad;
};

// ------------------------------------------------------------ EOS, src/spb6_physics_omp.h:71-111
SPB6G_DEV double eps_amp(const Phys& P, int k, double a, double m, double p) {
    const PhaseD& h = P.ph[k];
    return (p + h.g * h.pi) * (a - m * h.b) / (h.g - 1.0) + m * h.q;
}
SPB6G_DEV double p_ame(const Phys& P, int k, double a, double m, double e) {
    const PhaseD& h = P.ph[k];
    return (e - m * h.q) * (h.g - 1.0) / (a - m * h.b) - h.g * h.pi;
}
SPB6G_DEV double c2_rp(const Phys& P, int k, double r, double p) {
    const PhaseD& h = P.ph[k];
    return h.g * (p + h.pi) / (r * (1.0 - r * h.b));
}
SPB6G_DEV double dedp_am(const Phys& P, int k, double a, double m) {
    const PhaseD& h = P.ph[k];
    return (a - m * h.b) / (h.g - 1.0);
}
SPB6G_DEV double T_amp(const Phys& P, int k, double a, double m, double p) {
    const PhaseD& h = P.ph[k];
    return (a / m - h.b) * (p + h.pi) / ((h.g - 1.0) * h.cv);
}
SPB6G_DEV double p_mix(const Phys& P, double a1, double m1, double m2, double rhoe) {
    const double a[2] = {a1, 1.0 - a1}, m[2] = {m1, m2};
    double num = rhoe, den = 0.0;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        num -= m[k] * P.ph[k].q + P.ph[k].g * P.ph[k].pi * dedp_am(P, k, a[k], m[k]);
        den += dedp_am(P, k, a[k], m[k]);
    }
    return num / den;
}
SPB6G_DEV bool p_admissible(const Phys& P, int k, double p) { return p + P.ph[k].pi > 0; }
SPB6G_DEV double eps_round(const Phys& P, int k, double m) { return fabs(m * P.ph[k].q); }

// ------------------------------------------------------------ closure, :229-243, :430-548, :842-866
struct ClIn {
    double atr[2], mtr[2], etr[2], s, rhoeC, pguess, Qph[2];
};
struct ClOut {
    double a[2], e[2], pbar;
};

SPB6G_DEV double E_above(const Phys& P, const ClIn& in, int k) {  // :430-433
    const double v = in.etr[k] - in.mtr[k] * P.ph[k].q - (in.atr[k] - in.mtr[k] * P.ph[k].b) * P.ph[k].pi;
    return SMAX(0.0, v);
}

// Quantities of the p-closure that do not depend on the trial pressure (:481-489).
struct ClPre {
    double D0, lE[2], A0[2], Qb;
    bool byMass;
};
SPB6G_DEV void closure_pre(const Phys& P, const ClIn& in, ClPre& pr) {
    pr.D0 = in.rhoeC - in.etr[0] - in.etr[1];
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
// Bracketed safeguarded Newton on Phi (closure_p, :472-548), preceded by the
// admissibility checks of closure() (:842-866).  At most 400 iterations.
SPB6G_DEV bool closure(const Phys& P, const ClIn& in, ClOut& o) {
#pragma unroll
    for (int k = 0; k < 2; k++)
        if (!(in.atr[k] > 0) || !(in.mtr[k] > 0) || !isfinite(in.etr[k])) return false;
    if (!isfinite(in.rhoeC) || !isfinite(in.s)) return false;
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
    if (!(p_admissible(P, 0, p1) && p_admissible(P, 1, p2))) return false;
    w.cf = sqrt((m1 * c2_rp(P, 0, r1, p1) + m2 * c2_rp(P, 1, r2, p2)) / w.rho);
    return true;
}
SPB6G_DEV double pbar_of(const Phys& P, const double* Q) {
    const double a1 = Q[IA1];
    return a1 * p_ame(P, 0, a1, Q[IM1], Q[IE1]) + (1 - a1) * p_ame(P, 1, 1 - a1, Q[IM2], Q[IE2]);
}

// ------------------------------------------------------------ shock budget, :267-428
SPB6G_DEV bool eos_ok(const Phys& P, int k, double p, double v) {
    if (!(v > 0) || !isfinite(p)) return false;
    return v > P.ph[k].b && p + P.ph[k].pi > 0;
}
SPB6G_DEV double hug_v(const Phys& P, int k, double p0, double p1, double v0) {  // NASG closed form, :279-284
    const PhaseD& h = P.ph[k];
    const double x0 = p0 + h.pi, x1 = p1 + h.pi;
    return h.b + (v0 - h.b) * ((h.g - 1.0) * x1 + (h.g + 1.0) * x0) / ((h.g + 1.0) * x1 + (h.g - 1.0) * x0);
}
SPB6G_DEV void K_G(const Phys& P, int k, double p, double v, double& K, double& Gm) {  // :296-301
    K = c2_rp(P, k, 1.0 / v, p) / v;
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
SPB6G_DEV bool prof_rhs(const Phys& P, const ShockProf& S, double v, const double* y, double* dy) {  // :304-312
    const double p = y[0], v1 = y[1], v2 = (v - S.Y[0] * v1) * S.iY1, Pr = S.p0 + S.j2 * (S.v0 - v);
    if (!eos_ok(P, 0, p, v1) || !eos_ok(P, 1, p, v2)) return false;
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
            ok = prof_rhs(P, S, v + A[st] * h, yt, k[st]);
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
SPB6G_DEV double shoot_F(const Phys& P, ShockProf& S, const double vH[2], const double vpre[2], double t, double& qq) {
    const double c = 1.0 / (1.0 + exp(-t));
    double v1e;
    if (!prof_integrate(P, S, c, v1e, qq)) return NAN;
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
SPB6G_DEV bool shock_share_strong(const Phys& P, const double Y[2], const double vpre[2], double p0, double p1,
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
    double fa = shoot_F(P, S, vH, vpre, ta, qa), fb = shoot_F(P, S, vH, vpre, tb, qb);
    if (!isfinite(fa) || !isfinite(fb)) return false;
    for (double st = 2.0; fa >= 0 && ta > -40.0; st *= 2.0) {
        tb = ta; fb = fa; qb = qa;
        ta = SMAX(-40.0, ta - st);
        fa = shoot_F(P, S, vH, vpre, ta, qa);
        if (!isfinite(fa)) return false;
    }
    for (double st = 2.0; fb <= 0 && tb < 40.0; st *= 2.0) {
        ta = tb; fa = fb; qa = qb;
        tb = SMIN(40.0, tb + st);
        fb = shoot_F(P, S, vH, vpre, tb, qb);
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
            const double ft = shoot_F(P, S, vH, vpre, t, qt);
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
// stencil_state (:395-400): {a1, a2, m1, m2, p, u, v}; p = NaN when inadmissible.
SPB6G_DEV void stencil_state(const Phys& P, const double* c, double* st) {
    const double a1 = c[IA1], m1 = c[IM1], m2 = c[IM2], r = m1 + m2;
    st[0] = a1; st[1] = 1.0 - a1; st[2] = m1; st[3] = m2; st[4] = NAN;
    st[5] = r > 0 ? c[IMU] / r : 0.0;
    st[6] = r > 0 ? c[IMV] / r : 0.0;
    if (a1 > 0 && a1 < 1 && m1 > 0 && m2 > 0) {
        const double p = p_mix(P, a1, m1, m2, c[IE1] + c[IE2]);
        if (p_admissible(P, 0, p) && p_admissible(P, 1, p)) st[4] = p;
    }
}

}  // namespace spb6g
