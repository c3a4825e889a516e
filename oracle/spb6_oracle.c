/* ORACLE -- test infrastructure only, never part of the product.
 *
 * A serial C restatement of the reference SPB6_PC_IMEX stage loop (the OpenMP
 * path src/SPB6_PC_IMEX_omp.cpp with src/spb6_physics_omp.h) for the
 * mechanical (p) relaxation with stiffened-gas / NASG phases -- the scope the
 * GPU path implements.  Each function cites the reference lines it follows;
 * operation order is kept so that results agree with the compiled reference
 * (oracle/_ref) bit for bit, which tests/test_oracle.py checks.
 *
 * Used by tests/ (the CPU checker of the CUDA path), __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg.  Entry point: spb6_oracle_run (spb6_oracle.h).
 */
#define _POSIX_C_SOURCE 199309L
#include "spb6_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* Round-off perturbation variants (the reference's own acceptance criterion for a changed
 * implementation, docs/code/openmp_optimisation.md:81-82, is "no larger than the code's own
 * change under a round-off perturbation"):
 *   SPB6_ORACLE_ULP   exp / log / pow of the shock-profile shooting return the next double up;
 *   SPB6_ORACLE_FD    finite-difference Jacobian step 1.01e-7 instead of 1e-7 (the perturbation
 *                     the reference's report uses). */
#ifdef SPB6_ORACLE_ULP
static double sh_exp(double x) { return nextafter(exp(x), INFINITY); }
static double sh_log(double x) { return nextafter(log(x), INFINITY); }
static double sh_pow(double x, double y) { return nextafter(pow(x, y), INFINITY); }
#else
#define sh_exp exp
#define sh_log log
#define sh_pow pow
#endif
#ifdef SPB6_ORACLE_FD
#define FD_STEP 1.01e-7
#else
#define FD_STEP 1e-7
#endif

/* std::max / std::min semantics (the second argument wins only on a strict compare) */
#define SMAX(a, b) ((a) < (b) ? (b) : (a))
#define SMIN(a, b) ((b) < (a) ? (b) : (a))

enum { IA1 = 0, IM1, IM2, IMU, IMV, IE1, IE2, IEN, NV = 8 };
#define G 2 /* ghost layers, SPB6_PC_IMEX_omp.cpp:67 */

typedef struct { double g, pi, q, qp, cv, b; } Phase;

/* ------------------------------------------------------------------ solver context */
typedef struct {
    /* settings */
    int nx, ny, NXT, NYT, rk, ramp, rus_local, limiter, acdt, newton_iter, bicg_iter, share_mode;
    int bcs[4];
    double bcu[4], bcp[4];
    Phase ph[2];
    double x0, x1, y0, y1, dx, dy, cfl, cfl_ac, dtfix, newton_tol, bicg_tol, tend;
    /* time state */
    double t, dt, dtprev, adt, p_ref, vx_max, vy_max;
    int startup;
    /* counters (SPB6_PC_IMEX_omp.cpp:98-99) */
    long st_steps, st_reject, st_newton_it, st_stage, st_rk1, st_floor, st_bicg_it;
    double st_maxres;
    /* grids, AoS with ghosts like the reference Grid (:124-143) */
    double *u, *un, *qe, *qs, *ust, *wxl, *wxr, *wyl, *wyr, *hs[3];
    double *phx, *phy, *a2s, *ubx, *uby; /* Arrays with ghosts (:145-163) */
    double *vsc, *esc;
    /* pressure unknowns (interior) */
    double *P, *Pst;
    /* stage data (:591-608) */
    double *ustc, *vstc, *ubsx, *kpx, *wlx, *pvx, *ubsy, *kpy, *wly, *pvy, *kw, *qph, *cz, *pold;
    double *dxl, *dxr, *dyl, *dyr;
    double rx, ry, tau;
    /* Newton / BiCGStab work */
    double *Gv, *Gn, *lo, *di, *up, *sc, *cp, *dpv, *dP, *rhs, *Pn;
    int *acol; double *aval; int *an; /* rows of up to 5 entries (:734) */
    double *bdinv, *br, *br0, *bp, *bv, *bs, *bt, *bph, *bsh, *bax;
} Orc;

static Orc O; /* one case at a time */
/* stage-mode capture of the stage data (faces, residual scale, shock budget) right after the prep */
static double* g_prep_capture = NULL;
static size_t g_prep_len = 0;
static const double* g_qph_inject = NULL; /* stage mode: Q_1, Q_2 (2 blocks of nx*ny) replacing the shock budget */

static inline size_t cid(int i, int j) { return (size_t)i + (size_t)j * O.NXT; }
static inline double* cell(double* g, int i, int j) { return g + NV * cid(i, j); }

/* ------------------------------------------------------------------ EOS, src/spb6_physics_omp.h:71-111 */
static double eps_amp(int k, double a, double m, double p) {
    const Phase* P = &O.ph[k];
    return (p + P->g * P->pi) * (a - m * P->b) / (P->g - 1.0) + m * P->q;
}
static double p_ame(int k, double a, double m, double e) {
    const Phase* P = &O.ph[k];
    return (e - m * P->q) * (P->g - 1.0) / (a - m * P->b) - P->g * P->pi;
}
static double T_amp(int k, double a, double m, double p) {
    const Phase* P = &O.ph[k];
    return (a / m - P->b) * (p + P->pi) / ((P->g - 1.0) * P->cv);
}
static double c2_rp(int k, double r, double p) {
    const Phase* P = &O.ph[k];
    return P->g * (p + P->pi) / (r * (1.0 - r * P->b));
}
static double dedp_am(int k, double a, double m) {
    const Phase* P = &O.ph[k];
    return (a - m * P->b) / (P->g - 1.0);
}
static double p_mix(double a1, double m1, double m2, double rhoe) {
    const double a[2] = {a1, 1.0 - a1}, m[2] = {m1, m2};
    double num = rhoe, den = 0.0;
    for (int k = 0; k < 2; k++) {
        num -= m[k] * O.ph[k].q + O.ph[k].g * O.ph[k].pi * dedp_am(k, a[k], m[k]);
        den += dedp_am(k, a[k], m[k]);
    }
    return num / den;
}
static int p_admissible(int k, double p) { return p + O.ph[k].pi > 0; }
static double eps_round(int k, double m) { return fabs(m * O.ph[k].q); }

/* ------------------------------------------------------------------ closure, :229-243, :430-548, :842-866 */
typedef struct {
    double atr[2], mtr[2], etr[2], s, rhoeC, tau, pguess, Qph[2];
} ClIn;
typedef struct { double a[2], m[2], e[2], p[2], T[2], pbar; } ClOut;
typedef struct { double A[2], B[2], N[2], lam[2]; } PCoef;

static double E_above(const ClIn* in, int k) { /* :430-433 */
    const double v = in->etr[k] - in->mtr[k] * O.ph[k].q - (in->atr[k] - in->mtr[k] * O.ph[k].b) * O.ph[k].pi;
    return SMAX(0.0, v);
}
static void defect_split(const ClIn* in, double delta, double lam[2], double extra[2]) { /* :438-449 */
    if (O.share_mode == 2) {
        const double sm = in->mtr[0] + in->mtr[1];
        for (int k = 0; k < 2; k++) { lam[k] = sm > 0 ? in->mtr[k] / sm : 0.5; extra[k] = 0.0; }
        return;
    }
    double E[2], sE = 0.0;
    for (int k = 0; k < 2; k++) { E[k] = E_above(in, k); sE += E[k]; }
    double lE[2];
    if (sE > 0) for (int k = 0; k < 2; k++) lE[k] = E[k] / sE;
    else { const double sm = in->mtr[0] + in->mtr[1]; for (int k = 0; k < 2; k++) lE[k] = sm > 0 ? in->mtr[k] / sm : 0.5; }
    const double Q = O.share_mode == 1 ? 0.0 : in->Qph[0] + in->Qph[1];
    extra[0] = extra[1] = 0.0;
    if (!(delta > 0.0) || !(Q > 0.0)) { lam[0] = lE[0]; lam[1] = lE[1]; return; }
    if (delta < Q) { lam[0] = in->Qph[0] / Q; lam[1] = in->Qph[1] / Q; return; }
    for (int k = 0; k < 2; k++) { lam[k] = lE[k]; extra[k] = in->Qph[k] - Q * lE[k]; }
}
static int p_coef(const ClIn* in, PCoef* c, double pseg) { /* :453-464 */
    if (!(in->mtr[0] + in->mtr[1] > 0)) return 0;
    const double D0 = in->rhoeC - in->etr[0] - in->etr[1];
    double ex[2] = {0.0, 0.0};
    defect_split(in, D0 + (pseg > -1e299 ? pseg : in->pguess) * in->s, c->lam, ex);
    for (int k = 0; k < 2; k++) {
        c->A[k] = in->etr[k] - in->mtr[k] * O.ph[k].q + c->lam[k] * D0 + ex[k];
        c->B[k] = in->atr[k] + c->lam[k] * in->s;
        c->N[k] = c->A[k] - (c->B[k] - in->mtr[k] * O.ph[k].b) * O.ph[k].pi;
    }
    return 1;
}
static double alpha_p(const PCoef* c, const ClIn* in, int k, double p) { /* :465 */
    const Phase* P = &O.ph[k];
    return ((P->g - 1.0) * (c->A[k] + c->B[k] * p) + (p + P->g * P->pi) * in->mtr[k] * P->b) / (P->g * (p + P->pi));
}
static double dalpha_p(const PCoef* c, int k, double p) { /* :466 */
    const Phase* P = &O.ph[k];
    return -(P->g - 1.0) * c->N[k] / (P->g * (p + P->pi) * (p + P->pi));
}

/* Piecewise lambda selection shared by Phi and the final coefficients (:491-511). */
typedef struct { double D0, lE[2], A0[2], Qb; int byMass; } ClPre;
static void seg_lambda(const ClIn* in, const ClPre* pr, double p, double lam[2], double ex[2]) {
    ex[0] = ex[1] = 0.0;
    if (pr->byMass) { lam[0] = pr->lE[0]; lam[1] = pr->lE[1]; return; }
    const double delta = pr->D0 + p * in->s;
    if (!(delta > 0.0) || !(pr->Qb > 0.0)) { lam[0] = pr->lE[0]; lam[1] = pr->lE[1]; }
    else if (delta < pr->Qb) { lam[0] = in->Qph[0] / pr->Qb; lam[1] = in->Qph[1] / pr->Qb; }
    else for (int k = 0; k < 2; k++) { lam[k] = pr->lE[k]; ex[k] = in->Qph[k] - pr->Qb * pr->lE[k]; }
}
static double PhiD(const ClIn* in, const ClPre* pr, double p, double* df) { /* :502-519 */
    double lam[2], ex[2];
    seg_lambda(in, pr, p, lam, ex);
    double f = 0.0;
    *df = 0.0;
    for (int k = 0; k < 2; k++) {
        const Phase* P = &O.ph[k];
        const double A = pr->A0[k] + lam[k] * pr->D0 + ex[k], B = in->atr[k] + lam[k] * in->s,
                     N = A - (B - in->mtr[k] * P->b) * P->pi;
        f += ((P->g - 1.0) * (A + B * p) + (p + P->g * P->pi) * in->mtr[k] * P->b) / (P->g * (p + P->pi));
        *df += -(P->g - 1.0) * N / (P->g * (p + P->pi) * (p + P->pi));
    }
    return f - 1.0;
}
static int closure_p(const ClIn* in, ClOut* o) { /* :472-548 (SG/NASG branch) */
    if (!(in->mtr[0] + in->mtr[1] > 0)) return 0;
    const double plo = SMAX(-O.ph[0].pi, -O.ph[1].pi); /* plo_mix :468 */
    ClPre pr;
    pr.D0 = in->rhoeC - in->etr[0] - in->etr[1];
    const double sm = in->mtr[0] + in->mtr[1];
    pr.byMass = O.share_mode == 2;
    {
        double E[2], sE = 0.0;
        for (int k = 0; k < 2; k++) { E[k] = E_above(in, k); sE += E[k]; }
        if (pr.byMass) for (int k = 0; k < 2; k++) pr.lE[k] = sm > 0 ? in->mtr[k] / sm : 0.5;
        else if (sE > 0) for (int k = 0; k < 2; k++) pr.lE[k] = E[k] / sE;
        else for (int k = 0; k < 2; k++) pr.lE[k] = sm > 0 ? in->mtr[k] / sm : 0.5;
    }
    pr.Qb = (pr.byMass || O.share_mode == 1) ? 0.0 : in->Qph[0] + in->Qph[1];
    for (int k = 0; k < 2; k++) pr.A0[k] = in->etr[k] - in->mtr[k] * O.ph[k].q;
    double p = plo + SMAX(in->pguess - plo, 1e-3 * (fabs(plo) + 1.0));
    double lo = plo, hi = INFINITY;
    int conv = 0;
    for (int it = 0; it < 400; it++) {
        double df;
        const double f = PhiD(in, &pr, p, &df);
        if (f == 0.0) { conv = 1; break; }
        if (f > 0) lo = p; else hi = p;
        double pn = df < 0 ? p - f / df : NAN;
        if (fabs(pn - p) <= 2e-16 * (fabs(p) + fabs(plo))) { p = pn; conv = 1; break; }
        if (!(pn > lo && pn < hi)) {
            if (!isfinite(hi)) pn = plo + 4.0 * (p - plo);
            else if (lo == plo) pn = plo + 0.25 * (hi - plo);
            else pn = (hi - plo > 1e3 * (lo - plo + 1e-300) && lo > plo) ? plo + sqrt((lo - plo) * (hi - plo)) : 0.5 * (lo + hi);
        }
        if (fabs(pn - p) <= 2e-16 * (fabs(p) + fabs(plo)) || (hi < INFINITY && hi - lo <= 4e-16 * (fabs(hi) + fabs(lo)))) { p = pn; conv = 1; break; }
        p = pn;
    }
    if (!conv) return 0;
    PCoef c;
    {
        double ex[2];
        seg_lambda(in, &pr, p, c.lam, ex);
        for (int k = 0; k < 2; k++) {
            c.A[k] = pr.A0[k] + c.lam[k] * pr.D0 + ex[k];
            c.B[k] = in->atr[k] + c.lam[k] * in->s;
            c.N[k] = c.A[k] - (c.B[k] - in->mtr[k] * O.ph[k].b) * O.ph[k].pi;
        }
    }
    for (int k = 0; k < 2; k++) {
        o->a[k] = alpha_p(&c, in, k, p);
        o->m[k] = in->mtr[k];
        if (!(o->a[k] > o->m[k] * O.ph[k].b) || !(p + O.ph[k].pi > 0)) return 0;
        o->e[k] = eps_amp(k, o->a[k], o->m[k], p);
        o->p[k] = p;
        o->T[k] = T_amp(k, o->a[k], o->m[k], p);
    }
    o->pbar = p;
    return isfinite(p);
}
static int closure(const ClIn* in, ClOut* o) { /* :842-866, type CL_P */
    for (int k = 0; k < 2; k++)
        if (!(in->atr[k] > 0) || !(in->mtr[k] > 0) || !isfinite(in->etr[k])) return 0;
    if (!isfinite(in->rhoeC) || !isfinite(in->s)) return 0;
    const int ok = closure_p(in, o);
    return ok && isfinite(o->pbar);
}
static double closure_roundoff(const ClIn* in, double p) { /* SPB6_PC_IMEX_omp.cpp:657-664 */
    PCoef c;
    if (!p_coef(in, &c, p)) return 0.0;
    double dphi = 0.0, sens = 0.0;
    for (int k = 0; k < 2; k++) {
        dphi += dalpha_p(&c, k, p);
        sens += fabs(c.lam[k]) * (O.ph[k].g - 1.0) / (O.ph[k].g * (p + O.ph[k].pi));
    }
    const double en = 2.220446049250313e-16 * (fabs(in->rhoeC) + fabs(in->etr[0]) + fabs(in->etr[1]) +
                                              fabs(in->mtr[0] * O.ph[0].q) + fabs(in->mtr[1] * O.ph[1].q));
    return dphi < 0 ? en * sens / -dphi : 0.0;
}

/* ------------------------------------------------------------------ shock budget, :267-428 */
static void eos_ep_ev(int k, double p, double v, double* ep, double* evp) {
    const Phase* P = &O.ph[k];
    *ep = (v - P->b) / (P->g - 1.0);
    *evp = P->g * (p + P->pi) / (P->g - 1.0);
}
static int eos_ok(int k, double p, double v) {
    if (!(v > 0) || !isfinite(p)) return 0;
    return v > O.ph[k].b && p + O.ph[k].pi > 0;
}
static double hug_v(int k, double p0, double p1, double v0) { /* NASG closed form, :279-284 */
    const Phase* P = &O.ph[k];
    const double x0 = p0 + P->pi, x1 = p1 + P->pi;
    return P->b + (v0 - P->b) * ((P->g - 1.0) * x1 + (P->g + 1.0) * x0) / ((P->g + 1.0) * x1 + (P->g - 1.0) * x0);
}
static void K_G(int k, double p, double v, double* K, double* Gm) { /* :296-301 */
    *K = c2_rp(k, 1.0 / v, p) / v;
    *Gm = 0.5 * (O.ph[k].g + 1.0);
    if (O.ph[k].b != 0.0) *Gm *= v / (v - O.ph[k].b);
}
typedef struct { double Y[2], vk0[2], v0, p0, j2, vend; } ShockProf;
static int prof_rhs(const ShockProf* S, double c, double v, const double* y, double* dy) { /* :304-312 */
    const double p = y[0], v1 = y[1], v2 = (v - S->Y[0] * v1) / S->Y[1], Pr = S->p0 + S->j2 * (S->v0 - v);
    if (!eos_ok(0, p, v1) || !eos_ok(1, p, v2)) return 0;
    const double lam[2] = {c, 1.0 - c}, vk[2] = {v1, v2};
    double num = -1.0, den = 0.0, r[2], ep[2], evp[2];
    for (int k = 0; k < 2; k++) {
        eos_ep_ev(k, p, vk[k], &ep[k], &evp[k]);
        r[k] = lam[k] / S->Y[k] * (p - Pr);
        num += S->Y[k] * r[k] / evp[k];
        den += S->Y[k] * ep[k] / evp[k];
    }
    dy[0] = num / den;
    dy[1] = (r[0] - ep[0] * dy[0]) / evp[0];
    dy[2] = p - Pr;
    return isfinite(dy[0]) && isfinite(dy[1]);
}
/* Adaptive Cash-Karp RK45 (the published Cash & Karp 1990 embedded pair), :313-343 */
static int prof_integrate(const ShockProf* S, double c, double* v1end, double* qend) {
    static const double A[6] = {0, 0.2, 0.3, 0.6, 1.0, 0.875};
    static const double B[6][5] = {{0}, {0.2}, {3.0 / 40, 9.0 / 40}, {0.3, -0.9, 1.2}, {-11.0 / 54, 2.5, -70.0 / 27, 35.0 / 27},
                                   {1631.0 / 55296, 175.0 / 512, 575.0 / 13824, 44275.0 / 110592, 253.0 / 4096}};
    static const double C5[6] = {37.0 / 378, 0, 250.0 / 621, 125.0 / 594, 0, 512.0 / 1771};
    static const double C4[6] = {2825.0 / 27648, 0, 18575.0 / 48384, 13525.0 / 55296, 277.0 / 14336, 0.25};
    double y[3] = {S->p0, S->vk0[0], 0.0}, v = S->v0;
    const double L = S->vend - S->v0, sc[3] = {fabs(S->p0) + S->j2 * fabs(L), S->vk0[0], S->j2 * L * L + 1e-300};
    double h = L / 32.0;
    for (int it = 0; it < 4000; it++) {
        const int last = (L < 0 && v + h <= S->vend) || (L > 0 && v + h >= S->vend);
        if (last) h = S->vend - v;
        double k[6][3], yt[3];
        int ok = 1;
        for (int st = 0; st < 6 && ok; st++) {
            for (int n = 0; n < 3; n++) { yt[n] = y[n]; for (int q = 0; q < st; q++) yt[n] += h * B[st][q] * k[q][n]; }
            ok = prof_rhs(S, c, v + A[st] * h, yt, k[st]);
        }
        double err = 0.0, y5[3];
        if (ok)
            for (int n = 0; n < 3; n++) {
                double d5 = 0, d4 = 0;
                for (int st = 0; st < 6; st++) { d5 += C5[st] * k[st][n]; d4 += C4[st] * k[st][n]; }
                y5[n] = y[n] + h * d5;
                err = SMAX(err, fabs(h * (d5 - d4)) / sc[n]);
            }
        if (!ok || !(err <= 1e-8)) {
            h *= ok ? SMAX(0.1, 0.9 * sh_pow(1e-8 / err, 0.25)) : 0.25;
            if (fabs(h) < 1e-14 * fabs(L)) return 0;
            continue;
        }
        for (int n = 0; n < 3; n++) y[n] = y5[n];
        if (last) { *v1end = y[1]; *qend = y[2]; return 1; }
        v += h;
        h *= SMIN(5.0, 0.9 * sh_pow(1e-8 / SMAX(err, 1e-30), 0.2));
    }
    return 0;
}
static double shoot_F(const ShockProf* S, const double vH[2], const double vpre[2], double t, double* qq) {
    const double c = 1.0 / (1.0 + sh_exp(-t));
    double v1e;
    if (!prof_integrate(S, c, &v1e, qq)) return NAN;
    return (v1e - vH[0]) / vpre[0];
}
static int shock_share(const double Y[2], const double vpre[2], double p0, double p1, double lam[2], double* q) { /* :345-393 */
    double K[2], Gm[2], w[2], sw = 0.0, Kmin = INFINITY;
    for (int k = 0; k < 2; k++) {
        K_G(k, p0, vpre[k], &K[k], &Gm[k]);
        if (!(K[k] > 0)) return 0;
        Kmin = SMIN(Kmin, K[k]);
    }
    const double dp = p1 - p0;
    if (dp < 1e-2 * Kmin) {
        *q = 0.0;
        for (int k = 0; k < 2; k++) { w[k] = Y[k] * vpre[k] * Gm[k] / (K[k] * K[k]); sw += w[k]; }
        for (int k = 0; k < 2; k++) lam[k] = w[k] / sw;
        *q = sw * dp * dp * dp / 6.0;
        return 1;
    }
    ShockProf S;
    S.p0 = p0;
    double vH[2];
    for (int k = 0; k < 2; k++) {
        S.Y[k] = Y[k]; S.vk0[k] = vpre[k];
        vH[k] = hug_v(k, p0, p1, vpre[k]);
        if (!isfinite(vH[k])) return 0;
    }
    S.v0 = Y[0] * vpre[0] + Y[1] * vpre[1];
    S.vend = Y[0] * vH[0] + Y[1] * vH[1];
    if (!(S.vend < S.v0)) return 0;
    S.j2 = dp / (S.v0 - S.vend);
    double t0;
    {
        double ww[2];
        for (int k = 0; k < 2; k++) ww[k] = Y[k] * vpre[k] * Gm[k] / (K[k] * K[k]);
        const double c0 = SMIN(1.0 - 1e-12, SMAX(1e-12, ww[0] / (ww[0] + ww[1])));
        t0 = isfinite(c0) ? sh_log(c0 / (1.0 - c0)) : 0.0;
    }
    double ta = SMAX(-40.0, t0 - 1.0), tb = SMIN(40.0, t0 + 1.0), qa = 0, qb = 0;
    double fa = shoot_F(&S, vH, vpre, ta, &qa), fb = shoot_F(&S, vH, vpre, tb, &qb);
    if (!isfinite(fa) || !isfinite(fb)) return 0;
    for (double st = 2.0; fa >= 0 && ta > -40.0; st *= 2.0) {
        tb = ta; fb = fa; qb = qa;
        ta = SMAX(-40.0, ta - st);
        fa = shoot_F(&S, vH, vpre, ta, &qa);
        if (!isfinite(fa)) return 0;
    }
    for (double st = 2.0; fb <= 0 && tb < 40.0; st *= 2.0) {
        ta = tb; fa = fb; qa = qb;
        tb = SMIN(40.0, tb + st);
        fb = shoot_F(&S, vH, vpre, tb, &qb);
        if (!isfinite(fb)) return 0;
    }
    double t, qt;
    if (fa >= 0) { t = ta; qt = qa; }
    else if (fb <= 0) { t = tb; qt = qb; }
    else {
        int side = 0;
        t = ta; qt = qa;
        for (int it = 0; it < 100; it++) { /* Illinois false position */
            t = (ta * fb - tb * fa) / (fb - fa);
            if (!(t > ta && t < tb)) t = 0.5 * (ta + tb);
            const double ft = shoot_F(&S, vH, vpre, t, &qt);
            if (!isfinite(ft)) return 0;
            if (fabs(ft) < 1e-10 || tb - ta < 1e-10) break;
            if (ft < 0) { ta = t; fa = ft; if (side == -1) fb *= 0.5; side = -1; }
            else { tb = t; fb = ft; if (side == 1) fa *= 0.5; side = 1; }
        }
    }
    const double c = 1.0 / (1.0 + sh_exp(-t));
    lam[0] = c; lam[1] = 1.0 - c;
    *q = qt;
    return *q > 0;
}
static void stencil_state(const double* c, double* st) { /* :395-400 */
    const double a1 = c[IA1], m1 = c[IM1], m2 = c[IM2], r = m1 + m2;
    st[0] = a1; st[1] = 1.0 - a1; st[2] = m1; st[3] = m2; st[4] = NAN;
    st[5] = r > 0 ? c[IMU] / r : 0.0;
    st[6] = r > 0 ? c[IMV] / r : 0.0;
    if (a1 > 0 && a1 < 1 && m1 > 0 && m2 > 0) {
        const double p = p_mix(a1, m1, m2, c[IE1] + c[IE2]);
        if (p_admissible(0, p) && p_admissible(1, p)) st[4] = p;
    }
}
static void shock_budget(const double* X, int i, int j, int twoD, double Q[2]) { /* :405-428 */
    Q[0] = Q[1] = 0.0;
    double c0[7], st[7], lo[7] = {0, 0, 0, 0, 0, 0, 0}, plo = 1e300, phi = -1e300, div = 0.0;
    stencil_state(cell((double*)X, i, j), c0);
    for (int d = 0; d < (twoD ? 2 : 1); d++)
        for (int q = -1; q <= 1; q++) {
            if (d == 1 && q == 0) continue;
            stencil_state(cell((double*)X, i + (d == 0 ? q : 0), j + (d == 1 ? q : 0)), st);
            if (q == 1) div += st[5 + d];
            else if (q == -1) div -= st[5 + d];
            if (!isfinite(st[4])) continue;
            if (st[4] < plo) { plo = st[4]; for (int n = 0; n < 7; n++) lo[n] = st[n]; }
            if (st[4] > phi) phi = st[4];
        }
    if (!(div < 0.0) || !(phi > plo)) return;
    double Y[2], vpre[2], lam[2], q;
    const double rho = c0[2] + c0[3];
    if (!(rho > 0)) return;
    for (int k = 0; k < 2; k++) {
        Y[k] = c0[2 + k] / rho;
        vpre[k] = (lo[k] > 0 && lo[2 + k] > 0) ? lo[k] / lo[2 + k] : (c0[2 + k] > 0 ? c0[k] / c0[2 + k] : 0.0);
    }
    if (!(Y[0] > 0) || !(Y[1] > 0) || !(vpre[0] > 0) || !(vpre[1] > 0)) return;
    if (!shock_share(Y, vpre, plo, phi, lam, &q)) return;
    for (int k = 0; k < 2; k++) Q[k] = lam[k] * rho * q;
}

/* ------------------------------------------------------------------ primitives, :893-913 */
typedef struct { double a1, r1, r2, u, v, p1, p2, p, rho, cf; } Prim;
static int prim_of(const double* Q, Prim* w) {
    const double a1 = Q[IA1], a2 = 1 - a1, m1 = Q[IM1], m2 = Q[IM2];
    if (!(a1 > 0 && a2 > 0 && m1 > 0 && m2 > 0)) return 0;
    w->a1 = a1; w->rho = m1 + m2; w->r1 = m1 / a1; w->r2 = m2 / a2; w->u = Q[IMU] / w->rho; w->v = Q[IMV] / w->rho;
    w->p = p_mix(a1, m1, m2, Q[IEN] - 0.5 * w->rho * (w->u * w->u + w->v * w->v));
    w->p1 = p_ame(0, a1, m1, Q[IE1]);
    w->p2 = p_ame(1, a2, m2, Q[IE2]);
    if (!(p_admissible(0, w->p1) && p_admissible(1, w->p2))) return 0;
    w->cf = sqrt((m1 * c2_rp(0, w->r1, w->p1) + m2 * c2_rp(1, w->r2, w->p2)) / w->rho);
    return 1;
}
static double pbar_of(const double* Q) {
    const double a1 = Q[IA1];
    return a1 * p_ame(0, a1, Q[IM1], Q[IE1]) + (1 - a1) * p_ame(1, 1 - a1, Q[IM2], Q[IE2]);
}

/* ------------------------------------------------------------------ boundaries, physics :982-1013; driver :516-537 */
static void ghost_fill(double* u, int i, int j, int si, int sj, int side) {
    double* d = cell(u, i, j);
    const double* s = cell(u, si, sj);
    for (int k = 0; k < NV; k++) d[k] = s[k];
    if (O.bcs[side] == SPB6_BC_PRES) {
        const double a1 = d[IA1], e1 = eps_amp(0, a1, d[IM1], O.bcp[side]), e2 = eps_amp(1, 1 - a1, d[IM2], O.bcp[side]);
        d[IEN] += (e1 + e2) - (d[IE1] + d[IE2]);
        d[IE1] = e1; d[IE2] = e2;
        return;
    }
    if (O.bcs[side] != SPB6_BC_WALL) return;
    const int kn = side < 2 ? IMU : IMV;
    const double rho = d[IM1] + d[IM2];
    if (O.bcu[side] == 0.0) { d[kn] = -d[kn]; return; }
    const double mn = 2.0 * rho * O.bcu[side] - s[kn];
    d[IEN] += 0.5 * (mn * mn - s[kn] * s[kn]) / rho;
    d[kn] = mn;
}
static void bc_apply(double* u) {
    const int nx = O.nx, ny = O.ny;
    for (int j = 0; j < ny + 2 * G; j++)
        for (int q = 0; q < G; q++) {
            const int iL = G - 1 - q, iR = nx + G + q;
            const int sL = O.bcs[0] == SPB6_BC_PERIODIC ? nx + G - 1 - q : (O.bcs[0] == SPB6_BC_WALL ? G + q : G);
            const int sR = O.bcs[1] == SPB6_BC_PERIODIC ? G + q : (O.bcs[1] == SPB6_BC_WALL ? nx + G - 1 - q : nx + G - 1);
            ghost_fill(u, iL, j, sL, j, 0);
            ghost_fill(u, iR, j, sR, j, 1);
        }
    if (ny > 1 || O.bcs[2] == SPB6_BC_PERIODIC) {
        for (int i = 0; i < nx + 2 * G; i++)
            for (int q = 0; q < G; q++) {
                const int jL = G - 1 - q, jR = ny + G + q;
                const int sL = O.bcs[2] == SPB6_BC_PERIODIC ? ny + G - 1 - q : (O.bcs[2] == SPB6_BC_WALL ? G + q : G);
                const int sR = O.bcs[3] == SPB6_BC_PERIODIC ? G + q : (O.bcs[3] == SPB6_BC_WALL ? ny + G - 1 - q : ny + G - 1);
                ghost_fill(u, i, jL, i, sL, 2);
                ghost_fill(u, i, jR, i, sR, 3);
            }
    } else {
        for (int i = 0; i < nx + 2 * G; i++)
            for (int q = 0; q < G; q++)
                for (int k = 0; k < NV; k++) {
                    cell(u, i, G - 1 - q)[k] = cell(u, i, G)[k];
                    cell(u, i, G + 1 + q)[k] = cell(u, i, G)[k];
                }
    }
}
static void bc_src(int side, int q, int n, double sg, int* sL, double* fs) {
    *fs = 1.0;
    if (O.bcs[side] == SPB6_BC_PERIODIC) *sL = (side % 2 == 0) ? n + G - 1 - q : G + q;
    else if (O.bcs[side] == SPB6_BC_WALL) { *sL = (side % 2 == 0) ? G + q : n + G - 1 - q; *fs = sg; }
    else *sL = (side % 2 == 0) ? G : n + G - 1;
}
static void bound_cond_array(double* a, double sign_x, double sign_y) {
    const int nx = O.nx, ny = O.ny;
    for (int j = 0; j < ny + 2 * G; j++)
        for (int q = 0; q < G; q++) {
            int sL, sR; double fL, fR;
            bc_src(0, q, nx, sign_x, &sL, &fL);
            bc_src(1, q, nx, sign_x, &sR, &fR);
            a[cid(G - 1 - q, j)] = fL * a[cid(sL, j)];
            a[cid(nx + G + q, j)] = fR * a[cid(sR, j)];
        }
    for (int i = 0; i < nx + 2 * G; i++)
        for (int q = 0; q < G; q++) {
            int sL, sR; double fL, fR;
            if (ny == 1 && O.bcs[2] != SPB6_BC_PERIODIC) { sL = G; sR = G; fL = fR = 1.0; }
            else { bc_src(2, q, ny, sign_y, &sL, &fL); bc_src(3, q, ny, sign_y, &sR, &fR); }
            a[cid(i, G - 1 - q)] = fL * a[cid(i, sL)];
            a[cid(i, ny + G + q)] = fR * a[cid(i, sR)];
        }
}

/* ------------------------------------------------------------------ reconstruction, :369-471 */
static void tvd_reconstruction(const double* u) {
    const int NXT = O.NXT, NYT = O.NYT;
    const size_t ncell = (size_t)NXT * NYT;
    memcpy(O.wxl, u, ncell * NV * sizeof(double));
    memcpy(O.wxr, u, ncell * NV * sizeof(double));
    memcpy(O.wyl, u, ncell * NV * sizeof(double));
    memcpy(O.wyr, u, ncell * NV * sizeof(double));
    memset(O.phx, 0, ncell * sizeof(double));
    memset(O.phy, 0, ncell * sizeof(double));
    for (size_t c = 0; c < ncell; c++) O.vsc[c] = O.esc[c] = 0.0;
    const int j0 = O.ny == 1 ? G : 0, j1 = O.ny == 1 ? G + 1 : NYT;
    for (int j = j0; j < j1; j++)
        for (int i = 0; i < NXT; i++) {
            const double* q = cell((double*)u, i, j);
            Prim w;
            const double rho = q[IM1] + q[IM2], mm = hypot(q[IMU], q[IMV]);
            const size_t c = cid(i, j);
            O.vsc[c] = (rho > 0 ? mm / rho : 0.0) + (prim_of(q, &w) ? w.cf : 0.0);
            O.esc[c] = fabs(q[IE1]) + fabs(q[IE2]) + (rho > 0 ? 0.5 * mm * mm / rho : 0.0);
        }
    static const int VOL[5] = {IA1, IM1, IM2, IE1, IE2};
    for (int dir = 0; dir < (O.ny > 1 ? 2 : 1); dir++) {
        double *wL = dir == 0 ? O.wxl : O.wyl, *wR = dir == 0 ? O.wxr : O.wyr;
        double* phis = dir == 0 ? O.phx : O.phy;
        for (int j = j0; j < j1; j++)
            for (int i = 0; i < NXT; i++) {
                int ia = i, ja = j, ib = i, jb = j;
                if (dir == 0) { ia = i - 1; ib = i + 1; if (ia < 0 || ib >= NXT) continue; }
                else { ja = j - 1; jb = j + 1; if (ja < 0 || jb >= NYT) continue; }
                const size_t ca = cid(ia, ja), cc = cid(i, j), cb = cid(ib, jb);
                const double *Ua = u + NV * ca, *Uc = u + NV * cc, *Ub = u + NV * cb;
                double phi = 1.0;
                for (int q = 0; q < 5; q++) {
                    const int k = VOL[q];
                    const double xa = Ua[k], xc = Uc[k], xb = Ub[k];
                    double sc;
                    if (k == IA1) sc = 3.0;
                    else if (k == IM1 || k == IM2) sc = fabs(xa) + fabs(xc) + fabs(xb);
                    else sc = O.esc[ca] + O.esc[cc] + O.esc[cb];
                    const double a = xc - xa, b = xb - xc, tiny = 1e-12 * sc + 1e-300;
                    if (!O.limiter) break;
                    if (fabs(a) <= tiny && fabs(b) <= tiny) continue;
                    if (a * b <= 0) { phi = 0.0; break; }
                    const double c = 0.5 * (a + b), m = fabs(a) < fabs(b) ? a : b;
                    phi = SMIN(phi, m / c);
                }
                if (O.limiter && phi > 0.0) { /* face-state admissibility cap, :416-432 */
                    const double* cs[3] = {Ua, Uc, Ub};
                    for (int ph = 0; ph < 2; ph++) {
                        double L1[3], L2[3];
                        for (int n = 0; n < 3; n++) {
                            const double a = ph == 0 ? cs[n][IA1] : 1.0 - cs[n][IA1], m = cs[n][ph == 0 ? IM1 : IM2],
                                         e = cs[n][ph == 0 ? IE1 : IE2];
                            L1[n] = a - m * O.ph[ph].b;
                            L2[n] = e - m * O.ph[ph].q - L1[n] * O.ph[ph].pi;
                        }
                        const double* Ls[2] = {L1, L2};
                        for (int l = 0; l < 2; l++) {
                            const double dL = fabs(Ls[l][2] - Ls[l][0]);
                            if (Ls[l][1] > 0.0 && dL > 0.0) phi = SMIN(phi, 2.0 * Ls[l][1] / dL);
                        }
                    }
                }
                double *WL = wL + NV * cc, *WR = wR + NV * cc;
                for (int q = 0; q < 5; q++) {
                    const int k = VOL[q];
                    const double sig = phi * 0.5 * (Ub[k] - Ua[k]);
                    WL[k] = Uc[k] - 0.5 * sig;
                    WR[k] = Uc[k] + 0.5 * sig;
                }
                const double ra = Ua[IM1] + Ua[IM2], rc = Uc[IM1] + Uc[IM2], rb = Ub[IM1] + Ub[IM2];
                const double tiny = 1e-12 * (O.vsc[ca] + O.vsc[cc] + O.vsc[cb]) + 1e-300;
                double vL[2], vR[2], sm = 1.0;
                for (int d = 0; d < 2; d++) {
                    const int k = d == 0 ? IMU : IMV;
                    const double va = Ua[k] / ra, vc = Uc[k] / rc, vb = Ub[k] / rb, a = vc - va, b = vb - vc;
                    double sl = 0.0;
                    if (!O.limiter) sl = 0.5 * (a + b);
                    else if (!(fabs(a) <= tiny && fabs(b) <= tiny)) {
                        if (a * b > 0) { sl = fabs(a) < fabs(b) ? a : b; sm = SMIN(sm, sl / (0.5 * (a + b))); }
                        else sm = 0.0;
                    }
                    vL[d] = vc - 0.5 * sl;
                    vR[d] = vc + 0.5 * sl;
                }
                const double rL = WL[IM1] + WL[IM2], rR = WR[IM1] + WR[IM2];
                WL[IMU] = rL * vL[0]; WL[IMV] = rL * vL[1];
                WL[IEN] = WL[IE1] + WL[IE2] + 0.5 * rL * (vL[0] * vL[0] + vL[1] * vL[1]);
                WR[IMU] = rR * vR[0]; WR[IMV] = rR * vR[1];
                WR[IEN] = WR[IE1] + WR[IE2] + 0.5 * rR * (vR[0] * vR[0] + vR[1] * vR[1]);
                phis[cc] = SMIN(phi, sm);
            }
    }
}

/* ------------------------------------------------------------------ explicit update, :210-346 */
static void rusanov(double* flux, const double* QL, const double* QR, int d, double amax) {
    const int km = d == 0 ? IMU : IMV;
    const double vL = QL[km] / (QL[IM1] + QL[IM2]), vR = QR[km] / (QR[IM1] + QR[IM2]);
    const double a = O.rus_local ? SMAX(fabs(QL[km] / (QL[IM1] + QL[IM2])), fabs(QR[km] / (QR[IM1] + QR[IM2]))) : amax;
    for (int k = 0; k < NV; k++) flux[k] = 0.5 * (QL[k] * vL + QR[k] * vR) - 0.5 * a * (QR[k] - QL[k]);
}
static int update(double* uc, const double* Qe, const double* Qs) {
    const int nx = O.nx, ny = O.ny, NXT = O.NXT;
    double vxm = 0, vym = 0;
    int rok = 1;
    for (int j = 0; j < ny + 2 * G; j++)
        for (int i = 0; i < nx + 2 * G; i++) {
            const double* q = Qe + NV * cid(i, j);
            const double rho = q[IM1] + q[IM2];
            if (!(rho > 0)) { rok = 0; continue; }
            if (i >= G && i < nx + G && j >= G && j < ny + G) {
                vxm = SMAX(vxm, fabs(q[IMU] / rho));
                vym = SMAX(vym, fabs(q[IMV] / rho));
            }
        }
    if (!rok) return 0;
    for (int j = G; j < ny + G; j++)
        for (int i = G - 1; i < nx + G; i++) {
            const double *r = O.wxr + NV * cid(i, j), *l = O.wxl + NV * cid(i + 1, j);
            const double uL = r[IMU] / (r[IM1] + r[IM2]), uR = l[IMU] / (l[IM1] + l[IM2]);
            vxm = SMAX(vxm, SMAX(fabs(uL), fabs(uR)));
            O.ubx[cid(i, j)] = 0.5 * (uL + uR);
        }
    if (ny > 1)
        for (int j = G - 1; j < ny + G; j++)
            for (int i = G; i < nx + G; i++) {
                const double *r = O.wyr + NV * cid(i, j), *l = O.wyl + NV * cid(i, j + 1);
                const double vL = r[IMV] / (r[IM1] + r[IM2]), vR = l[IMV] / (l[IM1] + l[IM2]);
                vym = SMAX(vym, SMAX(fabs(vL), fabs(vR)));
                O.uby[cid(i, j)] = 0.5 * (vL + vR);
            }
    O.vx_max = vxm;
    O.vy_max = vym;
    for (int j = G; j < ny + G; j++)
        for (int i = G; i < nx + G; i++) {
            double fp[NV], fm[NV];
            double* out = uc + NV * cid(i, j);
            const double *qs = Qs + NV * cid(i, j), *qe = Qe + NV * cid(i, j);
            rusanov(fp, O.wxr + NV * cid(i, j), O.wxl + NV * cid(i + 1, j), 0, O.vx_max);
            rusanov(fm, O.wxr + NV * cid(i - 1, j), O.wxl + NV * cid(i, j), 0, O.vx_max);
            for (int k = 0; k < NV; k++) out[k] = qs[k] - O.adt / O.dx * (fp[k] - fm[k]);
            out[IA1] += O.adt / O.dx * qe[IA1] * (O.ubx[cid(i, j)] - O.ubx[cid(i - 1, j)]);
            if (ny > 1) {
                double gp[NV], gm[NV];
                rusanov(gp, O.wyr + NV * cid(i, j), O.wyl + NV * cid(i, j + 1), 1, O.vy_max);
                rusanov(gm, O.wyr + NV * cid(i, j - 1), O.wyl + NV * cid(i, j), 1, O.vy_max);
                for (int k = 0; k < NV; k++) out[k] -= O.adt / O.dy * (gp[k] - gm[k]);
                out[IA1] += O.adt / O.dy * qe[IA1] * (O.uby[cid(i, j)] - O.uby[cid(i, j - 1)]);
            }
            O.a2s[cid(i, j)] = 1.0 - out[IA1];
        }
    (void)NXT;
    bc_apply(uc);
    bound_cond_array(O.a2s, 1, 1);
    return 1;
}

/* ------------------------------------------------------------------ time step, :502-514 */
static double caldt(const double* u, int acoustic) {
    double ux = 0, uy = 0;
    for (int j = G; j < O.ny + G; j++)
        for (int i = G; i < O.nx + G; i++) {
            Prim w;
            if (!prim_of(u + NV * cid(i, j), &w)) continue;
            const double c = acoustic ? w.cf : 0.0;
            ux = SMAX(ux, fabs(w.u) + c);
            uy = SMAX(uy, fabs(w.v) + c);
        }
    const double rate = ux / O.dx + (O.ny > 1 ? uy / O.dy : 0.0);
    return rate > 0 ? 1.0 / rate : INFINITY;
}

/* ------------------------------------------------------------------ implicit part, :610-731 */
typedef struct { double uf, du, pf, wL, wR, utL, utR; const double *cL, *cR; } FaceVals;
static void face_weights(FaceVals* f, double ube) {
    f->wL = SMAX(f->uf, 0.0) - SMAX(ube, 0.0);
    f->wR = SMIN(f->uf, 0.0) - SMIN(ube, 0.0);
}
static int wall_x(int i) {
    if (i == G - 1 && O.bcs[0] == SPB6_BC_WALL) return 0;
    if (i == O.nx + G - 1 && O.bcs[1] == SPB6_BC_WALL) return 1;
    return -1;
}
static int wall_y(int j) {
    if (j == G - 1 && O.bcs[2] == SPB6_BC_WALL) return 2;
    if (j == O.ny + G - 1 && O.bcs[3] == SPB6_BC_WALL) return 3;
    return -1;
}
static void face_x(int i, int j, double PL, double PR, FaceVals* f) {
    const size_t c = cid(i, j);
    f->pf = O.wlx[c] * PL + (1.0 - O.wlx[c]) * PR - O.pvx[c];
    f->cL = O.dxl + 6 * c; f->cR = O.dxr + 6 * c;
    f->utL = O.vstc[c]; f->utR = O.vstc[cid(i + 1, j)];
    const int w = wall_x(i);
    if (w >= 0) {
        if (O.bcu[w] == 0.0) { f->uf = 0.0; f->du = 0.0; f->wL = f->wR = 0.0; return; }
        f->uf = O.bcu[w]; f->du = f->uf - O.ubx[c]; face_weights(f, O.ubx[c]); return;
    }
    f->uf = O.ubsx[c] - O.kpx[c] * (PR - PL);
    f->du = f->uf - O.ubx[c];
    face_weights(f, O.ubx[c]);
}
static void face_y(int i, int j, double PL, double PR, FaceVals* f) {
    const size_t c = cid(i, j);
    f->pf = O.wly[c] * PL + (1.0 - O.wly[c]) * PR - O.pvy[c];
    f->cL = O.dyl + 6 * c; f->cR = O.dyr + 6 * c;
    f->utL = O.ustc[c]; f->utR = O.ustc[cid(i, j + 1)];
    const int w = wall_y(j);
    if (w >= 0) {
        if (O.bcu[w] == 0.0) { f->uf = 0.0; f->du = 0.0; f->wL = f->wR = 0.0; return; }
        f->uf = O.bcu[w]; f->du = f->uf - O.uby[c]; face_weights(f, O.uby[c]); return;
    }
    f->uf = O.ubsy[c] - O.kpy[c] * (PR - PL);
    f->du = f->uf - O.uby[c];
    face_weights(f, O.uby[c]);
}
static double inc(const FaceVals* f, int k) { return f->cL[k] * f->wL + f->cR[k] * f->wR; }
typedef struct { double M, Mt, E; } FaceFlux;
static FaceFlux face_flux(const FaceVals* f) {
    const double ML = (f->cL[2] + f->cL[3]) * f->wL, MR = (f->cR[2] + f->cR[3]) * f->wR, M = ML + MR;
    FaceFlux F;
    F.M = M;
    F.Mt = f->utL * ML + f->utR * MR;
    F.E = inc(f, 4) + inc(f, 5) + 0.5 * f->uf * f->uf * M + 0.5 * (f->utL * f->utL * ML + f->utR * f->utR * MR) + (O.p_ref + f->pf) * f->uf;
    return F;
}
typedef struct { ClOut cl; double mx, my, E, s, sig; } CellOut;
static int cell_residual(int i, int j, double Pc, double PW, double PE, double PS, double PN, double* Gr, CellOut* out) { /* :666-704 */
    FaceVals fe, fw, fn, fs;
    face_x(i, j, Pc, PE, &fe);
    face_x(i - 1, j, PW, Pc, &fw);
    const int twoD = O.ny > 1;
    if (twoD) { face_y(i, j, Pc, PN, &fn); face_y(i, j - 1, PS, Pc, &fs); }
    const double* xs = O.ust + NV * cid(i, j); /* X* lives in the stage output grid */
    double X[6] = {xs[IA1], O.a2s[cid(i, j)], xs[IM1], xs[IM2], xs[IE1], xs[IE2]};
    for (int k = 2; k < 6; k++) {
        X[k] -= O.rx * (inc(&fe, k) - inc(&fw, k));
        if (twoD) X[k] -= O.ry * (inc(&fn, k) - inc(&fs, k));
    }
    X[1] = 1.0 - X[0];
    const double s = O.rx * (fe.uf - fw.uf) + (twoD ? O.ry * (fn.uf - fs.uf) : 0.0);
    X[0] *= 1.0 - s;
    X[1] *= 1.0 - s;
    const FaceFlux FEe = face_flux(&fe), FEw = face_flux(&fw);
    double mx = xs[IMU] - O.rx * (fe.pf - fw.pf) - O.rx * (fe.uf * FEe.M - fw.uf * FEw.M);
    double my = xs[IMV] - O.rx * (FEe.Mt - FEw.Mt);
    double E = xs[IEN] - O.rx * (FEe.E - FEw.E);
    if (twoD) {
        const FaceFlux FEn = face_flux(&fn), FEs = face_flux(&fs);
        my -= O.ry * (fn.pf - fs.pf) + O.ry * (fn.uf * FEn.M - fs.uf * FEs.M);
        mx -= O.ry * (FEn.Mt - FEs.Mt);
        E -= O.ry * (FEn.E - FEs.E);
    }
    const double rho = X[2] + X[3];
    if (!(rho > 0)) return 0;
    ClIn in;
    in.atr[0] = X[0]; in.atr[1] = X[1]; in.mtr[0] = X[2]; in.mtr[1] = X[3]; in.etr[0] = X[4]; in.etr[1] = X[5];
    in.s = s;
    in.rhoeC = E - 0.5 * (mx * mx + my * my) / rho;
    in.tau = O.tau;
    in.pguess = O.p_ref + Pc;
    in.Qph[0] = O.qph[cid(i, j) * 2];
    in.Qph[1] = O.qph[cid(i, j) * 2 + 1];
    ClOut o;
    if (!closure(&in, &o)) return 0;
    *Gr = (o.pbar - O.p_ref) - Pc;
    if (out) { out->cl = o; out->mx = mx; out->my = my; out->E = E; out->s = s; out->sig = closure_roundoff(&in, o.pbar); }
    return isfinite(*Gr);
}
static int M_P(int i, int j) { /* :709-718 */
    int I, J;
    const int xper = O.bcs[0] == SPB6_BC_PERIODIC, yper = O.bcs[2] == SPB6_BC_PERIODIC;
    if (i < G) I = xper ? O.nx + i : G;
    else if (i > O.nx + G - 1) I = xper ? i - O.nx : O.nx + G - 1;
    else I = i;
    if (j < G) J = (yper && O.ny > 1) ? O.ny + j : G;
    else if (j > O.ny + G - 1) J = (yper && O.ny > 1) ? j - O.ny : O.ny + G - 1;
    else J = j;
    return (I - G) + O.nx * (J - G);
}
static int residual_at(const double* P, int i, int j, double dc, int which, double dn, double* Gr, CellOut* out) { /* :720-731 */
    const double Pc = P[i + j * O.nx] + dc;
    double PW = P[M_P(i + G - 1, j + G)], PE = P[M_P(i + G + 1, j + G)], PS = P[M_P(i + G, j + G - 1)], PN = P[M_P(i + G, j + G + 1)];
    if (which == 0) PW += dn;
    if (which == 1) PE += dn;
    if (which == 2) PS += dn;
    if (which == 3) PN += dn;
    if (i == 0 && O.bcs[0] == SPB6_BC_PRES) PW = O.bcp[0] - O.p_ref;
    if (i == O.nx - 1 && O.bcs[1] == SPB6_BC_PRES) PE = O.bcp[1] - O.p_ref;
    return cell_residual(i + G, j + G, Pc, PW, PE, PS, PN, Gr, out);
}

/* ordered block sum, :744-749 */
static double block_sum_vec(int n, const double* a, const double* b) {
    const int B = 1024, nb = (n + B - 1) / B;
    double s = 0;
    for (int c = 0; c < nb; c++) {
        double part = 0;
        const int e = n < (c + 1) * B ? n : (c + 1) * B;
        for (int r = c * B; r < e; r++) part += b ? a[r] * b[r] : a[r];
        s += part;
    }
    return s;
}
static void spmv(double* Ax, const double* x) { /* :737-741 */
    const int n = O.nx * O.ny;
    for (int r = 0; r < n; r++) {
        double s = 0;
        for (int q = 0; q < O.an[r]; q++) s += O.aval[5 * r + q] * x[O.acol[5 * r + q]];
        Ax[r] = s;
    }
}
static int bicgstab(double* x, const double* b) { /* GMRES_Solver, :752-794 */
    const int n = O.nx * O.ny;
    for (int q = 0; q < n; q++) O.bdinv[q] = (O.an[q] > 0 && O.aval[5 * q] != 0) ? 1.0 / O.aval[5 * q] : 1.0;
    double E;
    {
        const int B = 1024, nb = (n + B - 1) / B;
        E = 0;
        for (int c = 0; c < nb; c++) {
            double part = 0;
            const int e = n < (c + 1) * B ? n : (c + 1) * B;
            for (int r = c * B; r < e; r++) {
                double t = 0;
                for (int q = 0; q < O.an[r]; q++) t += O.aval[5 * r + q];
                part += t;
            }
            E += part;
        }
    }
    const double Einv = (E != 0.0 && isfinite(E)) ? 1.0 / E : 0.0;
#define PREC(in, out)                                                        \
    do {                                                                     \
        const double cc_ = block_sum_vec(n, in, NULL) * Einv;                \
        for (int r_ = 0; r_ < n; r_++) out[r_] = O.bdinv[r_] * in[r_] + cc_; \
    } while (0)
    PREC(b, x);
    for (int q = 0; q < n; q++) { O.bp[q] = 0; O.bv[q] = 0; }
    spmv(O.bax, x);
    for (int q = 0; q < n; q++) { O.br[q] = b[q] - O.bax[q]; O.br0[q] = O.br[q]; }
    const double bn = sqrt(block_sum_vec(n, b, b)) + 1e-300;
    double rho = 1, alpha = 1, omega = 1;
    for (int it = 0; it < O.bicg_iter; it++) {
        if (sqrt(block_sum_vec(n, O.br, O.br)) <= O.bicg_tol * bn) { O.st_bicg_it += it; return 1; }
        const double rho1 = block_sum_vec(n, O.br0, O.br);
        if (rho1 == 0) { O.st_bicg_it += it; return 0; }
        const double beta = (rho1 / rho) * (alpha / omega);
        rho = rho1;
        for (int q = 0; q < n; q++) O.bp[q] = O.br[q] + beta * (O.bp[q] - omega * O.bv[q]);
        PREC(O.bp, O.bph);
        spmv(O.bv, O.bph);
        alpha = rho / block_sum_vec(n, O.br0, O.bv);
        for (int q = 0; q < n; q++) O.bs[q] = O.br[q] - alpha * O.bv[q];
        if (sqrt(block_sum_vec(n, O.bs, O.bs)) <= O.bicg_tol * bn) {
            for (int q = 0; q < n; q++) x[q] += alpha * O.bph[q];
            O.st_bicg_it += it + 1;
            return 1;
        }
        PREC(O.bs, O.bsh);
        spmv(O.bt, O.bsh);
        omega = block_sum_vec(n, O.bt, O.bs) / block_sum_vec(n, O.bt, O.bt);
        for (int q = 0; q < n; q++) { x[q] += alpha * O.bph[q] + omega * O.bsh[q]; O.br[q] = O.bs[q] - omega * O.bt[q]; }
    }
#undef PREC
    O.st_bicg_it += O.bicg_iter;
    return sqrt(block_sum_vec(n, O.br, O.br)) <= 1e3 * O.bicg_tol * bn;
}
static int eval_all(const double* Pq, double* R) {
    int ok = 1;
    const int n = O.nx * O.ny;
    for (int q = 0; q < n; q++) {
        double g;
        if (!residual_at(Pq, q % O.nx, q / O.nx, 0, -1, 0, &g, NULL)) ok = 0;
        else R[q] = g;
    }
    return ok;
}
static double res_norm(const double* R, const double* Pq) {
    double m = 0;
    const int n = O.nx * O.ny;
    for (int q = 0; q < n; q++) {
        const int i = q % O.nx, j = q / O.nx;
        m = SMAX(m, fabs(R[q]) / (fabs(O.p_ref + Pq[q]) + O.kw[cid(i + G, j + G)] + 1.0));
    }
    return m;
}
static int newton(double* P, double* resfinal) { /* Newton_Solver, :799-904 (jreuse = 0) */
    const int nx = O.nx, ny = O.ny, n = nx * ny;
    memcpy(O.Pn, P, (size_t)n * sizeof(double));
    if (!eval_all(P, O.Gv)) { *resfinal = INFINITY; return 0; }
    double res = res_norm(O.Gv, P);
    const int tri = (ny == 1 && O.bcs[0] != SPB6_BC_PERIODIC);
    for (int it = 0; it < O.newton_iter; it++) {
        *resfinal = res;
        if (res < O.newton_tol) return 1;
        for (int q = 0; q < n; q++) {
            const int I = q % nx + G, J = q / nx + G;
            const double K = O.kw[cid(I, J)];
            double D = O.rx * (O.kpx[cid(I, J)] + O.kpx[cid(I - 1, J)]);
            if (ny > 1) D += O.ry * (O.kpy[cid(I, J)] + O.kpy[cid(I, J - 1)]);
            O.sc[q] = (fabs(O.p_ref + P[q]) + K + 1.0) / (1.0 + K * D);
        }
        for (int r = 0; r < n; r++) {
            const int i = r % nx, j = r / nx;
            const double h = FD_STEP * O.sc[r];
            double g1;
            if (!residual_at(P, i, j, h, -1, 0, &g1, NULL)) return 0;
            int cnt = 0;
            O.acol[5 * r] = r; O.aval[5 * r] = (g1 - O.Gv[r]) / h; cnt = 1;
            static const int dd[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
            for (int w = 0; w < 4; w++) {
                if (ny == 1 && w >= 2) break;
                const int c = M_P(i + G + dd[w][0], j + G + dd[w][1]);
                const double hn = FD_STEP * O.sc[c];
                double g2;
                if (!residual_at(P, i, j, 0, w, hn, &g2, NULL)) return 0;
                O.acol[5 * r + cnt] = c; O.aval[5 * r + cnt] = (g2 - O.Gv[r]) / hn; cnt++;
            }
            O.an[r] = cnt;
        }
        for (int q = 0; q < n; q++) O.rhs[q] = -O.Gv[q];
        if (tri) { /* Thomas, :858-863 */
            for (int r = 0; r < n; r++) {
                O.lo[r] = O.up[r] = O.di[r] = 0;
                for (int q = 0; q < O.an[r]; q++) {
                    const int c = O.acol[5 * r + q];
                    if (c == r) O.di[r] += O.aval[5 * r + q];
                    else if (c == r - 1) O.lo[r] = O.aval[5 * r + q];
                    else if (c == r + 1) O.up[r] = O.aval[5 * r + q];
                }
            }
            O.cp[0] = O.up[0] / O.di[0];
            O.dpv[0] = O.rhs[0] / O.di[0];
            for (int r = 1; r < n; r++) {
                const double m = O.di[r] - O.lo[r] * O.cp[r - 1];
                O.cp[r] = O.up[r] / m;
                O.dpv[r] = (O.rhs[r] - O.lo[r] * O.dpv[r - 1]) / m;
            }
            O.dP[n - 1] = O.dpv[n - 1];
            for (int r = n - 2; r >= 0; r--) O.dP[r] = O.dpv[r] - O.cp[r] * O.dP[r + 1];
        } else {
            if (!bicgstab(O.dP, O.rhs)) return 0;
        }
        double sn = 0.0;
        for (int q = 0; q < n; q++) sn = SMAX(sn, fabs(O.dP[q]) / (fabs(P[q]) + O.sc[q]));
        if (sn < O.newton_tol) {
            for (int q = 0; q < n; q++) P[q] += O.dP[q];
            O.st_newton_it++;
            if (!eval_all(P, O.Gv)) return 0;
            *resfinal = res_norm(O.Gv, P);
            return 1;
        }
        double lam = 1.0;
        int acc = 0;
        for (int ls = 0; ls < 40; ls++) {
            for (int q = 0; q < n; q++) O.Pn[q] = P[q] + lam * O.dP[q];
            if (eval_all(O.Pn, O.Gn)) {
                const double rn = res_norm(O.Gn, O.Pn);
                if (rn < res * (1.0 - 1e-4 * lam) || rn < O.newton_tol) { acc = 1; res = rn; break; }
            }
            lam *= 0.5;
        }
        if (!acc) { /* round-off floor acceptance, :890-899 */
            *resfinal = res;
            int floor_ok = 1;
            for (int q = 0; q < n; q++) {
                const int i = q % nx, j = q / nx;
                double g;
                CellOut o;
                if (!residual_at(P, i, j, 0, -1, 0, &g, &o)) { floor_ok = 0; continue; }
                if (fabs(g) > O.newton_tol * (fabs(O.p_ref + P[q]) + O.kw[cid(i + G, j + G)] + 1.0) + o.sig) floor_ok = 0;
            }
            if (floor_ok) O.st_floor++;
            return floor_ok;
        }
        memcpy(P, O.Pn, (size_t)n * sizeof(double));
        { double* t = O.Gv; O.Gv = O.Gn; O.Gn = t; }
        O.st_newton_it++;
    }
    *resfinal = res;
    return res < O.newton_tol;
}

static double minmod(double a, double b) { return a * b <= 0 ? 0.0 : (fabs(a) < fabs(b) ? a : b); }
static double psi_face(double xm, double xL, double xR, double xp) { /* :978-982 */
    const double D = xR - xL;
    if (D == 0.0) return 1.0;
    if (!O.limiter) return SMIN(1.0, SMAX(0.0, 1.0 - 0.25 * ((xR - xm) + (xp - xL)) / D));
    return 1.0 - 0.5 * (minmod(xL - xm, D) + minmod(D, xp - xR)) / D;
}
static double dil_jump(int i, int j, int ydir) { /* :989-1000 */
    const double *u = O.ustc, *v = O.vstc;
    if (!ydir) {
        const double d = u[cid(i + 1, j)] - u[cid(i, j)];
        if (O.ny == 1 || j < 1 || j + 1 >= O.NYT) return d;
        return 0.25 * (2.0 * d + ((u[cid(i + 1, j + 1)] - u[cid(i, j + 1)]) + (u[cid(i + 1, j - 1)] - u[cid(i, j - 1)]))) +
               0.25 * (O.dx / O.dy) * ((v[cid(i, j + 1)] - v[cid(i, j - 1)]) + (v[cid(i + 1, j + 1)] - v[cid(i + 1, j - 1)]));
    }
    const double d = v[cid(i, j + 1)] - v[cid(i, j)];
    if (i < 1 || i + 1 >= O.NXT) return d;
    return 0.25 * (2.0 * d + ((v[cid(i + 1, j + 1)] - v[cid(i + 1, j)]) + (v[cid(i - 1, j + 1)] - v[cid(i - 1, j)]))) +
           0.25 * (O.dy / O.dx) * ((u[cid(i + 1, j)] - u[cid(i - 1, j)]) + (u[cid(i + 1, j + 1)] - u[cid(i - 1, j + 1)]));
}
static void set_face(int iL, int jL, int iR, int jR, double hh, int ydir, double* ubs, double* kp, double* wL, double* pv) { /* :1001-1023 */
    const double* X = O.ust;
    const double rL = cell((double*)X, iL, jL)[IM1] + cell((double*)X, iL, jL)[IM2];
    const double rR = cell((double*)X, iR, jR)[IM1] + cell((double*)X, iR, jR)[IM2];
    const double* V = ydir ? O.vstc : O.ustc;
    const double uL = V[cid(iL, jL)], uR = V[cid(iR, jR)];
    *ubs = 0.5 * (uL + uR);
    *kp = O.tau / hh / (0.5 * (rL + rR));
    *wL = rR / (rL + rR);
    *pv = 0.0;
    const double cL = O.cz[cid(iL, jL)], cR = O.cz[cid(iR, jR)];
    if (!(isfinite(cL) && isfinite(cR))) return;
    const double phi = SMAX(0.0, 1.0 - O.tau * SMIN(cL, cR) / hh);
    if (phi == 0.0) return;
    const int di = iR - iL, dj = jR - jL, im = iL - di, jm = jL - dj, ip = iR + di, jp = jR + dj;
    double psiP = 1.0, psiU = 1.0;
    if (im >= 0 && jm >= 0 && ip < O.NXT && jp < O.NYT) {
        const double* ph = ydir ? O.phy : O.phx;
        const double phis = SMIN(ph[cid(iL, jL)], ph[cid(iR, jR)]);
        psiP = 1.0 - (1.0 - psi_face(O.pold[cid(im, jm)], O.pold[cid(iL, jL)], O.pold[cid(iR, jR)], O.pold[cid(ip, jp)])) * phis;
        psiU = psi_face(V[cid(im, jm)], uL, uR, V[cid(ip, jp)]);
    }
    const double ZL = rL * cL, ZR = rR * cR;
    *kp += phi * psiP / (ZL + ZR);
    *pv = phi * psiU * ZL * ZR / (ZL + ZR) * dil_jump(iL, jL, ydir);
}
static double cfz(int i, int j) { /* :948-955 */
    const double* X = cell(O.ust, i, j);
    const double a1 = X[IA1], a2 = O.a2s[cid(i, j)], m1 = X[IM1], m2 = X[IM2];
    if (!(a1 > 0 && a2 > 0 && m1 > 0 && m2 > 0)) return INFINITY;
    const double p1 = p_ame(0, a1, m1, X[IE1]), p2 = p_ame(1, a2, m2, X[IE2]);
    if (!(p_admissible(0, p1) && p_admissible(1, p2))) return INFINITY;
    const double c21 = c2_rp(0, m1 / a1, p1), c22 = c2_rp(1, m2 / a2, p2);
    const double c2 = (m1 * c21 + m2 * c22) / (m1 + m2);
    return c2 > 0 ? sqrt(c2) : INFINITY;
}
/* PressureSubsystem :908-1074; X* is in O.ust (with ghosts), result written back to O.ust */
static int pressure_subsystem(double* P, double tau) {
    const int nx = O.nx, ny = O.ny, NXT = O.NXT, NYT = O.NYT;
    O.tau = tau; O.rx = tau / O.dx; O.ry = tau / O.dy;
    const int jr0 = ny == 1 ? G : 0, jr1 = ny == 1 ? G + 1 : NYT;
    int sok = 1;
    for (int j = jr0; j < jr1; j++)
        for (int i = 0; i < NXT; i++) {
            const double* X = cell(O.ust, i, j);
            const double sa = X[IA1] + O.a2s[cid(i, j)], rho = X[IM1] + X[IM2];
            if (!(sa > 0 && rho > 0)) { sok = 0; continue; }
            O.ustc[cid(i, j)] = X[IMU] / rho;
            O.vstc[cid(i, j)] = X[IMV] / rho;
        }
    if (!sok) return 0;
    {
        static const int VK[5] = {IA1, IM1, IM2, IE1, IE2};
#define PUT(d, w, ii, jj)                                                     \
    do {                                                                      \
        const double* w_ = cell(w, ii, jj);                                   \
        (d)[0] = w_[VK[0]]; (d)[1] = 1.0 - w_[VK[0]];                         \
        for (int q_ = 1; q_ < 5; q_++) (d)[q_ + 1] = w_[VK[q_]];              \
    } while (0)
        for (int j = jr0; j < jr1; j++)
            for (int i = 0; i < NXT - 1; i++) { PUT(O.dxl + 6 * cid(i, j), O.wxr, i, j); PUT(O.dxr + 6 * cid(i, j), O.wxl, i + 1, j); }
        if (ny > 1)
            for (int j = 0; j < NYT - 1; j++)
                for (int i = 0; i < NXT; i++) { PUT(O.dyl + 6 * cid(i, j), O.wyr, i, j); PUT(O.dyr + 6 * cid(i, j), O.wyl, i, j + 1); }
#undef PUT
    }
    for (int j = jr0; j < jr1; j++)
        for (int i = 0; i < NXT; i++) O.cz[cid(i, j)] = cfz(i, j);
    for (int j = jr0; j < jr1; j++)
        for (int i = 0; i < NXT; i++) { /* residual scale, :960-971 */
            const double* X = cell(O.ust, i, j);
            const double a1 = X[IA1], a2 = O.a2s[cid(i, j)], m1 = X[IM1], m2 = X[IM2], sa = a1 + a2;
            double K = SMAX(O.ph[0].pi, O.ph[1].pi), PE = 0.0;
            if (a1 > 0 && a2 > 0 && m1 > 0 && m2 > 0) {
                const double p1 = p_ame(0, a1, m1, X[IE1]), p2 = p_ame(1, a2, m2, X[IE2]);
                if (p_admissible(0, p1) && p_admissible(1, p2))
                    K = 1.0 / ((a1 / sa) / (m1 / a1 * c2_rp(0, m1 / a1, p1)) + (a2 / sa) / (m2 / a2 * c2_rp(1, m2 / a2, p2)));
                const double dd = dedp_am(0, a1, m1) + dedp_am(1, a2, m2);
                if (dd > 0) PE = (fabs(X[IE1]) + eps_round(0, m1) + fabs(X[IE2]) + eps_round(1, m2)) / dd;
            }
            O.kw[cid(i, j)] = K + PE;
        }
    for (int j = 0; j < NYT; j++)
        for (int i = 0; i < NXT; i++) O.pold[cid(i, j)] = P[M_P(i, j)];
    for (int j = jr0; j < jr1; j++)
        for (int i = 0; i < NXT - 1; i++) {
            const size_t c = cid(i, j);
            set_face(i, j, i + 1, j, O.dx, 0, &O.ubsx[c], &O.kpx[c], &O.wlx[c], &O.pvx[c]);
        }
    if (ny > 1)
        for (int j = 0; j < NYT - 1; j++)
            for (int i = 0; i < NXT; i++) {
                const size_t c = cid(i, j);
                set_face(i, j, i, j + 1, O.dy, 1, &O.ubsy[c], &O.kpy[c], &O.wly[c], &O.pvy[c]);
            }
    for (int q = 0; q < nx * ny; q++) {
        const int i = q % nx + G, j = q / nx + G;
        if (g_qph_inject) { /* stage data supplied by the caller (test hook) */
            O.qph[cid(i, j) * 2] = g_qph_inject[q];
            O.qph[cid(i, j) * 2 + 1] = g_qph_inject[nx * ny + q];
        } else
            shock_budget(O.ust, i, j, ny > 1, &O.qph[cid(i, j) * 2]);
    }
    if (g_prep_capture) { /* x faces i-1/2..nx-1/2 of interior rows, y faces, Kw, Qph */
        size_t w = 0;
        double* fxs[4] = {O.ubsx, O.kpx, O.wlx, O.pvx};
        double* fys[4] = {O.ubsy, O.kpy, O.wly, O.pvy};
        for (int a = 0; a < 4; a++)
            for (int j = 0; j < ny; j++)
                for (int i = -1; i < nx; i++) g_prep_capture[w++] = fxs[a][cid(i + G, j + G)];
        for (int a = 0; a < 4; a++)
            for (int j = -1; j < ny; j++)
                for (int i = 0; i < nx; i++) g_prep_capture[w++] = ny > 1 ? fys[a][cid(i + G, j + G)] : 0.0;
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) g_prep_capture[w++] = O.kw[cid(i + G, j + G)];
        for (int k = 0; k < 2; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) g_prep_capture[w++] = O.qph[cid(i + G, j + G) * 2 + k];
        g_prep_len = w;
        g_prep_capture = NULL;
    }
    double res;
    const int ok = newton(P, &res);
    if (ok) O.st_maxres = SMAX(O.st_maxres, res);
    if (!ok) return 0;
    /* final state, :1056-1073; X* is read from O.ust, so build the new state in O.un-sized scratch first */
    const size_t ncell = (size_t)NXT * NYT;
    double* fin = (double*)malloc(ncell * NV * sizeof(double));
    memcpy(fin, O.ust, ncell * NV * sizeof(double));
    int fok = 1;
    for (int q = 0; q < nx * ny; q++) {
        const int i = q % nx, j = q / nx;
        double Gv;
        CellOut o;
        if (!residual_at(P, i, j, 0, -1, 0, &Gv, &o)) { fok = 0; continue; }
        double* d = cell(fin, i + G, j + G);
        d[IA1] = o.cl.a[0]; d[IM1] = o.cl.m[0]; d[IM2] = o.cl.m[1]; d[IMU] = o.mx; d[IMV] = o.my;
        d[IE1] = o.cl.e[0]; d[IE2] = o.cl.e[1]; d[IEN] = o.E;
    }
    memcpy(O.ust, fin, ncell * NV * sizeof(double));
    free(fin);
    if (!fok) return 0;
    bc_apply(O.ust);
    O.st_stage++;
    return 1;
}

/* ------------------------------------------------------------------ driver, :1279-1384 */
static void set_tab(int rk, double Ae[3][3], double Ai[3][3]) {
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Ae[a][b] = Ai[a][b] = 0;
    if (rk == 1) Ai[0][0] = 1.0;
    else if (rk == 2) {
        const double bb = 1.0 - 1.0 / sqrt(2.0), cc = 1.0 / (2.0 * bb);
        Ae[1][0] = cc; Ai[0][0] = bb; Ai[1][0] = 1 - bb; Ai[1][1] = bb;
    } else if (rk == 3) {
        const double r12 = 0.5, r13 = 1.0 / 3.0, r14 = 1.0 / 4.0;
        Ae[1][0] = r12; Ae[2][0] = r12; Ae[2][1] = r12;
        Ai[0][0] = r14; Ai[1][1] = r14; Ai[2][0] = r13; Ai[2][1] = r13; Ai[2][2] = r13;
    }
}
/* one explicit predictor + implicit solve; X* written to O.ust */
static int run_stage(int rks, double Ae[3][3], double Ai[3][3], double* Pst) {
    const size_t ncell = (size_t)O.NXT * O.NYT, nb = ncell * NV * sizeof(double);
    memcpy(O.qe, O.un, nb);
    memcpy(O.qs, O.un, nb);
    for (int r = 0; r < rks; r++)
        for (int i = G; i < O.nx + G; i++)
            for (int j = G; j < O.ny + G; j++)
                for (int k = 0; k < NV; k++) {
                    const size_t x = NV * cid(i, j) + k;
                    O.qe[x] = O.qe[x] + Ae[rks][r] * O.dt * O.hs[r][x];
                    O.qs[x] = O.qs[x] + Ai[rks][r] * O.dt * O.hs[r][x];
                }
    bc_apply(O.qe);
    bc_apply(O.qs);
    O.adt = Ai[rks][rks] * O.dt;
    tvd_reconstruction(O.qe);
    int ok = update(O.ust, O.qe, O.qs);
    ok = ok && pressure_subsystem(Pst, O.adt);
    if (ok)
        for (int i = G; i < O.nx + G; i++)
            for (int j = G; j < O.ny + G; j++)
                for (int k = 0; k < NV; k++) {
                    const size_t x = NV * cid(i, j) + k;
                    O.hs[rks][x] = (O.ust[x] - O.qs[x]) / O.adt;
                }
    return ok;
}
static int step(void) {
    const size_t ncell = (size_t)O.NXT * O.NYT, nb = ncell * NV * sizeof(double);
    const size_t np = (size_t)O.nx * O.ny * sizeof(double);
    int ramping = 0;
    if (O.dtfix > 0) O.dt = O.dtfix;
    else {
        O.dt = O.cfl * caldt(O.u, O.acdt);
        if (O.ramp) {
            if (O.dtprev < 0) O.dtprev = O.cfl_ac * caldt(O.u, 1) / 1.2;
            if (O.dt > 1.2 * O.dtprev) { O.dt = 1.2 * O.dtprev; ramping = 1; }
        }
        if (!isfinite(O.dt)) O.dt = O.cfl_ac * caldt(O.u, 1);
    }
    O.dt = SMIN(O.dt, O.tend - O.t);
    if (!(O.dt > 1e-12 * O.tend)) return 2;
    int done = 0;
    double Ae[3][3], Ai[3][3];
    for (int attempt = 0; attempt < 30 && !done; attempt++) {
        const int first_order = O.ramp && ramping && O.startup;
        const int rk = first_order ? 1 : O.rk;
        if (rk == 1) O.st_rk1++;
        set_tab(rk, Ae, Ai);
        memcpy(O.un, O.u, nb);
        memcpy(O.Pst, O.P, np);
        int ok = 1;
        for (int rks = 0; rks < rk && ok; rks++) ok = run_stage(rks, Ae, Ai, O.Pst);
        if (ok) { memcpy(O.u, O.ust, nb); memcpy(O.P, O.Pst, np); done = 1; }
        if (!done) { O.st_reject++; O.dt *= 0.5; }
    }
    if (!done) return 2;
    O.t = O.t + O.dt;
    O.dtprev = O.dt;
    O.st_steps++;
    if (!ramping) O.startup = 0;
    return 0;
}

static double* zalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }
static void free_all(void) {
    double** ptrs[] = {&O.u, &O.un, &O.qe, &O.qs, &O.ust, &O.wxl, &O.wxr, &O.wyl, &O.wyr, &O.hs[0], &O.hs[1], &O.hs[2],
                       &O.phx, &O.phy, &O.a2s, &O.ubx, &O.uby, &O.vsc, &O.esc, &O.P, &O.Pst, &O.ustc, &O.vstc, &O.ubsx,
                       &O.kpx, &O.wlx, &O.pvx, &O.ubsy, &O.kpy, &O.wly, &O.pvy, &O.kw, &O.qph, &O.cz, &O.pold, &O.dxl,
                       &O.dxr, &O.dyl, &O.dyr, &O.Gv, &O.Gn, &O.lo, &O.di, &O.up, &O.sc, &O.cp, &O.dpv, &O.dP, &O.rhs,
                       &O.Pn, &O.aval, &O.bdinv, &O.br, &O.br0, &O.bp, &O.bv, &O.bs, &O.bt, &O.bph, &O.bsh, &O.bax};
    for (size_t k = 0; k < sizeof ptrs / sizeof ptrs[0]; k++) { free(*ptrs[k]); *ptrs[k] = NULL; }
    free(O.acol); O.acol = NULL;
    free(O.an); O.an = NULL;
}

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
static void totals(const double* u, double M[3]) {
    M[0] = M[1] = M[2] = 0;
    for (int j = G; j < O.ny + G; j++)
        for (int i = G; i < O.nx + G; i++) { const double* q = u + NV * cid(i, j); M[0] += q[IM1]; M[1] += q[IM2]; M[2] += q[IEN]; }
}

int spb6_oracle_run(const spb6_case* c, const double* U0, void* out, size_t cap) {
    if (!c || c->magic != SPB6_CASE_MAGIC || c->version != SPB6_CASE_VERSION || c->nx < 1 || c->ny < 1) return -1;
    if (c->kind[0] != 0 || c->kind[1] != 0) return -3;  /* Mie-Grueneisen phases: not restated here */
    if (c->relax != 0) return -3;                        /* thermal relaxation: not restated here */
    if (c->jreuse != 0) return -3;                       /* modified Newton: not restated here */
    if (c->order == 1) return -3;                        /* first order: not restated here */
    if (!isinf(c->mu_rate) || c->unify != 0 || c->nu_law != 0) return -3;  /* finite rates: not restated */
    const int nx = c->nx, ny = c->ny, n = nx * ny;
    const size_t nstage = (size_t)n * 8 + n + (size_t)(nx + 1) * ny + (size_t)nx * (ny + 1) + 2 * (size_t)n +
                          4 * (size_t)(nx + 1) * ny + 4 * (size_t)nx * (ny + 1) + 3 * (size_t)n;
    const size_t need = sizeof(spb6_result) + sizeof(double) * ((size_t)n * 8 + n + (c->mode == SPB6_MODE_STAGE ? nstage : 0));
    if (cap < need) return -2;
    memset(&O, 0, sizeof O);
    O.nx = nx; O.ny = ny; O.NXT = nx + 2 * G; O.NYT = ny + 2 * G;
    O.rk = c->rk; O.ramp = c->ramp; O.rus_local = c->rus_local; O.limiter = c->limiter; O.acdt = c->acdt;
    O.newton_iter = c->newton_iter; O.bicg_iter = c->bicg_iter; O.share_mode = c->share_mode;
    for (int q = 0; q < 4; q++) { O.bcs[q] = c->bc[q]; O.bcu[q] = c->bcu[q]; O.bcp[q] = c->bcp[q]; }
    for (int k = 0; k < 2; k++) { O.ph[k].g = c->g[k]; O.ph[k].pi = c->pinf[k]; O.ph[k].q = c->q[k]; O.ph[k].qp = c->qp[k]; O.ph[k].cv = c->cv[k]; O.ph[k].b = c->b[k]; }
    O.x0 = c->x0; O.x1 = c->x1; O.y0 = c->y0; O.y1 = c->y1;
    O.dx = (O.x1 - O.x0) / nx; O.dy = (O.y1 - O.y0) / ny;
    O.cfl = c->cfl; O.cfl_ac = c->cfl_ac; O.dtfix = c->dtfix; O.newton_tol = c->newton_tol; O.bicg_tol = c->bicg_tol; O.tend = c->tend;
    const size_t ncell = (size_t)O.NXT * O.NYT;
    O.u = zalloc(ncell * NV); O.un = zalloc(ncell * NV); O.qe = zalloc(ncell * NV); O.qs = zalloc(ncell * NV); O.ust = zalloc(ncell * NV);
    O.wxl = zalloc(ncell * NV); O.wxr = zalloc(ncell * NV); O.wyl = zalloc(ncell * NV); O.wyr = zalloc(ncell * NV);
    for (int r = 0; r < 3; r++) O.hs[r] = zalloc(ncell * NV);
    O.phx = zalloc(ncell); O.phy = zalloc(ncell); O.a2s = zalloc(ncell); O.ubx = zalloc(ncell); O.uby = zalloc(ncell);
    O.vsc = zalloc(ncell); O.esc = zalloc(ncell);
    O.P = zalloc(n); O.Pst = zalloc(n);
    O.ustc = zalloc(ncell); O.vstc = zalloc(ncell); O.ubsx = zalloc(ncell); O.kpx = zalloc(ncell); O.wlx = zalloc(ncell); O.pvx = zalloc(ncell);
    O.ubsy = zalloc(ncell); O.kpy = zalloc(ncell); O.wly = zalloc(ncell); O.pvy = zalloc(ncell);
    for (size_t q = 0; q < ncell; q++) { O.wlx[q] = 0.5; O.wly[q] = 0.5; }
    O.kw = zalloc(ncell); O.qph = zalloc(ncell * 2); O.cz = zalloc(ncell); O.pold = zalloc(ncell);
    O.dxl = zalloc(ncell * 6); O.dxr = zalloc(ncell * 6); O.dyl = zalloc(ncell * 6); O.dyr = zalloc(ncell * 6);
    O.Gv = zalloc(n); O.Gn = zalloc(n); O.lo = zalloc(n); O.di = zalloc(n); O.up = zalloc(n); O.sc = zalloc(n); O.cp = zalloc(n);
    O.dpv = zalloc(n); O.dP = zalloc(n); O.rhs = zalloc(n); O.Pn = zalloc(n);
    O.aval = zalloc((size_t)n * 5); O.acol = (int*)calloc((size_t)n * 5, sizeof(int)); O.an = (int*)calloc((size_t)n, sizeof(int));
    O.bdinv = zalloc(n); O.br = zalloc(n); O.br0 = zalloc(n); O.bp = zalloc(n); O.bv = zalloc(n); O.bs = zalloc(n); O.bt = zalloc(n);
    O.bph = zalloc(n); O.bsh = zalloc(n); O.bax = zalloc(n);

    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
            for (int k = 0; k < NV; k++) cell(O.u, i + G, j + G)[k] = U0[((size_t)j * nx + i) * NV + k];
    bc_apply(O.u);
    O.p_ref = INFINITY; /* :1309-1312 */
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) O.p_ref = SMIN(O.p_ref, pbar_of(cell(O.u, i + G, j + G)));
    if (!isfinite(O.p_ref)) O.p_ref = 0.0;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) O.P[i + j * nx] = pbar_of(cell(O.u, i + G, j + G)) - O.p_ref;
    O.dtprev = -1;
    O.startup = 1;
    double M0[3];
    totals(O.u, M0);

    char* o = (char*)out;
    spb6_result* r = (spb6_result*)o;
    memset(r, 0, sizeof *r);
    double* arr = (double*)(o + sizeof(spb6_result));
    size_t off = (size_t)n * 8 + n;
    double t0 = now_s();
    int rc = 0;
    if (c->mode == SPB6_MODE_STAGE) {
        double Ae[3][3], Ai[3][3];
        set_tab(O.rk, Ae, Ai);
        O.dt = c->dtfix;
        memcpy(O.un, O.u, ncell * NV * sizeof(double));
        memcpy(O.Pst, O.P, (size_t)n * sizeof(double));
        memcpy(O.qe, O.un, ncell * NV * sizeof(double));
        memcpy(O.qs, O.un, ncell * NV * sizeof(double));
        bc_apply(O.qe);
        bc_apply(O.qs);
        O.adt = Ai[0][0] * O.dt;
        tvd_reconstruction(O.qe);
        int ok = update(O.ust, O.qe, O.qs);
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++)
                for (int k = 0; k < NV; k++) arr[off++] = cell(O.ust, i + G, j + G)[k];
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) arr[off++] = O.a2s[cid(i + G, j + G)];
        for (int j = 0; j < ny; j++)
            for (int i = -1; i < nx; i++) arr[off++] = O.ubx[cid(i + G, j + G)];
        for (int j = -1; j < ny; j++)
            for (int i = 0; i < nx; i++) arr[off++] = ny > 1 ? O.uby[cid(i + G, j + G)] : 0.0;
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) arr[off++] = O.phx[cid(i + G, j + G)];
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) arr[off++] = O.phy[cid(i + G, j + G)];
        g_prep_capture = arr + off;
        g_prep_len = 0;
        g_qph_inject = c->inject_qph ? U0 + (size_t)n * NV : NULL;
        ok = ok && pressure_subsystem(O.Pst, O.adt);
        g_prep_capture = NULL;
        g_qph_inject = NULL;
        off += g_prep_len;
        if (ok) { memcpy(O.u, O.ust, ncell * NV * sizeof(double)); memcpy(O.P, O.Pst, (size_t)n * sizeof(double)); }
        rc = ok ? 0 : 2;
    } else {
        const int to_end = c->mode == SPB6_MODE_TEND;
        double tw = t0;
        long timed = 0;
        for (int s = 0; (to_end || s < c->nsteps) && rc == 0 && O.t < O.tend * (1 - 1e-12); s++) {
            if (s == c->warmup) tw = now_s();
            rc = step();
            if (s >= c->warmup) timed++;
            if (c->budget_s > 0 && s >= c->warmup && now_s() - tw > c->budget_s) break;
        }
        r->timed_steps = timed;
        (void)tw;
        t0 = tw;
    }
    const double wall = now_s() - t0;
    double M1[3];
    totals(O.u, M1);
    r->magic = SPB6_CASE_MAGIC; r->status = rc; r->nx = nx; r->ny = ny;
    r->steps = O.st_steps; r->rejects = O.st_reject; r->rk1 = O.st_rk1; r->stages = O.st_stage; r->newton_it = O.st_newton_it;
    r->floor_count = O.st_floor; r->bicg_it = O.st_bicg_it;
    r->t = O.t; r->dt = O.dt; r->maxres = O.st_maxres; r->p_ref = O.p_ref; r->wall_s = wall;
    for (int q = 0; q < 3; q++) r->dM[q] = (M1[q] - M0[q]) / M0[q];
    size_t w = 0;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
            for (int k = 0; k < NV; k++) arr[w++] = cell(O.u, i + G, j + G)[k];
    for (int q = 0; q < n; q++) arr[w++] = O.P[q];
    const size_t total = sizeof(spb6_result) + sizeof(double) * (c->mode == SPB6_MODE_STAGE ? off : w);
    free_all();
    return (int)total;
}
