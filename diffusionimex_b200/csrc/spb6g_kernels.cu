// Stage pipeline kernels of the SPB6 IMEX solver (one thread per cell / face /
// row; grid-stride loops; deterministic reductions).  Reference functions are
// cited per kernel; arithmetic follows them in operation order.
#include <cstdio>

#include <cuda_bf16.h>

#include "../../include/spb6g.h"
#include "spb6g_ctx.cuh"
#include "spb6g_mgfwd.cuh"

namespace spb6g {

constexpr int TPB = 256;

static int blocks_for(long n, int tpb = TPB) {
    long b = (n + tpb - 1) / tpb;
    if (b < 1) b = 1;
    if (b > 148L * 32) b = 148L * 32;
    return (int)b;
}
static inline void count(const Ctx& c, int k) {
    if (c.nlaunch) *c.nlaunch += k;
}
int red_blocks(int n, int threads) {
    long b = ((long)n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148L * 8) b = 148L * 8;
    return (int)b;
}

// ============================================================ stage data (PressureSubsystem prep :922-1039)
SPB6G_DEV void xs_at(const Ctx& c, int i, int j, double* q) {
    CState X;
    for (int k = 0; k < NV; k++) X.v[k] = c.Xs.v[k];
    load_state(c.phy, c.g, X, i, j, q);
}
// frozen sound speed c_f on X* (cfz :948-955)
SPB6G_DEV double cfz(const Phys& P, const double* X, double a2) {
    const double a1 = X[IA1], m1 = X[IM1], m2 = X[IM2];
    if (!(a1 > 0 && a2 > 0 && m1 > 0 && m2 > 0)) return INFINITY;
    const double p1 = p_ame(P, 0, a1, m1, X[IE1]), p2 = p_ame(P, 1, a2, m2, X[IE2]);
    if (!(p_admissible(P, 0, a1, m1, p1) && p_admissible(P, 1, a2, m2, p2))) return INFINITY;
    const double c21 = c2_rp(P, 0, m1 / a1, p1), c22 = c2_rp(P, 1, m2 / a2, p2);
    const double c2 = (m1 * c21 + m2 * c22) / (m1 + m2);
    return c2 > 0 ? sqrt(c2) : INFINITY;
}
SPB6G_DEV double minmod(double a, double b) { return a * b <= 0 ? 0.0 : (fabs(a) < fabs(b) ? a : b); }
SPB6G_DEV double psi_face(int limiter, double xm, double xL, double xR, double xp) {  // :978-982
    const double D = xR - xL;
    if (D == 0.0) return 1.0;
    if (!limiter) return SMIN(1.0, SMAX(0.0, 1.0 - 0.25 * ((xR - xm) + (xp - xL)) / D));
    return 1.0 - 0.5 * (minmod(xL - xm, D) + minmod(D, xp - xR)) / D;
}
SPB6G_DEV void vel_at(const Ctx& c, int i, int j, double& u, double& v) {
    double q[NV];
    xs_at(c, i, j, q);
    const double rho = q[IM1] + q[IM2];
    u = q[IMU] / rho;
    v = q[IMV] / rho;
}
SPB6G_DEV double pold_at(const Ctx& c, int i, int j) { return c.P[mp_index(c.g, i, j)]; }

// Per-cell quantities of the stage prep on the padded grid (cells -2..nx+1 x
// -2..ny+1, ghosts through the boundary maps): rho*, u* = rho u*/rho*, v*, and
// the frozen sound speed c_f (cfz :948-955); interior cells also get the
// residual scale K + P_E (:960-971) and the admissibility check (:928-929).
SPB6G_DEV int pad_index(const Geom& g, int i, int j) { return (i + 2) + (g.ny > 1 ? (j + 2) * (g.nx + 4) : 0); }  // 1D: one row
SPB6G_DEV long prep_cells(const Geom& g) { return (long)(g.nx + 4) * (g.ny > 1 ? g.ny + 4 : 1); }
SPB6G_DEV void prep_cell_at(const Ctx& c, long t) {
    const Geom& g = c.g;
    const int W = g.nx + 4;
    {
        const int i = (int)(t % W) - 2, j = g.ny > 1 ? (int)(t / W) - 2 : 0;
        double X[NV];
        xs_at(c, i, j, X);
        const double a2 = load_arr(g, c.a2s, i, j);
        const double rho = X[IM1] + X[IM2];
        const int p = pad_index(g, i, j);
        c.pad_rho[p] = rho;
        c.pad_u[p] = X[IMU] / rho;
        c.pad_v[p] = X[IMV] / rho;
        c.pad_cz[p] = cfz(c.phy, X, a2);
        if (i < 0 || i >= g.nx || j < 0 || j >= g.ny) return;
        const size_t x = (size_t)i + (size_t)j * g.nx;
        const double a1 = X[IA1], m1 = X[IM1], m2 = X[IM2], sa = a1 + a2;
        if (!(sa > 0 && rho > 0)) atomicOr(&c.ns->err, 2);
        double K = SMAX(c.phy.ph[0].pi, c.phy.ph[1].pi), PE = 0.0;
        if (a1 > 0 && a2 > 0 && m1 > 0 && m2 > 0) {
            const double p1 = p_ame(c.phy, 0, a1, m1, X[IE1]), p2 = p_ame(c.phy, 1, a2, m2, X[IE2]);
            if (p_admissible(c.phy, 0, a1, m1, p1) && p_admissible(c.phy, 1, a2, m2, p2))
                K = 1.0 / ((a1 / sa) / (m1 / a1 * c2_rp(c.phy, 0, m1 / a1, p1)) + (a2 / sa) / (m2 / a2 * c2_rp(c.phy, 1, m2 / a2, p2)));
            const double dd = dedp_am(c.phy, 0, a1, m1) + dedp_am(c.phy, 1, a2, m2);
            if (dd > 0) PE = (fabs(X[IE1]) + eps_round(c.phy, 0, a1, m1) + fabs(X[IE2]) + eps_round(c.phy, 1, a2, m2)) / dd;
        }
        c.kw[x] = K + PE;
    }
}
__global__ void __launch_bounds__(TPB, 3) k_prep_cell(Ctx c) {
    const long tot = prep_cells(c.g);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) prep_cell_at(c, t);
}

// Face coefficients of the implicit face velocity / pressure (set_face :1001-1023, dil_jump :989-1000)
// and the tangential velocities of the face's two cells.
SPB6G_DEV void set_face(const Ctx& c, int iL, int jL, int ydir, double& ubs, double& kp, double& wl, double& pv,
                        double& utL, double& utR) {
    const Geom& g = c.g;
    const int iR = iL + (ydir ? 0 : 1), jR = jL + (ydir ? 1 : 0);
    const double hh = ydir ? g.dy : g.dx;
    const int pL = pad_index(g, iL, jL), pR = pad_index(g, iR, jR);
    const double* U = c.pad_u;
    const double* V = c.pad_v;
    const double* N = ydir ? V : U;  // normal velocity
    const double rL = c.pad_rho[pL], rR = c.pad_rho[pR];
    const double uL = N[pL], uR = N[pR];
    utL = ydir ? U[pL] : V[pL];
    utR = ydir ? U[pR] : V[pR];
    ubs = 0.5 * (uL + uR);
    kp = c.tau / hh / (0.5 * (rL + rR));
    wl = rR / (rL + rR);
    pv = 0.0;
    const double cL = c.pad_cz[pL], cR = c.pad_cz[pR];
    if (!(isfinite(cL) && isfinite(cR))) return;
    const double phi = SMAX(0.0, 1.0 - c.tau * SMIN(cL, cR) / hh);
    if (phi == 0.0) return;
    const int di = iR - iL, dj = jR - jL, im = iL - di, jm = jL - dj, ip = iR + di, jp = jR + dj;
    // the reference's range test (im >= 0 && ... jp < NYT) holds for every face the residual reads
    const double phis = ydir ? SMIN(c.phis_y[ryi(g, iL, jL)], c.phis_y[ryi(g, iR, jR)])
                             : SMIN(c.phis_x[rxi(g, iL, jL)], c.phis_x[rxi(g, iR, jR)]);
    // first order: psi_face is 1 (:979) and phi_x, phi_y are 0 (:373)
    const bool o1 = c.phy.order == 1;
    const double psiP = o1 ? 1.0 : 1.0 - (1.0 - psi_face(c.phy.limiter, pold_at(c, im, jm), pold_at(c, iL, jL), pold_at(c, iR, jR), pold_at(c, ip, jp))) * phis;
    const double psiU = o1 ? 1.0 : psi_face(c.phy.limiter, N[pad_index(g, im, jm)], uL, uR, N[pad_index(g, ip, jp)]);
    double D;
    if (!ydir) {
        const double d = uR - uL;
        if (g.ny == 1) D = d;
        else {
            const int p0p = pad_index(g, iL, jL + 1), p1p = pad_index(g, iL + 1, jL + 1);
            const int p0m = pad_index(g, iL, jL - 1), p1m = pad_index(g, iL + 1, jL - 1);
            D = 0.25 * (2.0 * d + ((U[p1p] - U[p0p]) + (U[p1m] - U[p0m]))) + 0.25 * (g.dx / g.dy) * ((V[p0p] - V[p0m]) + (V[p1p] - V[p1m]));
        }
    } else {
        const double d = uR - uL;
        const int pp1 = pad_index(g, iL + 1, jL + 1), pp0 = pad_index(g, iL + 1, jL);
        const int pm1 = pad_index(g, iL - 1, jL + 1), pm0 = pad_index(g, iL - 1, jL);
        D = 0.25 * (2.0 * d + ((V[pp1] - V[pp0]) + (V[pm1] - V[pm0]))) + 0.25 * (g.dy / g.dx) * ((U[pp0] - U[pm0]) + (U[pp1] - U[pm1]));
    }
    const double ZL = rL * cL, ZR = rR * cR;
    kp += phi * psiP / (ZL + ZR);
    pv = phi * psiU * ZL * ZR / (ZL + ZR) * D;
}
SPB6G_DEV void prep_fx_at(const Ctx& c, long t) {
    const Geom& g = c.g;
    const long tot = (long)(g.nx + 1) * g.ny;
    {
        const int i = (int)(t % (g.nx + 1)) - 1, j = (int)(t / (g.nx + 1));
        double ubs, kp, wl, pv, utL, utR;
        set_face(c, i, j, 0, ubs, kp, wl, pv, utL, utR);
        const size_t f = fxi(g, i, j);
        c.fx_ubs[f] = ubs; c.fx_kp[f] = kp; c.fx_wl[f] = wl; c.fx_pv[f] = pv;
        c.fxd[8 * (size_t)tot + f] = utL;
        c.fxd[9 * (size_t)tot + f] = utR;
    }
}
__global__ void k_prep_fx(Ctx c) {
    const long tot = (long)(c.g.nx + 1) * c.g.ny;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) prep_fx_at(c, t);
}
__global__ void k_prep_fy(Ctx c) {
    const Geom& g = c.g;
    const long tot = (long)g.nx * (g.ny + 1);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.nx), j = (int)(t / g.nx) - 1;
        double ubs, kp, wl, pv, utL, utR;
        set_face(c, i, j, 1, ubs, kp, wl, pv, utL, utR);
        const size_t f = fyi(g, i, j);
        c.fy_ubs[f] = ubs; c.fy_kp[f] = kp; c.fy_wl[f] = wl; c.fy_pv[f] = pv;
        c.fyd[8 * (size_t)tot + f] = utL;
        c.fyd[9 * (size_t)tot + f] = utR;
    }
}
void launch_prep(const Ctx& c, cudaStream_t st) {
    SPB6G_MG_FORWARD_EOS(launch_prep, mg_view(c), st);
    const long pad = (long)(c.g.nx + 4) * (c.g.ny > 1 ? c.g.ny + 4 : 1);
    k_prep_cell<<<blocks_for(pad), TPB, 0, st>>>(c);
    k_prep_fx<<<blocks_for((long)(c.g.nx + 1) * c.g.ny), TPB, 0, st>>>(c);
    if (c.g.ny > 1) k_prep_fy<<<blocks_for((long)c.g.nx * (c.g.ny + 1)), TPB, 0, st>>>(c);
    count(c, c.g.ny > 1 ? 3 : 2);
}

// ============================================================ shock budget (shock_budget physics :405-428)
// Evaluates the compact-stencil budget; returns 0 (no budget), 1 (weak, Q set) or 2 (strong branch needed).
SPB6G_DEV int shock_cell(const Ctx& c, int i, int j, double Q[2], bool do_strong) {
    Q[0] = Q[1] = 0.0;
    const bool twoD = c.g.ny > 1;
    double q[NV], c0[7], st[7], lo[7] = {0, 0, 0, 0, 0, 0, 0}, plo = 1e300, phi = -1e300, div = 0.0;
    xs_at(c, i, j, q);
    stencil_state(c.phy, q, c0);
    for (int d = 0; d < (twoD ? 2 : 1); d++)
        for (int s = -1; s <= 1; s++) {
            if (d == 1 && s == 0) continue;
            xs_at(c, i + (d == 0 ? s : 0), j + (d == 1 ? s : 0), q);
            stencil_state(c.phy, q, st);
            if (s == 1) div += st[5 + d];
            else if (s == -1) div -= st[5 + d];
            if (!isfinite(st[4])) continue;
            if (st[4] < plo) { plo = st[4]; for (int n = 0; n < 7; n++) lo[n] = st[n]; }
            if (st[4] > phi) phi = st[4];
        }
    if (!(div < 0.0) || !(phi > plo)) return 0;
    double Y[2], vpre[2], lam[2], qq, K[2], Gm[2];
    const double rho = c0[2] + c0[3];
    if (!(rho > 0)) return 0;
    for (int k = 0; k < 2; k++) {
        Y[k] = c0[2 + k] / rho;
        vpre[k] = (lo[k] > 0 && lo[2 + k] > 0) ? lo[k] / lo[2 + k] : (c0[2 + k] > 0 ? c0[k] / c0[2 + k] : 0.0);
    }
    if (!(Y[0] > 0) || !(Y[1] > 0) || !(vpre[0] > 0) || !(vpre[1] > 0)) return 0;
    bool strong;
    if (shock_share_weak(c.phy, Y, vpre, plo, phi, lam, qq, strong, K, Gm)) {
        for (int k = 0; k < 2; k++) Q[k] = lam[k] * rho * qq;
        return 1;
    }
    if (!strong) return 0;
    if (!do_strong) return 2;
    if (!shock_share_strong(c.phy, Y, vpre, plo, phi, K, Gm, lam, qq)) return 0;
    for (int k = 0; k < 2; k++) Q[k] = lam[k] * rho * qq;
    return 1;
}
__global__ void k_shock_weak(Ctx c) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        double Q[2];
        const int r = shock_cell(c, x % c.g.nx, x / c.g.nx, Q, false);
        c.qph0[x] = Q[0];
        c.qph1[x] = Q[1];
        c.smask[x] = r == 2 ? 1 : 0;
        if (r == 2) {
            const int slot = atomicAdd(&c.ns->nstrong, 1);
            c.strong_list[slot] = x;
        }
    }
}
// One worklist cell per thread: the grid covers the largest possible worklist (every cell) and
// blocks past the worklist's end return at once, so no thread integrates two cells in a row.
__global__ void k_shock_strong(Ctx c) {
    const int cnt = *(volatile int*)&c.ns->nstrong;
    if ((long)blockIdx.x * blockDim.x >= cnt) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int x = c.strong_list[t];
        double Q[2];
        shock_cell(c, x % c.g.nx, x / c.g.nx, Q, true);
        c.qph0[x] = Q[0];
        c.qph1[x] = Q[1];
    }
}
// Weak-shock cells are finished in place; strong-shock cells (Kapila profile
// shooting, 6-9 RK45 integrations each) go through a compacted worklist.
void launch_shock_weak(const Ctx& c, cudaStream_t st) {
    SPB6G_MG_FORWARD_EOS(launch_shock_weak, mg_view(c), st);
    k_shock_weak<<<blocks_for(c.n), TPB, 0, st>>>(c);
    count(c, 1);
}
void launch_shock_strong(const Ctx& c, cudaStream_t st) {
    SPB6G_MG_FORWARD_EOS(launch_shock_strong, mg_view(c), st);
    k_shock_strong<<<(c.n + 31) / 32, 32, 0, st>>>(c);
    count(c, 1);
}

// ============================================================ implicit residual (:610-731)
struct FaceV {
    double uf, pf, wL, wR, utL, utR, cL[4], cR[4];  // donors: m1, m2, e1, e2
};
SPB6G_DEV void face_weights(FaceV& f, double ube) {
    f.wL = SMAX(f.uf, 0.0) - SMAX(ube, 0.0);
    f.wR = SMIN(f.uf, 0.0) - SMIN(ube, 0.0);
}
// face_x / face_y (:623-642) for the face between (i, j) and its +x / +y neighbour.
SPB6G_DEV void face_eval(const Ctx& c, int i, int j, int ydir, double PL, double PR, FaceV& f) {
    const Geom& g = c.g;
    size_t fi;
    double wl, pv, ubs, kp, ube;
    if (!ydir) {
        fi = fxi(g, i, j);
        wl = c.fx_wl[fi]; pv = c.fx_pv[fi]; ubs = c.fx_ubs[fi]; kp = c.fx_kp[fi]; ube = c.ube_x[fi];
    } else {
        fi = fyi(g, i, j);
        wl = c.fy_wl[fi]; pv = c.fy_pv[fi]; ubs = c.fy_ubs[fi]; kp = c.fy_kp[fi]; ube = c.ube_y[fi];
    }
    f.pf = wl * PL + (1.0 - wl) * PR - pv;
    {
        const double* pl = ydir ? c.fyd : c.fxd;
        const size_t st = ydir ? (size_t)g.nx * (g.ny + 1) : (size_t)(g.nx + 1) * g.ny;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            f.cL[q] = pl[q * st + fi];
            f.cR[q] = pl[(4 + q) * st + fi];
        }
        f.utL = pl[8 * st + fi];
        f.utR = pl[9 * st + fi];
    }
    int w = -1;
    if (!ydir) { if (i == -1 && g.bcs[0] == BC_WALL) w = 0; else if (i == g.nx - 1 && g.bcs[1] == BC_WALL) w = 1; }
    else { if (j == -1 && g.bcs[2] == BC_WALL) w = 2; else if (j == g.ny - 1 && g.bcs[3] == BC_WALL) w = 3; }
    if (w >= 0) {
        if (g.bcu[w] == 0.0) { f.uf = 0.0; f.wL = f.wR = 0.0; return; }
        f.uf = g.bcu[w];
        face_weights(f, ube);
        return;
    }
    f.uf = ubs - kp * (PR - PL);
    face_weights(f, ube);
}
SPB6G_DEV double finc(const FaceV& f, int q) { return f.cL[q] * f.wL + f.cR[q] * f.wR; }
struct FFlux {
    double M, Mt, E;
};
SPB6G_DEV FFlux face_flux(const FaceV& f, double p_ref) {  // :646-651
    const double ML = (f.cL[0] + f.cL[1]) * f.wL, MR = (f.cR[0] + f.cR[1]) * f.wR, M = ML + MR;
    FFlux F;
    F.M = M;
    F.Mt = f.utL * ML + f.utR * MR;
    F.E = finc(f, 2) + finc(f, 3) + 0.5 * f.uf * f.uf * M + 0.5 * (f.utL * f.utL * ML + f.utR * f.utR * MR) + (p_ref + f.pf) * f.uf;
    return F;
}
struct CellRes {
    ClIn in;
    ClOut o;
    double mx, my, E;
};
// cell_residual (:666-704): G = pbar_closure(P) - P_REF - Pc.  The faces are
// evaluated in pairs (x: east/west, then y: north/south) so only two face records
// are live; each conservative quantity still receives its x difference before its
// y difference, exactly the reference's order.
SPB6G_DEV bool cell_residual(const Ctx& c, int i, int j, double Pc, double PW, double PE, double PS, double PN, double& Gr,
                             CellRes* out) {
    const Geom& g = c.g;
    const size_t x = (size_t)i + (size_t)j * g.nx;
    const bool twoD = g.ny > 1;
    double X[6] = {c.Xs.v[IA1][x], c.a2s[x], c.Xs.v[IM1][x], c.Xs.v[IM2][x], c.Xs.v[IE1][x], c.Xs.v[IE2][x]};
    double s, mx, my, E;
    {
        FaceV fe, fw;
        face_eval(c, i, j, 0, Pc, PE, fe);
        face_eval(c, i - 1, j, 0, PW, Pc, fw);
#pragma unroll
        for (int k = 2; k < 6; k++) X[k] -= c.rx * (finc(fe, k - 2) - finc(fw, k - 2));
        s = c.rx * (fe.uf - fw.uf);
        const FFlux FEe = face_flux(fe, c.p_ref), FEw = face_flux(fw, c.p_ref);
        mx = c.Xs.v[IMU][x] - c.rx * (fe.pf - fw.pf) - c.rx * (fe.uf * FEe.M - fw.uf * FEw.M);
        my = c.Xs.v[IMV][x] - c.rx * (FEe.Mt - FEw.Mt);
        E = c.Xs.v[IEN][x] - c.rx * (FEe.E - FEw.E);
    }
    if (twoD) {
        FaceV fn, fs;
        face_eval(c, i, j, 1, Pc, PN, fn);
        face_eval(c, i, j - 1, 1, PS, Pc, fs);
#pragma unroll
        for (int k = 2; k < 6; k++) X[k] -= c.ry * (finc(fn, k - 2) - finc(fs, k - 2));
        s = s + c.ry * (fn.uf - fs.uf);
        const FFlux FEn = face_flux(fn, c.p_ref), FEs = face_flux(fs, c.p_ref);
        my -= c.ry * (fn.pf - fs.pf) + c.ry * (fn.uf * FEn.M - fs.uf * FEs.M);
        mx -= c.ry * (FEn.Mt - FEs.Mt);
        E -= c.ry * (FEn.E - FEs.E);
    } else {
        s = s + 0.0;
    }
    X[1] = 1.0 - X[0];
    X[0] *= 1.0 - s;
    X[1] *= 1.0 - s;
    const double rho = X[2] + X[3];
    if (!(rho > 0)) return false;
    ClIn in;
    in.atr[0] = X[0]; in.atr[1] = X[1]; in.mtr[0] = X[2]; in.mtr[1] = X[3]; in.etr[0] = X[4]; in.etr[1] = X[5];
    in.s = s;
    in.rhoeC = E - 0.5 * (mx * mx + my * my) / rho;
    in.pguess = c.p_ref + Pc;
    in.Qph[0] = c.qph0[x];
    in.Qph[1] = c.qph1[x];
    // S.type (:695): the activation's type, frozen per step; without relaxation the mechanical one
    in.type = SPB6G_MG ? (c.phy.relax ? (int)c.ctype[x] : c.phy.mech) : CL_P;
    in.tau = c.tau;
    in.Z[0] = in.Z[1] = 1.0;
    in.nu = (SPB6G_MG && c.step_nu) ? c.step_nu[x] : -1.0;
    if (SPB6G_MG && in.type == CL_MU) {  // impedances of the stage's unit contents X* / (a1 + a2) (:1036-1037)
        const double sa = c.Xs.v[IA1][x] + c.a2s[x];
        for (int k = 0; k < 2; k++) {
            const double a = (k == 0 ? c.Xs.v[IA1][x] : c.a2s[x]) / sa, m = c.Xs.v[k == 0 ? IM1 : IM2][x] / sa;
            const double pk = p_ame(c.phy, k, a, m, c.Xs.v[k == 0 ? IE1 : IE2][x] / sa), r = m / a;
            in.Z[k] = r * sqrt(SMAX(c2_rp(c.phy, k, r, pk), 1e-30));
        }
    }
    ClOut o;
    if (!closure(c.phy, in, o)) return false;
    Gr = (o.pbar - c.p_ref) - Pc;
    if (out) { out->in = in; out->o = o; out->mx = mx; out->my = my; out->E = E; }
    return isfinite(Gr);
}

// The five pressures of row (i, j): self, W, E, S, N through M_P.
struct Nb5 {
    double c, w, e, s, n;
};
template <class F>
SPB6G_DEV Nb5 gather_p(const Geom& g, int i, int j, F pv) {
    Nb5 p;
    p.c = pv(i + j * g.nx);
    p.w = pv(mp_index(g, i - 1, j));
    p.e = pv(mp_index(g, i + 1, j));
    p.s = pv(mp_index(g, i, j - 1));
    p.n = pv(mp_index(g, i, j + 1));
    return p;
}
// residual_at (:720-731): dc perturbs the own cell, `which` (0 W, 1 E, 2 S, 3 N) one neighbour by dn.
SPB6G_DEV bool residual_at(const Ctx& c, int i, int j, const Nb5& p, double dc, int which, double dn, double& Gr, CellRes* out) {
    const double Pc = p.c + dc;
    double PW = p.w, PE = p.e, PS = p.s, PN = p.n;
    if (which == 0) PW += dn;
    if (which == 1) PE += dn;
    if (which == 2) PS += dn;
    if (which == 3) PN += dn;
    if (i == 0 && c.g.bcs[0] == BC_PRES) PW = c.g.bcp[0] - c.p_ref;
    if (i == c.g.nx - 1 && c.g.bcs[1] == BC_PRES) PE = c.g.bcp[1] - c.p_ref;
    return cell_residual(c, i, j, Pc, PW, PE, PS, PN, Gr, out);
}
SPB6G_DEV double row_scale(const Ctx& c, int i, int j, double Pc) {  // natural scale s_q (:832-836)
    const Geom& g = c.g;
    const size_t x = (size_t)i + (size_t)j * g.nx;
    const double K = c.kw[x];
    double D = c.rx * (c.fx_kp[fxi(g, i, j)] + c.fx_kp[fxi(g, i - 1, j)]);
    if (g.ny > 1) D += c.ry * (c.fy_kp[fyi(g, i, j)] + c.fy_kp[fyi(g, i, j - 1)]);
    return (fabs(c.p_ref + Pc) + K + 1.0) / (1.0 + K * D);
}

// evalAll + norm (:805-814), optionally at Pn = P + lam dP (line search :880-886).
// skip_strong (mode 0 only): cells whose strong-shock budget is still being computed on
// the side stream get their row scale only; k_residual_strong finishes them.
__global__ void __launch_bounds__(RED_THREADS, 3) k_residual(Ctx c, int mode, double lam, int skip_strong) {
    const Geom& g = c.g;
    double m[1] = {0.0};
    const double* P = c.P;
    const double* dP = c.dP;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
        if (skip_strong && c.smask[x]) {
            c.sc[x] = row_scale(c, i, j, P[x]);
            continue;
        }
        Nb5 p = mode == 0 ? gather_p(g, i, j, [&](int q) { return P[q]; })
                          : gather_p(g, i, j, [&](int q) { return P[q] + lam * dP[q]; });
        double Gr;
        const bool ok = residual_at(c, i, j, p, 0, -1, 0, Gr, nullptr);
        const double sc = row_scale(c, i, j, p.c);
        if (mode == 0) { c.G[x] = Gr; c.sc[x] = sc; }
        else { c.Gn[x] = Gr; c.scn[x] = sc; c.Pn[x] = p.c; }
        if (!ok) atomicOr(&c.ns->fail, 1);
        else m[0] = SMAX(m[0], SMAX(0.0, fabs(Gr) / (fabs(c.p_ref + p.c) + c.kw[x] + 1.0)));
    }
    double tot[1];
    if (grid_fold<RedMax, 1>(m, c.partials, &c.counters[0], tot) && threadIdx.x == 0) c.ns->res = tot[0];
}
void launch_residual(const Ctx& c, cudaStream_t st, int mode, double lam, int skip_strong) {
    SPB6G_MG_FORWARD(launch_residual, mg_view(c), st, mode, lam, skip_strong);
    k_residual<<<red_blocks(c.n), RED_THREADS, 0, st>>>(c, mode, lam, skip_strong);
    count(c, 1);
}
// Mode-0 residual of the strong-shock cells (the worklist), folded into the
// max-norm that k_residual(skip_strong) left in ns->res.
__global__ void __launch_bounds__(RED_THREADS, 3) k_residual_strong(Ctx c) {
    const Geom& g = c.g;
    double m[1] = {0.0};
    const double* P = c.P;
    const int cnt = c.ns->nstrong;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += gridDim.x * blockDim.x) {
        const int x = c.strong_list[t];
        const int i = x % g.nx, j = x / g.nx;
        const Nb5 p = gather_p(g, i, j, [&](int q) { return P[q]; });
        double Gr;
        const bool ok = residual_at(c, i, j, p, 0, -1, 0, Gr, nullptr);
        c.G[x] = Gr;
        if (!ok) atomicOr(&c.ns->fail, 1);
        else m[0] = SMAX(m[0], SMAX(0.0, fabs(Gr) / (fabs(c.p_ref + p.c) + c.kw[x] + 1.0)));
    }
    double tot[1];
    if (grid_fold<RedMax, 1>(m, c.partials, &c.counters[10], tot) && threadIdx.x == 0) c.ns->res = SMAX(c.ns->res, tot[0]);
}
void launch_residual_strong(const Ctx& c, cudaStream_t st) {
    SPB6G_MG_FORWARD(launch_residual_strong, mg_view(c), st);
    k_residual_strong<<<148 * 2, RED_THREADS, 0, st>>>(c);
    count(c, 1);
}

// FD Jacobian (:837-853).  One thread per matrix entry: entry 0 perturbs the own
// cell by h = 1e-7 s_r, entries 1-4 the W, E, S, N neighbour by 1e-7 s_col; each is
// one residual evaluation, so the 5 closures of a row run in 5 independent threads.
SPB6G_DEV void jac_entry(const Ctx& c, int x, int w) {
    const Geom& g = c.g;
    const int i = x % g.nx, j = x / g.nx;
    const Nb5 p = gather_p(g, i, j, [&](int q) { return c.P[q]; });
    const double G0 = c.G[x];
    double gv, a;
    bool ok;
    if (w == 0) {
        const double h = 1e-7 * c.sc[x];
        ok = residual_at(c, i, j, p, h, -1, 0, gv, nullptr);
        a = (gv - G0) / h;
    } else {
        const int di = w == 1 ? -1 : (w == 2 ? 1 : 0), dj = w == 3 ? -1 : (w == 4 ? 1 : 0);
        const int col = mp_index(g, i + di, j + dj);
        const double hn = 1e-7 * c.sc[col];
        ok = residual_at(c, i, j, p, 0, w - 1, hn, gv, nullptr);
        a = (gv - G0) / hn;
    }
    if (!ok) atomicOr(&c.ns->fail, 2);
    double* plane = w == 0 ? c.aC : w == 1 ? c.aW : w == 2 ? c.aE : w == 3 ? c.aS : c.aN;
    plane[x] = a;
}
// skip_strong: rows of strong-shock cells are left to k_jac_strong.
__global__ void __launch_bounds__(RED_THREADS, 3) k_jac_entries(Ctx c, int skip_strong) {
    const int nw = c.g.ny > 1 ? 5 : 3;
    // blocks nw*r .. nw*r + nw-1 evaluate the nw entries of the same 256 rows: they run side by
    // side, so the rows' stage data comes from DRAM once and from L2 for the other entries,
    // while every warp follows one entry's code path
    const int w = blockIdx.x % nw, rb = blockIdx.x / nw;
    const int x = rb * blockDim.x + threadIdx.x;
    if (x >= c.n || (skip_strong && c.smask[x])) return;
    jac_entry(c, x, w);
}
// The nw entries of every strong-shock row (the worklist).
__global__ void __launch_bounds__(RED_THREADS, 3) k_jac_strong(Ctx c) {
    const int nw = c.g.ny > 1 ? 5 : 3;
    const long cnt = (long)c.ns->nstrong * nw;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < cnt; t += (long)gridDim.x * blockDim.x)
        jac_entry(c, c.strong_list[t / nw], (int)(t % nw));
}
// Row sums A 1 (summed in the row's entry order, as block_sum's terms :763), Jacobi
// inverse, and the set-up sums E = 1^T A 1, 1^T b, b^T b with b = -G.
__global__ void __launch_bounds__(RED_THREADS) k_jac_finish(Ctx c) {
    const bool twoD = c.g.ny > 1;
    double acc[3] = {0.0, 0.0, 0.0};
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < c.n) {
        const double aC = c.aC[x];
        double e = 0;
        e += aC; e += c.aW[x]; e += c.aE[x];
        if (twoD) { e += c.aS[x]; e += c.aN[x]; }
        c.A1[x] = e;
        c.dinv[x] = aC != 0 ? 1.0 / aC : 1.0;
        if (c.prec) {  // precision form: the SpMV's FP32 copy of the diagonals
            c.fC[x] = (float)aC; c.fW[x] = (float)c.aW[x]; c.fE[x] = (float)c.aE[x];
            if (twoD) { c.fS[x] = (float)c.aS[x]; c.fN[x] = (float)c.aN[x]; }
        }
        const double b = -c.G[x];
        acc[0] = e;
        acc[1] = b;
        acc[2] = b * b;
    }
    double tot[3];
    if (grid_fold<RedSum, 3>(acc, c.partials, &c.counters[1], tot) && threadIdx.x == 0) {
        c.ns->E = tot[0]; c.ns->sumb = tot[1]; c.ns->bb = tot[2];
    }
}
void launch_jac_entries(const Ctx& c, cudaStream_t st, int skip_strong) {
    SPB6G_MG_FORWARD(launch_jac_entries, mg_view(c), st, skip_strong);
    const int nw = c.g.ny > 1 ? 5 : 3;
    k_jac_entries<<<nw * ((c.n + RED_THREADS - 1) / RED_THREADS), RED_THREADS, 0, st>>>(c, skip_strong);
    count(c, 1);
}
void launch_jac_strong(const Ctx& c, cudaStream_t st) {
    SPB6G_MG_FORWARD(launch_jac_strong, mg_view(c), st);
    k_jac_strong<<<148 * 4, RED_THREADS, 0, st>>>(c);
    count(c, 1);
}
void launch_jac_finish(const Ctx& c, cudaStream_t st) {
    k_jac_finish<<<(c.n + RED_THREADS - 1) / RED_THREADS, RED_THREADS, 0, st>>>(c);
    count(c, 1);
}
void launch_jacobian(const Ctx& c, cudaStream_t st) {
    SPB6G_MG_FORWARD(launch_jacobian, mg_view(c), st);
    launch_jac_entries(c, st, 0);
    launch_jac_finish(c, st);
}

// ============================================================ BiCGStab (GMRES_Solver :752-794)
// Jacobi + Nicolaides preconditioner M^-1 r = D^-1 r + 1 (1^T r)/E.  The coarse
// term is carried through the matrix as A M^-1 r = A (D^-1 r) + (1^T r / E) A 1,
// so each iteration is four passes: p & q = A D^-1 p; v, s & u = A D^-1 s; t; x & r.
// Every pass runs one row per thread on a (nx/256, ny) grid.
struct Nbr {
    int w, e, s, n;
};
SPB6G_DEV Nbr neighbours(const Geom& g, int i, int j, int x) {
    Nbr r;
    if (i > 0 && i < g.nx - 1) { r.w = x - 1; r.e = x + 1; }
    else { r.w = mp_index(g, i - 1, j); r.e = mp_index(g, i + 1, j); }
    if (j > 0 && j < g.ny - 1) { r.s = x - g.nx; r.n = x + g.nx; }
    else { r.s = mp_index(g, i, j - 1); r.n = mp_index(g, i, j + 1); }
    return r;
}
// Row of the SpMV in the reference's entry order: self, W, E, S, N (Pressure_Subsystem_AX :737-741).
template <class F>
SPB6G_DEV double spmv_row(const Ctx& c, const Nbr& nb, int x, F val) {
    double s = 0;
    s += c.aC[x] * val(x);
    s += c.aW[x] * val(nb.w);
    s += c.aE[x] * val(nb.e);
    if (c.g.ny > 1) {
        s += c.aS[x] * val(nb.s);
        s += c.aN[x] * val(nb.n);
    }
    return s;
}
// Each block covers 256 columns of ROWS_PER_BLOCK rows; a thread folds its rows
// in row order, so every sum below is deterministic for a given grid.
constexpr int ROWS_PER_BLOCK = 4;
#define ROW_LOOP_BEGIN                                                           \
    const int i = blockIdx.x * blockDim.x + threadIdx.x;                         \
    if (i < c.g.nx)                                                              \
        for (int jj = 0; jj < ROWS_PER_BLOCK; jj++) {                            \
            const int j = blockIdx.y * ROWS_PER_BLOCK + jj;                      \
            if (j >= c.g.ny) break;                                              \
            const int x = i + j * c.g.nx;
#define ROW_LOOP_END }

__global__ void __launch_bounds__(RED_THREADS) k_bicg_init(Ctx c, double tol, int maxit) {
    const NewtonScalars ns = *c.ns;
    const double Einv = (ns.E != 0.0 && isfinite(ns.E)) ? 1.0 / ns.E : 0.0;
    const double cb = ns.sumb * Einv;
    double acc[2] = {0.0, 0.0};
    ROW_LOOP_BEGIN
        const Nbr nb = neighbours(c.g, i, j, x);
        auto xv = [&](int q) { return c.dinv[q] * (-c.G[q]) + cb; };
        const double Ax = spmv_row(c, nb, x, xv);
        const double r = -c.G[x] - Ax;
        c.dP[x] = xv(x);
        c.br[x] = r;
        c.br0[x] = r;
        c.bp[x] = 0.0;
        c.bv[x] = 0.0;
        acc[0] += r * r;
        acc[1] += r * c.A1[x];
    ROW_LOOP_END
    double tot[2];
    if (grid_fold<RedSum, 2>(acc, c.partials, &c.counters[2], tot) && threadIdx.x == 0) {
        BicgScalars& b = *c.bs_;
        b.rho = b.alpha = b.omega = 1.0;
        b.Einv = Einv;
        b.cb = cb;
        b.bn = sqrt(ns.bb) + 1e-300;
        b.rr = tot[0];
        b.r0r = tot[0];
        b.r0A1 = tot[1];
        b.tol = tol;
        b.maxit = maxit;
        b.iters = 0;
        // a failed Jacobian (closure failure) ends the solve before it starts
        b.status = ns.fail ? BICG_FAIL : (sqrt(b.rr) <= tol * b.bn ? BICG_CONV : (b.r0r == 0 ? BICG_FAIL : BICG_RUNNING));
    }
}
// pass 1: p = r + beta (p - omega v); q = A D^-1 p; sums 1^T p, r0^T q
__global__ void __launch_bounds__(RED_THREADS) k_bicg_p(Ctx c, const double* __restrict__ p_old, double* __restrict__ p_new) {
    const BicgScalars b = *c.bs_;
    if (b.status != BICG_RUNNING) return;
    const double beta = (b.r0r / b.rho) * (b.alpha / b.omega), om = b.omega;
    const double* __restrict__ br = c.br;
    const double* __restrict__ bv = c.bv;
    const double* __restrict__ dinv = c.dinv;
    double acc[2] = {0.0, 0.0};
    ROW_LOOP_BEGIN
        const Nbr nb = neighbours(c.g, i, j, x);
        auto pn = [&](int q) { return br[q] + beta * (p_old[q] - om * bv[q]); };
        const double p = pn(x);
        const double q = spmv_row(c, nb, x, [&](int k) { return dinv[k] * pn(k); });
        p_new[x] = p;
        c.bq[x] = q;
        acc[0] += p;
        acc[1] += c.br0[x] * q;
    ROW_LOOP_END
    double tot[2];
    if (grid_fold<RedSum, 2>(acc, c.partials, &c.counters[3], tot) && threadIdx.x == 0) {
        BicgScalars& B = *c.bs_;
        B.rho = B.r0r;
        B.cc = tot[0] * B.Einv;
        B.alpha = B.rho / (tot[1] + B.cc * B.r0A1);
    }
}
// pass 2: v = q + cc A1; s = r - alpha v; u = A D^-1 s; sums s^T s, 1^T s
__global__ void __launch_bounds__(RED_THREADS) k_bicg_s(Ctx c) {
    const BicgScalars b = *c.bs_;
    if (b.status != BICG_RUNNING) return;
    const double al = b.alpha, cc = b.cc;
    const double* __restrict__ br = c.br;
    const double* __restrict__ bq = c.bq;
    const double* __restrict__ A1 = c.A1;
    const double* __restrict__ dinv = c.dinv;
    double acc[2] = {0.0, 0.0};
    ROW_LOOP_BEGIN
        const Nbr nb = neighbours(c.g, i, j, x);
        auto sv = [&](int q) { return br[q] - al * (bq[q] + cc * A1[q]); };
        const double v = bq[x] + cc * A1[x];
        const double s = br[x] - al * v;
        const double u = spmv_row(c, nb, x, [&](int k) { return dinv[k] * sv(k); });
        c.bv[x] = v;
        c.bs[x] = s;
        c.bu[x] = u;
        acc[0] += s * s;
        acc[1] += s;
    ROW_LOOP_END
    double tot[2];
    if (grid_fold<RedSum, 2>(acc, c.partials, &c.counters[4], tot) && threadIdx.x == 0) {
        BicgScalars& B = *c.bs_;
        B.ss = tot[0];
        B.cs = tot[1] * B.Einv;
        if (sqrt(tot[0]) <= B.tol * B.bn) B.status = BICG_CONV_HALF;
    }
}
// pass 3: t = u + cs A1; sums t^T s, t^T t
__global__ void __launch_bounds__(RED_THREADS) k_bicg_t(Ctx c) {
    const BicgScalars b = *c.bs_;
    if (b.status != BICG_RUNNING) return;
    double acc[2] = {0.0, 0.0};
    ROW_LOOP_BEGIN
        const double t = c.bu[x] + b.cs * c.A1[x];
        c.bt[x] = t;
        acc[0] += t * c.bs[x];
        acc[1] += t * t;
    ROW_LOOP_END
    double tot[2];
    if (grid_fold<RedSum, 2>(acc, c.partials, &c.counters[5], tot) && threadIdx.x == 0) {
        BicgScalars& B = *c.bs_;
        B.ts = tot[0];
        B.tt = tot[1];
        B.omega = tot[0] / tot[1];
    }
}
// pass 4: x += alpha ph + omega sh; r = s - omega t; sums r^T r, r0^T r
__global__ void __launch_bounds__(RED_THREADS) k_bicg_x(Ctx c, const double* __restrict__ p) {
    const BicgScalars b = *c.bs_;
    if (b.status != BICG_RUNNING && b.status != BICG_CONV_HALF) return;
    const bool half = b.status == BICG_CONV_HALF;
    double acc[2] = {0.0, 0.0};
    ROW_LOOP_BEGIN
        const double ph = c.dinv[x] * p[x] + b.cc;
        if (half) {
            c.dP[x] += b.alpha * ph;
        } else {
            const double sh = c.dinv[x] * c.bs[x] + b.cs;
            c.dP[x] += b.alpha * ph + b.omega * sh;
            const double r = c.bs[x] - b.omega * c.bt[x];
            c.br[x] = r;
            acc[0] += r * r;
            acc[1] += c.br0[x] * r;
        }
    ROW_LOOP_END
    double tot[2];
    if (grid_fold<RedSum, 2>(acc, c.partials, &c.counters[6], tot) && threadIdx.x == 0) {
        BicgScalars& B = *c.bs_;
        B.iters += 1;
        if (half) { B.status = BICG_CONV; return; }
        B.rr = tot[0];
        B.r0r = tot[1];
        if (sqrt(B.rr) <= B.tol * B.bn) B.status = BICG_CONV;
        else if (B.iters >= B.maxit) B.status = sqrt(B.rr) <= 1e3 * B.tol * B.bn ? BICG_CONV : BICG_FAIL;
        else if (B.r0r == 0) B.status = BICG_FAIL;
        else if (!isfinite(B.rr)) B.status = BICG_FAIL;  // NaN never converges; the reference loops to GMRESiter and fails
    }
}
// Loop condition of the device-side iteration: continue while the solve is running.
__global__ void k_bicg_cond(const BicgScalars* b, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, b->status == BICG_RUNNING ? 1u : 0u);
}
static dim3 row_grid(const Ctx& c) {
    return dim3((unsigned)((c.g.nx + RED_THREADS - 1) / RED_THREADS), (unsigned)((c.g.ny + ROWS_PER_BLOCK - 1) / ROWS_PER_BLOCK));
}
void launch_bicg_init(const Ctx& c, cudaStream_t st, double tol, int maxit) {
    k_bicg_init<<<row_grid(c), RED_THREADS, 0, st>>>(c, tol, maxit);
    count(c, 1);
}
static void enqueue_iteration(const Ctx& c, cudaStream_t st, const dim3& gr, double* p_old, double* p_new) {
    k_bicg_p<<<gr, RED_THREADS, 0, st>>>(c, p_old, p_new);
    k_bicg_s<<<gr, RED_THREADS, 0, st>>>(c);
    k_bicg_t<<<gr, RED_THREADS, 0, st>>>(c);
    k_bicg_x<<<gr, RED_THREADS, 0, st>>>(c, p_new);
}
// `count` iterations.  p is double-buffered (pass 1 reads neighbours' old p
// while writing the new one); `parity` selects the buffer holding the current p.
void launch_bicg_iters(const Ctx& c, cudaStream_t st, int count_, int& parity) {
    const dim3 gr = row_grid(c);
    for (int k = 0; k < count_; k++) {
        double* p0 = parity ? c.tcp : c.bp;  // tcp is the Thomas scratch, free on the BiCGStab path
        double* p1 = parity ? c.bp : c.tcp;
        enqueue_iteration(c, st, gr, p0, p1);
        parity ^= 1;
    }
    count(c, 4 * count_);
}
// The whole BiCGStab loop as one graph launch: a while-node whose body is two
// iterations (the p buffers alternate) and the condition kernel.  The loop ends
// on the device when the status leaves RUNNING (converged, failed, or GMRESiter
// reached); no host round trip per iteration.  Kernel arguments are the solver's
// fixed buffers, so the graph is built once per solver.
int build_bicg_graph(const Ctx& c, cudaStream_t st, cudaGraphExec_t* exec) {
    cudaGraph_t graph = nullptr;
    if (cudaGraphCreate(&graph, 0) != cudaSuccess) return -1;
    cudaGraphConditionalHandle h;
    if (cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault) != cudaSuccess) return -2;
    cudaGraphNodeParams params = {};
    params.type = cudaGraphNodeTypeConditional;
    params.conditional.handle = h;
    params.conditional.type = cudaGraphCondTypeWhile;
    params.conditional.size = 1;
    cudaGraphNode_t node;
    if (cudaGraphAddNode(&node, graph, nullptr, 0, &params) != cudaSuccess) return -3;
    cudaGraph_t body = params.conditional.phGraph_out[0];
    if (cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return -4;
    const dim3 gr = row_grid(c);
    enqueue_iteration(c, st, gr, c.bp, c.tcp);
    enqueue_iteration(c, st, gr, c.tcp, c.bp);
    k_bicg_cond<<<1, 1, 0, st>>>(c.bs_, h);
    cudaGraph_t captured = nullptr;
    if (cudaStreamEndCapture(st, &captured) != cudaSuccess) return -5;
    if (cudaGraphInstantiate(exec, graph, 0) != cudaSuccess) return -6;
    cudaGraphDestroy(graph);
    return 0;
}
void launch_bicg_graph(const Ctx& c, cudaStream_t st, cudaGraphExec_t exec, int expected_iters) {
    cudaGraphLaunch(exec, st);
    count(c, 4 * (expected_iters + (expected_iters & 1)) + (expected_iters + 2) / 2);
}

// ============================================================ BiCGStab, persistent form
// The whole solve (set-up and every iteration of GMRES_Solver :752-794) in one
// cooperative launch: every block stays resident, owns the row chunks
// blockIdx.x, blockIdx.x + G, ... (PB_THREADS rows each) for the whole solve, and
// the four passes of an iteration are separated by a software grid barrier.
// Each barrier carries one reduction: blocks publish their partial sums, and
// after the barrier every block folds all G partials in block order, so every
// block holds bit-identical scalars without a further round trip.  The
// arithmetic per row is the one of the four-pass kernels above.
constexpr unsigned BARRIER_SPIN_LIMIT = 1u << 21;  // polls of >= 0.3 us each: gives up after about a second

SPB6G_DEV unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
SPB6G_DEV int ld_relaxed_gpu(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Grid barrier on a monotone arrival counter: thread 0 of every block adds 1
// with release semantics, and barrier number e of a launch is complete once the
// counter reaches e * G (acquire polls).  The counter is cleared before every
// launch.  The wait is bounded: past BARRIER_SPIN_LIMIT polls, or once another
// block has given up, the block records the failure and returns false.
SPB6G_DEV bool barrier_arrive_wait(GridBarrier* gb, unsigned target) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&gb->count) : "memory");
    unsigned it = 0;
    while (ld_acquire_gpu(&gb->count) < target) {
        if (++it > BARRIER_SPIN_LIMIT || ld_relaxed_gpu(&gb->err)) {
            atomicExch(&gb->err, 1);
            return false;
        }
    }
    return true;
}

// Publishes this block's NQ partial sums (records of PB_SLOT_Q), waits for every
// block, and folds all G records in block order in warp 0; `tot` is then the same
// in every thread of every block.  `epoch` counts the barriers of the launch.
template <int NQ>
SPB6G_DEV bool sync_fold(double (&acc)[NQ], double* slot, unsigned G, GridBarrier* gb, unsigned& epoch, double (&tot)[NQ]) {
    static_assert(NQ <= PB_SLOT_Q, "a barrier record holds PB_SLOT_Q sums");
    __shared__ double sh[NQ * 32];
    __shared__ double bc[NQ];
    __shared__ int s_ok;
    block_fold<RedSum, NQ>(acc, sh);
    epoch += 1;
    if (threadIdx.x < 32) {
        int ok = 1;
        if (threadIdx.x == 0) {
#pragma unroll
            for (int q = 0; q < NQ; q++) slot[PB_SLOT_Q * blockIdx.x + q] = acc[q];
            ok = barrier_arrive_wait(gb, epoch * G) ? 1 : 0;
        }
        ok = __shfl_sync(0xffffffffu, ok, 0);
        __syncwarp();
        if (ok) {
            double f[NQ];
#pragma unroll
            for (int q = 0; q < NQ; q++) f[q] = 0.0;
            for (unsigned b = threadIdx.x; b < G; b += 32) {
#pragma unroll
                for (int q = 0; q < NQ; q++) f[q] += __ldcg(slot + PB_SLOT_Q * b + q);
            }
#pragma unroll
            for (int q = 0; q < NQ; q++) f[q] = warp_fold<RedSum>(f[q]);
            if (threadIdx.x == 0) {
#pragma unroll
                for (int q = 0; q < NQ; q++) bc[q] = f[q];
            }
        }
        if (threadIdx.x == 0) s_ok = ok;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NQ; q++) tot[q] = bc[q];
    return s_ok != 0;
}

// Work unit of the persistent passes: a strip of 32 columns x J rows owned by one
// warp for the whole solve.  Lane l holds column i0 + l and walks the rows
// upward; west / east neighbours come from the row's values in shared memory,
// south / north ones from the rows below and above, which the walk loads anyway.
// Rows arrive through a PS_D-deep cp.async pipeline (loads for row t + PS_D - 1
// are in flight while row t is used), so each warp keeps several rows of every
// operand in flight instead of one.
constexpr int PB_WARPS = PB_THREADS / 32;
constexpr int PS_D = 4;                           // rows in flight per warp
constexpr int PS_HV = 4;                          // operands needed at the neighbours (34 columns)
constexpr int PS_RV = 6;                          // operands needed at the row itself (32 columns)
constexpr int PS_STAGE = PS_HV * 34 + PS_RV * 32;  // doubles per row stage
constexpr int PS_WARP = PS_D * PS_STAGE + 3 * 34;  // + three rows of scaled stencil values
constexpr size_t PB_SMEM = (size_t)PB_WARPS * PS_WARP * sizeof(double);

struct Strip {
    int i0, j0, J;
};
struct StripGrid {
    int ncols, J, nstrips;
};
SPB6G_DEV StripGrid strip_grid(const Geom& g, int warps) {
    StripGrid s;
    s.ncols = (g.nx + 31) / 32;
    const long cells = (long)g.ny * s.ncols;
    s.J = (int)((cells + warps - 1) / warps);
    if (s.J < 1) s.J = 1;
    s.nstrips = s.ncols * ((g.ny + s.J - 1) / s.J);
    return s;
}
SPB6G_DEV Strip strip_at(const Geom& g, const StripGrid& sg, int s) {
    Strip st;
    st.i0 = (s % sg.ncols) * 32;
    st.j0 = (s / sg.ncols) * sg.J;
    st.J = min(sg.J, g.ny - st.j0);
    return st;
}
// Column / row of the pressure-unknown map M_P (mp_index is separable); columns
// beyond the east neighbour of the last cell are never used and read column 0.
SPB6G_DEV int map_col(const Geom& g, int i) {
    if (i < -1 || i > g.nx) return 0;
    const bool xp = g.bcs[0] == BC_PERIODIC;
    if (i < 0) return xp ? g.nx + i : 0;
    if (i > g.nx - 1) return xp ? i - g.nx : g.nx - 1;
    return i;
}
SPB6G_DEV int map_row(const Geom& g, int j) {
    const bool yp = g.bcs[2] == BC_PERIODIC && g.ny > 1;
    if (j < 0) return yp ? g.ny + j : 0;
    if (j > g.ny - 1) return yp ? j - g.ny : g.ny - 1;
    return j;
}
SPB6G_DEV void cp_async8(double* s, const double* gp) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(s)), "l"(gp) : "memory");
}
SPB6G_DEV void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
SPB6G_DEV void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Five-point pass over one strip.  hv: the PS_HV operands of the scaled stencil
// value ph(k) (rows j0-1 .. j0+J, columns i0-1 .. i0+32, boundary-mapped);
// mat: the five matrix diagonals (self, W, E, S, N) at the row itself, of type MT
// (FP64, or FP32 in the precision form); ex: NEX FP64 operands at the row itself.
// phf(stage, col) gives ph from a row stage; out(a, e, stage, col, phS, phW, phC,
// phE, phN, x) consumes a row, a[m * 32] being diagonal m and e[v * 32] operand v.
constexpr int PS_HV_BYTES = PS_HV * 34 * 8;
template <class MT>
SPB6G_DEV void cp_async_el(MT* s, const MT* gp) {
    if constexpr (sizeof(MT) == 8) cp_async8((double*)s, (const double*)gp);
    else asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(s)), "l"(gp) : "memory");
}
template <class MT, int NEX, class PH, class OUT>
SPB6G_DEV void stencil_strip(const Geom& g, const Strip& st, double* ws, const double* const (&hv)[PS_HV],
                             const MT* const (&mat)[5], const double* const* ex, PH phf, OUT out) {
    const int lane = threadIdx.x & 31;
    const int nload = st.J + 2;
    double* stages = ws;
    double* phr = ws + PS_D * PS_STAGE;
    const int ic_own = map_col(g, st.i0 + lane);
    const int ic_halo = lane == 0 ? map_col(g, st.i0 - 1) : map_col(g, st.i0 + 32);
    const bool own = st.i0 + lane < g.nx;
    auto matp = [&](double* sp) { return (MT*)((char*)sp + PS_HV_BYTES); };
    auto exp_ = [&](double* sp) { return (double*)((char*)sp + PS_HV_BYTES + 5 * 32 * sizeof(MT)); };
    auto issue = [&](int t) {
        if (t < nload) {
            double* sp = stages + (t % PS_D) * PS_STAGE;
            const size_t rb = (size_t)map_row(g, st.j0 - 1 + t) * g.nx;
#pragma unroll
            for (int v = 0; v < PS_HV; v++) cp_async8(sp + v * 34 + lane + 1, hv[v] + rb + ic_own);
            if (lane < 2) {
#pragma unroll
                for (int v = 0; v < PS_HV; v++) cp_async8(sp + v * 34 + (lane ? 33 : 0), hv[v] + rb + ic_halo);
            }
            if (own && t >= 1 && t <= st.J) {
                MT* mp = matp(sp);
#pragma unroll
                for (int m = 0; m < 5; m++) cp_async_el<MT>(mp + m * 32 + lane, mat[m] + rb + ic_own);
                double* ep = exp_(sp);
#pragma unroll
                for (int v = 0; v < NEX; v++) cp_async8(ep + v * 32 + lane, ex[v] + rb + ic_own);
            }
        }
        cp_commit();
    };
#pragma unroll
    for (int t = 0; t < PS_D - 1; t++) issue(t);
    for (int t = 0; t < nload; t++) {
        cp_wait<PS_D - 2>();
        __syncwarp();
        const double* sp = stages + (t % PS_D) * PS_STAGE;
        double* pr = phr + (t % 3) * 34;
        pr[lane + 1] = phf(sp, lane + 1);
        if (lane < 2) pr[lane ? 33 : 0] = phf(sp, lane ? 33 : 0);
        __syncwarp();
        if (t >= 2 && own) {
            double* so = stages + ((t - 1) % PS_D) * PS_STAGE;
            const double* pS = phr + ((t - 2) % 3) * 34;
            const double* pC = phr + ((t - 1) % 3) * 34;
            out((const MT*)matp(so) + lane, (const double*)exp_(so) + lane, (const double*)so, lane + 1, pS[lane + 1],
                pC[lane], pC[lane + 1], pC[lane + 2], pr[lane + 1], (st.j0 + t - 2) * g.nx + st.i0 + lane);
        }
        __syncwarp();
        issue(t + PS_D - 1);
    }
    cp_wait<0>();
    __syncwarp();
}
// Row-local pass over one strip: NRV operands of each own cell through the same pipeline.
template <int NRV, class OUT>
SPB6G_DEV void row_strip(const Geom& g, const Strip& st, double* ws, const double* const (&rv)[NRV], OUT out) {
    const int lane = threadIdx.x & 31;
    const bool own = st.i0 + lane < g.nx;
    auto issue = [&](int t) {
        if (t < st.J && own) {
            double* sp = ws + (t % PS_D) * PS_STAGE;
            const size_t x = (size_t)(st.j0 + t) * g.nx + st.i0 + lane;
#pragma unroll
            for (int v = 0; v < NRV; v++) cp_async8(sp + v * 32 + lane, rv[v] + x);
        }
        cp_commit();
    };
#pragma unroll
    for (int t = 0; t < PS_D - 1; t++) issue(t);
    for (int t = 0; t < st.J; t++) {
        cp_wait<PS_D - 2>();
        __syncwarp();
        if (own) out(ws + (t % PS_D) * PS_STAGE, lane, (st.j0 + t) * g.nx + st.i0 + lane);
        __syncwarp();
        issue(t + PS_D - 1);
    }
    cp_wait<0>();
    __syncwarp();
}

// The five diagonals in the SpMV's precision.
template <class MT>
SPB6G_DEV const MT* diag(const Ctx& c, int m);
template <>
SPB6G_DEV const double* diag<double>(const Ctx& c, int m) {
    return m == 0 ? c.aC : m == 1 ? c.aW : m == 2 ? c.aE : m == 3 ? c.aS : c.aN;
}
template <>
SPB6G_DEV const float* diag<float>(const Ctx& c, int m) {
    return m == 0 ? c.fC : m == 1 ? c.fW : m == 2 ? c.fE : m == 3 ? c.fS : c.fN;
}

#define PB_STRIPS_BEGIN                                                         \
    for (int s_ = wid; s_ < sg.nstrips; s_ += nwarps) {                         \
        const Strip st = strip_at(c.g, sg, s_);
#define PB_STRIPS_END }

// Three passes per iteration.  Besides the A 1 trick of the four-pass kernels
// (A M^-1 r = A (D^-1 r) + (1^T r / E) A 1), the coarse coefficient of s is
// formed from sums the first barrier already carries: 1^T s = 1^T r - alpha 1^T v
// with 1^T v = 1^T q + cc 1^T A1, so t = A M^-1 s and its two inner products are
// finished in the same pass as s (the reference sums s itself; the identity is
// exact, the rounding of this one scalar differs).
template <class MT>
__global__ void __launch_bounds__(PB_THREADS, 1) k_bicg_solve(Ctx c, double tol, int maxit) {
    extern __shared__ double pb_smem[];
    const int n = c.n, nx = c.g.nx;
    const unsigned G = gridDim.x;
    const int nwarps = G * PB_WARPS, wid = blockIdx.x * PB_WARPS + (threadIdx.x >> 5);
    double* ws = pb_smem + (threadIdx.x >> 5) * PS_WARP;
    const StripGrid sg = strip_grid(c.g, nwarps);
    const bool two_d = c.g.ny > 1;
    GridBarrier* gb = c.gbar;
    unsigned epoch = 0;
    double* slots = c.gpart;  // G records of PB_SLOT_Q per barrier, two barriers apart
    const double* __restrict__ dinv = c.dinv;
    const double* __restrict__ A1 = c.A1;
    double* __restrict__ br = c.br;
    double* __restrict__ bv = c.bv;
    double* __restrict__ bq = c.bq;
    double* __restrict__ bs = c.bs;
    double* __restrict__ bt = c.bt;
    double* __restrict__ dP = c.dP;
    auto slot = [&](int k) { return slots + (size_t)(k & 1) * PB_SLOT_Q * G; };
    const MT* const mat[5] = {diag<MT>(c, 0), diag<MT>(c, 1), diag<MT>(c, 2), diag<MT>(c, 3), diag<MT>(c, 4)};

    const NewtonScalars ns = *c.ns;
    const double Einv = (ns.E != 0.0 && isfinite(ns.E)) ? 1.0 / ns.E : 0.0;
    const double cb = ns.sumb * Einv;
    const double* __restrict__ x0l = c.x0l;
    int bar = 0;
    // Learned first iterate (no counterpart in the reference): the start is x0 = a M^-1 b + c xl,
    // (a, c) minimising ||b - A x0||_2 over that plane, used only when its residual is below
    // 0.99 of the plain start's ||b - A M^-1 b||; otherwise the plain start x0 = M^-1 b stands.
    // A pass forms u = A M^-1 b and w = A xl (kept in br and bq) and the five inner products.
    bool use_l = false;
    double la = 1.0, lc = 0.0;
    if (x0l) {
        double a5[5] = {0.0, 0.0, 0.0, 0.0, 0.0}, t5[5];
        for (int x = blockIdx.x * PB_THREADS + threadIdx.x; x < n; x += G * PB_THREADS) {
            const int j = x / nx, i = x - j * nx;
            const Nbr nb = neighbours(c.g, i, j, x);
            const double u = spmv_row(c, nb, x, [&](int q) { return dinv[q] * (-c.G[q]) + cb; });
            const double w = spmv_row(c, nb, x, [&](int q) { return x0l[q]; });
            const double b = -c.G[x];
            br[x] = u;
            bq[x] = w;
            a5[0] += b * u;
            a5[1] += u * u;
            a5[2] += b * w;
            a5[3] += u * w;
            a5[4] += w * w;
        }
        if (!sync_fold<5>(a5, slot(bar++), G, gb, epoch, t5)) goto timeout;
        const double bu = t5[0], uu = t5[1], bw = t5[2], uw = t5[3], ww = t5[4];
        const double det = uu * ww - uw * uw;
        if (isfinite(det) && det > 1e-12 * uu * ww) {
            const double a = (bu * ww - bw * uw) / det, cl = (bw * uu - bu * uw) / det;
            // squared residuals: the plane's minimum and the plain start's
            const double r_l = ns.bb - (a * bu + cl * bw), r_p = ns.bb - 2.0 * bu + uu;
            if (isfinite(a) && isfinite(cl) && r_l < 0.99 * r_p) {
                use_l = true;
                la = a;
                lc = cl;
            }
        }
    }
    {
    // set-up: x = x0, r = r0 = b - A x, p = v = 0 (plain row loop, once per solve)
    double a4[4] = {0.0, 0.0, 0.0, 0.0}, t4[4];
    for (int x = blockIdx.x * PB_THREADS + threadIdx.x; x < n; x += G * PB_THREADS) {
        const int j = x / nx, i = x - j * nx;
        auto xv = [&](int q) { return dinv[q] * (-c.G[q]) + cb; };
        double r;
        if (!x0l) {
            const Nbr nb = neighbours(c.g, i, j, x);
            const double Ax = spmv_row(c, nb, x, xv);
            r = -c.G[x] - Ax;
            dP[x] = xv(x);
        } else if (!use_l) {
            r = -c.G[x] - br[x];
            dP[x] = xv(x);
        } else {
            r = -c.G[x] - la * br[x] - lc * bq[x];
            dP[x] = la * xv(x) + lc * x0l[x];
        }
        br[x] = r;
        c.br0[x] = r;
        c.bp[x] = 0.0;
        bv[x] = 0.0;
        a4[0] += r * r;
        a4[1] += r * A1[x];
        a4[2] += r;
        a4[3] += A1[x];
    }
    if (!sync_fold<4>(a4, slot(bar++), G, gb, epoch, t4)) goto timeout;
    {
        double rho = 1.0, alpha = 1.0, omega = 1.0, cc = 0.0, cs = 0.0, ss = 0.0, ts = 0.0, tt = 0.0;
        const double bn = sqrt(ns.bb) + 1e-300;
        double rr = t4[0], r0r = t4[0], sr = t4[2];
        const double r0A1 = t4[1], sA1 = t4[3];
        int status = ns.fail ? BICG_FAIL : (sqrt(rr) <= tol * bn ? BICG_CONV : (r0r == 0 ? BICG_FAIL : BICG_RUNNING));
        int iters = 0, parity = 0;
        double a3[3], t3[3];
        while (status == BICG_RUNNING) {
            const double* p_old = parity ? c.tcp : c.bp;
            double* p_new = parity ? c.bp : c.tcp;
            // pass 1: p = r + beta (p - omega v); q = A D^-1 p; sums 1^T p, r0^T q, 1^T q
            {
                const double beta = (r0r / rho) * (alpha / omega), om = omega;
                const double* const hv[PS_HV] = {br, p_old, bv, dinv};
                const double* const ex[1] = {c.br0};
                auto pn = [&](const double* sp, int k) { return sp[k] + beta * (sp[34 + k] - om * sp[68 + k]); };
                auto phf = [&](const double* sp, int k) { return sp[102 + k] * pn(sp, k); };
                a3[0] = a3[1] = a3[2] = 0.0;
                PB_STRIPS_BEGIN
                    stencil_strip<MT, 1>(c.g, st, ws, hv, mat, ex, phf,
                        [&](const MT* a, const double* e, const double* so, int k, double phS, double phW, double phC,
                            double phE, double phN, int x) {
                            const double p = pn(so, k);
                            MT qm = 0;  // the SpMV row in the matrix precision
                            qm += a[0] * (MT)phC;
                            qm += a[32] * (MT)phW;
                            qm += a[64] * (MT)phE;
                            if (two_d) {
                                qm += a[96] * (MT)phS;
                                qm += a[128] * (MT)phN;
                            }
                            const double q = (double)qm;
                            p_new[x] = p;
                            bq[x] = q;
                            a3[0] += p;
                            a3[1] += e[0] * q;
                            a3[2] += q;
                        });
                PB_STRIPS_END
            }
            if (!sync_fold<3>(a3, slot(bar++), G, gb, epoch, t3)) goto timeout;
            rho = r0r;
            cc = t3[0] * Einv;
            alpha = rho / (t3[1] + cc * r0A1);
            cs = (sr - alpha * (t3[2] + cc * sA1)) * Einv;
            // pass 2: v = q + cc A1; s = r - alpha v; t = A D^-1 s + cs A1; sums s^T s, t^T s, t^T t
            {
                const double al = alpha, ccv = cc, csv = cs;
                const double* const hv[PS_HV] = {br, bq, A1, dinv};
                auto sv = [&](const double* sp, int k) { return sp[k] - al * (sp[34 + k] + ccv * sp[68 + k]); };
                auto phf = [&](const double* sp, int k) { return sp[102 + k] * sv(sp, k); };
                a3[0] = a3[1] = a3[2] = 0.0;
                PB_STRIPS_BEGIN
                    stencil_strip<MT, 0>(c.g, st, ws, hv, mat, nullptr, phf,
                        [&](const MT* a, const double*, const double* so, int k, double phS, double phW, double phC,
                            double phE, double phN, int x) {
                            const double v = so[34 + k] + ccv * so[68 + k];
                            const double s = so[k] - al * v;
                            MT um = 0;
                            um += a[0] * (MT)phC;
                            um += a[32] * (MT)phW;
                            um += a[64] * (MT)phE;
                            if (two_d) {
                                um += a[96] * (MT)phS;
                                um += a[128] * (MT)phN;
                            }
                            const double u = (double)um;
                            const double tv = u + csv * so[68 + k];
                            bv[x] = v;
                            bs[x] = s;
                            bt[x] = tv;
                            a3[0] += s * s;
                            a3[1] += tv * s;
                            a3[2] += tv * tv;
                        });
                PB_STRIPS_END
            }
            if (!sync_fold<3>(a3, slot(bar++), G, gb, epoch, t3)) goto timeout;
            ss = t3[0];
            const bool half = sqrt(ss) <= tol * bn;
            if (!half) {
                ts = t3[1];
                tt = t3[2];
                omega = ts / tt;
            }
            // pass 3: x += alpha ph + omega sh; r = s - omega t; sums r^T r, r0^T r, 1^T r
            a3[0] = a3[1] = a3[2] = 0.0;
            if (half) {
                const double al = alpha, ccv = cc;
                const double* const rv[3] = {dinv, p_new, dP};
                PB_STRIPS_BEGIN
                    row_strip<3>(c.g, st, ws, rv, [&](const double* sp, int k, int x) {
                        const double ph = sp[k] * sp[32 + k] + ccv;
                        dP[x] = sp[64 + k] + al * ph;
                    });
                PB_STRIPS_END
            } else {
                const double al = alpha, om = omega, ccv = cc, csv = cs;
                const double* const rv[6] = {dinv, p_new, bs, bt, dP, c.br0};
                PB_STRIPS_BEGIN
                    row_strip<6>(c.g, st, ws, rv, [&](const double* sp, int k, int x) {
                        const double ph = sp[k] * sp[32 + k] + ccv;
                        const double sh = sp[k] * sp[64 + k] + csv;
                        dP[x] = sp[128 + k] + (al * ph + om * sh);
                        const double r = sp[64 + k] - om * sp[96 + k];
                        br[x] = r;
                        a3[0] += r * r;
                        a3[1] += sp[160 + k] * r;
                        a3[2] += r;
                    });
                PB_STRIPS_END
            }
            iters += 1;
            if (half) { status = BICG_CONV; break; }
            if (!sync_fold<3>(a3, slot(bar++), G, gb, epoch, t3)) goto timeout;
            rr = t3[0];
            r0r = t3[1];
            sr = t3[2];
            if (sqrt(rr) <= tol * bn) status = BICG_CONV;
            else if (iters >= maxit) status = sqrt(rr) <= 1e3 * tol * bn ? BICG_CONV : BICG_FAIL;
            else if (r0r == 0) status = BICG_FAIL;
            else if (!isfinite(rr)) status = BICG_FAIL;  // NaN never converges; the reference loops to GMRESiter and fails
            parity ^= 1;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            BicgScalars& B = *c.bs_;
            B.rho = rho; B.alpha = alpha; B.omega = omega; B.bn = bn; B.Einv = Einv; B.cb = cb;
            B.r0A1 = r0A1; B.cc = cc; B.cs = cs; B.rr = rr; B.r0r = r0r; B.ts = ts; B.tt = tt; B.ss = ss;
            B.tol = tol; B.maxit = maxit; B.iters = iters; B.status = status; B.x0_learned = use_l ? 1 : 0;
        }
        return;
    }
    }
timeout:
    if (threadIdx.x == 0) c.bs_->status = BICG_TIMEOUT;
}
#undef PB_STRIPS_BEGIN
#undef PB_STRIPS_END

int bicg_solve_blocks(int device, int n) {
    int per_sm = 0, sms = 0, coop = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device) != cudaSuccess || !coop) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    if (cudaFuncSetAttribute(k_bicg_solve<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PB_SMEM) != cudaSuccess ||
        cudaFuncSetAttribute(k_bicg_solve<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PB_SMEM) != cudaSuccess)
        return 0;
    int per_sm_f = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bicg_solve<double>, PB_THREADS, PB_SMEM) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f, k_bicg_solve<float>, PB_THREADS, PB_SMEM) != cudaSuccess)
        return 0;
    if (per_sm_f < per_sm) per_sm = per_sm_f;
    // about four rows per thread at least: small grids use fewer blocks (cheaper barriers)
    const long want = ((long)n + 4L * PB_THREADS - 1) / (4L * PB_THREADS);
    long G = (long)per_sm * sms;
    if (G > want) G = want;
    return G > 0 ? (int)G : 0;
}
int launch_bicg_solve(const Ctx& c, cudaStream_t st, double tol, int maxit, int G) {
    void* args[] = {(void*)&c, (void*)&tol, (void*)&maxit};
    count(c, 1);
    const void* fn = c.prec ? (const void*)k_bicg_solve<float> : (const void*)k_bicg_solve<double>;
    return cudaLaunchCooperativeKernel(fn, dim3(G), dim3(PB_THREADS), args, PB_SMEM, st) == cudaSuccess ? 0 : -1;
}

// ============================================================ learned warm start (no counterpart in the reference)
// Scale of the pressure rate: sigma = RMS of R over the cells (rate_sc[0]), or the
// normalisation's target scale before the first converged stage.
SPB6G_DEV double rate_scale(const Ctx& c, double tscale) {
    const double s = c.rate_sc ? c.rate_sc[0] : 0.0;
    return s > 0.0 ? s : tscale;
}
// Feature row of cell (i, j): for each field f of (rho, rho u, rho v, alpha1, E*, P, R / sigma)
// -- the first five from the explicit predictor X* (boundary-mapped like every
// stencil read), P the stage's starting pressure and R the pressure rate of the
// last converged stage (both through M_P; R = 0 before the first) -- the centre
// value normalised as (v - mean_f) / std_f, then the 8 neighbours (rows below,
// same row, above; west to east) as differences to the centre over dstd_f; the
// 64th value is the centre's last rate change (R - R2) / sigma.  BF16.
constexpr double FEAT_CLAMP = 1024.0;
// One block per FT_X x FT_Y tile: the seven fields of the tile and its one-cell ring go to shared
// memory once (each through the boundary maps, as every stencil read), then every thread forms its
// cell's row from there.  Neighbour m = 1..8 of the row runs over the rows below, the same row and
// the rows above, west to east.
constexpr int FT_X = 32, FT_Y = 8;
__global__ void __launch_bounds__(FT_X * FT_Y, 3) k_features(Ctx c, FeatureNorm nm, __nv_bfloat16* __restrict__ X) {
    __shared__ double F[NFIELD][FT_Y + 2][FT_X + 2];
    const Geom& g = c.g;
    const double isig = 1.0 / rate_scale(c, nm.tscale);
    const int i0 = blockIdx.x * FT_X, j0 = blockIdx.y * FT_Y;
    for (int t = threadIdx.x; t < (FT_X + 2) * (FT_Y + 2); t += FT_X * FT_Y) {
        const int lx = t % (FT_X + 2), ly = t / (FT_X + 2);
        const int i = i0 - 1 + lx, j = j0 - 1 + ly;
        if (i > g.nx || j > g.ny) continue;  // beyond the ring of the last cells
        double q[NV];
        xs_at(c, i, j, q);
        const int m = mp_index(g, i, j);
        F[0][ly][lx] = q[IM1] + q[IM2];
        F[1][ly][lx] = q[IMU];
        F[2][ly][lx] = q[IMV];
        F[3][ly][lx] = q[IA1];
        F[4][ly][lx] = q[IEN];
        F[5][ly][lx] = c.P[m];
        F[6][ly][lx] = c.Prate ? c.Prate[m] * isig : 0.0;
    }
    __syncthreads();
    const int li = threadIdx.x % FT_X, lj = threadIdx.x / FT_X;
    const int i = i0 + li, j = j0 + lj;
    if (i >= g.nx || j >= g.ny) return;
    const size_t x = (size_t)j * g.nx + i;
    // normalised values are clamped to +-FEAT_CLAMP (a field that was constant in the pilot
    // run has a tiny scale), and a non-finite value reads as 0
    auto fb = [](double z) {
        z = z == z ? fmin(fmax(z, -FEAT_CLAMP), FEAT_CLAMP) : 0.0;
        return __float2bfloat16_rn((float)z);
    };
    constexpr int DI[9] = {0, -1, 0, 1, -1, 1, -1, 0, 1}, DJ[9] = {0, -1, -1, -1, 0, 0, 1, 1, 1};
    auto value = [&](int idx) -> __nv_bfloat16 {
        if (idx == 63) return fb(c.Prate ? (c.Prate[x] - c.Prate2[x]) * isig : 0.0);
        const int f = idx / 9, m = idx % 9;
        const double v0 = F[f][lj + 1][li + 1];
        if (m == 0) return fb((v0 - nm.mean[f]) * nm.istd[f]);
        return fb((F[f][lj + 1 + DJ[m]][li + 1 + DI[m]] - v0) * nm.idstd[f]);
    };
    uint4* dst = (uint4*)(X + x * 64);
#pragma unroll
    for (int q = 0; q < 8; q++) {
        unsigned w[4];
#pragma unroll
        for (int h = 0; h < 4; h++) {
            const __nv_bfloat162 p2 = __halves2bfloat162(value(8 * q + 2 * h), value(8 * q + 2 * h + 1));
            w[h] = *reinterpret_cast<const unsigned*>(&p2);
        }
        dst[q] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}
void launch_features(const Ctx& c, cudaStream_t st, const FeatureNorm& nm, void* X) {
    SPB6G_MG_FORWARD(launch_features, mg_view(c), st, mg_view(nm), X);
    const dim3 grid((unsigned)((c.g.nx + FT_X - 1) / FT_X), (unsigned)((c.g.ny + FT_Y - 1) / FT_Y));
    k_features<<<grid, FT_X * FT_Y, 0, st>>>(c, nm, (__nv_bfloat16*)X);
    count(c, 1);
}
// Step towards a predicted pressure.  The network predicts how far the stage's pressure
// rate departs from the last stage's, in units of sigma: the learned guess is
// P_start + sdt (R + sigma y), the extrapolation (y = 0) P_start + sdt R.
// Step from the current start to a candidate: dP = sdt (a_r R + a_q (R - R2) + a_c (R2 - R3) +
// a_y sigma y), R the pressure rate of the last converged stage, R2 and R3 those of the two before.
__global__ void k_guess(Ctx c, const float* __restrict__ y, double tscale, double a_r, double a_q, double a_c, double a_y) {
    const double sig = rate_scale(c, tscale);
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const double r = c.Prate ? c.Prate[x] : 0.0;
        const double r2 = c.Prate2 ? c.Prate2[x] : r;
        const double r3 = c.Prate3 ? c.Prate3[x] : r2;
        const double d = y ? a_y * (double)y[x] * sig : 0.0;
        c.dP[x] = c.sdt * (a_r * r + a_q * (r - r2) + a_c * (r2 - r3) + d);
    }
}
void launch_guess(const Ctx& c, cudaStream_t st, const float* y, double tscale, double a_r, double a_q, double a_c,
                  double a_y) {
    k_guess<<<blocks_for(c.n), TPB, 0, st>>>(c, y, tscale, a_r, a_q, a_c, a_y);
    count(c, 1);
}
// Jacobi step on the nonlinear residual with the diagonal of the last Jacobian built:
// dP = coef D^-1 (-G).
__global__ void k_jacobi_dir(Ctx c, double coef) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x)
        c.dP[x] = coef * (c.dinv[x] * (-c.G[x]));
}
void launch_jacobi_dir(const Ctx& c, cudaStream_t st, double coef) {
    k_jacobi_dir<<<blocks_for(c.n), TPB, 0, st>>>(c, coef);
    count(c, 1);
}
// Inner products of the residual-minimising start: with g[0] the residual at the plain start and
// w_j = g[j] - g[base_j] (j = 1..K, K <= GRAM_K) the residual changes along the candidate
// directions, the Gram matrix <w_j, w_k> (j <= k, row by row) and <w_j, g[0]>; per-block partials,
// folded by k_gram_fold in block order.
__global__ void __launch_bounds__(RED_THREADS) k_gram(int n, GramIn in, double* __restrict__ part) {
    __shared__ double sh[GRAM_Q * 32];
    double acc[GRAM_Q];
#pragma unroll
    for (int q = 0; q < GRAM_Q; q++) acc[q] = 0.0;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
        double w[GRAM_K];
#pragma unroll
        for (int j = 0; j < GRAM_K; j++) w[j] = j < in.K ? in.g[j + 1][x] - in.g[in.base[j + 1]][x] : 0.0;
        const double g0 = in.g[0][x];
        int q = 0;
#pragma unroll
        for (int j = 0; j < GRAM_K; j++)
#pragma unroll
            for (int k = j; k < GRAM_K; k++) acc[q++] += w[j] * w[k];
#pragma unroll
        for (int j = 0; j < GRAM_K; j++) acc[q++] += w[j] * g0;
    }
    block_fold<RedSum, GRAM_Q>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < GRAM_Q; q++) part[(size_t)blockIdx.x * GRAM_Q + q] = acc[q];
    }
}
__global__ void k_gram_fold(const double* __restrict__ part, int nb, double* __restrict__ out) {
    double f[GRAM_Q];
#pragma unroll
    for (int q = 0; q < GRAM_Q; q++) f[q] = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) {
#pragma unroll
        for (int q = 0; q < GRAM_Q; q++) f[q] += part[(size_t)b * GRAM_Q + q];
    }
#pragma unroll
    for (int q = 0; q < GRAM_Q; q++) f[q] = warp_fold<RedSum>(f[q]);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < GRAM_Q; q++) out[q] = f[q];
    }
}
int launch_gram(const Ctx& c, cudaStream_t st, const GramIn& in, double* part, double* out) {
    const int nb = red_blocks(c.n, RED_THREADS);
    k_gram<<<nb, RED_THREADS, 0, st>>>(c.n, in, part);
    k_gram_fold<<<1, 32, 0, st>>>(part, nb, out);
    count(c, 2);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// Box average of radius r along x (dir 0) or y (dir 1) of a per-cell field, boundary-mapped like
// every stencil read (periodic wrap, else the edge cell): the separable smoothing of the network's
// output, so that its step carries only the smooth part of the prediction.
__global__ void k_smooth(Ctx c, const float* __restrict__ in, float* __restrict__ out, int r, int dir) {
    const Geom& g = c.g;
    const float w = 1.0f / (2 * r + 1);
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
        float s = 0.0f;
        for (int d = -r; d <= r; d++) s += in[dir == 0 ? mp_index(g, i + d, j) : mp_index(g, i, j + d)];
        out[x] = s * w;
    }
}
void launch_smooth(const Ctx& c, cudaStream_t st, float* y, float* tmp, int r) {
    k_smooth<<<blocks_for(c.n), TPB, 0, st>>>(c, y, tmp, r, 0);
    if (c.g.ny > 1) {
        k_smooth<<<blocks_for(c.n), TPB, 0, st>>>(c, tmp, y, r, 1);
        count(c, 2);
    } else {
        cudaMemcpyAsync(y, tmp, (size_t)c.n * sizeof(float), cudaMemcpyDeviceToDevice, st);
        count(c, 1);
    }
}
// After a converged stage: the new rate R' = (P_converged - P_start) / sdt, the training
// target (R' - R) / sigma (when t is not null), R2 = R, R = R', and sigma' = RMS of R'
// (folded by the last block, after every block has read sigma).
__global__ void __launch_bounds__(TPB) k_rate(Ctx c, const double* __restrict__ P0, double tscale, float* __restrict__ t) {
    const double idt = 1.0 / c.sdt;
    const double isig = 1.0 / rate_scale(c, tscale);
    double acc[1] = {0.0};
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const double r = (c.P[x] - P0[x]) * idt;
        const double r0 = c.Prate[x];
        if (t) t[x] = (float)((r - r0) * isig);
        if (c.Prate3) c.Prate3[x] = c.Prate2[x];
        c.Prate2[x] = r0;
        c.Prate[x] = r;
        acc[0] += r * r;
    }
    double tot[1];
    if (grid_fold<RedSum, 1>(acc, c.partials, &c.counters[13], tot) && threadIdx.x == 0) {
        const double s = sqrt(tot[0] / c.n);
        c.rate_sc[0] = isfinite(s) ? s : 0.0;
    }
}
void launch_rate(const Ctx& c, cudaStream_t st, const double* P0, double tscale, float* t) {
    k_rate<<<red_blocks(c.n, TPB), TPB, 0, st>>>(c, P0, tscale, t);
    count(c, 1);
}

// ============================================================ Thomas (1D non-periodic, :858-863)
SPB6G_DEV void thomas_solve(const Ctx& c) {
    // One thread; the loads of row r + 2 are issued while row r is eliminated (the pointers do not
    // alias), so the division chain, not a memory round trip, sets the pace.  Same arithmetic as
    // the sweep re-reading cp, dp and dP from memory.
    const Geom& g = c.g;
    const int n = g.nx;
    double* __restrict__ cp = c.tcp;
    double* __restrict__ dp = c.tdp;
    double* __restrict__ x = c.dP;
    const double* __restrict__ aC = c.aC;
    const double* __restrict__ aW = c.aW;
    const double* __restrict__ aE = c.aE;
    const double* __restrict__ G = c.G;
    struct Row {
        double c, w, e, g;
    };
    auto load = [&](int r) { return r < n ? Row{aC[r], aW[r], aE[r], G[r]} : Row{0.0, 0.0, 0.0, 0.0}; };
    auto coef = [&](int r, const Row& q, double& lo, double& di, double& up) {
        lo = up = di = 0;
        di += q.c;
        const int cw = mp_index(g, r - 1, 0), ce = mp_index(g, r + 1, 0);
        const double vw = q.w, ve = q.e;
        if (cw == r) di += vw; else if (cw == r - 1) lo = vw; else if (cw == r + 1) up = vw;
        if (ce == r) di += ve; else if (ce == r - 1) lo = ve; else if (ce == r + 1) up = ve;
    };
    double lo, di, up;
    Row q0 = load(0), q1 = load(1), q2 = load(2);
    coef(0, q0, lo, di, up);
    double cpv = up / di, dpv = -q0.g / di;
    cp[0] = cpv;
    dp[0] = dpv;
    for (int r = 1; r < n; r++) {
        const Row q = q1;
        q1 = q2;
        q2 = load(r + 2);
        coef(r, q, lo, di, up);
        const double m = di - lo * cpv;
        cpv = up / m;
        dpv = (-q.g - lo * dpv) / m;
        cp[r] = cpv;
        dp[r] = dpv;
    }
    double xv = dpv;  // dp[n - 1]
    x[n - 1] = xv;
    double c1 = n > 1 ? cp[n - 2] : 0.0, d1 = n > 1 ? dp[n - 2] : 0.0;
    double c2 = n > 2 ? cp[n - 3] : 0.0, d2 = n > 2 ? dp[n - 3] : 0.0;
    for (int r = n - 2; r >= 0; r--) {
        const double cr = c1, dr = d1;
        c1 = c2;
        d1 = d2;
        if (r >= 2) { c2 = cp[r - 2]; d2 = dp[r - 2]; }
        xv = dr - cr * xv;
        x[r] = xv;
    }
}
__global__ void k_thomas(Ctx c) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    thomas_solve(c);
}
// The same elimination with the rows staged in shared memory: every thread of the block forms the
// rows' coefficients and right-hand sides (coalesced loads), one thread runs the two sweeps with
// the next row's operands already in registers -- the chain is then the divisions' latency, not
// a global-memory round trip per row -- and the block writes dP back.  The arithmetic and its
// order are thomas_solve's, so the result is bitwise the same.
constexpr int THOMAS_THREADS = 512;
constexpr int THOMAS_SMEM_MAX_ROWS = (224 * 1024) / (4 * (int)sizeof(double));  // lo, di, up/cp, rhs/dp/x
__global__ void __launch_bounds__(THOMAS_THREADS) k_thomas_smem(Ctx c) {
    extern __shared__ __align__(16) double tsm[];
    const Geom& g = c.g;
    const int n = g.nx;
    double* lo = tsm;
    double* di = lo + n;
    double* up = di + n;   // becomes cp
    double* rhs = up + n;  // becomes dp, then the solution
    for (int r = threadIdx.x; r < n; r += blockDim.x) {
        double l = 0, d = 0, u = 0;
        d += c.aC[r];
        const int cw = mp_index(g, r - 1, 0), ce = mp_index(g, r + 1, 0);
        const double vw = c.aW[r], ve = c.aE[r];
        if (cw == r) d += vw; else if (cw == r - 1) l = vw; else if (cw == r + 1) u = vw;
        if (ce == r) d += ve; else if (ce == r - 1) l = ve; else if (ce == r + 1) u = ve;
        lo[r] = l;
        di[r] = d;
        up[r] = u;
        rhs[r] = c.G[r];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double cpv = up[0] / di[0], dpv = -rhs[0] / di[0];
        up[0] = cpv;
        rhs[0] = dpv;
        double ln = n > 1 ? lo[1] : 0.0, dn = n > 1 ? di[1] : 0.0, un = n > 1 ? up[1] : 0.0, gn = n > 1 ? rhs[1] : 0.0;
        for (int r = 1; r < n; r++) {
            const double l = ln, d = dn, u = un, gr = gn;
            if (r + 1 < n) { ln = lo[r + 1]; dn = di[r + 1]; un = up[r + 1]; gn = rhs[r + 1]; }
            const double m = d - l * cpv;
            cpv = u / m;
            dpv = (-gr - l * dpv) / m;
            up[r] = cpv;
            rhs[r] = dpv;
        }
        double xv = rhs[n - 1];
        double cn = n > 1 ? up[n - 2] : 0.0, pn = n > 1 ? rhs[n - 2] : 0.0;
        for (int r = n - 2; r >= 0; r--) {
            const double cr = cn, pr = pn;
            if (r > 0) { cn = up[r - 1]; pn = rhs[r - 1]; }
            xv = pr - cr * xv;
            rhs[r] = xv;
        }
    }
    __syncthreads();
    for (int r = threadIdx.x; r < n; r += blockDim.x) c.dP[r] = rhs[r];
}
void launch_thomas(const Ctx& c, cudaStream_t st) {
    const int n = c.g.nx;
    if (n <= THOMAS_SMEM_MAX_ROWS) {
        static unsigned long long configured = 0;  // one bit per device: the attribute is per device
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 64 && !(configured & (1ull << dev))) {
            cudaFuncSetAttribute(k_thomas_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, 224 * 1024);
            configured |= 1ull << dev;
        }
        k_thomas_smem<<<1, THOMAS_THREADS, (size_t)n * 4 * sizeof(double), st>>>(c);
    } else {
        k_thomas<<<1, 32, 0, st>>>(c);
    }
    count(c, 1);
}

// ============================================================ Newton step control (:870-879, :890-899)
__global__ void __launch_bounds__(RED_THREADS) k_stepnorm(Ctx c) {
    double m[1] = {0.0};
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x)
        m[0] = SMAX(m[0], SMAX(0.0, fabs(c.dP[x]) / (fabs(c.P[x]) + c.sc[x])));
    double tot[1];
    if (grid_fold<RedMax, 1>(m, c.partials, &c.counters[7], tot) && threadIdx.x == 0) c.ns->sn = tot[0];
}
void launch_stepnorm(const Ctx& c, cudaStream_t st) {
    k_stepnorm<<<red_blocks(c.n), RED_THREADS, 0, st>>>(c);
    count(c, 1);
}
__global__ void k_apply_step(Ctx c) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) c.P[x] += c.dP[x];
}
void launch_apply_step(const Ctx& c, cudaStream_t st) {
    k_apply_step<<<blocks_for(c.n), TPB, 0, st>>>(c);
    count(c, 1);
}
SPB6G_DEV void floor_at(const Ctx& c, int x, double tol) {
    const Geom& g = c.g;
    const int i = x % g.nx, j = x / g.nx;
    const Nb5 p = gather_p(g, i, j, [&](int q) { return c.P[q]; });
    double Gr;
    CellRes o;
    if (!residual_at(c, i, j, p, 0, -1, 0, Gr, &o)) { atomicOr(&c.ns->fail, 4); return; }
    const double sig = closure_roundoff(c.phy, o.in, o.o.pbar);
    if (fabs(Gr) > tol * (fabs(c.p_ref + p.c) + c.kw[x] + 1.0) + sig) atomicOr(&c.ns->fail, 4);
}
__global__ void k_floor(Ctx c, double tol) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) floor_at(c, x, tol);
}
void launch_floor(const Ctx& c, cudaStream_t st, double tol) {
    SPB6G_MG_FORWARD(launch_floor, mg_view(c), st, tol);
    k_floor<<<blocks_for(c.n), TPB, 0, st>>>(c, tol);
    count(c, 1);
}

// ============================================================ final state (:1056-1073) and H_s (:1363-1371)
// RelaxationActivation (:563-586) with the rates infinite: the closure type of every cell for the
// step (closure_type_of :870-886).  Outside the interface zone eps_I <= alpha1 <= 1 - eps_I, and
// for RELAX_LEVEL 0, the p closure.  In the zone: level 1 pT; level 2 pT, or pTg where the pT
// state's temperature is above Tsat(p); level 3 pTg where a phase temperature of the p closure
// without the energy defect is above Tsat(p), else p.  U^n of a pT / pTg cell is projected on that
// manifold (project_cell :549-561: the closure at s = 0 from the conservative state; alpha, the
// phase masses and energies change, the momentum and E do not); a cell whose projection has no
// solution takes the p closure.  The level-2 test's pT state is the pT projection itself (the
// same closure of the same input).
#if SPB6G_MG
__global__ void k_relax_activate(Ctx c, State U) {
    const Phys& P = c.phy;
    const int therm = isinf(P.theta_rate) ? CL_PT : CL_THETA, chem = isinf(P.nu_rate) ? CL_PTG : CL_NU;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const double a1 = U.v[IA1][x];
        int ty = P.mech;
        double nu = 0.0;
        if (P.relax > 0 && a1 >= P.eps_i && a1 <= 1.0 - P.eps_i) {
            const double m1 = U.v[IM1][x], m2 = U.v[IM2][x], mu = U.v[IMU][x], mv = U.v[IMV][x];
            const double rho = m1 + m2;
            ClIn in;
            in.atr[0] = a1; in.atr[1] = 1.0 - a1; in.mtr[0] = m1; in.mtr[1] = m2;
            in.etr[0] = U.v[IE1][x]; in.etr[1] = U.v[IE2][x];
            in.s = 0.0;
            in.rhoeC = U.v[IEN][x] - 0.5 * (mu * mu + mv * mv) / rho;
            in.pguess = SMAX(p_mix(P, in.atr[0], in.mtr[0], in.mtr[1], in.rhoeC), 1.0);
            in.Qph[0] = in.Qph[1] = 0.0;
            in.tau = 0.0;
            in.Z[0] = in.Z[1] = 1.0;
            in.nu = -1.0;
            ClOut o;
            if (P.relax == 3) {  // a phase above Tsat in the p closure without the energy defect
                in.type = CL_PND;
                if (closure(P, in, o)) {
                    const double p = o.pbar, Ts = sat_temperature(P, p);
                    if (isfinite(Ts) && (T_amp(P, 0, o.a[0], m1, p) > Ts || T_amp(P, 1, o.a[1], m2, p) > Ts)) ty = chem;
                }
            } else {  // levels 1, 2: thermal, or chemical where the pT state is above Tsat (level 2)
                ty = therm;
                if (P.relax == 2) {
                    const ClMg r = closure_pT(P, m1, m2, in.rhoeC, in.pguess);
                    if (r.ok) {
                        const double Ts = sat_temperature(P, r.o.pbar);
                        if (isfinite(Ts) && r.o.Tk[0] > Ts) ty = chem;
                    }
                }
            }
            if (ty == CL_PT || ty == CL_PTG) {  // project_cell: the closure is also the feasibility test
                in.type = ty;
                if (!closure(P, in, o)) {
                    ty = P.mech;
                } else if (P.unify_proj) {
                    U.v[IA1][x] = o.a[0];
                    U.v[IM1][x] = o.m[0];
                    U.v[IM2][x] = o.m[1];
                    U.v[IE1][x] = o.e[0];
                    U.v[IE2][x] = o.e[1];
                }
            }
            if (P.nu_law && ty == CL_NU) {  // the rate at the cell's pT state (no mass transfer), :574-581
                in.atr[0] = U.v[IA1][x]; in.atr[1] = 1.0 - in.atr[0];
                in.mtr[0] = U.v[IM1][x]; in.mtr[1] = U.v[IM2][x];
                in.etr[0] = U.v[IE1][x]; in.etr[1] = U.v[IE2][x];
                in.pguess = SMAX(p_mix(P, in.atr[0], in.mtr[0], in.mtr[1], in.rhoeC), 1.0);
                in.type = CL_PT;
                if (closure(P, in, o)) nu = nu_law(P, o.pbar, o.Tk[0], o.a[1]);
            }
        }
        c.ctype[x] = (unsigned char)ty;
        if (c.step_nu) c.step_nu[x] = nu;
    }
}
#endif
void launch_relax_activate(const Ctx& c, cudaStream_t st, State U) {
#if SPB6G_MG
    k_relax_activate<<<blocks_for(c.n), TPB, 0, st>>>(c, U);
    count(c, 1);
#else
    spb6g_mg::launch_relax_activate(mg_view(c), st, mg_view(U));
#endif
}

SPB6G_DEV void final_at(const Ctx& c, int x, double* tm = nullptr) {
    const Geom& g = c.g;
    {
        const int i = x % g.nx, j = x / g.nx;
        const Nb5 p = gather_p(g, i, j, [&](int q) { return c.P[q]; });
        double Gr;
        CellRes o;
        if (!residual_at(c, i, j, p, 0, -1, 0, Gr, &o)) { atomicOr(&c.ns->fail, 8); return; }
        // the phase masses are the closure's (:1063): pTg and nu cells exchange mass
        const int ty = o.in.type;
        const bool xm = SPB6G_MG && (ty == CL_PTG || ty == CL_NU || (ty == CL_PT && c.phy.unify == 1));
        const double mk[2] = {xm ? o.o.m[0] : o.in.mtr[0], xm ? o.o.m[1] : o.in.mtr[1]};
        double U[NV];
        U[IA1] = o.o.a[0]; U[IM1] = mk[0]; U[IM2] = mk[1]; U[IMU] = o.mx; U[IMV] = o.my;
        U[IE1] = o.o.e[0]; U[IE2] = o.o.e[1]; U[IEN] = o.E;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double qs = c.Un.v[k][x];  // Qs of this stage, formed as the explicit kernel forms it
            for (int r = 0; r < c.nH; r++) qs = qs + c.ci[r] * c.Hprev[((size_t)r * NV + k) * c.n + x];
            c.Ust.v[k][x] = U[k];
            c.H[(size_t)k * c.n + x] = (U[k] - qs) / c.adt;
        }
        if (tm) {  // st_Tmax (:1064-1065): the phase temperatures where the phase is present
#pragma unroll
            for (int k = 0; k < 2; k++) {  // the closure's phase temperatures (o.cl.T :1066-1067)
                const bool own = SPB6G_MG && (ty != CL_P || c.phy.unify == 1);
                const double T = own ? o.o.Tk[k] : T_amp(c.phy, k, o.o.a[k], mk[k], o.o.pbar);
                if (o.o.a[k] > 1e-9 && isfinite(T)) tm[k] = SMAX(tm[k], T);
            }
        }
    }
}
// 3 blocks of 256 per SM (80 registers, a small spill) beat 2 blocks without spills by 11 % on
// the 1024^2 bubble field; the extended build's out-of-line closures keep 2.
__global__ void __launch_bounds__(RED_THREADS, SPB6G_MG ? 2 : 3) k_final(Ctx c) {
    double m[2] = {0.0, 0.0};
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) final_at(c, x, m);
    double tot[2];
    if (grid_fold<RedMax, 2>(m, c.partials, &c.counters[12], tot) && threadIdx.x == 0) {
        c.ns->tmax[0] = tot[0];
        c.ns->tmax[1] = tot[1];
    }
}
void launch_final(const Ctx& c, cudaStream_t st) {
    SPB6G_MG_FORWARD(launch_final, mg_view(c), st);
    k_final<<<red_blocks(c.n), RED_THREADS, 0, st>>>(c);
    count(c, 1);
}

// ============================================================ caldt (:502-514) and P_REF (:1309-1312)
__global__ void __launch_bounds__(RED_THREADS, 3) k_caldt(Ctx c, CState U, int acoustic) {
    double m[2] = {0.0, 0.0};
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        double q[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) q[k] = U.v[k][x];
        Prim w;
        if (!prim_of(c.phy, q, w)) continue;
        const double cs = acoustic ? w.cf : 0.0;
        m[0] = SMAX(m[0], SMAX(0.0, fabs(w.u) + cs));
        m[1] = SMAX(m[1], SMAX(0.0, fabs(w.v) + cs));
    }
    double tot[2];
    if (grid_fold<RedMax, 2>(m, c.partials, &c.counters[8], tot) && threadIdx.x == 0) {
        c.ns->rate_x = tot[0];
        c.ns->rate_y = tot[1];
    }
}
void launch_caldt(const Ctx& c, cudaStream_t st, CState U, int acoustic) {
    SPB6G_MG_FORWARD_EOS(launch_caldt, mg_view(c), st, mg_view(U), acoustic);
    k_caldt<<<red_blocks(c.n), RED_THREADS, 0, st>>>(c, U, acoustic);
    count(c, 1);
}
__global__ void __launch_bounds__(RED_THREADS) k_pbar_min(Ctx c, CState U) {
    double m[1] = {INFINITY};
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        double q[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) q[k] = U.v[k][x];
        m[0] = SMIN(m[0], SMIN(INFINITY, pbar_of(c.phy, q)));
    }
    double tot[1];
    if (grid_fold<RedMin, 1>(m, c.partials, &c.counters[9], tot) && threadIdx.x == 0) c.ns->pmin = tot[0];
}
void launch_pbar_min(const Ctx& c, cudaStream_t st, CState U) {
    SPB6G_MG_FORWARD_EOS(launch_pbar_min, mg_view(c), st, mg_view(U));
    k_pbar_min<<<red_blocks(c.n), RED_THREADS, 0, st>>>(c, U);
    count(c, 1);
}
__global__ void k_pbar_init(Ctx c, CState U, double p_ref, double* P) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        double q[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) q[k] = U.v[k][x];
        P[x] = pbar_of(c.phy, q) - p_ref;
    }
}
void launch_pbar_init(const Ctx& c, cudaStream_t st, CState U, double p_ref, double* P) {
    SPB6G_MG_FORWARD_EOS(launch_pbar_init, mg_view(c), st, mg_view(U), p_ref, P);
    k_pbar_init<<<blocks_for(c.n), TPB, 0, st>>>(c, U, p_ref, P);
    count(c, 1);
}


// ============================================================ batched form (no counterpart in the reference)
// Hundreds of independent 1D instances in one persistent launch: block b runs
// instance b's time loop -- the host driver's do_step / run_stage / Newton_Solver
// decision for decision -- with every grid pass done by the block's threads
// through the same per-cell functions as the single-grid kernels, so each
// instance computes exactly what a single-grid solver on it computes.
struct BatchShared {
    Ctx c;
    double red[64];
    double bc;
};
SPB6G_DEV double b_max(double v, BatchShared& s) {
    double a[1] = {v};
    block_fold<RedMax, 1>(a, s.red);
    if (threadIdx.x == 0) s.bc = a[0];
    __syncthreads();
    const double r = s.bc;
    __syncthreads();
    return r;
}
SPB6G_DEV int b_flag(const int* p) {
    __syncthreads();
    const int v = *(volatile const int*)p;
    __syncthreads();
    return v;
}
SPB6G_DEV void b_clear(int* p, int nwords) {
    __syncthreads();
    if ((int)threadIdx.x < nwords) atomicExch(p + threadIdx.x, 0);
    __syncthreads();
}
// evalAll + norm (mode 0: at P into G, sc; mode 1: at Pn = P + lam dP into Gn, scn, Pn)
SPB6G_DEV double b_residual(BatchShared& s, int mode, double lam) {
    const Ctx& c = s.c;
    const Geom& g = c.g;
    double m = 0.0;
    for (int x = threadIdx.x; x < c.n; x += blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
        Nb5 p = mode == 0 ? gather_p(g, i, j, [&](int q) { return c.P[q]; })
                          : gather_p(g, i, j, [&](int q) { return c.P[q] + lam * c.dP[q]; });
        double Gr;
        const bool ok = residual_at(c, i, j, p, 0, -1, 0, Gr, nullptr);
        const double sc = row_scale(c, i, j, p.c);
        if (mode == 0) { c.G[x] = Gr; c.sc[x] = sc; }
        else { c.Gn[x] = Gr; c.scn[x] = sc; c.Pn[x] = p.c; }
        if (!ok) atomicOr(&c.ns->fail, 1);
        else m = SMAX(m, SMAX(0.0, fabs(Gr) / (fabs(c.p_ref + p.c) + c.kw[x] + 1.0)));
    }
    return b_max(m, s);
}
SPB6G_DEV double b_inv_rate(BatchShared& s, const BatchInst& B, int acoustic) {  // caldt (:502-514)
    const Ctx& c = s.c;
    double m = 0.0;
    for (int x = threadIdx.x; x < c.n; x += blockDim.x) {
        double q[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) q[k] = B.U[k][x];
        Prim w;
        if (!prim_of(c.phy, q, w)) continue;
        m = SMAX(m, SMAX(0.0, fabs(w.u) + (acoustic ? w.cf : 0.0)));
    }
    const double rate = b_max(m, s) / c.g.dx;
    return rate > 0 ? 1.0 / rate : INFINITY;
}
SPB6G_DEV int b_newton(BatchShared& s, BatchInst& B, double& resfinal) {  // Newton_Solver (:799-904), Thomas path
    Ctx& c = s.c;
    const int tid = threadIdx.x, nth = blockDim.x;
    const double tol = B.newton_tol;
    b_clear(&c.ns->fail, 1);
    double res = b_residual(s, 0, 0.0);
    if (b_flag(&c.ns->err)) return SPB6G_INADMISSIBLE;
    if (b_flag(&c.ns->fail)) { resfinal = INFINITY; return SPB6G_NEWTON_FAIL; }
    for (int it = 0; it < B.newton_iter; it++) {
        resfinal = res;
        if (res < tol) return SPB6G_OK;
        b_clear(&c.ns->fail, 1);
        for (int t = tid; t < 3 * c.n; t += nth) jac_entry(c, t / 3, t % 3);
        __syncthreads();
        if (tid == 0) thomas_solve(c);
        __syncthreads();
        if (b_flag(&c.ns->fail)) return SPB6G_NEWTON_FAIL;
        b_clear(&c.ns->fail, 1);
        double m = 0.0;  // step criterion (:870-879)
        for (int x = tid; x < c.n; x += nth) m = SMAX(m, SMAX(0.0, fabs(c.dP[x]) / (fabs(c.P[x]) + c.sc[x])));
        const double sn = b_max(m, s);
        double rn = b_residual(s, 1, 1.0);
        if (sn < tol) {
            for (int x = tid; x < c.n; x += nth) c.P[x] += c.dP[x];
            if (tid == 0) B.newton_it++;
            b_clear(&c.ns->fail, 1);
            res = b_residual(s, 0, 0.0);
            if (b_flag(&c.ns->fail)) return SPB6G_NEWTON_FAIL;
            resfinal = res;
            return SPB6G_OK;
        }
        double lam = 1.0;
        bool acc = false;
        for (int ls = 0; ls < 40; ls++) {  // line search (:880-888)
            if (ls > 0) {
                b_clear(&c.ns->fail, 1);
                rn = b_residual(s, 1, lam);
            }
            if (!b_flag(&c.ns->fail)) {
                if (rn < res * (1.0 - 1e-4 * lam) || rn < tol) { acc = true; res = rn; break; }
            }
            lam *= 0.5;
        }
        if (!acc) {  // round-off floor acceptance (:890-899)
            resfinal = res;
            b_clear(&c.ns->fail, 1);
            for (int x = tid; x < c.n; x += nth) floor_at(c, x, tol);
            if (b_flag(&c.ns->fail)) return SPB6G_NEWTON_FAIL;
            if (tid == 0) B.floor_count++;
            return SPB6G_OK;
        }
        __syncthreads();
        if (tid == 0) {
            double* q;
            q = c.P; c.P = c.Pn; c.Pn = q;
            q = c.G; c.G = c.Gn; c.Gn = q;
            q = c.sc; c.sc = c.scn; c.scn = q;
            B.newton_it++;
        }
        __syncthreads();
    }
    resfinal = res;
    return res < tol ? SPB6G_OK : SPB6G_NEWTON_FAIL;
}
SPB6G_DEV void b_set_tab(int rk, double Ae[3][3], double Ai[3][3]) {  // main's set_tab, :1281-1303
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Ae[a][b] = Ai[a][b] = 0;
    if (rk == 1) {
        Ai[0][0] = 1.0;
    } else if (rk == 2) {
        const double bb = 1.0 - 1.0 / sqrt(2.0), cc = 1.0 / (2.0 * bb);
        Ae[1][0] = cc;
        Ai[0][0] = bb;
        Ai[1][0] = 1 - bb;
        Ai[1][1] = bb;
    } else if (rk == 3) {
        const double r12 = 0.5, r13 = 1.0 / 3.0, r14 = 1.0 / 4.0;
        Ae[1][0] = r12; Ae[2][0] = r12; Ae[2][1] = r12;
        Ai[0][0] = r14; Ai[1][1] = r14; Ai[2][0] = r13; Ai[2][1] = r13; Ai[2][2] = r13;
    }
}
template <int TW>
SPB6G_DEV int b_stage(BatchShared& s, BatchInst& B, int rks, double Ae[3][3], double Ai[3][3], double dt, unsigned char* fsm) {
    Ctx& c = s.c;
    const int tid = threadIdx.x, nth = blockDim.x;
    __syncthreads();
    if (tid == 0) {
        for (int k = 0; k < NV; k++) c.Un.v[k] = B.U[k];
        c.Hprev = B.Hs;
        c.nH = rks;
        for (int r = 0; r < 2; r++) {
            c.ce[r] = r < rks ? Ae[rks][r] * dt : 0.0;
            c.ci[r] = r < rks ? Ai[rks][r] * dt : 0.0;
        }
        c.adt = Ai[rks][rks] * dt;
        c.tau = c.adt;
        c.rx = c.tau / c.g.dx;
        c.ry = c.tau / c.g.dy;
        c.H = B.Hs + (size_t)rks * NV * c.n;
    }
    b_clear(&c.ns->fail, 3);  // fail, err, nstrong
    const int ntiles = (c.g.nx + TW - 1) / TW;
    for (int tl = 0; tl < ntiles; tl++) {
        flux_tile<double, TW, 1, false>(c, tl, 0, fsm, tid, nth);
        __syncthreads();
    }
    const long npad = prep_cells(c.g);
    for (long q = tid; q < npad; q += nth) prep_cell_at(c, q);
    __syncthreads();
    for (long q = tid; q < c.g.nx + 1; q += nth) prep_fx_at(c, q);
    __syncthreads();
    for (int x = tid; x < c.n; x += nth) {
        double Q[2];
        shock_cell(c, x % c.g.nx, x / c.g.nx, Q, true);
        c.qph0[x] = Q[0];
        c.qph1[x] = Q[1];
    }
    __syncthreads();
    double res = 0;
    const int rc = b_newton(s, B, res);
    if (rc != SPB6G_OK) return rc;
    if (tid == 0 && res > B.maxres) B.maxres = res;
    b_clear(&c.ns->fail, 1);
    double tm[2] = {0.0, 0.0};  // st_Tmax of the stage's final state (:1064-1070)
    for (int x = tid; x < c.n; x += nth) final_at(c, x, tm);
    block_fold<RedMax, 2>(tm, s.red);
    if (b_flag(&c.ns->fail)) return SPB6G_NEWTON_FAIL;
    if (tid == 0) {
        B.stages++;
        B.tmax[0] = SMAX(B.tmax[0], tm[0]);
        B.tmax[1] = SMAX(B.tmax[1], tm[1]);
    }
    return SPB6G_OK;
}
template <int TW>
SPB6G_DEV int b_step(BatchShared& s, BatchInst& B, unsigned char* fsm) {  // main's loop body (:1316-1384)
    Ctx& c = s.c;
    const int tid = threadIdx.x, nth = blockDim.x;
    bool ramping = false;
    double dt = B.dt, dtprev = B.dtprev;
    if (B.dtfix > 0) dt = B.dtfix;
    else {
        dt = B.cfl * b_inv_rate(s, B, B.acdt);
        if (B.ramp) {
            if (dtprev < 0) dtprev = B.cfl_ac * b_inv_rate(s, B, 1) / 1.2;
            if (dt > 1.2 * dtprev) { dt = 1.2 * dtprev; ramping = true; }
        }
        if (!isfinite(dt)) dt = B.cfl_ac * b_inv_rate(s, B, 1);
    }
    dt = SMIN(dt, B.tend - B.t);
    if (!(dt > 1e-12 * B.tend)) return SPB6G_DT_UNDERFLOW;
    bool done = false;
    double Ae[3][3], Ai[3][3];
    for (int attempt = 0; attempt < 30 && !done; attempt++) {
        const bool first_order = B.ramp && ramping && B.startup;
        const int rk = first_order ? 1 : B.rk;
        __syncthreads();
        if (tid == 0 && rk == 1) B.rk1++;
        b_set_tab(rk, Ae, Ai);
        // begin_attempt_pressure: the Newton iterate starts as a copy of the accepted pressure
        int other[2], k = 0;
        for (int b = 0; b < 3; b++)
            if (b != B.pmain) other[k++] = b;
        for (int x = tid; x < c.n; x += nth) B.Pbuf[other[0]][x] = B.Pbuf[B.pmain][x];
        __syncthreads();
        if (tid == 0) { c.P = B.Pbuf[other[0]]; c.Pn = B.Pbuf[other[1]]; }
        __syncthreads();
        bool ok = true;
        for (int rks = 0; rks < rk && ok; rks++) ok = b_stage<TW>(s, B, rks, Ae, Ai, dt, fsm) == SPB6G_OK;
        __syncthreads();
        if (ok) {
            int pm = 0;
            for (int b = 0; b < 3; b++)
                if (B.Pbuf[b] == c.P) pm = b;
            __syncthreads();
            if (tid == 0) {
                for (int q = 0; q < NV; q++) {
                    double* u = B.U[q];
                    B.U[q] = B.Ust[q];
                    B.Ust[q] = u;
                    c.Ust.v[q] = B.Ust[q];
                }
                B.pmain = pm;
            }
            done = true;
        }
        __syncthreads();
        if (!done) {
            if (tid == 0) B.rejects++;
            dt *= 0.5;
        }
    }
    if (!done) return SPB6G_STEP_FAILED;
    __syncthreads();
    if (tid == 0) {
        B.t = B.t + dt;
        B.dt = dt;
        B.dtprev = dt;
        B.steps++;
        if (!ramping) B.startup = 0;
    }
    __syncthreads();
    return SPB6G_OK;
}
// Blocks take the grids list[0..count) (all of insts when list is NULL) in order.
template <int TW>
__global__ void __launch_bounds__(256) k_batch(BatchInst* insts, const int* list, int count, int nsteps) {
    extern __shared__ __align__(16) unsigned char batch_smem[];
    __shared__ BatchShared s;
    for (int k = blockIdx.x; k < count; k += gridDim.x) {
        BatchInst& B = insts[list ? list[k] : k];
        __syncthreads();
        if (threadIdx.x == 0) s.c = B.c;
        __syncthreads();
        for (int k = 0; k < nsteps; k++) {
            const bool stop = B.status != SPB6G_OK || !(B.t < B.tend * (1 - 1e-12));  // as spb6g_advance
            __syncthreads();
            if (stop) break;
            const int rc = b_step<TW>(s, B, batch_smem);
            __syncthreads();
            if (rc != SPB6G_OK) {
                if (threadIdx.x == 0) B.status = rc;
                __syncthreads();
                break;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) B.c = s.c;
        __syncthreads();
    }
}
int batch_max_blocks(int threads, int tw, int device) {
    int per_sm = 0, sms = 0;
    const size_t smem = flux_tile_bytes_1d(tw);
    const void* fn = tw == 128 ? (const void*)k_batch<128> : (const void*)k_batch<256>;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) return 0;
    return per_sm * sms;
}
int launch_batch(BatchInst* insts, const int* list, int count, int nsteps, int threads, int tw, int grid, cudaStream_t st) {
    const size_t smem = flux_tile_bytes_1d(tw);
    if (tw == 128) k_batch<128><<<grid, threads, smem, st>>>(insts, list, count, nsteps);
    else k_batch<256><<<grid, threads, smem, st>>>(insts, list, count, nsteps);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace spb6g
