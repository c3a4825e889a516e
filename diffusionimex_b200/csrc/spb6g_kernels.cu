// Stage pipeline kernels of the SPB6 IMEX solver (one thread per cell / face /
// row; grid-stride loops; deterministic reductions).  Reference functions are
// cited per kernel; arithmetic follows them in operation order.
#include <cstdio>

#include "spb6g_ctx.cuh"

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

// ============================================================ stage combination (main :1341-1351)
__global__ void k_combine(int n, CState U, const double* __restrict__ Hs, int nH, double c0e, double c1e, double c0i,
                          double c1i, State Qe, State Qs) {
    const double ce[2] = {c0e, c1e}, ci[2] = {c0i, c1i};
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < n; x += gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double e = U.v[k][x], s = e;
            for (int r = 0; r < nH; r++) {
                const double h = Hs[((size_t)r * NV + k) * n + x];
                e = e + ce[r] * h;
                s = s + ci[r] * h;
            }
            Qe.v[k][x] = e;
            Qs.v[k][x] = s;
        }
    }
}

void launch_combine(const Ctx& c, cudaStream_t st, const double* const* U, const double* Hs, int nH, const double* ae,
                    const double* ai, double dt, double* const* Qe, double* const* Qs) {
    CState u;
    State qe, qs;
    for (int k = 0; k < NV; k++) { u.v[k] = U[k]; qe.v[k] = Qe[k]; qs.v[k] = Qs[k]; }
    // coefficients Ae[s][r] * dt and Ai[s][r] * dt, as the reference forms them (Ae * dt * H)
    const double c0e = nH > 0 ? ae[0] * dt : 0, c1e = nH > 1 ? ae[1] * dt : 0;
    const double c0i = nH > 0 ? ai[0] * dt : 0, c1i = nH > 1 ? ai[1] * dt : 0;
    k_combine<<<blocks_for(c.n), TPB, 0, st>>>(c.n, u, Hs, nH, c0e, c1e, c0i, c1i, qe, qs);
    count(c, 1);
}

// ============================================================ reconstruction (TVDReconstruction :369-471)
SPB6G_DEV void cell_scales(const Phys& P, const double* q, double& vsc, double& esc) {
    Prim w;
    const double rho = q[IM1] + q[IM2], mm = hypot(q[IMU], q[IMV]);
    vsc = (rho > 0 ? mm / rho : 0.0) + (prim_of(P, q, w) ? w.cf : 0.0);
    esc = fabs(q[IE1]) + fabs(q[IE2]) + (rho > 0 ? 0.5 * mm * mm / rho : 0.0);
}

// Shared limiter phi of the volume-transported quantities with the face
// admissibility cap (:399-432), and the velocity minmod slopes (:450-463).
SPB6G_DEV void recon_dir(const Phys& P, const double* Ua, const double* Uc, const double* Ub, double vsa, double vsc,
                         double vsb, double esa, double esc, double esb, double& phi_out, double& phis_out, double& slu,
                         double& slv) {
    const int VOL[5] = {IA1, IM1, IM2, IE1, IE2};
    double phi = 1.0;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int k = VOL[q];
        const double xa = Ua[k], xc = Uc[k], xb = Ub[k];
        double sc;
        if (k == IA1) sc = 3.0;
        else if (k == IM1 || k == IM2) sc = fabs(xa) + fabs(xc) + fabs(xb);
        else sc = esa + esc + esb;
        const double a = xc - xa, b = xb - xc, tiny = 1e-12 * sc + 1e-300;
        if (!P.limiter) break;
        if (fabs(a) <= tiny && fabs(b) <= tiny) continue;
        if (a * b <= 0) { phi = 0.0; break; }
        const double c = 0.5 * (a + b), m = fabs(a) < fabs(b) ? a : b;
        phi = SMIN(phi, m / c);
    }
    if (P.limiter && phi > 0.0) {
        const double* cs[3] = {Ua, Uc, Ub};
#pragma unroll
        for (int ph = 0; ph < 2; ph++) {
            double L1[3], L2[3];
#pragma unroll
            for (int n = 0; n < 3; n++) {
                const double a = ph == 0 ? cs[n][IA1] : 1.0 - cs[n][IA1], m = cs[n][ph == 0 ? IM1 : IM2],
                             e = cs[n][ph == 0 ? IE1 : IE2];
                L1[n] = a - m * P.ph[ph].b;
                L2[n] = e - m * P.ph[ph].q - L1[n] * P.ph[ph].pi;
            }
            {
                const double dL = fabs(L1[2] - L1[0]);
                if (L1[1] > 0.0 && dL > 0.0) phi = SMIN(phi, 2.0 * L1[1] / dL);
            }
            {
                const double dL = fabs(L2[2] - L2[0]);
                if (L2[1] > 0.0 && dL > 0.0) phi = SMIN(phi, 2.0 * L2[1] / dL);
            }
        }
    }
    const double ra = Ua[IM1] + Ua[IM2], rc = Uc[IM1] + Uc[IM2], rb = Ub[IM1] + Ub[IM2];
    const double tiny = 1e-12 * (vsa + vsc + vsb) + 1e-300;
    double sm = 1.0, sl[2];
#pragma unroll
    for (int d = 0; d < 2; d++) {
        const int k = d == 0 ? IMU : IMV;
        const double va = Ua[k] / ra, vc = Uc[k] / rc, vb = Ub[k] / rb, a = vc - va, b = vb - vc;
        double s = 0.0;
        if (!P.limiter) s = 0.5 * (a + b);
        else if (!(fabs(a) <= tiny && fabs(b) <= tiny)) {
            if (a * b > 0) { s = fabs(a) < fabs(b) ? a : b; sm = SMIN(sm, s / (0.5 * (a + b))); }
            else sm = 0.0;
        }
        sl[d] = s;
    }
    phi_out = phi;
    phis_out = SMIN(phi, sm);
    slu = sl[0];
    slv = sl[1];
}

// Cells i in [-1, nx], j in [-1, ny]: x-reconstruction on interior rows, y on interior columns.
__global__ void k_recon(Ctx c) {
    const Geom& g = c.g;
    const int W = g.nx + 2, Hh = g.ny > 1 ? g.ny + 2 : 1;
    const long tot = (long)W * Hh;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % W) - 1, j = g.ny > 1 ? (int)(t / W) - 1 : 0;
        double qc[NV], qa[NV], qb[NV], vs_c, es_c, vs_a, es_a, vs_b, es_b;
        load_state(c.phy, g, c.Qe, i, j, qc);
        cell_scales(c.phy, qc, vs_c, es_c);
        if (j >= 0 && j < g.ny) {
            load_state(c.phy, g, c.Qe, i - 1, j, qa);
            load_state(c.phy, g, c.Qe, i + 1, j, qb);
            cell_scales(c.phy, qa, vs_a, es_a);
            cell_scales(c.phy, qb, vs_b, es_b);
            double phi, phis, slu, slv;
            recon_dir(c.phy, qa, qc, qb, vs_a, vs_c, vs_b, es_a, es_c, es_b, phi, phis, slu, slv);
            const size_t x = rxi(g, i, j);
            c.phiv_x[x] = phi; c.phis_x[x] = phis; c.slu_x[x] = slu; c.slv_x[x] = slv;
        }
        if (g.ny > 1 && i >= 0 && i < g.nx) {
            load_state(c.phy, g, c.Qe, i, j - 1, qa);
            load_state(c.phy, g, c.Qe, i, j + 1, qb);
            cell_scales(c.phy, qa, vs_a, es_a);
            cell_scales(c.phy, qb, vs_b, es_b);
            double phi, phis, slu, slv;
            recon_dir(c.phy, qa, qc, qb, vs_a, vs_c, vs_b, es_a, es_c, es_b, phi, phis, slu, slv);
            const size_t x = ryi(g, i, j);
            c.phiv_y[x] = phi; c.phis_y[x] = phis; c.slu_y[x] = slu; c.slv_y[x] = slv;
        }
    }
}
void launch_recon(const Ctx& c, cudaStream_t st) {
    const long tot = (long)(c.g.nx + 2) * (c.g.ny > 1 ? c.g.ny + 2 : 1);
    k_recon<<<blocks_for(tot), TPB, 0, st>>>(c);
    count(c, 1);
}

// Face state of cell (ci, cj) on its left (right = false) or right side in direction dir (:433-467).
SPB6G_DEV void face_state(const Ctx& c, int ci, int cj, int dir, bool right, double* w) {
    double qa[NV], qc[NV], qb[NV];
    const int di = dir == 0, dj = dir == 1;
    load_state(c.phy, c.g, c.Qe, ci - di, cj - dj, qa);
    load_state(c.phy, c.g, c.Qe, ci, cj, qc);
    load_state(c.phy, c.g, c.Qe, ci + di, cj + dj, qb);
    double phi, slu, slv;
    if (dir == 0) {
        const size_t x = rxi(c.g, ci, cj);
        phi = c.phiv_x[x]; slu = c.slu_x[x]; slv = c.slv_x[x];
    } else {
        const size_t x = ryi(c.g, ci, cj);
        phi = c.phiv_y[x]; slu = c.slu_y[x]; slv = c.slv_y[x];
    }
    const int VOL[5] = {IA1, IM1, IM2, IE1, IE2};
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int k = VOL[q];
        const double sig = phi * 0.5 * (qb[k] - qa[k]);
        w[k] = right ? qc[k] + 0.5 * sig : qc[k] - 0.5 * sig;
    }
    const double rc = qc[IM1] + qc[IM2];
    const double vcu = qc[IMU] / rc, vcv = qc[IMV] / rc;
    const double v0 = right ? vcu + 0.5 * slu : vcu - 0.5 * slu, v1 = right ? vcv + 0.5 * slv : vcv - 0.5 * slv;
    const double r = w[IM1] + w[IM2];
    w[IMU] = r * v0;
    w[IMV] = r * v1;
    w[IEN] = w[IE1] + w[IE2] + 0.5 * r * (v0 * v0 + v1 * v1);
}
// Rusanov flux at the material speed (RusanovC_x/y :237-259), local speed per face.
SPB6G_DEV void rusanov(const double* QL, const double* QR, int d, double* flux) {
    const int km = d == 0 ? IMU : IMV;
    const double vL = QL[km] / (QL[IM1] + QL[IM2]), vR = QR[km] / (QR[IM1] + QR[IM2]);
    const double a = SMAX(fabs(QL[km] / (QL[IM1] + QL[IM2])), fabs(QR[km] / (QR[IM1] + QR[IM2])));
#pragma unroll
    for (int k = 0; k < NV; k++) flux[k] = 0.5 * (QL[k] * vL + QR[k] * vR) - 0.5 * a * (QR[k] - QL[k]);
}

// Explicit update X* = Qs - tau div F(Qe) with the path-conservative alpha term (Update :264-346).
__global__ void k_update(Ctx c) {
    const Geom& g = c.g;
    const int nx = g.nx, ny = g.ny;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % nx, j = x / nx;
        const double rho = c.Qe.v[IM1][x] + c.Qe.v[IM2][x];
        if (!(rho > 0)) atomicOr(&c.ns->err, 1);
        double wRm[NV], wLc[NV], wRc[NV], wLp[NV], fp[NV], fm[NV], X[NV];
        face_state(c, i - 1, j, 0, true, wRm);
        face_state(c, i, j, 0, false, wLc);
        face_state(c, i, j, 0, true, wRc);
        face_state(c, i + 1, j, 0, false, wLp);
        const double ubr = 0.5 * (wRc[IMU] / (wRc[IM1] + wRc[IM2]) + wLp[IMU] / (wLp[IM1] + wLp[IM2]));
        const double ubl = 0.5 * (wRm[IMU] / (wRm[IM1] + wRm[IM2]) + wLc[IMU] / (wLc[IM1] + wLc[IM2]));
        c.ube_x[fxi(g, i, j)] = ubr;
        if (i == 0) c.ube_x[fxi(g, -1, j)] = ubl;
        rusanov(wRc, wLp, 0, fp);
        rusanov(wRm, wLc, 0, fm);
        const double qe_a1 = c.Qe.v[IA1][x];
#pragma unroll
        for (int k = 0; k < NV; k++) X[k] = c.Qs.v[k][x] - c.adt / g.dx * (fp[k] - fm[k]);
        X[IA1] += c.adt / g.dx * qe_a1 * (ubr - ubl);
        if (ny > 1) {
            face_state(c, i, j - 1, 1, true, wRm);
            face_state(c, i, j, 1, false, wLc);
            face_state(c, i, j, 1, true, wRc);
            face_state(c, i, j + 1, 1, false, wLp);
            const double vbr = 0.5 * (wRc[IMV] / (wRc[IM1] + wRc[IM2]) + wLp[IMV] / (wLp[IM1] + wLp[IM2]));
            const double vbl = 0.5 * (wRm[IMV] / (wRm[IM1] + wRm[IM2]) + wLc[IMV] / (wLc[IM1] + wLc[IM2]));
            c.ube_y[fyi(g, i, j)] = vbr;
            if (j == 0) c.ube_y[fyi(g, i, -1)] = vbl;
            rusanov(wRc, wLp, 1, fp);
            rusanov(wRm, wLc, 1, fm);
#pragma unroll
            for (int k = 0; k < NV; k++) X[k] -= c.adt / g.dy * (fp[k] - fm[k]);
            X[IA1] += c.adt / g.dy * qe_a1 * (vbr - vbl);
        }
#pragma unroll
        for (int k = 0; k < NV; k++) c.Xs.v[k][x] = X[k];
        c.a2s[x] = 1.0 - X[IA1];
    }
}
void launch_update(const Ctx& c, cudaStream_t st) {
    k_update<<<blocks_for(c.n), TPB, 0, st>>>(c);
    count(c, 1);
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
    if (!(p_admissible(P, 0, p1) && p_admissible(P, 1, p2))) return INFINITY;
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

__global__ void k_prep_cell(Ctx c) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        double X[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) X[k] = c.Xs.v[k][x];
        const double a1 = X[IA1], a2 = c.a2s[x], m1 = X[IM1], m2 = X[IM2], sa = a1 + a2, rho = m1 + m2;
        if (!(sa > 0 && rho > 0)) atomicOr(&c.ns->err, 2);
        c.ust[x] = X[IMU] / rho;
        c.vst[x] = X[IMV] / rho;
        // residual scale K + P_E (:960-971)
        double K = SMAX(c.phy.ph[0].pi, c.phy.ph[1].pi), PE = 0.0;
        if (a1 > 0 && a2 > 0 && m1 > 0 && m2 > 0) {
            const double p1 = p_ame(c.phy, 0, a1, m1, X[IE1]), p2 = p_ame(c.phy, 1, a2, m2, X[IE2]);
            if (p_admissible(c.phy, 0, p1) && p_admissible(c.phy, 1, p2))
                K = 1.0 / ((a1 / sa) / (m1 / a1 * c2_rp(c.phy, 0, m1 / a1, p1)) + (a2 / sa) / (m2 / a2 * c2_rp(c.phy, 1, m2 / a2, p2)));
            const double dd = dedp_am(c.phy, 0, a1, m1) + dedp_am(c.phy, 1, a2, m2);
            if (dd > 0) PE = (fabs(X[IE1]) + eps_round(c.phy, 0, m1) + fabs(X[IE2]) + eps_round(c.phy, 1, m2)) / dd;
        }
        c.kw[x] = K + PE;
    }
}

// Face coefficients of the implicit face velocity / pressure (set_face :1001-1023, dil_jump :989-1000).
SPB6G_DEV void set_face(const Ctx& c, int iL, int jL, int ydir, double& ubs, double& kp, double& wl, double& pv) {
    const Geom& g = c.g;
    const int iR = iL + (ydir ? 0 : 1), jR = jL + (ydir ? 1 : 0);
    const double hh = ydir ? g.dy : g.dx;
    double XL[NV], XR[NV];
    xs_at(c, iL, jL, XL);
    xs_at(c, iR, jR, XR);
    const double rL = XL[IM1] + XL[IM2], rR = XR[IM1] + XR[IM2];
    const double uL = (ydir ? XL[IMV] : XL[IMU]) / rL, uR = (ydir ? XR[IMV] : XR[IMU]) / rR;
    ubs = 0.5 * (uL + uR);
    kp = c.tau / hh / (0.5 * (rL + rR));
    wl = rR / (rL + rR);
    pv = 0.0;
    const double cL = cfz(c.phy, XL, load_arr(g, c.a2s, iL, jL)), cR = cfz(c.phy, XR, load_arr(g, c.a2s, iR, jR));
    if (!(isfinite(cL) && isfinite(cR))) return;
    const double phi = SMAX(0.0, 1.0 - c.tau * SMIN(cL, cR) / hh);
    if (phi == 0.0) return;
    const int di = iR - iL, dj = jR - jL, im = iL - di, jm = jL - dj, ip = iR + di, jp = jR + dj;
    // the reference's range test (im >= 0 && ... jp < NYT) holds for every face the residual reads
    const double phis = ydir ? SMIN(c.phis_y[ryi(g, iL, jL)], c.phis_y[ryi(g, iR, jR)])
                             : SMIN(c.phis_x[rxi(g, iL, jL)], c.phis_x[rxi(g, iR, jR)]);
    const double psiP = 1.0 - (1.0 - psi_face(c.phy.limiter, pold_at(c, im, jm), pold_at(c, iL, jL), pold_at(c, iR, jR), pold_at(c, ip, jp))) * phis;
    double um, vm, up, vp;
    vel_at(c, im, jm, um, vm);
    vel_at(c, ip, jp, up, vp);
    const double psiU = psi_face(c.phy.limiter, ydir ? vm : um, uL, uR, ydir ? vp : up);
    // dil_jump
    double D;
    if (!ydir) {
        const double d = uR - uL;
        if (g.ny == 1) D = d;
        else {
            double u0p, v0p, u1p, v1p, u0m, v0m, u1m, v1m;
            vel_at(c, iL, jL + 1, u0p, v0p);
            vel_at(c, iL + 1, jL + 1, u1p, v1p);
            vel_at(c, iL, jL - 1, u0m, v0m);
            vel_at(c, iL + 1, jL - 1, u1m, v1m);
            D = 0.25 * (2.0 * d + ((u1p - u0p) + (u1m - u0m))) + 0.25 * (g.dx / g.dy) * ((v0p - v0m) + (v1p - v1m));
        }
    } else {
        const double d = uR - uL;  // v(i, j+1) - v(i, j)
        double up1, vp1, up0, vp0, um1, vm1, um0, vm0;
        vel_at(c, iL + 1, jL + 1, up1, vp1);
        vel_at(c, iL + 1, jL, up0, vp0);
        vel_at(c, iL - 1, jL + 1, um1, vm1);
        vel_at(c, iL - 1, jL, um0, vm0);
        D = 0.25 * (2.0 * d + ((vp1 - vp0) + (vm1 - vm0))) + 0.25 * (g.dy / g.dx) * ((up0 - um0) + (up1 - um1));
    }
    const double ZL = rL * cL, ZR = rR * cR;
    kp += phi * psiP / (ZL + ZR);
    pv = phi * psiU * ZL * ZR / (ZL + ZR) * D;
}
SPB6G_DEV void donor(const Ctx& c, int ci, int cj, int dir, bool right, double* d);
// Donors and tangential velocities of one face (fixed for the stage).
SPB6G_DEV void face_fixed(const Ctx& c, int i, int j, int ydir, double* plane, size_t f, size_t stride) {
    double dl[4], dr[4], u, v;
    donor(c, i, j, ydir, true, dl);
    donor(c, i + (ydir ? 0 : 1), j + (ydir ? 1 : 0), ydir, false, dr);
#pragma unroll
    for (int q = 0; q < 4; q++) {
        plane[q * stride + f] = dl[q];
        plane[(4 + q) * stride + f] = dr[q];
    }
    vel_at(c, i, j, u, v);
    plane[8 * stride + f] = ydir ? u : v;
    vel_at(c, i + (ydir ? 0 : 1), j + (ydir ? 1 : 0), u, v);
    plane[9 * stride + f] = ydir ? u : v;
}
__global__ void k_prep_fx(Ctx c) {
    const Geom& g = c.g;
    const long tot = (long)(g.nx + 1) * g.ny;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % (g.nx + 1)) - 1, j = (int)(t / (g.nx + 1));
        double ubs, kp, wl, pv;
        set_face(c, i, j, 0, ubs, kp, wl, pv);
        const size_t f = fxi(g, i, j);
        c.fx_ubs[f] = ubs; c.fx_kp[f] = kp; c.fx_wl[f] = wl; c.fx_pv[f] = pv;
        face_fixed(c, i, j, 0, c.fxd, f, (size_t)tot);
    }
}
__global__ void k_prep_fy(Ctx c) {
    const Geom& g = c.g;
    const long tot = (long)g.nx * (g.ny + 1);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < tot; t += (long)gridDim.x * blockDim.x) {
        const int i = (int)(t % g.nx), j = (int)(t / g.nx) - 1;
        double ubs, kp, wl, pv;
        set_face(c, i, j, 1, ubs, kp, wl, pv);
        const size_t f = fyi(g, i, j);
        c.fy_ubs[f] = ubs; c.fy_kp[f] = kp; c.fy_wl[f] = wl; c.fy_pv[f] = pv;
        face_fixed(c, i, j, 1, c.fyd, f, (size_t)tot);
    }
}
void launch_prep(const Ctx& c, cudaStream_t st) {
    k_prep_cell<<<blocks_for(c.n), TPB, 0, st>>>(c);
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
        if (r == 2) {
            const int slot = atomicAdd(&c.ns->nstrong, 1);
            c.strong_list[slot] = x;
        }
    }
}
__global__ void k_shock_strong(Ctx c) {
    const int cnt = *(volatile int*)&c.ns->nstrong;
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
void launch_shock(const Ctx& c, cudaStream_t st) {
    k_shock_weak<<<blocks_for(c.n), TPB, 0, st>>>(c);
    k_shock_strong<<<148 * 4, 32, 0, st>>>(c);
    count(c, 2);
}

// ============================================================ implicit residual (:610-731)
struct FaceV {
    double uf, pf, wL, wR, utL, utR, cL[4], cR[4];  // donors: m1, m2, e1, e2
};
// Donor m1, m2, e1, e2 of the reconstructed face value of cell (ci, cj): right (+) or left (-) face.
SPB6G_DEV void donor(const Ctx& c, int ci, int cj, int dir, bool right, double* d) {
    double qa[NV], qc[NV], qb[NV];
    const int di = dir == 0, dj = dir == 1;
    load_state(c.phy, c.g, c.Qe, ci - di, cj - dj, qa);
    load_state(c.phy, c.g, c.Qe, ci, cj, qc);
    load_state(c.phy, c.g, c.Qe, ci + di, cj + dj, qb);
    const double phi = dir == 0 ? c.phiv_x[rxi(c.g, ci, cj)] : c.phiv_y[ryi(c.g, ci, cj)];
    const int K[4] = {IM1, IM2, IE1, IE2};
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int k = K[q];
        const double sig = phi * 0.5 * (qb[k] - qa[k]);
        d[q] = right ? qc[k] + 0.5 * sig : qc[k] - 0.5 * sig;
    }
}
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
__global__ void __launch_bounds__(RED_THREADS, 2) k_residual(Ctx c, int mode, double lam) {
    const Geom& g = c.g;
    double m[1] = {0.0};
    const double* P = c.P;
    const double* dP = c.dP;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
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
void launch_residual(const Ctx& c, cudaStream_t st, int mode, double lam) {
    k_residual<<<red_blocks(c.n), RED_THREADS, 0, st>>>(c, mode, lam);
    count(c, 1);
}

// FD Jacobian rows (:837-853) with the BiCGStab set-up sums E = 1^T A 1, 1^T b, b^T b.
constexpr int JAC_THREADS = 128;
__global__ void __launch_bounds__(JAC_THREADS, 3) k_jacobian(Ctx c) {
    const Geom& g = c.g;
    double acc[3] = {0.0, 0.0, 0.0};
    const bool twoD = g.ny > 1;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
        const Nb5 p = gather_p(g, i, j, [&](int q) { return c.P[q]; });
        const double G0 = c.G[x];
        bool ok = true;
        double g1;
        const double h = 1e-7 * c.sc[x];
        ok = ok && residual_at(c, i, j, p, h, -1, 0, g1, nullptr);
        const double aC = (g1 - G0) / h;
        double av[4] = {0, 0, 0, 0};
        const int nb[4][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}};
        for (int w = 0; w < (twoD ? 4 : 2); w++) {
            const int col = mp_index(g, i + nb[w][0], j + nb[w][1]);
            const double hn = 1e-7 * c.sc[col];
            double g2;
            ok = ok && residual_at(c, i, j, p, 0, w, hn, g2, nullptr);
            av[w] = (g2 - G0) / hn;
        }
        if (!ok) atomicOr(&c.ns->fail, 2);
        c.aC[x] = aC; c.aW[x] = av[0]; c.aE[x] = av[1]; c.aS[x] = av[2]; c.aN[x] = av[3];
        double e = 0;
        e += aC; e += av[0]; e += av[1];
        if (twoD) { e += av[2]; e += av[3]; }
        c.A1[x] = e;
        c.dinv[x] = aC != 0 ? 1.0 / aC : 1.0;
        const double b = -G0;
        acc[0] += e;
        acc[1] += b;
        acc[2] += b * b;
    }
    double tot[3];
    if (grid_fold<RedSum, 3>(acc, c.partials, &c.counters[1], tot) && threadIdx.x == 0) {
        c.ns->E = tot[0]; c.ns->sumb = tot[1]; c.ns->bb = tot[2];
    }
}
void launch_jacobian(const Ctx& c, cudaStream_t st) {
    k_jacobian<<<red_blocks(c.n, JAC_THREADS), JAC_THREADS, 0, st>>>(c);
    count(c, 1);
}

// ============================================================ BiCGStab (GMRES_Solver :752-794)
// Jacobi + Nicolaides preconditioner M^-1 r = D^-1 r + 1 (1^T r)/E.  The coarse
// term is carried through the matrix as A M^-1 r = A (D^-1 r) + (1^T r / E) A 1,
// so each iteration is four passes: p & q = A D^-1 p; v, s & u = A D^-1 s; t; x & r.
template <class F>
SPB6G_DEV double spmv_row(const Ctx& c, int i, int j, int x, F val) {
    const Geom& g = c.g;
    double s = 0;
    s += c.aC[x] * val(x);
    s += c.aW[x] * val(mp_index(g, i - 1, j));
    s += c.aE[x] * val(mp_index(g, i + 1, j));
    if (g.ny > 1) {
        s += c.aS[x] * val(mp_index(g, i, j - 1));
        s += c.aN[x] * val(mp_index(g, i, j + 1));
    }
    return s;
}

__global__ void __launch_bounds__(RED_THREADS) k_bicg_init(Ctx c, double tol, int maxit) {
    const Geom& g = c.g;
    const NewtonScalars ns = *c.ns;
    const double Einv = (ns.E != 0.0 && isfinite(ns.E)) ? 1.0 / ns.E : 0.0;
    const double cb = ns.sumb * Einv;
    double acc[2] = {0.0, 0.0};
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
        auto xv = [&](int q) { return c.dinv[q] * (-c.G[q]) + cb; };
        const double Ax = spmv_row(c, i, j, x, xv);
        const double r = -c.G[x] - Ax;
        c.dP[x] = xv(x);
        c.br[x] = r;
        c.br0[x] = r;
        c.bp[x] = 0.0;
        c.bv[x] = 0.0;
        acc[0] += r * r;
        acc[1] += r * c.A1[x];
    }
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
        b.status = sqrt(b.rr) <= tol * b.bn ? BICG_CONV : (b.r0r == 0 ? BICG_FAIL : BICG_RUNNING);
    }
}
// pass 1: p = r + beta (p - omega v); q = A D^-1 p; sums 1^T p, r0^T q
__global__ void __launch_bounds__(RED_THREADS) k_bicg_p(Ctx c, const double* __restrict__ p_old, double* __restrict__ p_new) {
    const BicgScalars b = *c.bs_;
    if (b.status != BICG_RUNNING) return;
    const Geom& g = c.g;
    const double beta = (b.r0r / b.rho) * (b.alpha / b.omega), om = b.omega;
    double acc[2] = {0.0, 0.0};
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
        auto pn = [&](int q) { return c.br[q] + beta * (p_old[q] - om * c.bv[q]); };
        const double p = pn(x);
        const double q = spmv_row(c, i, j, x, [&](int k) { return c.dinv[k] * pn(k); });
        p_new[x] = p;
        c.bq[x] = q;
        acc[0] += p;
        acc[1] += c.br0[x] * q;
    }
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
    const Geom& g = c.g;
    const double al = b.alpha, cc = b.cc;
    double acc[2] = {0.0, 0.0};
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
        auto sv = [&](int q) { return c.br[q] - al * (c.bq[q] + cc * c.A1[q]); };
        const double v = c.bq[x] + cc * c.A1[x];
        const double s = c.br[x] - al * v;
        const double u = spmv_row(c, i, j, x, [&](int k) { return c.dinv[k] * sv(k); });
        c.bv[x] = v;
        c.bs[x] = s;
        c.bu[x] = u;
        acc[0] += s * s;
        acc[1] += s;
    }
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
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const double t = c.bu[x] + b.cs * c.A1[x];
        c.bt[x] = t;
        acc[0] += t * c.bs[x];
        acc[1] += t * t;
    }
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
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
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
    }
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
    }
}
void launch_bicg_init(const Ctx& c, cudaStream_t st, double tol, int maxit) {
    k_bicg_init<<<red_blocks(c.n), RED_THREADS, 0, st>>>(c, tol, maxit);
    count(c, 1);
}
// `count` iterations.  p is double-buffered (pass 1 reads neighbours' old p
// while writing the new one); `parity` selects the buffer holding the current p.
void launch_bicg_iters(const Ctx& c, cudaStream_t st, int count_, int& parity) {
    const int nb = red_blocks(c.n);
    for (int k = 0; k < count_; k++) {
        double* p0 = parity ? c.tcp : c.bp;  // tcp is the Thomas scratch, free on the BiCGStab path
        double* p1 = parity ? c.bp : c.tcp;
        k_bicg_p<<<nb, RED_THREADS, 0, st>>>(c, p0, p1);
        k_bicg_s<<<nb, RED_THREADS, 0, st>>>(c);
        k_bicg_t<<<nb, RED_THREADS, 0, st>>>(c);
        k_bicg_x<<<nb, RED_THREADS, 0, st>>>(c, p1);
        parity ^= 1;
    }
    count(c, 4 * count_);
}

// ============================================================ Thomas (1D non-periodic, :858-863)
__global__ void k_thomas(Ctx c) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const Geom& g = c.g;
    const int n = g.nx;
    double* cp = c.tcp;
    double* dp = c.tdp;
    auto coef = [&](int r, double& lo, double& di, double& up) {
        lo = up = di = 0;
        di += c.aC[r];
        const int cw = mp_index(g, r - 1, 0), ce = mp_index(g, r + 1, 0);
        const double vw = c.aW[r], ve = c.aE[r];
        if (cw == r) di += vw; else if (cw == r - 1) lo = vw; else if (cw == r + 1) up = vw;
        if (ce == r) di += ve; else if (ce == r - 1) lo = ve; else if (ce == r + 1) up = ve;
    };
    double lo, di, up;
    coef(0, lo, di, up);
    cp[0] = up / di;
    dp[0] = -c.G[0] / di;
    for (int r = 1; r < n; r++) {
        coef(r, lo, di, up);
        const double m = di - lo * cp[r - 1];
        cp[r] = up / m;
        dp[r] = (-c.G[r] - lo * dp[r - 1]) / m;
    }
    c.dP[n - 1] = dp[n - 1];
    for (int r = n - 2; r >= 0; r--) c.dP[r] = dp[r] - cp[r] * c.dP[r + 1];
}
void launch_thomas(const Ctx& c, cudaStream_t st) {
    k_thomas<<<1, 32, 0, st>>>(c);
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
__global__ void k_floor(Ctx c, double tol) {
    const Geom& g = c.g;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
        const Nb5 p = gather_p(g, i, j, [&](int q) { return c.P[q]; });
        double Gr;
        CellRes o;
        if (!residual_at(c, i, j, p, 0, -1, 0, Gr, &o)) { atomicOr(&c.ns->fail, 4); continue; }
        const double sig = closure_roundoff(c.phy, o.in, o.o.pbar);
        if (fabs(Gr) > tol * (fabs(c.p_ref + p.c) + c.kw[x] + 1.0) + sig) atomicOr(&c.ns->fail, 4);
    }
}
void launch_floor(const Ctx& c, cudaStream_t st, double tol) {
    k_floor<<<blocks_for(c.n), TPB, 0, st>>>(c, tol);
    count(c, 1);
}

// ============================================================ final state (:1056-1073) and H_s (:1363-1371)
__global__ void k_final(Ctx c) {
    const Geom& g = c.g;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < c.n; x += gridDim.x * blockDim.x) {
        const int i = x % g.nx, j = x / g.nx;
        const Nb5 p = gather_p(g, i, j, [&](int q) { return c.P[q]; });
        double Gr;
        CellRes o;
        if (!residual_at(c, i, j, p, 0, -1, 0, Gr, &o)) { atomicOr(&c.ns->fail, 8); continue; }
        double U[NV];
        U[IA1] = o.o.a[0]; U[IM1] = o.in.mtr[0]; U[IM2] = o.in.mtr[1]; U[IMU] = o.mx; U[IMV] = o.my;
        U[IE1] = o.o.e[0]; U[IE2] = o.o.e[1]; U[IEN] = o.E;
#pragma unroll
        for (int k = 0; k < NV; k++) {
            c.Ust.v[k][x] = U[k];
            c.H[(size_t)k * c.n + x] = (U[k] - c.Qs.v[k][x]) / c.adt;
        }
    }
}
void launch_final(const Ctx& c, cudaStream_t st) {
    k_final<<<blocks_for(c.n), TPB, 0, st>>>(c);
    count(c, 1);
}

// ============================================================ caldt (:502-514) and P_REF (:1309-1312)
__global__ void __launch_bounds__(RED_THREADS) k_caldt(Ctx c, CState U, int acoustic) {
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
    k_pbar_init<<<blocks_for(c.n), TPB, 0, st>>>(c, U, p_ref, P);
    count(c, 1);
}

}  // namespace spb6g
