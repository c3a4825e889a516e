// Fused explicit stage kernel: stage combination, MUSCL reconstruction with the
// shared minmod limiter, Rusanov fluxes at the material speed, the explicit
// update X* = Qs - tau div F(Qe) with the path-conservative alpha term, and the
// per-face donor states the implicit part needs.
//
// Reference: main's stage combination (src/SPB6_PC_IMEX_omp.cpp:1341-1351),
// TVDReconstruction (:369-471), RusanovC_x/y (:237-259), Update (:264-346) and
// the donor copy of PressureSubsystem (:936-944).  Arithmetic per cell and per
// face is the reference's, in its order; each quantity is computed once per
// tile from shared memory instead of once per use.
//
// One CTA owns a TX x TY tile of interior cells.  It stages Qe for the tile plus
// a two-cell halo (cross-shaped) in shared memory -- ghost cells through the
// boundary maps -- then computes per-cell scales, the reconstruction of every
// cell one layer around the tile, every face flux of the tile once, and the
// update of the tile's cells.
#include "spb6g_ctx.cuh"
#include "spb6g_mgfwd.cuh"

namespace spb6g {

namespace {

template <class R, int TX, int TY, bool TWO_D>
struct FluxTile {
    static constexpr int HY = TWO_D ? 2 : 0;
    static constexpr int NLX = TX + 4, NLY = TY + 2 * HY;
    static constexpr int NRX = TX + 2;                      // x-reconstructed cells -1..TX
    static constexpr int NRY = TWO_D ? TY + 2 : 1;          // y-reconstructed cells -1..TY
    static constexpr int NFX = TX + 1, NFY = TWO_D ? TY + 1 : 1;
    static constexpr int Q_SZ = NV * NLX * NLY;
    static constexpr int S_SZ = 4 * NLX * NLY;              // vsc, esc, u, v per staged cell
    static constexpr int RX_SZ = 3 * NRX * TY;              // phi (volume), slope u, slope v
    static constexpr int RY_SZ = TWO_D ? 3 * TX * NRY : 0;
    static constexpr int FX_SZ = 9 * NFX * TY;              // 8 fluxes + face velocity
    static constexpr int FY_SZ = TWO_D ? 9 * TX * NFY : 0;
    // precision form only: the admissibility terms L1, L2 of both phases per staged cell,
    // formed in FP64 from the FP64 state (they subtract p_inf-sized values)
    static constexpr int L_SZ = sizeof(R) == sizeof(double) ? 0 : 4 * NLX * NLY;
    static constexpr int TOTAL = Q_SZ + S_SZ + RX_SZ + RY_SZ + FX_SZ + FY_SZ + L_SZ;
    static constexpr size_t BYTES = (size_t)TOTAL * sizeof(R);
};

// Qe of a (possibly ghost) cell: the stage combination at the mapped source, then the ghost transforms.
SPB6G_DEV void load_qe(const Ctx& c, int i, int j, double* q) {
    int sx, sy;
    const int si = src_x(c.g, i, sx), sj = src_y(c.g, j, sy);
    const size_t x = (size_t)si + (size_t)sj * c.g.nx;
#pragma unroll
    for (int k = 0; k < NV; k++) {
        double e = c.Un.v[k][x];
        for (int r = 0; r < c.nH; r++) e = e + c.ce[r] * c.Hprev[((size_t)r * NV + k) * c.n + x];
        q[k] = e;
    }
    if (sx >= 0) ghost_transform(c.phy, c.g, sx, q);
    if (sy >= 0) ghost_transform(c.phy, c.g, sy, q);
}

// Frozen sound speed of prim_of (physics :893-902) without the velocity and mixture pressure,
// which the scales do not use; false where prim_of is false.
SPB6G_DEV bool frozen_cf(const Phys& P, const double* Q, double& cf) {
    const double a1 = Q[IA1], a2 = 1 - a1, m1 = Q[IM1], m2 = Q[IM2];
    if (!(a1 > 0 && a2 > 0 && m1 > 0 && m2 > 0)) return false;
    const double rho = m1 + m2, r1 = m1 / a1, r2 = m2 / a2;
    const double p1 = p_ame(P, 0, a1, m1, Q[IE1]), p2 = p_ame(P, 1, a2, m2, Q[IE2]);
    if (!(p_admissible(P, 0, a1, m1, p1) && p_admissible(P, 1, a2, m2, p2))) return false;
    cf = sqrt((m1 * c2_rp(P, 0, r1, p1) + m2 * c2_rp(P, 1, r2, p2)) / rho);
    return true;
}
// Round-off scales of TVDReconstruction (:379-385): |u| + c_f and sum |eps| + kinetic energy.
SPB6G_DEV void scales_of(const Phys& P, const double* q, double& vsc, double& esc) {
    double cf;
    const double rho = q[IM1] + q[IM2], mm = hypot(q[IMU], q[IMV]);
    vsc = (rho > 0 ? mm / rho : 0.0) + (frozen_cf(P, q, cf) ? cf : 0.0);
    esc = fabs(q[IE1]) + fabs(q[IE2]) + (rho > 0 ? 0.5 * mm * mm / rho : 0.0);
}

// Shared limiter, face-admissibility cap and velocity slopes (TVDReconstruction :399-463).
// Precision form (R = float): the same arithmetic in FP32, except the admissibility
// terms L1, L2, which arrive precomputed in FP64 (Lx[4] = L1, L2 of phase 1, then phase 2)
// because they subtract p_inf-sized energies; round-off thresholds scale with FP32's epsilon.
template <class R>
SPB6G_DEV R tiny_rel() { return sizeof(R) == sizeof(double) ? R(1e-12) : R(1e-5); }
template <class R>
SPB6G_DEV R tiny_abs() { return sizeof(R) == sizeof(double) ? R(1e-300) : R(1e-30); }

template <class R>
SPB6G_DEV void recon3(const Phys& P, const R* Ua, const R* Uc, const R* Ub, R vsa, R vsc,
                      R vsb, R esa, R esc, R esb, const R* va_, const R* vc_,
                      const R* vb_, R& phi_out, R& phis_out, R& slu, R& slv,
                      const R* La = nullptr, const R* Lc = nullptr, const R* Lb = nullptr) {
    const int VOL[5] = {IA1, IM1, IM2, IE1, IE2};
    R phi = 1.0;
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int k = VOL[q];
        const R xa = Ua[k], xc = Uc[k], xb = Ub[k];
        R sc;
        if (k == IA1) sc = 3.0;
        else if (k == IM1 || k == IM2) sc = fabs(xa) + fabs(xc) + fabs(xb);
        else sc = esa + esc + esb;
        const R a = xc - xa, b = xb - xc, tiny = tiny_rel<R>() * sc + tiny_abs<R>();
        if (!P.limiter) break;
        if (fabs(a) <= tiny && fabs(b) <= tiny) continue;
        if (a * b <= 0) { phi = 0.0; break; }
        const R cc = R(0.5) * (a + b), m = fabs(a) < fabs(b) ? a : b;
        phi = SMIN(phi, m / cc);
    }
    if (P.limiter && phi > R(0.0)) {
#pragma unroll
        for (int ph = 0; ph < 2; ph++) {
            if (SPB6G_MG && P.ph[ph].kind) continue;  // the face-admissibility bound is for NASG / SG phases (:419)
            R L1[3], L2[3];
            if constexpr (sizeof(R) == sizeof(double)) {
                const R* cs[3] = {Ua, Uc, Ub};
#pragma unroll
                for (int n = 0; n < 3; n++) {
                    const R a = ph == 0 ? cs[n][IA1] : 1.0 - cs[n][IA1], m = cs[n][ph == 0 ? IM1 : IM2],
                            e = cs[n][ph == 0 ? IE1 : IE2];
                    L1[n] = a - m * P.ph[ph].b;
                    L2[n] = e - m * P.ph[ph].q - L1[n] * P.ph[ph].pi;
                }
            } else {
                const R* ls[3] = {La, Lc, Lb};
#pragma unroll
                for (int n = 0; n < 3; n++) { L1[n] = ls[n][2 * ph]; L2[n] = ls[n][2 * ph + 1]; }
            }
            {
                const R dL = fabs(L1[2] - L1[0]);
                if (L1[1] > R(0.0) && dL > R(0.0)) phi = SMIN(phi, R(2.0) * L1[1] / dL);
            }
            {
                const R dL = fabs(L2[2] - L2[0]);
                if (L2[1] > R(0.0) && dL > R(0.0)) phi = SMIN(phi, R(2.0) * L2[1] / dL);
            }
        }
    }
    // va_, vc_, vb_: the cells' velocities (u, v) = (rho u, rho v) / (m1 + m2), computed once per cell
    const R tiny = tiny_rel<R>() * (vsa + vsc + vsb) + tiny_abs<R>();
    R sm = 1.0, sl[2];
#pragma unroll
    for (int d = 0; d < 2; d++) {
        const R va = va_[d], vc = vc_[d], vb = vb_[d], a = vc - va, b = vb - vc;
        R s = 0.0;
        if (!P.limiter) s = R(0.5) * (a + b);
        else if (!(fabs(a) <= tiny && fabs(b) <= tiny)) {
            if (a * b > 0) { s = fabs(a) < fabs(b) ? a : b; sm = SMIN(sm, s / (R(0.5) * (a + b))); }
            else sm = 0.0;
        }
        sl[d] = s;
    }
    phi_out = phi;
    phis_out = SMIN(phi, sm);
    slu = sl[0];
    slv = sl[1];
}

// Face value of a cell on its right (+) or left (-) side from the cell's stencil and its reconstruction.
template <class R>
SPB6G_DEV void face_value(const R* Ua, const R* Uc, const R* Ub, R vcu, R vcv, R phi,
                          R slu, R slv, bool right, R* w) {
    const int VOL[5] = {IA1, IM1, IM2, IE1, IE2};
#pragma unroll
    for (int q = 0; q < 5; q++) {
        const int k = VOL[q];
        const R sig = phi * R(0.5) * (Ub[k] - Ua[k]);
        w[k] = right ? Uc[k] + R(0.5) * sig : Uc[k] - R(0.5) * sig;
    }
    const R v0 = right ? vcu + R(0.5) * slu : vcu - R(0.5) * slu, v1 = right ? vcv + R(0.5) * slv : vcv - R(0.5) * slv;
    const R r = w[IM1] + w[IM2];
    w[IMU] = r * v0;
    w[IMV] = r * v1;
    w[IEN] = w[IE1] + w[IE2] + R(0.5) * r * (v0 * v0 + v1 * v1);
}

// Rusanov flux (RusanovC_x/y :237-259); returns the normal face-state velocities, which are
// also the terms of the face velocity ube (Update :283-294).  The dissipation speed is the face's
// max(|vL|, |vR|) (RUS_LOCAL = 1) or, for aglob >= 0, the grid-wide maximum aglob (RUS_LOCAL = 0).
template <class R>
SPB6G_DEV void rusanov_flux(const R* QL, const R* QR, int d, R aglob, R* flux, R& vL, R& vR) {
    const int km = d == 0 ? IMU : IMV;
    vL = QL[km] / (QL[IM1] + QL[IM2]);
    vR = QR[km] / (QR[IM1] + QR[IM2]);
    const R a = aglob >= R(0) ? aglob : SMAX(fabs(vL), fabs(vR));
#pragma unroll
    for (int k = 0; k < NV; k++) flux[k] = R(0.5) * (QL[k] * vL + QR[k] * vR) - R(0.5) * a * (QR[k] - QL[k]);
}

}  // namespace

// Non-negative doubles order as their bit patterns: the grid-wide maxima are reduced with an
// integer atomicMax on the bits.
SPB6G_DEV void atomic_max_nonneg(unsigned long long* dst, double v) {
    atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

// One TX x TY tile (tile coordinates bx, by) computed by `nth` threads of a block
// (thread index tid); `smem_bytes` holds FluxTile<...>::BYTES.  Used by k_flux
// (one tile per block) and by the batched driver (a block walks its instance's tiles).
// SPEED = true is the pre-pass of RUS_LOCAL = 0: the same reconstruction and face states,
// reduced to the grid-wide dissipation speeds a_x, a_y of Update :266-298 (max of |u|, |v| over
// the interior cells of Qe, then over the normal velocities of every face state) in
// c.ns->rus_v; it writes nothing else.
template <class R, int TX, int TY, bool TWO_D, bool SPEED>
__device__ void flux_tile(const Ctx& c, int bx, int by, unsigned char* smem_bytes, int tid, int nth) {
    using T = FluxTile<R, TX, TY, TWO_D>;
    constexpr bool MIXED = sizeof(R) != sizeof(double);
    constexpr int HY = T::HY, NLX = T::NLX, NLY = T::NLY, NRX = T::NRX, NRY = T::NRY, NFX = T::NFX, NFY = T::NFY;
    R* Qs_ = (R*)smem_bytes;                 // [NV][NLY][NLX]
    R* VS = Qs_ + T::Q_SZ;                   // [NLY][NLX]
    R* ES = VS + NLX * NLY;
    R* VU = ES + NLX * NLY;                  // cell velocity u
    R* VV = VU + NLX * NLY;                  // cell velocity v
    R* RX = VV + NLX * NLY;                  // [3][TY][NRX]
    R* RY = RX + T::RX_SZ;                   // [3][NRY][TX]
    R* FX = RY + T::RY_SZ;                   // [9][TY][NFX]
    R* FY = FX + T::FX_SZ;                   // [9][NFY][TX]
    R* LS = FY + T::FY_SZ;                   // precision form: [NLY][NLX][4] admissibility terms
    const Geom& g = c.g;
    const int i0 = bx * TX, j0 = TWO_D ? by * TY : 0;
    auto Q = [&](int k, int ly, int lx) -> R& { return Qs_[(k * NLY + ly) * NLX + lx]; };
    auto in_cross = [&](int lx, int ly) {
        if (!TWO_D) return true;
        const bool cx = lx >= 2 && lx < TX + 2, cy = ly >= HY && ly < HY + TY;
        return cx || cy;
    };
    auto exists = [&](int gi, int gj) {
        return gi >= -2 && gi <= g.nx + 1 && (TWO_D ? (gj >= -2 && gj <= g.ny + 1) : true);
    };

    double smax_x = 0.0, smax_y = 0.0;  // SPEED: this thread's maxima

    // 1. Qe of the tile and its halo; per-cell scales
    for (int t = tid; t < NLX * NLY; t += nth) {
        const int lx = t % NLX, ly = t / NLX;
        const int gi = i0 - 2 + lx, gj = TWO_D ? j0 - HY + ly : 0;
        if (!in_cross(lx, ly) || !exists(gi, gj)) continue;
        double q[NV];
        load_qe(c, gi, gj, q);
#pragma unroll
        for (int k = 0; k < NV; k++) Q(k, ly, lx) = (R)q[k];
        if (SPEED && gi >= i0 && gi < i0 + TX && gi < g.nx && (!TWO_D || (gj >= j0 && gj < j0 + TY && gj < g.ny))) {
            const double rho = q[IM1] + q[IM2];
            smax_x = fmax(smax_x, fabs(q[IMU] / rho));
            smax_y = fmax(smax_y, fabs(q[IMV] / rho));
        }
        double vs, es;
        scales_of(c.phy, q, vs, es);
        VS[ly * NLX + lx] = (R)vs;
        ES[ly * NLX + lx] = (R)es;
        const double rho = q[IM1] + q[IM2];
        VU[ly * NLX + lx] = (R)(q[IMU] / rho);
        VV[ly * NLX + lx] = (R)(q[IMV] / rho);
        if constexpr (MIXED) {
#pragma unroll
            for (int ph = 0; ph < 2; ph++) {
                const double a = ph == 0 ? q[IA1] : 1.0 - q[IA1], m = q[ph == 0 ? IM1 : IM2], e = q[ph == 0 ? IE1 : IE2];
                const double L1 = a - m * c.phy.ph[ph].b, L2 = e - m * c.phy.ph[ph].q - L1 * c.phy.ph[ph].pi;
                LS[(ly * NLX + lx) * 4 + 2 * ph] = (R)L1;
                LS[(ly * NLX + lx) * 4 + 2 * ph + 1] = (R)L2;
            }
        }
    }
    auto vel = [&](int ly, int lx, R* v) { v[0] = VU[ly * NLX + lx]; v[1] = VV[ly * NLX + lx]; };
    auto lterms = [&](int ly, int lx) -> const R* { return MIXED ? LS + (ly * NLX + lx) * 4 : nullptr; };
    __syncthreads();

    // 2. reconstruction of cells -1..TX (x) and -1..TY (y); at first order none, phi = 0 (:372-375)
    const bool first_order = c.phy.order == 1;
    for (int t = tid; t < NRX * TY; t += nth) {
        const int rx = t % NRX, ry = t / NRX;  // cell i0 - 1 + rx, row j0 + ry
        const int gi = i0 - 1 + rx, gj = j0 + ry;
        if (gi > g.nx || gj >= g.ny) continue;
        if (first_order) {
            if (!SPEED && ((gi >= i0 && gi < i0 + TX) || gi == -1 || gi == g.nx)) c.phis_x[rxi(g, gi, gj)] = 0.0;
            continue;
        }
        const int lx = rx + 1, ly = ry + HY;
        R Ua[NV], Uc[NV], Ub[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) { Ua[k] = Q(k, ly, lx - 1); Uc[k] = Q(k, ly, lx); Ub[k] = Q(k, ly, lx + 1); }
        R phi, phis, slu, slv, va[2], vc[2], vb[2];
        vel(ly, lx - 1, va); vel(ly, lx, vc); vel(ly, lx + 1, vb);
        recon3<R>(c.phy, Ua, Uc, Ub, VS[ly * NLX + lx - 1], VS[ly * NLX + lx], VS[ly * NLX + lx + 1], ES[ly * NLX + lx - 1],
                  ES[ly * NLX + lx], ES[ly * NLX + lx + 1], va, vc, vb, phi, phis, slu, slv, lterms(ly, lx - 1),
                  lterms(ly, lx), lterms(ly, lx + 1));
        RX[(0 * TY + ry) * NRX + rx] = phi;
        RX[(1 * TY + ry) * NRX + rx] = slu;
        RX[(2 * TY + ry) * NRX + rx] = slv;
        const bool own = (gi >= i0 && gi < i0 + TX) || gi == -1 || gi == g.nx;
        if (own && !SPEED) c.phis_x[rxi(g, gi, gj)] = (double)phis;
    }
    if (TWO_D) {
        for (int t = tid; t < TX * NRY; t += nth) {
            const int rx = t % TX, ry = t / TX;  // cell i0 + rx, row j0 - 1 + ry
            const int gi = i0 + rx, gj = j0 - 1 + ry;
            if (gi >= g.nx || gj > g.ny) continue;
            if (first_order) {
                if (!SPEED && ((gj >= j0 && gj < j0 + TY) || gj == -1 || gj == g.ny)) c.phis_y[ryi(g, gi, gj)] = 0.0;
                continue;
            }
            const int lx = rx + 2, ly = ry + 1;
            R Ua[NV], Uc[NV], Ub[NV];
#pragma unroll
            for (int k = 0; k < NV; k++) { Ua[k] = Q(k, ly - 1, lx); Uc[k] = Q(k, ly, lx); Ub[k] = Q(k, ly + 1, lx); }
            R phi, phis, slu, slv, va[2], vc[2], vb[2];
            vel(ly - 1, lx, va); vel(ly, lx, vc); vel(ly + 1, lx, vb);
            recon3<R>(c.phy, Ua, Uc, Ub, VS[(ly - 1) * NLX + lx], VS[ly * NLX + lx], VS[(ly + 1) * NLX + lx],
                      ES[(ly - 1) * NLX + lx], ES[ly * NLX + lx], ES[(ly + 1) * NLX + lx], va, vc, vb, phi, phis, slu, slv,
                      lterms(ly - 1, lx), lterms(ly, lx), lterms(ly + 1, lx));
            RY[(0 * NRY + ry) * TX + rx] = phi;
            RY[(1 * NRY + ry) * TX + rx] = slu;
            RY[(2 * NRY + ry) * TX + rx] = slv;
            const bool own = (gj >= j0 && gj < j0 + TY) || gj == -1 || gj == g.ny;
            if (own && !SPEED) c.phis_y[ryi(g, gi, gj)] = (double)phis;
        }
    }
    __syncthreads();

    // 3. face fluxes, face velocities ube and donors, once per face
    const size_t nfx = (size_t)(g.nx + 1) * g.ny, nfy = (size_t)g.nx * (g.ny + 1);
    R ax = R(-1), ay = R(-1);  // local dissipation speeds unless RUS_LOCAL = 0
    if (!SPEED && !c.phy.rus_local) {
        ax = (R)__longlong_as_double((long long)c.ns->rus_v[0]);
        ay = (R)__longlong_as_double((long long)c.ns->rus_v[1]);
    }
    for (int t = tid; t < NFX * TY; t += nth) {
        const int f = t % NFX, ry = t / NFX;  // face between cells i0 - 1 + f and i0 + f
        const int gl = i0 - 1 + f, gj = j0 + ry;
        if (gl > g.nx - 1 || gj >= g.ny) continue;
        const int ly = ry + HY, la = f + 1;   // local column of the left cell
        R Ua[NV], Uc[NV], Ub[NV], wR[NV], wL[NV], fl[NV];
        if (first_order) {  // the cells' own values on the face
#pragma unroll
            for (int k = 0; k < NV; k++) { wR[k] = Q(k, ly, la); wL[k] = Q(k, ly, la + 1); }
        } else {
            // right face value of the left cell
#pragma unroll
            for (int k = 0; k < NV; k++) { Ua[k] = Q(k, ly, la - 1); Uc[k] = Q(k, ly, la); Ub[k] = Q(k, ly, la + 1); }
            face_value(Ua, Uc, Ub, VU[ly * NLX + la], VV[ly * NLX + la], RX[(0 * TY + ry) * NRX + f],
                       RX[(1 * TY + ry) * NRX + f], RX[(2 * TY + ry) * NRX + f], true, wR);
            // left face value of the right cell
#pragma unroll
            for (int k = 0; k < NV; k++) { Ua[k] = Uc[k]; Uc[k] = Ub[k]; Ub[k] = Q(k, ly, la + 2); }
            face_value(Ua, Uc, Ub, VU[ly * NLX + la + 1], VV[ly * NLX + la + 1], RX[(0 * TY + ry) * NRX + f + 1],
                       RX[(1 * TY + ry) * NRX + f + 1], RX[(2 * TY + ry) * NRX + f + 1], false, wL);
        }
        R uL, uR;
        rusanov_flux<R>(wR, wL, 0, ax, fl, uL, uR);
        if (SPEED) {
            smax_x = fmax(smax_x, fmax(fabs((double)uL), fabs((double)uR)));
            continue;
        }
        const R ube = R(0.5) * (uL + uR);
#pragma unroll
        for (int k = 0; k < NV; k++) FX[(k * TY + ry) * NFX + f] = fl[k];
        FX[(8 * TY + ry) * NFX + f] = ube;
        if (f >= 1 || i0 == 0) {  // faces i0 .. i0+TX-1 belong to this tile, face -1/2 to the first
            const size_t fi = fxi(g, gl, gj);
            c.ube_x[fi] = (double)ube;
            const int K[4] = {IM1, IM2, IE1, IE2};
#pragma unroll
            for (int q = 0; q < 4; q++) {
                c.fxd[q * nfx + fi] = (double)wR[K[q]];
                c.fxd[(4 + q) * nfx + fi] = (double)wL[K[q]];
            }
        }
    }
    if (TWO_D) {
        for (int t = tid; t < TX * NFY; t += nth) {
            const int rx = t % TX, f = t / TX;  // face between rows j0 - 1 + f and j0 + f
            const int gi = i0 + rx, gl = j0 - 1 + f;
            if (gi >= g.nx || gl > g.ny - 1) continue;
            const int lx = rx + 2, la = f + 1;
            R Ua[NV], Uc[NV], Ub[NV], wR[NV], wL[NV], fl[NV];
            if (first_order) {
#pragma unroll
                for (int k = 0; k < NV; k++) { wR[k] = Q(k, la, lx); wL[k] = Q(k, la + 1, lx); }
            } else {
#pragma unroll
                for (int k = 0; k < NV; k++) { Ua[k] = Q(k, la - 1, lx); Uc[k] = Q(k, la, lx); Ub[k] = Q(k, la + 1, lx); }
                face_value(Ua, Uc, Ub, VU[la * NLX + lx], VV[la * NLX + lx], RY[(0 * NRY + f) * TX + rx],
                           RY[(1 * NRY + f) * TX + rx], RY[(2 * NRY + f) * TX + rx], true, wR);
#pragma unroll
                for (int k = 0; k < NV; k++) { Ua[k] = Uc[k]; Uc[k] = Ub[k]; Ub[k] = Q(k, la + 2, lx); }
                face_value(Ua, Uc, Ub, VU[(la + 1) * NLX + lx], VV[(la + 1) * NLX + lx], RY[(0 * NRY + f + 1) * TX + rx],
                           RY[(1 * NRY + f + 1) * TX + rx], RY[(2 * NRY + f + 1) * TX + rx], false, wL);
            }
            R vL, vR;
            rusanov_flux<R>(wR, wL, 1, ay, fl, vL, vR);
            if (SPEED) {
                smax_y = fmax(smax_y, fmax(fabs((double)vL), fabs((double)vR)));
                continue;
            }
            const R ube = R(0.5) * (vL + vR);
#pragma unroll
            for (int k = 0; k < NV; k++) FY[(k * NFY + f) * TX + rx] = fl[k];
            FY[(8 * NFY + f) * TX + rx] = ube;
            if (f >= 1 || j0 == 0) {
                const size_t fi = fyi(g, gi, gl);
                c.ube_y[fi] = (double)ube;
                const int K[4] = {IM1, IM2, IE1, IE2};
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    c.fyd[q * nfy + fi] = (double)wR[K[q]];
                    c.fyd[(4 + q) * nfy + fi] = (double)wL[K[q]];
                }
            }
        }
    }
    if (SPEED) {  // warp maxima, one atomic per warp and direction
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            smax_x = fmax(smax_x, __shfl_xor_sync(0xffffffffu, smax_x, o));
            smax_y = fmax(smax_y, __shfl_xor_sync(0xffffffffu, smax_y, o));
        }
        if ((tid & 31) == 0) {
            atomic_max_nonneg(&c.ns->rus_v[0], smax_x);
            atomic_max_nonneg(&c.ns->rus_v[1], smax_y);
        }
        return;
    }
    __syncthreads();

    // 4. explicit update of the tile's cells (Update :300-341)
    const double rx_ = c.adt / g.dx, ry_ = c.adt / g.dy;  // adt / dx, formed as the reference forms it per use
    for (int t = tid; t < TX * TY; t += nth) {
        const int rx = t % TX, ry = t / TX;
        const int gi = i0 + rx, gj = j0 + ry;
        if (gi >= g.nx || gj >= g.ny) continue;
        const size_t x = (size_t)gi + (size_t)gj * g.nx;
        const int lx = rx + 2, ly = ry + HY;
        if (!(Q(IM1, ly, lx) + Q(IM2, ly, lx) > 0)) atomicOr(&c.ns->err, 1);
        double X[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) {
            double s = c.Un.v[k][x];
            for (int r = 0; r < c.nH; r++) s = s + c.ci[r] * c.Hprev[((size_t)r * NV + k) * c.n + x];
            X[k] = s - rx_ * (double)(FX[(k * TY + ry) * NFX + rx + 1] - FX[(k * TY + ry) * NFX + rx]);
        }
        const double qa1 = (double)Q(IA1, ly, lx);
        X[IA1] += rx_ * qa1 * (double)(FX[(8 * TY + ry) * NFX + rx + 1] - FX[(8 * TY + ry) * NFX + rx]);
        if (TWO_D) {
#pragma unroll
            for (int k = 0; k < NV; k++)
                X[k] -= ry_ * (double)(FY[(k * NFY + ry + 1) * TX + rx] - FY[(k * NFY + ry) * TX + rx]);
            X[IA1] += ry_ * qa1 * (double)(FY[(8 * NFY + ry + 1) * TX + rx] - FY[(8 * NFY + ry) * TX + rx]);
        }
#pragma unroll
        for (int k = 0; k < NV; k++) c.Xs.v[k][x] = X[k];
        c.a2s[x] = 1.0 - X[IA1];
    }
}

template __device__ void flux_tile<double, 128, 1, false, false>(const Ctx&, int, int, unsigned char*, int, int);
template __device__ void flux_tile<double, 256, 1, false, false>(const Ctx&, int, int, unsigned char*, int, int);

namespace {

template <class R, int TX, int TY, bool TWO_D, bool SPEED>
__global__ void __launch_bounds__(TX * TY) k_flux(Ctx c) {
    extern __shared__ __align__(16) unsigned char flux_smem[];
    flux_tile<R, TX, TY, TWO_D, SPEED>(c, blockIdx.x, blockIdx.y, flux_smem, threadIdx.x, TX * TY);
}

template <class R, int TX, int TY, bool TWO_D>
void launch_tile(const Ctx& c, cudaStream_t st) {
    using T = FluxTile<R, TX, TY, TWO_D>;
    static unsigned long long configured = 0;  // one bit per device: the attribute is per device
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !(configured & (1ull << dev))) {
        cudaFuncSetAttribute(k_flux<R, TX, TY, TWO_D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::BYTES);
        cudaFuncSetAttribute(k_flux<R, TX, TY, TWO_D, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::BYTES);
        configured |= 1ull << dev;
    }
    const dim3 grid((unsigned)((c.g.nx + TX - 1) / TX), TWO_D ? (unsigned)((c.g.ny + TY - 1) / TY) : 1u);
    if (!c.phy.rus_local) {  // RUS_LOCAL = 0: the grid-wide speeds first (Update :266-298)
        cudaMemsetAsync(c.ns->rus_v, 0, sizeof(c.ns->rus_v), st);
        k_flux<R, TX, TY, TWO_D, true><<<grid, TX * TY, T::BYTES, st>>>(c);
        if (c.nlaunch) *c.nlaunch += 1;
    }
    k_flux<R, TX, TY, TWO_D, false><<<grid, TX * TY, T::BYTES, st>>>(c);
}

}  // namespace

size_t flux_tile_bytes_1d(int tx) {
    return tx == 128 ? FluxTile<double, 128, 1, false>::BYTES : FluxTile<double, 256, 1, false>::BYTES;
}

void launch_flux(const Ctx& c, cudaStream_t st) {
    SPB6G_MG_FORWARD_EOS(launch_flux, mg_view(c), st);
    if (c.prec) {  // precision form: reconstruction and fluxes in FP32
        if (c.g.ny > 1) launch_tile<float, 32, 8, true>(c, st);
        else launch_tile<float, 256, 1, false>(c, st);
    } else {
        if (c.g.ny > 1) launch_tile<double, 32, 8, true>(c, st);
        else launch_tile<double, 256, 1, false>(c, st);
    }
    if (c.nlaunch) *c.nlaunch += 1;
}

}  // namespace spb6g
