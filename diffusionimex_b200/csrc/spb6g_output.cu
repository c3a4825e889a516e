// Output formats of the reference's main() (host code); see spb6g_output.h.
#include "spb6g_output.h"

#include <algorithm>
#include <cmath>
#include <cstdio>

namespace spb6g {
namespace out {
namespace {

enum { IA1 = 0, IM1 = 1, IM2 = 2, IMU = 3, IMV = 4, IE1 = 5, IE2 = 6, IEN = 7 };

// Relations of phase k (physics :60-106), as the reference writes them: stiffened gas / NASG, or
// Mie-Grueneisen with the Cochran-Chan (kind 1) or JWL (kind 2) reference curves.
struct PhaseH {
    double g, pi, q, qp, cv, b;
    int kind;
    double G, rr, c1, c2, e1, e2, e0;
};
PhaseH phase(const spb6g_config& cf, int k) {
    return {cf.gamma[k], cf.pinf[k], cf.q[k], cf.qp[k], cf.cv[k], cf.b[k], cf.kind[k],
            cf.mg_G[k], cf.mg_rr[k], cf.mg_c1[k], cf.mg_c2[k], cf.mg_e1[k], cf.mg_e2[k], cf.mg_e0[k]};
}
void mg_ref(const PhaseH& P, double r, double& pr, double& dpr, double& er) {  // :60-69
    if (P.kind == 1) {
        const double x = r / P.rr, t1 = P.c1 * std::pow(x, P.e1), t2 = P.c2 * std::pow(x, P.e2);
        pr = t1 - t2;
        dpr = (P.e1 * t1 - P.e2 * t2) / r;
        er = (t1 / (P.e1 - 1.0) - t2 / (P.e2 - 1.0)) / r;
    } else {
        const double t1 = P.c1 * std::exp(-P.e1 * P.rr / r), t2 = P.c2 * std::exp(-P.e2 * P.rr / r);
        pr = t1 + t2;
        dpr = (P.e1 * t1 + P.e2 * t2) * P.rr / (r * r);
        er = t1 / (P.e1 * P.rr) + t2 / (P.e2 * P.rr) - P.e0;
    }
}
double p_ame(const PhaseH& P, double a, double m, double e) {
    if (P.kind) {
        double pr, dpr, er;
        mg_ref(P, m / a, pr, dpr, er);
        return P.G * (e - m * er) / a + pr;
    }
    return (e - m * P.q) * (P.g - 1.0) / (a - m * P.b) - P.g * P.pi;
}
double T_amp(const PhaseH& P, double a, double m, double p) {
    if (P.kind) {
        if (!(P.cv > 0)) return NAN;
        double pr, dpr, er;
        mg_ref(P, m / a, pr, dpr, er);
        return (a * (p - pr) / (P.G * m)) / P.cv;
    }
    return (a / m - P.b) * (p + P.pi) / ((P.g - 1.0) * P.cv);
}
double s_pT(const PhaseH& P, double p, double T) {
    return P.cv * (P.g * std::log(T) - (P.g - 1.0) * std::log(p + P.pi)) + P.qp;
}
double g_pT(const PhaseH& P, double p, double T) { return P.g * P.cv * T + P.b * p + P.q - T * s_pT(P, p, T); }
double c2_rp(const PhaseH& P, double r, double p) {
    if (P.kind) {
        double pr, dpr, er;
        mg_ref(P, r, pr, dpr, er);
        return (P.G + 1.0) * (p - pr) / r + dpr;
    }
    return P.g * (p + P.pi) / (r * (1.0 - r * P.b));
}
bool p_admissible(const PhaseH& P, double a, double m, double p) {  // :103-106
    if (P.kind) return std::isfinite(p) && c2_rp(P, m / a, p) > 0;
    return p + P.pi > 0;
}

struct Prim {
    double a1, r1, r2, u, v, p1, p2, rho, cf;
};
// prim_of (:893-902) without the mixture pressure, which cell_diag does not print.
bool prim_of(const PhaseH (&ph)[2], const double* Q, Prim& w) {
    const double a1 = Q[IA1], a2 = 1 - a1, m1 = Q[IM1], m2 = Q[IM2];
    if (!(a1 > 0 && a2 > 0 && m1 > 0 && m2 > 0)) return false;
    w.a1 = a1;
    w.rho = m1 + m2;
    w.r1 = m1 / a1;
    w.r2 = m2 / a2;
    w.u = Q[IMU] / w.rho;
    w.v = Q[IMV] / w.rho;
    w.p1 = p_ame(ph[0], a1, m1, Q[IE1]);
    w.p2 = p_ame(ph[1], a2, m2, Q[IE2]);
    if (!(p_admissible(ph[0], a1, m1, w.p1) && p_admissible(ph[1], a2, m2, w.p2))) return false;
    w.cf = std::sqrt((m1 * c2_rp(ph[0], w.r1, w.p1) + m2 * c2_rp(ph[1], w.r2, w.p2)) / w.rho);
    return true;
}
double spacing(double lo, double hi, int n) { return (hi - lo) / n; }

}  // namespace

void cell_diag(const spb6g_config& cf, const double* Q, double* o) {
    const PhaseH ph[2] = {phase(cf, 0), phase(cf, 1)};
    Prim w;
    const bool ok = prim_of(ph, Q, w);
    const double a1 = Q[IA1], m1 = Q[IM1], m2 = Q[IM2], rho = m1 + m2;
    double cw = NAN, T1 = NAN, T2 = NAN, dg = NAN;
    if (ok) {
        cw = std::sqrt(1.0 / (rho * (a1 / (w.r1 * c2_rp(ph[0], w.r1, w.p1)) + (1 - a1) / (w.r2 * c2_rp(ph[1], w.r2, w.p2)))));
        T1 = T_amp(ph[0], a1, m1, w.p1);
        T2 = T_amp(ph[1], 1 - a1, m2, w.p2);
        if (T1 > 0 && T2 > 0 && ph[0].cv > 0 && !ph[0].kind && !ph[1].kind) dg = g_pT(ph[0], w.p1, T1) - g_pT(ph[1], w.p2, T2);
    }
    o[0] = ok ? a1 * w.p1 + (1 - a1) * w.p2 : NAN;
    o[1] = ok ? w.u : NAN;
    o[2] = ok ? w.v : NAN;
    o[3] = rho;
    o[4] = 1 - a1;
    o[5] = m2 / rho;
    o[6] = ok ? w.r1 : NAN;
    o[7] = ok ? w.r2 : NAN;
    o[8] = ok ? w.cf : NAN;
    o[9] = cw;
    o[10] = T1;
    o[11] = T2;
    o[12] = ok ? w.p1 : NAN;
    o[13] = ok ? w.p2 : NAN;
    o[14] = dg;
}

int write_profile(const spb6g_config& cf, const double* U, const char* path, int prec) {
    FILE* f = std::fopen(path, "w");
    if (!f) return SPB6G_BAD_ARG;
    const double dx = spacing(cf.x0, cf.x1, cf.nx), dy = spacing(cf.y0, cf.y1, cf.ny);
    std::fprintf(f, "# x y p u v rho alpha2 Y2 rho1 rho2 c_frozen c_wood T1 T2 p1 p2 g1-g2\n");
    const int P = prec, Q = std::min(prec, 8), R = std::min(prec, 10);
    for (int j = 0; j < cf.ny; j++)
        for (int i = 0; i < cf.nx; i++) {
            double o[15];
            cell_diag(cf, U + ((size_t)j * cf.nx + i) * 8, o);
            std::fprintf(f, "%.10e %.10e %.*e %.*e %.*e %.*e %.*e %.*e %.*e %.*e %.*e %.*e %.*e %.*e %.*e %.*e %.*e\n",
                         cf.x0 + (i + 0.5) * dx, cf.y0 + (j + 0.5) * dy, P, o[0], P, o[1], P, o[2], P, o[3], P, o[4], P, o[5],
                         P, o[6], P, o[7], Q, o[8], Q, o[9], R, o[10], R, o[11], P, o[12], P, o[13], Q, o[14]);
        }
    return std::fclose(f) == 0 ? SPB6G_OK : SPB6G_BAD_ARG;
}

int write_probe(const spb6g_config& cf, const double* U, double t, double px, double py, const std::string& path, bool first) {
    const double dx = spacing(cf.x0, cf.x1, cf.nx), dy = spacing(cf.y0, cf.y1, cf.ny);
    const int i = std::min(cf.nx - 1, std::max(0, (int)std::floor((px - cf.x0) / dx)));
    const int j = std::min(cf.ny - 1, std::max(0, (int)std::floor((py - cf.y0) / dy)));
    double o[15];
    cell_diag(cf, U + ((size_t)j * cf.nx + i) * 8, o);
    FILE* f = std::fopen(path.c_str(), first ? "w" : "a");
    if (!f) return SPB6G_BAD_ARG;
    std::fprintf(f, "%.10e %.10e %.10e %.10e %.10e\n", t, o[0], o[5], o[4], o[10]);
    return std::fclose(f) == 0 ? SPB6G_OK : SPB6G_BAD_ARG;
}

std::string snap_name(const std::string& out, size_t k) {
    std::string b = out;
    if (b.size() > 4 && b.substr(b.size() - 4) == ".dat") b = b.substr(0, b.size() - 4);
    return b + "_s" + std::to_string(k) + ".dat";
}

void conserved_totals(const spb6g_config& cf, const double* U, double M[3]) {
    M[0] = M[1] = M[2] = 0;
    for (int j = 0; j < cf.ny; j++)
        for (int i = 0; i < cf.nx; i++) {
            const double* Q = U + ((size_t)j * cf.nx + i) * 8;
            M[0] += Q[IM1];
            M[1] += Q[IM2];
            M[2] += Q[IEN];
        }
}

}  // namespace out
}  // namespace spb6g
