// Saturation line of a stiffened-gas / NASG phase pair, built on the host once per solver.
//
// Chemical relaxation (RELAX_LEVEL 2 and 3) needs the saturation temperature Tsat(p), the root in
// T of g_1(p, T) = g_2(p, T) on the branch where the vapour (phase 2) has the larger entropy.  The
// device solves it by Newton from a first guess interpolated in ln p from this table; the table
// itself is built as the reference builds it (build_sat, src/spb6_physics_omp.h:127-153), with
// glibc's log / exp / pow, so the first guesses, the critical pressure and the critical volume
// are the reference's numbers:
//   * 1600 pressures evenly spaced in ln p over [0.1, 5e9] Pa;
//   * the first pressure: the first sign change of g_1 - g_2 on 4000 geometric temperatures over
//     [20, 5000] K, refined by 200 bisections; every later pressure: Newton from the previous
//     temperature (sat_newton :116-126);
//   * the table ends at the first pressure without a root or where the liquid volume reaches the
//     vapour's (the critical point), which 100 geometric bisections then refine.
#include <cmath>
#include <vector>

#include "../../include/spb6g.h"
#include "spb6g_ctx.cuh"

namespace spb6g {
namespace {

struct PhasePT {
    double g, pi, q, qp, cv, b;
    double v(double p, double T) const { return (g - 1.0) * cv * T / (p + pi) + b; }                 // v_pT :80
    double s(double p, double T) const { return cv * (g * std::log(T) - (g - 1.0) * std::log(p + pi)) + qp; }  // :82
    double gibbs(double p, double T) const { return g * cv * T + b * p + q - T * s(p, T); }          // g_pT :83
};

struct PhasePair {
    PhasePT liq, vap;
    double gap(double p, double T) const { return liq.gibbs(p, T) - vap.gibbs(p, T); }
    // Newton on gap(p, .) from T with the step held within [T/2, 2T]; `ok` when it met the
    // relative step 1e-14, or, after 60 iterations, when the gap is within 1e-8 (|g_1| + 1).
    double newton(double p, double T, bool& ok) const {
        ok = false;
        for (int it = 0; it < 60; it++) {
            const double f = gap(p, T), d = vap.s(p, T) - liq.s(p, T);
            if (!(d > 0) || !std::isfinite(f)) return T;
            double Tn = T - f / d;
            if (Tn < 0.5 * T) Tn = 0.5 * T;
            if (Tn > 2.0 * T) Tn = 2.0 * T;
            if (std::fabs(Tn - T) < 1e-14 * T) {
                ok = true;
                return Tn;
            }
            T = Tn;
        }
        ok = std::fabs(gap(p, T)) < 1e-8 * std::fabs(liq.gibbs(p, T)) + 1e-8;
        return T;
    }
    // The first root in T: scan geometric temperatures for the sign change, then bisect.
    double first_root(double p) const {
        double Ta = 20.0, fa = gap(p, Ta);
        for (int m = 1; m <= 4000; m++) {
            const double Tb = 20.0 * std::pow(250.0, m / 4000.0), fb = gap(p, Tb);
            if (fa < 0 && fb >= 0) {
                double a = Ta, b = Tb;
                for (int it = 0; it < 200; it++) {
                    const double c = 0.5 * (a + b);
                    if (gap(p, c) < 0) a = c; else b = c;
                }
                return 0.5 * (a + b);
            }
            Ta = Tb;
            fa = fb;
        }
        return -1.0;
    }
};

}  // namespace

std::vector<double> saturation_table(const spb6g_config* cfg) {
    PhasePair P;
    PhasePT* ph[2] = {&P.liq, &P.vap};
    for (int k = 0; k < 2; k++) *ph[k] = PhasePT{cfg->gamma[k], cfg->pinf[k], cfg->q[k], cfg->qp[k], cfg->cv[k], cfg->b[k]};
    const int NP = 1600;
    const double l0 = std::log(1e-1), l1 = std::log(5e9);
    std::vector<double> lp, Ts;
    double pcrit = INFINITY, vcrit = 0.0, pmin = 0.0, Tprev = -1.0;
    for (int n = 0; n < NP; n++) {
        const double l = l0 + (l1 - l0) * n / (NP - 1), p = std::exp(l);
        double Tr = -1.0;
        if (Tprev < 0) {
            Tr = P.first_root(p);
        } else {
            bool ok;
            const double T = P.newton(p, Tprev, ok);
            if (ok) Tr = T;
        }
        if (Tr < 0) {
            if (n > 0) pcrit = std::exp(lp.back());
            break;
        }
        if (!(P.vap.v(p, Tr) > P.liq.v(p, Tr))) {  // the critical point: v_liquid = v_vapour
            pcrit = p;
            vcrit = P.liq.v(p, Tr);
            break;
        }
        lp.push_back(l);
        Ts.push_back(Tr);
        Tprev = Tr;
    }
    if (!lp.empty()) pmin = std::exp(lp.front());
    if (vcrit == 0.0 && !Ts.empty()) vcrit = P.liq.v(std::exp(lp.back()), Ts.back());
    if (std::isfinite(pcrit) && !lp.empty()) {  // the end point, by bisection in ln p
        double a = std::exp(lp.back()), b = pcrit, Ta = Ts.back();
        for (int it = 0; it < 100; it++) {
            const double c = std::sqrt(a * b);
            bool ok;
            const double T = P.newton(c, Ta, ok);
            if (ok && P.vap.v(c, T) > P.liq.v(c, T)) {
                a = c;
                Ta = T;
            } else {
                b = c;
            }
        }
        pcrit = a;
        vcrit = P.liq.v(a, Ta);
    }
    std::vector<double> out = {(double)lp.size(), pcrit, vcrit, pmin};
    out.insert(out.end(), lp.begin(), lp.end());
    out.insert(out.end(), Ts.begin(), Ts.end());
    return out;
}

}  // namespace spb6g

extern "C" int spb6g_saturation_table(const spb6g_config* cfg, double* out, int cap, int* len) {
    if (!cfg || !len) return SPB6G_BAD_ARG;
    if (cfg->kind[0] != 0 || cfg->kind[1] != 0) return SPB6G_UNSUPPORTED;
    const std::vector<double> t = spb6g::saturation_table(cfg);
    *len = (int)t.size();
    if (out) {
        if (cap < (int)t.size()) return SPB6G_TOO_LARGE;
        for (size_t i = 0; i < t.size(); i++) out[i] = t[i];
    }
    return SPB6G_OK;
}
