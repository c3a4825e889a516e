// The launchers of the extended-physics build of the kernels: the same sources compiled a second
// time with SPB6G_MG = 1 into namespace spb6g_mg (Mie-Grueneisen phases, p-pT relaxation).  The
// default (stiffened-gas / NASG, mechanical relaxation) launchers of every kernel that evaluates
// the equations of state forward to them when the configuration needs either, so the default
// kernels carry none of that code.  The
// two builds' types are the same source, hence the same layout.
#pragma once
#include <cuda_runtime.h>

#if !SPB6G_MG
namespace spb6g_mg {
struct Ctx;
struct FeatureNorm;
struct CState {
    const double* v[8];
};
struct State {
    double* v[8];
};
void launch_relax_activate(const Ctx& c, cudaStream_t st, State U);
void launch_flux(const Ctx& c, cudaStream_t st);
void launch_prep(const Ctx& c, cudaStream_t st);
void launch_shock_weak(const Ctx& c, cudaStream_t st);
void launch_shock_strong(const Ctx& c, cudaStream_t st);
void launch_residual(const Ctx& c, cudaStream_t st, int mode, double lam, int skip_strong);
void launch_residual_strong(const Ctx& c, cudaStream_t st);
void launch_jacobian(const Ctx& c, cudaStream_t st);
void launch_jac_entries(const Ctx& c, cudaStream_t st, int skip_strong);
void launch_jac_strong(const Ctx& c, cudaStream_t st);
void launch_features(const Ctx& c, cudaStream_t st, const FeatureNorm& nm, void* X);
void launch_floor(const Ctx& c, cudaStream_t st, double tol);
void launch_final(const Ctx& c, cudaStream_t st);
void launch_caldt(const Ctx& c, cudaStream_t st, CState U, int acoustic);
void launch_pbar_min(const Ctx& c, cudaStream_t st, CState U);
void launch_pbar_init(const Ctx& c, cudaStream_t st, CState U, double p_ref, double* P);
}  // namespace spb6g_mg

namespace spb6g {
inline const spb6g_mg::Ctx& mg_view(const Ctx& c) { return reinterpret_cast<const spb6g_mg::Ctx&>(c); }
inline const spb6g_mg::FeatureNorm& mg_view(const FeatureNorm& f) { return reinterpret_cast<const spb6g_mg::FeatureNorm&>(f); }
inline spb6g_mg::State mg_view(const State& u) {
    spb6g_mg::State o;
    for (int k = 0; k < 8; k++) o.v[k] = u.v[k];
    return o;
}
inline spb6g_mg::CState mg_view(const CState& u) {
    spb6g_mg::CState o;
    for (int k = 0; k < 8; k++) o.v[k] = u.v[k];
    return o;
}
}  // namespace spb6g
// First statement of a default launcher: run the extended build's launcher instead.
// SPB6G_MG_FORWARD: kernels that evaluate the closure (its type is per cell under relaxation)
// and so need the extended build for a Mie-Grueneisen phase, relax > 0, a finite mu or unify = 1.
// SPB6G_MG_FORWARD_EOS: kernels that evaluate the equations of state but never the closure;
// with stiffened-gas / NASG phases they are the same in both builds, so only a
// Mie-Grueneisen phase sends them to the extended build.
#define SPB6G_MG_FORWARD(name, ...)                      \
    do {                                                 \
        if (c.phy.mg || c.phy.relax || c.phy.rates) {    \
            spb6g_mg::name(__VA_ARGS__);                 \
            return;                                      \
        }                                                \
    } while (0)
#define SPB6G_MG_FORWARD_EOS(name, ...)                  \
    do {                                                 \
        if (c.phy.mg) {                                  \
            spb6g_mg::name(__VA_ARGS__);                 \
            return;                                      \
        }                                                \
    } while (0)
#else
#define SPB6G_MG_FORWARD(name, ...) \
    do {                            \
    } while (0)
#define SPB6G_MG_FORWARD_EOS(name, ...) \
    do {                                \
    } while (0)
#endif
