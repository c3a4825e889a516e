// Device views of one solver's buffers, passed by value to every kernel of the
// stage pipeline, and the launchers the host driver calls.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "../../include/spb6g.h"
#include "spb6g_common.cuh"

namespace spb6g {

// Device-resident scalars of one BiCGStab solve (GMRES_Solver, src/SPB6_PC_IMEX_omp.cpp:752-794).
struct BicgScalars {
    double rho, alpha, omega, bn, Einv, cb, r0A1, cc, cs, rr, r0r, ts, tt, ss;
    double tol;
    int maxit, iters, status;
    int x0_learned;  // 1: the solve started from the learned first iterate
};
enum { BICG_RUNNING = 0, BICG_CONV = 1, BICG_FAIL = 2, BICG_CONV_HALF = 3, BICG_TIMEOUT = 4 };

// State of the software grid barrier of the persistent BiCGStab kernel.
struct GridBarrier {
    unsigned count, gen;
    int err, pad;
};
constexpr int PB_THREADS = 512;  // threads (and rows per chunk) of a persistent BiCGStab block
constexpr int PB_SLOT_Q = 8;     // partial sums per block in one grid-barrier record

// Reduction results read back by the host after a Newton decision point.
struct NewtonScalars {
    double res;    // residual max-norm of the last evaluation
    double sn;     // Newton step criterion
    double pmin;   // min pbar (P_REF) / caldt rates
    double rate_x, rate_y;
    double E, sumb, bb;  // Jacobian sums for the BiCGStab set-up
    double tmax[2];      // phase temperature maxima of the last final state (st_Tmax)
    unsigned long long rus_v[2];  // RUS_LOCAL = 0: bits of the grid-wide speeds vx_max, vy_max (:92)
    int fail;            // a residual / closure evaluation failed
    int err;             // inadmissible state in the explicit part or stage prep
    int nstrong;         // strong-shock worklist length
    int pad;
};

// Phases and scheme switches of a configuration (host side).
inline void phys_from_config(const spb6g_config* cfg, Phys& P) {
    P = Phys{};
    for (int k = 0; k < 2; k++) {
        PhaseD& h = P.ph[k];
        h.g = cfg->gamma[k]; h.pi = cfg->pinf[k]; h.q = cfg->q[k];
        h.qp = cfg->qp[k]; h.cv = cfg->cv[k]; h.b = cfg->b[k];
        h.kind = cfg->kind[k];
        h.G = cfg->mg_G[k]; h.rr = cfg->mg_rr[k]; h.c1 = cfg->mg_c1[k]; h.c2 = cfg->mg_c2[k];
        h.e1 = cfg->mg_e1[k]; h.e2 = cfg->mg_e2[k]; h.e0 = cfg->mg_e0[k];
    }
    P.share_mode = cfg->share_mode;
    P.limiter = cfg->limiter;
    P.rus_local = cfg->rus_local;
    P.mg = cfg->kind[0] != 0 || cfg->kind[1] != 0;
    P.relax = cfg->relax;
    P.eps_i = cfg->eps_i;
    // rates as main() resolves them (:1233-1235)
    P.mu_rate = cfg->mu_rate;
    P.theta_rate = cfg->theta_rate < 0 ? (cfg->relax >= 1 ? INFINITY : 0.0) : cfg->theta_rate;
    P.nu_rate = cfg->nu_rate < 0 ? ((cfg->relax == 2 || cfg->relax == 3) ? INFINITY : 0.0) : cfg->nu_rate;
    if (cfg->nu_law) P.nu_rate = 0.0;
    P.nu_cr = cfg->nu_cr;
    P.nu_pc = cfg->nu_pc;
    P.relax_form = cfg->relax_form;
    P.unify = cfg->unify;
    P.unify_proj = cfg->unify_proj;
    P.nu_law = cfg->nu_law;
    P.mech = isinf(cfg->mu_rate) ? CL_P : CL_MU;
    P.order = cfg->order == 1 ? 1 : 2;
    P.rates = (!isinf(cfg->mu_rate) || cfg->unify == 1) ? 1 : 0;
}

struct Ctx {
    Phys phy;
    Geom g;
    unsigned char* ctype;
    double* step_nu;  // nu law: each cell's mass transfer rate for the step (STEP_NU :175), else null  // per-cell closure type of the step (p-pT relaxation only)
    int n;
    int prec;  // 1: precision form (FP32 reconstruction, fluxes and SpMV), 0: FP64
    double tau, rx, ry, p_ref, adt;
    // explicit stage: Qe = Un + sum_r ce[r] H_r, Qs = Un + sum_r ci[r] H_r (main :1341-1351),
    // formed on the fly from the step's initial state and the previous stages' H
    CState Un;
    const double* Hprev;  // 8*n per earlier stage
    int nH;
    double ce[2], ci[2];
    State Xs;
    double* a2s;
    double *ube_x, *ube_y;  // (nx+1)*ny, nx*(ny+1)
    double* phis_x;         // min(phi, velocity smoothness) of cells -1..nx, (nx+2)*ny
    double* phis_y;         // nx*(ny+2)
    // stage data
    double *kw, *qph0, *qph1;
    double *pad_rho, *pad_u, *pad_v, *pad_cz;  // per-cell prep data on the padded grid (nx+4)*(ny+4)
    double *fx_ubs, *fx_kp, *fx_wl, *fx_pv;
    double *fy_ubs, *fy_kp, *fy_wl, *fy_pv;
    // per face, fixed for the stage: donors m1, m2, eps1, eps2 of the reconstructed left / right
    // face values (the reference's dxL/dxR, :936-944) and the tangential velocities of the two
    // cells (vst / ust): planes 0-3 left donor, 4-7 right donor, 8 utL, 9 utR
    double *fxd, *fyd;  // 10 planes of (nx+1)*ny / nx*(ny+1)
    int* strong_list;
    unsigned char* smask;  // 1 for cells on the strong-shock worklist of the stage
    // Newton
    double *P, *Pn, *G, *Gn, *sc, *scn, *dP;
    double *aC, *aW, *aE, *aS, *aN, *A1, *dinv;
    float *fC, *fW, *fE, *fS, *fN;  // precision form: FP32 diagonals for the SpMV
    double *br, *br0, *bp, *bv, *bq, *bs, *bu, *bt;
    double *tcp, *tdp;
    // learned warm start (no counterpart in the reference)
    double* Prate;     // pressure rate (P_converged - P_start) / sdt of the last converged stage, or null
    double* Prate2;    // the rate of the stage before it
    double* Prate3;    // and the one before that (NULL: not tracked)
    double* rate_sc;   // [0]: sigma, the RMS of Prate over the cells (0 before the first stage)
    const double* x0l; // learned first BiCGStab iterate of this solve, or null (the plain start M^-1 b)
    double sdt;        // time span of the stage: (c_s - c_{s-1}) dt, c the implicit tableau's row sums
    // final state
    State Ust;
    double* H;  // 8*n, this stage's derivative (U_s - Qs)/adt
    // reductions
    double* partials;
    unsigned* counters;  // [16]
    NewtonScalars* ns;
    BicgScalars* bs_;
    GridBarrier* gbar;  // persistent BiCGStab: barrier state (zero at start)
    double* gpart;      // persistent BiCGStab: 2 slots x G blocks x PB_SLOT_Q partial sums
    long long* nlaunch;  // host-side count of kernel launches (never dereferenced on the device)
};

SPB6G_DEV size_t fxi(const Geom& g, int i, int j) { return (size_t)(i + 1) + (size_t)j * (g.nx + 1); }
SPB6G_DEV size_t fyi(const Geom& g, int i, int j) { return (size_t)i + (size_t)(j + 1) * g.nx; }
SPB6G_DEV size_t rxi(const Geom& g, int i, int j) { return (size_t)(i + 1) + (size_t)j * (g.nx + 2); }
SPB6G_DEV size_t ryi(const Geom& g, int i, int j) { return (size_t)i + (size_t)(j + 1) * g.nx; }

// Normalisation of the warm-start features (mean / 1/std of the centre values,
// 1/std of the neighbour differences, per field) and the target scale.
constexpr int NFIELD = 7;  // rho, rho u, rho v, alpha1, E*, P, the previous stage's pressure rate / sigma
struct FeatureNorm {
    double mean[NFIELD], istd[NFIELD], idstd[NFIELD];
    double tscale;
};

// One instance of the batched form (1D, non-periodic: the Thomas path): its stage
// context and the time-loop state that the host driver keeps for a single grid.
struct BatchInst {
    Ctx c;
    double* U[NV];
    double* Ust[NV];
    double* Hs;
    double* Pbuf[3];
    int pmain;  // index of the accepted pressure in Pbuf
    int status;
    double t, dt, dtprev;
    int startup;
    // configuration
    double cfl, cfl_ac, dtfix, tend, newton_tol;
    int ramp, acdt, rk, newton_iter;
    // statistics
    long long steps, rejects, rk1, stages, newton_it, floor_count;
    double maxres;
    double tmax[2];
};

// ------------------------------------------------------------ launchers (spb6g_kernels.cu)
int red_blocks(int n, int threads = RED_THREADS);
// fused stage combination + reconstruction + Rusanov update + face donors (replaces combine/recon/update)
void launch_flux(const Ctx& c, cudaStream_t st);
// the fused explicit kernel's tile as a block-level device function (spb6g_flux.cu), and the
// shared-memory bytes of a 1D tile of width tx (128 or 256)
template <class R, int TX, int TY, bool TWO_D, bool SPEED = false>
__device__ void flux_tile(const Ctx& c, int bx, int by, unsigned char* smem_bytes, int tid, int nth);
size_t flux_tile_bytes_1d(int tx);
void launch_prep(const Ctx& c, cudaStream_t st);
// weak-shock budget + strong-shock worklist (and smask); strong-shock budget of the worklist
void launch_shock_weak(const Ctx& c, cudaStream_t st);
void launch_shock_strong(const Ctx& c, cudaStream_t st);
// mode 0: evaluate at P (writes G, sc);  mode 1: at Pn = P + lam dP (writes Pn, Gn, scn)
// skip_strong = 1 (mode 0): rows on the strong-shock worklist get only their scale s_q
void launch_residual(const Ctx& c, cudaStream_t st, int mode, double lam, int skip_strong = 0);
void launch_residual_strong(const Ctx& c, cudaStream_t st);
void launch_jacobian(const Ctx& c, cudaStream_t st);
void launch_jac_entries(const Ctx& c, cudaStream_t st, int skip_strong);
void launch_jac_strong(const Ctx& c, cudaStream_t st);
void launch_jac_finish(const Ctx& c, cudaStream_t st);
void launch_bicg_init(const Ctx& c, cudaStream_t st, double tol, int maxit);
void launch_bicg_iters(const Ctx& c, cudaStream_t st, int count, int& parity);
int build_bicg_graph(const Ctx& c, cudaStream_t st, cudaGraphExec_t* exec);
void launch_bicg_graph(const Ctx& c, cudaStream_t st, cudaGraphExec_t exec, int expected_iters);
// persistent form: number of co-resident blocks (0 when cooperative launch is unavailable) and the launch
int bicg_solve_blocks(int device, int n);
int launch_bicg_solve(const Ctx& c, cudaStream_t st, double tol, int maxit, int G);
void launch_thomas(const Ctx& c, cudaStream_t st);
// batched form: `count` instances, `nsteps` time steps each, one block of `threads` per instance,
// flux tiles of width tw (128 or 256); one persistent launch
int launch_batch(BatchInst* insts, const int* list, int count, int nsteps, int threads, int tw, int grid, cudaStream_t st);
int batch_max_blocks(int threads, int tw, int device);
// learned warm start: BF16 feature rows (n x 64), dP = sdt (Prate + y tscale), and after a converged
// stage the training target (if t) and the new pressure rate
void launch_features(const Ctx& c, cudaStream_t st, const FeatureNorm& nm, void* X);
// base_extrap = 0: dP = sdt (R + sigma y) from the stage's starting pressure; 1: dP = sdt sigma y from
// the extrapolated pressure P_start + sdt R; y = null: the extrapolation dP = sdt R
void launch_guess(const Ctx& c, cudaStream_t st, const float* y, double tscale, double a_r, double a_q, double a_c,
                  double a_y);
// residual vectors of the residual-minimising start (g[0] at the plain start, g[j] at candidate j):
// the Gram matrix of up to GRAM_K directions (upper triangle, row by row), then the right-hand side
constexpr int GRAM_K = 4;
constexpr int GRAM_Q = GRAM_K * (GRAM_K + 1) / 2 + GRAM_K;
struct GramIn {
    const double* g[GRAM_K + 1];
    int base[GRAM_K + 1];
    int K;
};
int launch_gram(const Ctx& c, cudaStream_t st, const GramIn& in, double* part, double* out);
void launch_jacobi_dir(const Ctx& c, cudaStream_t st, double coef);
void launch_rate(const Ctx& c, cudaStream_t st, const double* P0, double itscale, float* t);
// separable box average of radius r (0 < r <= nx, ny) of y, in place (tmp: n floats)
void launch_smooth(const Ctx& c, cudaStream_t st, float* y, float* tmp, int r);
void launch_stepnorm(const Ctx& c, cudaStream_t st);
void launch_apply_step(const Ctx& c, cudaStream_t st);
void launch_floor(const Ctx& c, cudaStream_t st, double tol);
void launch_final(const Ctx& c, cudaStream_t st);
void launch_relax_activate(const Ctx& c, cudaStream_t st, State U);
// Host: the packed saturation table of cfg's phases (spb6g_saturation.cu).
std::vector<double> saturation_table(const spb6g_config* cfg);
void launch_caldt(const Ctx& c, cudaStream_t st, CState U, int acoustic);
void launch_pbar_min(const Ctx& c, cudaStream_t st, CState U);
void launch_pbar_init(const Ctx& c, cudaStream_t st, CState U, double p_ref, double* P);

}  // namespace spb6g
