// Host driver of the B200 SPB6 IMEX solver and the C ABI of include/spb6g.h.
//
// The time loop, attempt/halving logic, stage combination and Newton control
// follow main() (src/SPB6_PC_IMEX_omp.cpp:1316-1384) and Newton_Solver
// (:799-904) decision for decision.  All field data stays on the device; the
// host reads back only the scalars a decision needs (residual norm, step
// criterion, BiCGStab status), through one pinned record per sync point.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/spb6g.h"
#include "spb6g_ctx.cuh"
#include "spb6g_output.h"

using namespace spb6g;

namespace {

enum TimerGroup { TG_EXPLICIT = 0, TG_PREP, TG_SHOCK, TG_RESIDUAL, TG_JACOBIAN, TG_LINEAR, TG_FINAL, TG_CALDT, TG_WARM, TG_COUNT };
const char* kTimerNames[TG_COUNT] = {"explicit", "prep", "shock", "residual", "jacobian", "linear", "final", "caldt", "warmstart"};

struct Pinned {
    NewtonScalars ns;
    BicgScalars bs;
};

}  // namespace

struct spb6g_solver {
    spb6g_config cfg;
    Phys P;
    Geom g;
    int n = 0;
    cudaStream_t st = nullptr;
    std::vector<void*> allocs;
    // state
    double *U[NV], *Ust[NV], *Xs[NV];
    double* Hs = nullptr;  // 3 stages x 8 x n
    double* Pbuf[3] = {nullptr, nullptr, nullptr};
    double* Pmain = nullptr;  // accepted pressure unknown; the other two buffers hold the Newton iterate and trial
    double* sc_build = nullptr;  // jreuse: the row scales s_q of the last Jacobian build (:831-836)
    Ctx c{};
    Pinned* pin = nullptr;
    // time state
    double t = 0, dt = 0, dtprev = -1, p_ref = 0;
    bool startup = true;
    spb6g_stats stats{};
    int bicg_parity = 0;
    // timing: events recorded around kernel groups, resolved at the next host sync
    bool timing = false;
    std::vector<cudaEvent_t> ev_pool;
    struct Pending { int group; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    cudaEvent_t open_ev = nullptr;
    double tms[TG_COUNT] = {};
    int64_t tcnt[TG_COUNT] = {};
    cudaEvent_t region[2] = {nullptr, nullptr};
    long long nlaunch = 0;
    int bicg_G = 0;                       // blocks of the persistent BiCGStab launch (0: not available)
    cudaGraphExec_t bicg_exec = nullptr;  // device-side BiCGStab loop (built once per solver)
    cudaStream_t st2 = nullptr;           // side stream: shock budget, overlapped with the stage prep
    cudaEvent_t ev_flux = nullptr, ev_weak = nullptr, ev_shock = nullptr;
    int last_bicg_iters = 8;
    // learned warm start (no counterpart in the reference)
    spb6g_mlp* warm = nullptr;          // network giving the first Newton guess (NULL: plain guess only)
    FeatureNorm norm{};                 // feature normalisation and target scale
    void* featbuf = nullptr;            // n x 64 BF16 feature rows of the current stage
    float* ybuf = nullptr;              // network output per cell
    double* Pstart = nullptr;           // stage's starting pressure (pressure rate, training targets)
    double* Prate = nullptr;            // pressure rate of the last converged stage (a feature and the extrapolation)
    double* Prate2 = nullptr;           // the rate of the stage before it
    double* Prate3 = nullptr;           // and the one before that
    double* rate_sc = nullptr;          // RMS of Prate (device scalar)
    bool rate_ready = false;            // a stage has converged since the tracking began (R exists)
    double span1 = 0.0, span2 = 0.0;    // time spans of the stages behind Prate and Prate2 (0: none yet)
    double span3 = 0.0;                 // and behind Prate3
    bool jac_ready = false;             // a Jacobian has been built (its diagonal's inverse is in dinv)
    double* x0buf = nullptr;            // learned first BiCGStab iterate of a stage
    double* gstore = nullptr;           // (GRAM_K + 1) x n residuals of the residual-minimising start
    double* scstore = nullptr;          // GRAM_K x n row scales of its candidates
    NewtonScalars* cand_ns = nullptr;   // and their norms and failure flags
    double* gram_part = nullptr;        // its per-block inner products
    double* gram = nullptr;             // and their totals
    int warm_mode = 15;                 // bits: 1 learned Newton start, 2 learned first BiCGStab iterate,
                                        // 4 the last Newton correction as the next solve's first iterate,
                                        // 8 residual-minimising combination, 16 Jacobi sweeps of the start,
                                        // 32 the older rate change as a fourth direction
    int warm_smooth = 0;                // radius of the box average of the network's output (0: none)
    float* ytmp = nullptr;              // scratch of the smoothing
    double stage_c = 0;                 // implicit stage time c_s of the last stage run (for the next stage's span)
    int attempt_stage = -1;             // stage-level API: the last stage of the attempt that converged (-1: none)
    void* rows_cur = nullptr;           // where this stage's feature rows were written
    void* dumpX = nullptr;              // caller's buffers for (feature row, target) pairs
    float* dumpT = nullptr;
    int64_t dump_cap = 0, dump_count = 0;
    bool dump_stage = false;
    // output of main() (snap=, probe=, prec=, the final profile; :1325, :1380-1387)
    std::string out_file;
    std::vector<double> snaps;
    size_t snapi = 0;
    bool probe = false;
    double probe_x = 0, probe_y = 0;
    int prec = 16;
    double M0[3] = {0, 0, 0};           // conserved totals at the start of the run (:1251)
    std::vector<double> host_U;         // AoS staging of the state for the writers
    int verbose = 0;                    // SPB6G_VERBOSE >= 3: one line per Newton iteration (VERBOSE, :810)
};

namespace {

#define CK(x)                                                                                        \
    do {                                                                                             \
        cudaError_t e_ = (x);                                                                        \
        if (e_ != cudaSuccess) {                                                                     \
            fprintf(stderr, "spb6g: CUDA error %s at %s:%d\n", cudaGetErrorString(e_), __FILE__, __LINE__); \
            return SPB6G_CUDA_ERROR;                                                                 \
        }                                                                                            \
    } while (0)

// Keep [p, p + bytes) in the persisting part of L2 for the solver's kernels: the set-aside is the
// smaller of the block and the device's maximum (a limit of this process's context, gone with
// it), the window covers as much of the block as one window may, and its hit ratio is the part
// of the window the set-aside holds.  Without persisting L2 the accesses stay normal.
static void persist_in_l2(spb6g_solver* s, void* p, size_t bytes) {
    int dev = 0, max_persist = 0, max_window = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev) != cudaSuccess ||
        max_persist <= 0 || max_window <= 0) {
        cudaGetLastError();
        return;
    }
    const size_t set_aside = bytes < (size_t)max_persist ? bytes : (size_t)max_persist;
    const size_t window = bytes < (size_t)max_window ? bytes : (size_t)max_window;
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, set_aside) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    cudaStreamAttrValue a = {};
    a.accessPolicyWindow.base_ptr = p;
    a.accessPolicyWindow.num_bytes = window;
    a.accessPolicyWindow.hitRatio = (float)((double)set_aside / (double)window < 1.0 ? (double)set_aside / (double)window : 1.0);
    a.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    a.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    for (cudaStream_t st : {s->st, s->st2})
        if (st && cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &a) != cudaSuccess) cudaGetLastError();
}

double* dalloc(spb6g_solver* s, size_t count) {
    void* p = nullptr;
    if (cudaMalloc(&p, (count ? count : 1) * sizeof(double)) != cudaSuccess) return nullptr;
    cudaMemsetAsync(p, 0, (count ? count : 1) * sizeof(double), s->st);
    s->allocs.push_back(p);
    return (double*)p;
}

cudaEvent_t pool_event(spb6g_solver* s) {
    if (s->ev_pool.empty()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        return e;
    }
    cudaEvent_t e = s->ev_pool.back();
    s->ev_pool.pop_back();
    return e;
}
void tbegin(spb6g_solver* s, int, cudaStream_t st = nullptr) {
    if (!s->timing) return;
    s->open_ev = pool_event(s);
    if (s->open_ev) cudaEventRecord(s->open_ev, st ? st : s->st);
}
void tend_(spb6g_solver* s, int g, cudaStream_t st = nullptr) {
    if (!s->timing || !s->open_ev) return;
    cudaEvent_t b = pool_event(s);
    if (!b) return;
    cudaEventRecord(b, st ? st : s->st);
    s->pending.push_back({g, s->open_ev, b});
    s->open_ev = nullptr;
}
// Stage prep on the main stream while the shock budget (whose strong-shock cells each
// integrate a shock profile serially) runs on the side stream; joined before Newton.
// Stage data on the main stream, shock budget on the side stream.  The main
// stream joins the side stream inside newton(): its first residual and the
// Jacobian rows of cells without a strong-shock budget run while the
// strong-shock worklist is still being integrated.
void prep_and_shock(spb6g_solver* s) {
    Ctx& c = s->c;
    cudaEventRecord(s->ev_flux, s->st);
    cudaStreamWaitEvent(s->st2, s->ev_flux, 0);
    tbegin(s, TG_SHOCK, s->st2);
    launch_shock_weak(c, s->st2);
    cudaEventRecord(s->ev_weak, s->st2);
    launch_shock_strong(c, s->st2);
    tend_(s, TG_SHOCK, s->st2);
    cudaEventRecord(s->ev_shock, s->st2);
    tbegin(s, TG_PREP);
    launch_prep(c, s->st);
    tend_(s, TG_PREP);
}
// Accumulates every completed group (called after a stream synchronisation).
void resolve_timing(spb6g_solver* s) {
    for (auto& p : s->pending) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            s->tms[p.group] += ms;
            s->tcnt[p.group] += 1;
        }
        s->ev_pool.push_back(p.a);
        s->ev_pool.push_back(p.b);
    }
    s->pending.clear();
}

int sync_read(spb6g_solver* s, bool bicg) {
    CK(cudaMemcpyAsync(&s->pin->ns, s->c.ns, sizeof(NewtonScalars), cudaMemcpyDeviceToHost, s->st));
    if (bicg) CK(cudaMemcpyAsync(&s->pin->bs, s->c.bs_, sizeof(BicgScalars), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (!s->pending.empty()) resolve_timing(s);
    return SPB6G_OK;
}
int reset_flags(spb6g_solver* s) {
    // fail, err, nstrong are contiguous ints at the end of NewtonScalars
    CK(cudaMemsetAsync(&s->c.ns->fail, 0, 3 * sizeof(int), s->st));
    return SPB6G_OK;
}
int reset_fail(spb6g_solver* s) {
    CK(cudaMemsetAsync(&s->c.ns->fail, 0, sizeof(int), s->st));
    return SPB6G_OK;
}

// Newton iterate and line-search trial live in the two buffers that are not Pmain.
int begin_attempt_pressure(spb6g_solver* s) {
    double* other[2];
    int k = 0;
    for (int b = 0; b < 3; b++)
        if (s->Pbuf[b] != s->Pmain) other[k++] = s->Pbuf[b];
    CK(cudaMemcpyAsync(other[0], s->Pmain, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    s->c.P = other[0];
    s->c.Pn = other[1];
    return SPB6G_OK;
}

void set_tab(int rk, double Ae[3][3], double Ai[3][3]) {  // main's set_tab, :1281-1303
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) Ae[a][b] = Ai[a][b] = 0;
    if (rk == 1) {
        Ai[0][0] = 1.0;
    } else if (rk == 2) {
        const double bb = 1.0 - 1.0 / std::sqrt(2.0), cc = 1.0 / (2.0 * bb);
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

int caldt(spb6g_solver* s, bool acoustic, double& inv) {
    CState u;
    for (int k = 0; k < NV; k++) u.v[k] = s->U[k];
    tbegin(s, TG_CALDT);
    launch_caldt(s->c, s->st, u, acoustic ? 1 : 0);
    tend_(s, TG_CALDT);
    int rc = sync_read(s, false);
    if (rc) return rc;
    const double rate = s->pin->ns.rate_x / s->g.dx + (s->g.ny > 1 ? s->pin->ns.rate_y / s->g.dy : 0.0);
    inv = rate > 0 ? 1.0 / rate : INFINITY;
    return SPB6G_OK;
}

// Coefficients x minimising ||g0 + sum_j x_j w_j||_2 from the Gram sums m (k_gram's layout):
// the normal equations by Cholesky, with a relative ridge of 1e-12 on the diagonal, over the
// directions of `mask` whose ||w_j||^2 is above 1e-24 of the largest (the others get 0: a zero
// network output adds no direction).  False when nothing is left or the system is not finite.
static bool solve_gram(const double* m, int K, double* x, unsigned mask = ~0u) {
    int idx[GRAM_K][GRAM_K];
    for (int j = 0, q = 0; j < GRAM_K; j++)
        for (int k = j; k < GRAM_K; k++, q++) idx[j][k] = idx[k][j] = q;
    const double* rhs = m + GRAM_K * (GRAM_K + 1) / 2;
    double dmax = 0.0;
    for (int i = 0; i < K; i++)
        if ((mask >> i) & 1u) dmax = std::max(dmax, m[idx[i][i]]);
    if (!(dmax > 0.0) || !std::isfinite(dmax)) return false;
    int act[GRAM_K], na = 0;
    for (int i = 0; i < K; i++) {
        x[i] = 0.0;
        if (((mask >> i) & 1u) && m[idx[i][i]] > 1e-24 * dmax) act[na++] = i;
    }
    double L[GRAM_K][GRAM_K] = {}, y[GRAM_K], z[GRAM_K];
    for (int i = 0; i < na; i++) {
        for (int j = 0; j <= i; j++) {
            double v = m[idx[act[i]][act[j]]] * (i == j ? 1.0 + 1e-12 : 1.0);
            for (int k = 0; k < j; k++) v -= L[i][k] * L[j][k];
            if (i == j) {
                if (!(v > 0.0) || !std::isfinite(v)) return false;
                L[i][i] = std::sqrt(v);
            } else {
                L[i][j] = v / L[j][j];
            }
        }
    }
    for (int i = 0; i < na; i++) {
        double v = -rhs[act[i]];
        for (int k = 0; k < i; k++) v -= L[i][k] * y[k];
        y[i] = v / L[i][i];
    }
    for (int i = na - 1; i >= 0; i--) {
        double v = y[i];
        for (int k = i + 1; k < na; k++) v -= L[k][i] * z[k];
        z[i] = v / L[i][i];
    }
    for (int i = 0; i < na; i++) {
        if (!std::isfinite(z[i])) return false;
        x[act[i]] = z[i];
    }
    return true;
}

// Evaluates the residual at P + dP (into Pn, Gn, scn), copying Gn to `keep` if given; r is the
// max-norm, or infinity where a closure failed.
static int eval_warm(spb6g_solver* s, Ctx& c, const char* what, double* keep, double best, double& r,
                     double* keep_sc = nullptr) {
    launch_residual(c, s->st, 1, 1.0);
    if (keep && cudaMemcpyAsync(keep, c.Gn, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st) != cudaSuccess)
        return -1;
    if (keep_sc && cudaMemcpyAsync(keep_sc, c.scn, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st) != cudaSuccess)
        return -1;
    if (sync_read(s, false)) return -1;
    r = s->pin->ns.fail ? INFINITY : s->pin->ns.res;
    if (s->verbose >= 3) fprintf(stderr, "    %s guess res %.3e, best so far %.3e\n", what, r, best);
    if (reset_fail(s)) return -1;
    return 0;
}
// The evaluated guess (Pn, Gn, scn) becomes the start.
static void take_warm(Ctx& c, double& res, double r) {
    std::swap(c.P, c.Pn);
    std::swap(c.G, c.Gn);
    std::swap(c.sc, c.scn);
    res = r;
}

// Newton_Solver (:799-904), jreuse = 0.  P lives in s->c.P (the stage pressure).
int newton(spb6g_solver* s, double& resfinal) {
    Ctx& c = s->c;
    const bool tri = s->g.ny == 1 && s->g.bcs[0] != BC_PERIODIC;
    const double tol = s->cfg.newton_tol;
    if (reset_fail(s)) return SPB6G_CUDA_ERROR;
    // First evaluation (evalAll + norm).  Rows whose strong-shock budget is still
    // being integrated on the side stream are skipped, and the Jacobian rows of all
    // other cells are formed ahead (used only if the first norm is above tolerance);
    // after the join the worklist rows follow.  Residual failures set bit 1 of
    // ns.fail, Jacobian failures bit 2.
    // (With a warm start the first iterate may change, so no rows are formed ahead.)
    const bool ahead = s->warm == nullptr;
    CK(cudaStreamWaitEvent(s->st, s->ev_weak, 0));
    tbegin(s, TG_RESIDUAL);
    launch_residual(c, s->st, 0, 0.0, 1);
    tend_(s, TG_RESIDUAL);
    if (ahead) {
        tbegin(s, TG_JACOBIAN);
        launch_jac_entries(c, s->st, 1);
        tend_(s, TG_JACOBIAN);
    }
    CK(cudaStreamWaitEvent(s->st, s->ev_shock, 0));
    tbegin(s, TG_RESIDUAL);
    launch_residual_strong(c, s->st);
    tend_(s, TG_RESIDUAL);
    if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
    if (s->pin->ns.err) return SPB6G_INADMISSIBLE;  // Update / prep admissibility (:272, :929)
    if (s->pin->ns.fail & 1) { resfinal = INFINITY; return SPB6G_NEWTON_FAIL; }
    double res = s->pin->ns.res;
    bool x0_pending = false;
    // learned prediction of the stage's pressure: P_start + sdt (R + sigma MLP(features))
    bool have_pred = false, warm_start = false;
    if (s->warm && s->rate_ready) {
        tbegin(s, TG_WARM);
        if (spb6g_mlp_forward(s->warm, s->rows_cur, s->n, s->ybuf, s->st) != SPB6G_OK) return SPB6G_CUDA_ERROR;
        if (s->warm_smooth > 0) launch_smooth(c, s->st, s->ybuf, s->ytmp, s->warm_smooth);
        have_pred = true;
        // the start on the rate model: P = P_start + sdt (b_r R + b_q (R - R2) + b_c (R2 - R3) + b_y sigma y)
        double b_r = 0.0, b_q = 0.0, b_c = 0.0, b_y = 0.0;
        warm_start = (s->warm_mode & 1) != 0;
        if (s->warm_mode & 1) {
            auto eval_guess = [&](const char* what, double* keep, double& r) { return eval_warm(s, c, what, keep, res, r); };
            auto take = [&](double r) { take_warm(c, res, r); };
            const double kq = s->span2 > 0.0 ? (s->span1 + c.sdt) / (s->span2 + s->span1) : 0.0;
            if (s->warm_mode & 8) {
                // Residual-minimising start: from the plain start P0 the candidates -- the
                // extrapolation, the second-order extrapolation, with bit 32 the extrapolation plus
                // the older rate change, and the network's guess -- give the residual's change along
                // the directions sdt R, sdt kq (R - R2), sdt (R2 - R3) and sdt sigma y; the start
                // combining them that minimises ||G||_2 of the residual taken linear in P is
                // evaluated too, and the candidate of smallest max-norm starts Newton.
                constexpr int NC = 4;
                double* const gst = s->gstore;
                CK(cudaMemcpyAsync(gst, c.G, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
                const double coef[NC][4] = {{1.0, 0.0, 0.0, 0.0}, {1.0, kq, 0.0, 0.0}, {1.0, 0.0, 1.0, 0.0}, {1.0, 0.0, 0.0, 1.0}};
                const bool avail[NC] = {true, kq > 0.0, (s->warm_mode & 32) && s->span3 > 0.0, true};
                const char* names[NC] = {"extrapolated", "second-order extrapolated", "older rate change", "learned"};
                auto guess = [&](const double* k) {
                    launch_guess(c, s->st, k[3] != 0.0 ? s->ybuf : nullptr, s->norm.tscale, k[0], k[1], k[2], k[3]);
                };
                // the candidates' residuals (kept with their row scales and norms), then the Gram
                // sums over all of them, with one read-back for everything
                double cres[NC];
                for (int k = 0; k < NC; k++) {
                    cres[k] = INFINITY;
                    if (!avail[k]) continue;
                    guess(coef[k]);
                    launch_residual(c, s->st, 1, 1.0);
                    CK(cudaMemcpyAsync(gst + (size_t)(k + 1) * s->n, c.Gn, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
                    CK(cudaMemcpyAsync(s->scstore + (size_t)k * s->n, c.scn, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
                    CK(cudaMemcpyAsync(s->cand_ns + k, c.ns, sizeof(NewtonScalars), cudaMemcpyDeviceToDevice, s->st));
                    if (reset_fail(s)) return SPB6G_CUDA_ERROR;
                }
                // directions: the extrapolation from P0, the other terms from the extrapolation;
                // g[0] the residual at P0, g[1] at the extrapolation, w_j = g[j] - g[base_j]
                GramIn gi{};
                double dir[NC][4];
                int K = 0, cand_of[NC];
                gi.g[0] = gst;
                for (int k = 0; k < NC; k++) {
                    if (!avail[k]) continue;
                    gi.g[K + 1] = gst + (size_t)(k + 1) * s->n;
                    gi.base[K + 1] = k == 0 ? 0 : 1;
                    for (int q = 0; q < 4; q++) dir[K][q] = coef[k][q] - (k == 0 ? 0.0 : coef[0][q]);
                    cand_of[K++] = k;
                }
                gi.K = K;
                if (launch_gram(c, s->st, gi, s->gram_part, s->gram) != 0) return SPB6G_CUDA_ERROR;
                NewtonScalars cns[NC];
                double m[GRAM_Q];
                CK(cudaMemcpyAsync(cns, s->cand_ns, sizeof cns, cudaMemcpyDeviceToHost, s->st));
                CK(cudaMemcpyAsync(m, s->gram, sizeof m, cudaMemcpyDeviceToHost, s->st));
                CK(cudaStreamSynchronize(s->st));
                for (int k = 0; k < NC; k++) {
                    if (!avail[k]) continue;
                    cres[k] = cns[k].fail ? INFINITY : cns[k].res;
                    if (s->verbose >= 3) fprintf(stderr, "    %s guess res %.3e, best so far %.3e\n", names[k], cres[k], res);
                }
                // the combination over the directions whose candidates' closures succeeded (each
                // is taken from the extrapolation, so that one has to)
                unsigned mask = 0;
                if (std::isfinite(cres[0]))
                    for (int j = 0; j < K; j++)
                        if (std::isfinite(cres[cand_of[j]])) mask |= 1u << j;
                double cc[4] = {0.0, 0.0, 0.0, 0.0}, cres_ls = INFINITY;
                double x[GRAM_K];
                if (mask && solve_gram(m, K, x, mask)) {
                    for (int j = 0; j < K; j++)
                        for (int q = 0; q < 4; q++) cc[q] += x[j] * dir[j][q];
                    guess(cc);
                    if (eval_guess("combined", nullptr, cres_ls) < 0) return SPB6G_CUDA_ERROR;
                }
                // the smallest max-norm among the plain start, the candidates and the combination
                int best = -1;
                double rb = res;
                for (int k = 0; k < NC; k++)
                    if (cres[k] < rb) { rb = cres[k]; best = k; }
                const double* pick = nullptr;
                if (cres_ls < rb) {
                    take(cres_ls);
                    pick = cc;
                    s->stats.combined++;
                } else if (best >= 0) {
                    // the candidate's trial state from its kept residual and row scales: Pn = P0 + dP
                    // (as the residual's trial forms it), Gn, scn
                    const size_t nb = (size_t)s->n * sizeof(double);
                    guess(coef[best]);
                    CK(cudaMemcpyAsync(c.Pn, c.P, nb, cudaMemcpyDeviceToDevice, s->st));
                    Ctx cp = c;
                    cp.P = c.Pn;
                    launch_apply_step(cp, s->st);
                    CK(cudaMemcpyAsync(c.Gn, gst + (size_t)(best + 1) * s->n, nb, cudaMemcpyDeviceToDevice, s->st));
                    CK(cudaMemcpyAsync(c.scn, s->scstore + (size_t)best * s->n, nb, cudaMemcpyDeviceToDevice, s->st));
                    take(cres[best]);
                    pick = coef[best];
                    if (best == 3) s->stats.learned++;
                    else if (best == 0) s->stats.extrapolated++;
                    else s->stats.extrapolated2++;
                }
                if (pick) { b_r = pick[0]; b_q = pick[1]; b_c = pick[2]; b_y = pick[3]; }
            } else {
                // the candidates in sequence, each tried against the best so far: the extrapolation
                // P_start + sdt R (the network's y = 0), the second-order extrapolation, then the
                // network's guess
                double r = 0;
                launch_guess(c, s->st, nullptr, s->norm.tscale, 1.0, 0.0, 0.0, 0.0);
                if (eval_guess("extrapolated", nullptr, r) < 0) return SPB6G_CUDA_ERROR;
                const bool ex = r < res;
                if (ex) { take(r); b_r = 1.0; }
                // second order: the rate taken linear in time through the midpoints of the last two
                // stages (R at the last one's, R2 at the one before), averaged over this stage
                bool eq = false;
                if (kq > 0.0) {
                    launch_guess(c, s->st, nullptr, s->norm.tscale, 1.0 - b_r, kq, 0.0, 0.0);
                    if (eval_guess("second-order extrapolated", nullptr, r) < 0) return SPB6G_CUDA_ERROR;
                    eq = r < res;
                    if (eq) { take(r); b_r = 1.0; b_q = kq; }
                }
                // the network's guess P_start + sdt (R + sigma y), from the chosen start
                launch_guess(c, s->st, s->ybuf, s->norm.tscale, 1.0 - b_r, -b_q, 0.0, 1.0);
                if (eval_guess("learned", nullptr, r) < 0) return SPB6G_CUDA_ERROR;
                if (r < res) {
                    take(r);
                    b_r = 1.0; b_q = 0.0; b_y = 1.0;
                    s->stats.learned++;
                } else if (eq) {
                    s->stats.extrapolated2++;
                } else if (ex) {
                    s->stats.extrapolated++;
                }
            }
        }
        // mode bit 16: up to two Jacobi sweeps on the nonlinear residual from the chosen start, with
        // the diagonal of the last Jacobian built (the previous stage's) and the step length that
        // minimises ||G||_2 of the residual taken linear along the step; a sweep stands when it
        // lowers the max-norm.  Only for a start within 30 tolerances: a sweep cuts the max-norm
        // by 4-10x, which can spare the stage its Newton iterations there, and not elsewhere.
        bool refined = false;
        if ((s->warm_mode & 16) && s->jac_ready && !tri && res < 30.0 * tol) {
            double* const gst = s->gstore;
            for (int sweep = 0; sweep < 2 && res >= tol; sweep++) {
                double r1 = INFINITY, r2 = INFINITY, x = 0.0;
                CK(cudaMemcpyAsync(gst, c.G, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
                launch_jacobi_dir(c, s->st, 1.0);
                if (eval_warm(s, c, "jacobi", gst + s->n, res, r1) < 0) return SPB6G_CUDA_ERROR;
                if (std::isfinite(r1)) {
                    GramIn gi{};
                    gi.g[0] = gst;
                    gi.g[1] = gst + s->n;
                    gi.K = 1;
                    if (launch_gram(c, s->st, gi, s->gram_part, s->gram) != 0) return SPB6G_CUDA_ERROR;
                    double m[GRAM_Q];
                    CK(cudaMemcpyAsync(m, s->gram, sizeof m, cudaMemcpyDeviceToHost, s->st));
                    CK(cudaStreamSynchronize(s->st));
                    if (solve_gram(m, 1, &x) && x != 1.0) {
                        launch_jacobi_dir(c, s->st, x);
                        if (eval_warm(s, c, "jacobi, step length", nullptr, res, r2) < 0) return SPB6G_CUDA_ERROR;
                    }
                }
                if (r2 < res && r2 <= r1) {
                    take_warm(c, res, r2);
                } else if (r1 < res) {
                    launch_jacobi_dir(c, s->st, 1.0);
                    if (eval_warm(s, c, "jacobi", nullptr, res, r1) < 0) return SPB6G_CUDA_ERROR;
                    take_warm(c, res, r1);
                } else {
                    break;
                }
                refined = true;
            }
            if (refined) s->stats.refined++;
        }
        tend_(s, TG_WARM);
        // the network's step from the chosen start is the first BiCGStab iterate's candidate,
        // unless the start is the network's guess itself or Jacobi sweeps moved it
        const bool is_net = b_r == 1.0 && b_q == 0.0 && b_c == 0.0 && b_y == 1.0;
        x0_pending = have_pred && !is_net && !refined && (s->warm_mode & 2) && !tri && s->bicg_G > 0;
        if (x0_pending) {
            launch_guess(c, s->st, s->ybuf, s->norm.tscale, 1.0 - b_r, -b_q, -b_c, 1.0 - b_y);
            CK(cudaMemcpyAsync(s->x0buf, c.dP, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
        }
    }
    // jreuse (modified Newton, :826-830, :887): the Jacobian is rebuilt at the first iteration, after
    // a damped step or a contraction above 0.25 (fresh_ok :797), and when the kept one lets the
    // line search fail; the step criterion meanwhile uses the scales of the last build
    const bool jreuse = s->cfg.jreuse != 0;
    double ratio = 1.0, lamprev = 1.0;
    bool fresh = false;
    // mode bit 4: from the second solve of the stage on, the last Newton correction dP (the last
    // solve's solution, still in dP) is the first iterate's candidate, combined with M^-1 b the same way
    const bool hist_x0 = s->warm && (s->warm_mode & 4) && !tri && s->bicg_G > 0;
    for (int it = 0; it < s->cfg.newton_iter; it++) {
        resfinal = res;
        if (s->verbose >= 3) fprintf(stderr, "    newton it %d res %.3e\n", it, res);
        // a warm start below the tolerance still takes one Newton step: the solve, not the
        // prediction, ends every stage (a start accepted as it is would stop the stage at the
        // tolerance's edge, where the plain path's last step lands far inside it)
        if (res < tol && !(warm_start && it == 0)) return SPB6G_OK;
        const bool build = !jreuse || it == 0 || !(lamprev == 1.0 && ratio <= 0.25);
        tbegin(s, TG_JACOBIAN);
        if (!build) {  // the kept diagonals; the BiCGStab set-up sums of the new right-hand side
            if (reset_fail(s)) return SPB6G_CUDA_ERROR;
            launch_jac_finish(c, s->st);
        } else if (it == 0 && ahead) {  // the rows formed ahead stand; add the worklist rows
            launch_jac_strong(c, s->st);
            launch_jac_finish(c, s->st);
        } else {
            if (reset_fail(s)) return SPB6G_CUDA_ERROR;
            launch_jacobian(c, s->st);
        }
        if (jreuse && build) CK(cudaMemcpyAsync(s->sc_build, c.sc, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
        s->jac_ready = true;
        fresh = build;
        tend_(s, TG_JACOBIAN);
        tbegin(s, TG_LINEAR);
        if (tri) {
            launch_thomas(c, s->st);
            if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
            if (s->pin->ns.fail) { tend_(s, TG_LINEAR); return SPB6G_NEWTON_FAIL; }
        } else {
            if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
            if (s->pin->ns.fail) { tend_(s, TG_LINEAR); return SPB6G_NEWTON_FAIL; }
            if (s->bicg_G > 0) {  // the whole solve in one persistent launch
                CK(cudaMemsetAsync(c.gbar, 0, sizeof(GridBarrier), s->st));
                Ctx cl = c;
                cl.x0l = (x0_pending && it == 0) ? s->x0buf : nullptr;
                if (hist_x0 && it > 0) {
                    CK(cudaMemcpyAsync(s->x0buf, c.dP, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
                    cl.x0l = s->x0buf;
                }
                if (launch_bicg_solve(cl, s->st, s->cfg.bicg_tol, s->cfg.bicg_iter, s->bicg_G) != 0) return SPB6G_CUDA_ERROR;
                if (sync_read(s, true)) return SPB6G_CUDA_ERROR;
                if (cl.x0l && s->pin->bs.x0_learned) s->stats.learned_x0++;
                if (s->pin->bs.status == BICG_TIMEOUT) {  // a grid barrier gave up (blocks not co-resident)
                    fprintf(stderr, "spb6g: BiCGStab grid barrier timed out\n");
                    tend_(s, TG_LINEAR);
                    return SPB6G_CUDA_ERROR;
                }
            } else {
            launch_bicg_init(c, s->st, s->cfg.bicg_tol, s->cfg.bicg_iter);
            s->bicg_parity = 0;
            if (s->bicg_exec) {
                launch_bicg_graph(c, s->st, s->bicg_exec, s->last_bicg_iters);
                if (sync_read(s, true)) return SPB6G_CUDA_ERROR;
            } else {  // host-polled chunks (used when the graph could not be built)
                int chunk = 4;
                for (;;) {
                    launch_bicg_iters(c, s->st, chunk, s->bicg_parity);
                    if (sync_read(s, true)) return SPB6G_CUDA_ERROR;
                    if (s->pin->bs.status != BICG_RUNNING) break;
                    if (chunk < 32) chunk *= 2;
                }
            }
            }
            s->last_bicg_iters = s->pin->bs.iters;
            s->stats.bicg_it += s->pin->bs.iters;
            if (s->pin->bs.status == BICG_FAIL) { tend_(s, TG_LINEAR); return SPB6G_LINEAR_FAIL; }
        }
        tend_(s, TG_LINEAR);
        // step criterion (:870-879) and the first line-search trial (lam = 1) in one sync
        if (reset_fail(s)) return SPB6G_CUDA_ERROR;
        tbegin(s, TG_RESIDUAL);
        {
            Ctx cs = c;  // the scales of the last build (the current ones unless the Jacobian is kept)
            if (jreuse) cs.sc = s->sc_build;
            launch_stepnorm(cs, s->st);
        }
        launch_residual(c, s->st, 1, 1.0);
        tend_(s, TG_RESIDUAL);
        if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
        if (s->verbose >= 3)
            fprintf(stderr, "      linear its %d  step %.3e  trial res %.3e%s\n", tri ? 0 : s->pin->bs.iters, s->pin->ns.sn,
                    s->pin->ns.res, s->pin->ns.fail ? " (closure failed)" : "");
        if (s->pin->ns.sn < tol) {
            launch_apply_step(c, s->st);
            s->stats.newton_it++;
            if (reset_fail(s)) return SPB6G_CUDA_ERROR;
            tbegin(s, TG_RESIDUAL);
            launch_residual(c, s->st, 0, 0.0);
            tend_(s, TG_RESIDUAL);
            if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
            if (s->pin->ns.fail) return SPB6G_NEWTON_FAIL;
            resfinal = s->pin->ns.res;
            return SPB6G_OK;
        }
        double lam = 1.0;
        bool acc = false;
        const double res0 = res;
        for (int ls = 0; ls < 40; ls++) {
            if (ls > 0) {
                if (reset_fail(s)) return SPB6G_CUDA_ERROR;
                tbegin(s, TG_RESIDUAL);
                launch_residual(c, s->st, 1, lam);
                tend_(s, TG_RESIDUAL);
                if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
            }
            if (!s->pin->ns.fail) {
                const double rn = s->pin->ns.res;
                if (rn < res * (1.0 - 1e-4 * lam) || rn < tol) { acc = true; res = rn; break; }
            }
            lam *= 0.5;
        }
        if (!acc && !fresh) {  // a kept Jacobian that does not descend: rebuild at the same P (:887)
            ratio = 1.0;
            lamprev = 0.0;
            continue;
        }
        ratio = res / res0;
        lamprev = lam;
        if (s->verbose >= 3) fprintf(stderr, "      line search lam %.4g res %.3e%s\n", lam, res, acc ? "" : " (not accepted)");
        if (!acc) {  // round-off floor acceptance (:890-899)
            resfinal = res;
            if (reset_fail(s)) return SPB6G_CUDA_ERROR;
            launch_floor(c, s->st, tol);
            if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
            if (s->pin->ns.fail) return SPB6G_NEWTON_FAIL;
            s->stats.floor_count++;
            return SPB6G_OK;
        }
        std::swap(c.P, c.Pn);
        std::swap(c.G, c.Gn);
        std::swap(c.sc, c.scn);
        s->stats.newton_it++;
    }
    resfinal = res;
    return res < tol ? SPB6G_OK : SPB6G_NEWTON_FAIL;
}

// One stage: combination, explicit predictor, stage data, Newton, final state and H_s.
// Ae_row[r], Ai_row[r] (r < rks) combine the earlier stages; Ai_row[rks] * dt is the stage's
// implicit step adt (main :1341-1350).
int run_stage(spb6g_solver* s, int rks, const double* Ae_row, const double* Ai_row, double dt) {
    Ctx& c = s->c;
    tbegin(s, TG_EXPLICIT);
    for (int k = 0; k < NV; k++) c.Un.v[k] = s->U[k];
    c.Hprev = s->Hs;
    c.nH = rks;
    for (int r = 0; r < 2; r++) {  // Ae[s][r] * dt and Ai[s][r] * dt, as main forms them (:1346-1347)
        c.ce[r] = r < rks ? Ae_row[r] * dt : 0.0;
        c.ci[r] = r < rks ? Ai_row[r] * dt : 0.0;
    }
    c.adt = Ai_row[rks] * dt;
    c.tau = c.adt;
    {  // time span of the stage, from the implicit tableau's row sums (the stage times c_s)
        double cs = 0;
        for (int r = 0; r <= rks; r++) cs += Ai_row[r];
        const double cp = rks > 0 ? s->stage_c : 0.0;
        c.sdt = (cs - cp) * dt > 0.05 * c.adt ? (cs - cp) * dt : c.adt;
        s->stage_c = cs;
    }
    c.rx = c.tau / s->g.dx;
    c.ry = c.tau / s->g.dy;
    c.H = s->Hs + (size_t)rks * NV * s->n;
    if (reset_flags(s)) return SPB6G_CUDA_ERROR;
    launch_flux(c, s->st);
    tend_(s, TG_EXPLICIT);
    // warm-start features of the stage (X* and the starting pressure), into the caller's
    // dump buffer when one has room, else into the solver's own rows
    // a stage is dumped once a pressure rate exists (its target is relative to the last rate)
    s->dump_stage = s->dumpX && s->rate_ready && s->dump_count + s->n <= s->dump_cap;
    // the pressure rate is tracked once a feature normalisation has been set (a feature, and the
    // extrapolation), so that it stays current on steps without a dump
    const bool track = s->Prate != nullptr;
    c.Prate = track ? s->Prate : nullptr;
    c.Prate2 = s->Prate2;
    c.Prate3 = s->Prate3;
    c.rate_sc = s->rate_sc;
    c.x0l = nullptr;
    if (s->warm || s->dump_stage) {
        tbegin(s, TG_WARM);
        s->rows_cur = s->dump_stage ? (void*)((char*)s->dumpX + (size_t)s->dump_count * 128) : s->featbuf;
        launch_features(c, s->st, s->norm, s->rows_cur);
        tend_(s, TG_WARM);
    }
    if (track) CK(cudaMemcpyAsync(s->Pstart, c.P, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice, s->st));
    prep_and_shock(s);
    double res = 0;
    const int rc = newton(s, res);
    if (rc != SPB6G_OK) return rc;
    if (track) {  // the new pressure rate, and the training pair (features, (R' - R) / sigma)
        launch_rate(c, s->st, s->Pstart, s->norm.tscale, s->dump_stage ? s->dumpT + s->dump_count : nullptr);
        if (s->dump_stage) s->dump_count += s->n;
        s->rate_ready = true;
        s->span3 = s->span2;
        s->span2 = s->span1;
        s->span1 = c.sdt;
    }
    if (res > s->stats.maxres) s->stats.maxres = res;
    if (reset_fail(s)) return SPB6G_CUDA_ERROR;
    tbegin(s, TG_FINAL);
    launch_final(c, s->st);
    tend_(s, TG_FINAL);
    if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
    if (s->pin->ns.fail) return SPB6G_NEWTON_FAIL;
    s->stats.stages++;
    for (int k = 0; k < 2; k++) s->stats.tmax[k] = SMAX(s->stats.tmax[k], s->pin->ns.tmax[k]);  // st_Tmax (:1070)
    return SPB6G_OK;
}

// main()'s loop body (:1316-1384).
int do_step(spb6g_solver* s) {
    const spb6g_config& cf = s->cfg;
    bool ramping = false;
    double inv;
    int rc;
    if (cf.dtfix > 0) s->dt = cf.dtfix;
    else {
        if ((rc = caldt(s, cf.acdt != 0, inv))) return rc;
        s->dt = cf.cfl * inv;
        if (cf.ramp) {
            if (s->dtprev < 0) {
                if ((rc = caldt(s, true, inv))) return rc;
                s->dtprev = cf.cfl_ac * inv / 1.2;
            }
            if (s->dt > 1.2 * s->dtprev) { s->dt = 1.2 * s->dtprev; ramping = true; }
        }
        if (!std::isfinite(s->dt)) {
            if ((rc = caldt(s, true, inv))) return rc;
            s->dt = cf.cfl_ac * inv;
        }
    }
    s->dt = SMIN(s->dt, cf.tend - s->t);
    if (s->snapi < s->snaps.size() && s->t + s->dt > s->snaps[s->snapi]) s->dt = s->snaps[s->snapi] - s->t;
    if (!(s->dt > 1e-12 * cf.tend)) return SPB6G_DT_UNDERFLOW;
    bool done = false;
    double Ae[3][3], Ai[3][3];
    for (int attempt = 0; attempt < 30 && !done; attempt++) {
        const bool first_order = cf.ramp && ramping && s->startup;
        const int rk = first_order ? 1 : cf.rk;
        if (rk == 1) s->stats.rk1++;
        set_tab(rk, Ae, Ai);
        if (cf.relax) {  // RelaxationActivation at every attempt (:1333): closure types, U^n projected
            State u;
            for (int k = 0; k < NV; k++) u.v[k] = s->U[k];
            launch_relax_activate(s->c, s->st, u);
        }
        if (begin_attempt_pressure(s)) return SPB6G_CUDA_ERROR;
        bool ok = true;
        for (int rks = 0; rks < rk && ok; rks++) {
            rc = run_stage(s, rks, Ae[rks], Ai[rks], s->dt);
            if (rc == SPB6G_CUDA_ERROR) return rc;
            ok = rc == SPB6G_OK;
        }
        if (ok) {
            for (int k = 0; k < NV; k++) {
                std::swap(s->U[k], s->Ust[k]);
                s->c.Ust.v[k] = s->Ust[k];
            }
            s->Pmain = s->c.P;  // the converged stage pressure becomes P (main :1374)
            done = true;
        }
        if (!done) { s->stats.rejects++; s->dt *= 0.5; }
    }
    if (!done) return SPB6G_STEP_FAILED;
    s->t = s->t + s->dt;
    s->dtprev = s->dt;
    s->stats.steps++;
    if (!ramping) s->startup = false;
    return SPB6G_OK;
}

}  // namespace

// ============================================================ C ABI
extern "C" {

void spb6g_default_config(spb6g_config* cfg) {
    if (!cfg) return;
    memset(cfg, 0, sizeof *cfg);
    cfg->nx = 1000; cfg->ny = 1;
    cfg->x0 = 0; cfg->x1 = 1; cfg->y0 = 0; cfg->y1 = 1;
    cfg->gamma[0] = 4.4; cfg->pinf[0] = 6e8; cfg->gamma[1] = 1.4; cfg->pinf[1] = 0;
    cfg->cv[0] = cfg->cv[1] = 1000.0;
    cfg->eps_i = 1e-4;
    cfg->mu_rate = INFINITY;
    cfg->theta_rate = -1.0;
    cfg->nu_rate = -1.0;
    cfg->nu_cr = 1.0;
    cfg->nu_pc = 22.064e6;
    cfg->relax_form = 0;
    cfg->unify = 0;
    cfg->unify_proj = 1;
    cfg->nu_law = 0;
    cfg->order = 2;
    cfg->rk = 2; cfg->cfl = 0.2; cfg->cfl_ac = 0.4; cfg->ramp = 1; cfg->rus_local = 1; cfg->limiter = 1;
    cfg->newton_tol = 1e-13; cfg->newton_iter = 60; cfg->bicg_tol = 1e-13; cfg->bicg_iter = 4000;
    cfg->tend = 240e-6;
}

int spb6g_create(const spb6g_config* cfg, spb6g_solver** out) {
    if (!cfg || !out) return SPB6G_BAD_ARG;
    *out = nullptr;
    if (cfg->nx < 1 || cfg->ny < 1 || cfg->rk < 1 || cfg->rk > 3 || !(cfg->x1 > cfg->x0) || !(cfg->y1 > cfg->y0))
        return SPB6G_BAD_ARG;
    for (int q = 0; q < 4; q++)
        if (cfg->bc[q] < 0 || cfg->bc[q] > 3) return SPB6G_BAD_ARG;
    if ((cfg->bc[0] == SPB6G_BC_PERIODIC) != (cfg->bc[1] == SPB6G_BC_PERIODIC)) return SPB6G_BAD_ARG;
    if ((cfg->bc[2] == SPB6G_BC_PERIODIC) != (cfg->bc[3] == SPB6G_BC_PERIODIC)) return SPB6G_BAD_ARG;
    if (cfg->rus_local != 0 && cfg->rus_local != 1) return SPB6G_BAD_ARG;
    if (cfg->jreuse != 0 && cfg->jreuse != 1) return SPB6G_BAD_ARG;
    if (cfg->order != 0 && cfg->order != 1 && cfg->order != 2) return SPB6G_BAD_ARG;
    for (int k = 0; k < 2; k++) {
        if (cfg->kind[k] < 0 || cfg->kind[k] > 2) return SPB6G_BAD_ARG;
        if (cfg->kind[k] && !(cfg->mg_G[k] > 0 && cfg->mg_rr[k] > 0)) return SPB6G_BAD_ARG;
    }
    if (cfg->relax < 0 || cfg->relax > 3) return SPB6G_BAD_ARG;
    if (!(cfg->mu_rate >= 0) || !(cfg->nu_cr >= 0) || !(cfg->nu_pc > 0) || cfg->relax_form < 0 || cfg->relax_form > 1 ||
        cfg->unify < 0 || cfg->unify > 2 || cfg->unify_proj < 0 || cfg->unify_proj > 1 || cfg->nu_law < 0 || cfg->nu_law > 1)
        return SPB6G_BAD_ARG;
    // Mie-Grueneisen phases relax mechanically and instantaneously only (closure :846); unify does
    // not apply to them (:848), as the closure dispatch leaves it
    if ((cfg->relax || !std::isinf(cfg->mu_rate)) && (cfg->kind[0] || cfg->kind[1])) return SPB6G_UNSUPPORTED;
    if (cfg->relax && !(cfg->eps_i >= 0 && cfg->eps_i < 0.5)) return SPB6G_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= cfg->device) return SPB6G_NO_DEVICE;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return SPB6G_NO_DEVICE;
    spb6g_solver* s = new (std::nothrow) spb6g_solver();
    if (!s) return SPB6G_BAD_ARG;
    s->cfg = *cfg;
    if (const char* v = getenv("SPB6G_VERBOSE")) s->verbose = atoi(v);
    phys_from_config(cfg, s->P);
    s->g.nx = cfg->nx; s->g.ny = cfg->ny;
    for (int q = 0; q < 4; q++) { s->g.bcs[q] = cfg->bc[q]; s->g.bcu[q] = cfg->bcu[q]; s->g.bcp[q] = cfg->bcp[q]; }
    s->g.dx = (cfg->x1 - cfg->x0) / cfg->nx;
    s->g.dy = (cfg->y1 - cfg->y0) / cfg->ny;
    const int nx = cfg->nx, ny = cfg->ny;
    const size_t n = (size_t)nx * ny;
    s->n = (int)n;
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s->st2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_flux, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_weak, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->ev_shock, cudaEventDisableTiming) != cudaSuccess) {
        spb6g_destroy(s);
        return SPB6G_CUDA_ERROR;
    }
    bool ok = true;
    auto A = [&](size_t cnt) { double* p = dalloc(s, cnt); if (!p) ok = false; return p; };
    for (int k = 0; k < NV; k++) { s->U[k] = A(n); s->Ust[k] = A(n); s->Xs[k] = A(n); }
    s->Hs = A(3 * NV * n);
    for (int b = 0; b < 3; b++) s->Pbuf[b] = A(n);
    s->Pmain = s->Pbuf[0];
    Ctx& c = s->c;
    c.P = s->Pbuf[1];
    c.Pn = s->Pbuf[2];
    c.g = s->g;
    c.phy = s->P;
    c.n = (int)n;
    for (int k = 0; k < NV; k++) c.Xs.v[k] = s->Xs[k];
    c.a2s = A(n);
    c.ube_x = A((size_t)(nx + 1) * ny); c.ube_y = A((size_t)nx * (ny + 1));
    const size_t nrx = (size_t)(nx + 2) * ny, nry = (size_t)nx * (ny + 2);
    c.phis_x = A(nrx);
    c.phis_y = A(nry);
    c.kw = A(n); c.qph0 = A(n); c.qph1 = A(n);
    {
        const size_t npad = (size_t)(nx + 4) * (ny > 1 ? ny + 4 : 1);
        c.pad_rho = A(npad); c.pad_u = A(npad); c.pad_v = A(npad); c.pad_cz = A(npad);
    }
    const size_t nfx = (size_t)(nx + 1) * ny, nfy = (size_t)nx * (ny + 1);
    c.fx_ubs = A(nfx); c.fx_kp = A(nfx); c.fx_wl = A(nfx); c.fx_pv = A(nfx);
    c.fy_ubs = A(nfy); c.fy_kp = A(nfy); c.fy_wl = A(nfy); c.fy_pv = A(nfy);
    c.fxd = A(10 * nfx); c.fyd = A(10 * nfy);
    c.strong_list = (int*)A(n / 2 + 1);
    c.smask = (unsigned char*)A(n / 8 + 1);
    c.ctype = cfg->relax ? (unsigned char*)A(n / 8 + 1) : nullptr;  // n bytes
    c.step_nu = (cfg->relax && cfg->nu_law) ? A(n) : nullptr;
    s->sc_build = cfg->jreuse ? A(n) : nullptr;
    if (cfg->relax >= 2) {  // the saturation line (build_sat, physics :127-153; main :1236)
        const std::vector<double> sat = saturation_table(cfg);
        double* d = A(sat.size());
        if (d && cudaMemcpy(d, sat.data(), sat.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) ok = false;
        c.phy.sat = d;
        s->P.sat = d;
    }
    c.G = A(n); c.Gn = A(n); c.sc = A(n); c.scn = A(n); c.dP = A(n);
    {  // the five diagonals, A 1 and D^-1 -- what every BiCGStab pass re-reads -- in one block
        const size_t stride = (n + 31) & ~(size_t)31;
        double* mb = A(7 * stride);
        if (mb) {
            c.aC = mb; c.aW = mb + stride; c.aE = mb + 2 * stride; c.aS = mb + 3 * stride; c.aN = mb + 4 * stride;
            c.A1 = mb + 5 * stride; c.dinv = mb + 6 * stride;
            // the diagonals only: also holding A 1 and D^-1 gained nothing in the solve and cost
            // the state-streaming kernels more L2
            if (ny > 1) persist_in_l2(s, mb, 5 * stride * sizeof(double));
        }
    }
    c.prec = cfg->precision ? 1 : 0;
    if (c.prec) {
        auto Af = [&](size_t cnt) { return (float*)A(cnt / 2 + 1); };
        c.fC = Af(n); c.fW = Af(n); c.fE = Af(n); c.fS = Af(n); c.fN = Af(n);
    }
    c.br = A(n); c.br0 = A(n); c.bp = A(n); c.bv = A(n); c.bq = A(n); c.bs = A(n); c.bu = A(n); c.bt = A(n);
    c.tcp = A(n); c.tdp = A(n);
    for (int k = 0; k < NV; k++) c.Ust.v[k] = s->Ust[k];
    // one partial record per block of the widest reduction launch (one row of 256 per block, or one 256-thread block per 256 cells)
    c.partials = A(((size_t)n / 32 + (size_t)ny * 2 + 4096) * MAXQ);
    c.counters = (unsigned*)A(16);
    c.ns = (NewtonScalars*)A(sizeof(NewtonScalars) / sizeof(double) + 1);
    c.bs_ = (BicgScalars*)A(sizeof(BicgScalars) / sizeof(double) + 1);
    c.gbar = (GridBarrier*)A(sizeof(GridBarrier) / sizeof(double) + 1);
    if (!(ny == 1 && cfg->bc[0] != SPB6G_BC_PERIODIC)) s->bicg_G = bicg_solve_blocks(cfg->device, (int)n);
    c.gpart = A(2 * PB_SLOT_Q * (size_t)(s->bicg_G > 0 ? s->bicg_G : 1));
    if (ok && cudaMallocHost((void**)&s->pin, sizeof(Pinned)) != cudaSuccess) ok = false;
    if (ok)
        for (int e = 0; e < 2; e++)
            if (cudaEventCreate(&s->region[e]) != cudaSuccess) ok = false;
    c.nlaunch = &s->nlaunch;
    c.p_ref = 0;
    if (!ok || cudaStreamSynchronize(s->st) != cudaSuccess) { spb6g_destroy(s); return SPB6G_CUDA_ERROR; }
    if (!(ny == 1 && cfg->bc[0] != SPB6G_BC_PERIODIC) && s->bicg_G == 0) {  // no cooperative launch: capture the loop as a graph
        if (build_bicg_graph(c, s->st, &s->bicg_exec) != 0) {
            s->bicg_exec = nullptr;
            cudaGetLastError();
        }
    }
    *out = s;
    return SPB6G_OK;
}

int spb6g_destroy(spb6g_solver* s) {
    if (!s) return SPB6G_BAD_ARG;
    if (s->st) cudaStreamSynchronize(s->st);
    if (s->bicg_exec) cudaGraphExecDestroy(s->bicg_exec);
    for (void* p : s->allocs) cudaFree(p);
    if (s->pin) cudaFreeHost(s->pin);
    resolve_timing(s);
    for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
    for (int e = 0; e < 2; e++)
        if (s->region[e]) cudaEventDestroy(s->region[e]);
    if (s->st2) { cudaStreamSynchronize(s->st2); cudaStreamDestroy(s->st2); }
    if (s->ev_flux) cudaEventDestroy(s->ev_flux);
    if (s->ev_weak) cudaEventDestroy(s->ev_weak);
    if (s->ev_shock) cudaEventDestroy(s->ev_shock);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
    return SPB6G_OK;
}

static int copy_state(spb6g_solver* s, double* const* dev, double* host_dst, const double* host_src, int layout);
// The current state in the AoS layout, in the handle's host staging buffer (for the writers).
static int stage_host_state(spb6g_solver* s) {
    s->host_U.resize((size_t)s->n * NV);
    return copy_state(s, s->U, s->host_U.data(), nullptr, SPB6G_LAYOUT_AOS);
}
static int copy_state(spb6g_solver* s, double* const* dev, double* host_dst, const double* host_src, int layout) {
    const int n = s->n;
    std::vector<double> tmp;
    if (layout != SPB6G_LAYOUT_AOS && layout != SPB6G_LAYOUT_SOA) return SPB6G_BAD_ARG;
    if (host_src) {
        if (layout == SPB6G_LAYOUT_SOA) {
            for (int k = 0; k < NV; k++)
                CK(cudaMemcpyAsync(dev[k], host_src + (size_t)k * n, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s->st));
        } else {
            tmp.resize((size_t)n * NV);
            for (int x = 0; x < n; x++)
                for (int k = 0; k < NV; k++) tmp[(size_t)k * n + x] = host_src[(size_t)x * NV + k];
            for (int k = 0; k < NV; k++)
                CK(cudaMemcpyAsync(dev[k], tmp.data() + (size_t)k * n, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s->st));
        }
        CK(cudaStreamSynchronize(s->st));
    } else {
        if (layout == SPB6G_LAYOUT_SOA) {
            for (int k = 0; k < NV; k++)
                CK(cudaMemcpyAsync(host_dst + (size_t)k * n, dev[k], (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
            CK(cudaStreamSynchronize(s->st));
        } else {
            tmp.resize((size_t)n * NV);
            for (int k = 0; k < NV; k++)
                CK(cudaMemcpyAsync(tmp.data() + (size_t)k * n, dev[k], (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
            CK(cudaStreamSynchronize(s->st));
            for (int x = 0; x < n; x++)
                for (int k = 0; k < NV; k++) host_dst[(size_t)x * NV + k] = tmp[(size_t)k * n + x];
        }
    }
    return SPB6G_OK;
}

int spb6g_upload_state(spb6g_solver* s, const double* U, int layout) {
    if (!s || !U) return SPB6G_BAD_ARG;
    return copy_state(s, s->U, nullptr, U, layout);
}
int spb6g_download_state(spb6g_solver* s, double* U, int layout) {
    if (!s || !U) return SPB6G_BAD_ARG;
    return copy_state(s, s->U, U, nullptr, layout);
}

int spb6g_init_pressure(spb6g_solver* s) {
    if (!s) return SPB6G_BAD_ARG;
    CState u;
    for (int k = 0; k < NV; k++) u.v[k] = s->U[k];
    launch_pbar_min(s->c, s->st, u);
    if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
    double pr = s->pin->ns.pmin;
    if (!std::isfinite(pr)) pr = 0.0;
    s->p_ref = pr;
    s->c.p_ref = pr;
    s->stats.p_ref = pr;
    launch_pbar_init(s->c, s->st, u, pr, s->Pmain);
    CK(cudaStreamSynchronize(s->st));
    s->t = 0; s->dt = 0; s->dtprev = -1; s->startup = true;
    // conserved totals of the initial state, the stats line's reference (:1251)
    const int rc = stage_host_state(s);
    if (rc != SPB6G_OK) return rc;
    out::conserved_totals(s->cfg, s->host_U.data(), s->M0);
    return SPB6G_OK;
}
int spb6g_set_pressure(spb6g_solver* s, const double* P, double p_ref) {
    if (!s || !P) return SPB6G_BAD_ARG;
    CK(cudaMemcpyAsync(s->Pmain, P, (size_t)s->n * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    s->p_ref = p_ref; s->c.p_ref = p_ref; s->stats.p_ref = p_ref;
    return SPB6G_OK;
}
int spb6g_get_pressure(spb6g_solver* s, double* P, double* p_ref) {
    if (!s) return SPB6G_BAD_ARG;
    if (P) {
        CK(cudaMemcpyAsync(P, s->Pmain, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    if (p_ref) *p_ref = s->p_ref;
    return SPB6G_OK;
}
int spb6g_caldt(spb6g_solver* s, int acoustic, double* inv_rate) {
    if (!s || !inv_rate) return SPB6G_BAD_ARG;
    return caldt(s, acoustic != 0, *inv_rate);
}
int spb6g_step(spb6g_solver* s) {
    if (!s) return SPB6G_BAD_ARG;
    const int rc = do_step(s);
    s->stats.t = s->t;
    s->stats.dt = s->dt;
    if (rc == SPB6G_OK && !s->out_file.empty()) {  // snapshot and probe after the accepted step (:1380-1381)
        const bool snap = s->snapi < s->snaps.size() && s->t >= s->snaps[s->snapi] * (1 - 1e-12);
        if (snap || s->probe) {
            const int r = stage_host_state(s);
            if (r != SPB6G_OK) return r;
        }
        if (snap) {
            const int r = out::write_profile(s->cfg, s->host_U.data(), out::snap_name(s->out_file, s->snapi).c_str(), s->prec);
            if (r != SPB6G_OK) return r;
            s->snapi++;
        }
        if (s->probe) {
            const int r = out::write_probe(s->cfg, s->host_U.data(), s->t, s->probe_x, s->probe_y, s->out_file + ".probe", false);
            if (r != SPB6G_OK) return r;
        }
    }
    return rc;
}
int spb6g_advance(spb6g_solver* s, int nsteps) {
    if (!s) return SPB6G_BAD_ARG;
    int rc = SPB6G_OK;
    for (int k = 0; (nsteps <= 0 || k < nsteps) && s->t < s->cfg.tend * (1 - 1e-12); k++) {
        rc = spb6g_step(s);
        if (rc != SPB6G_OK) break;
    }
    // the profile main() writes at the end of the run or when a step fails (:1326, :1379, :1388)
    const bool failed = rc == SPB6G_STEP_FAILED || rc == SPB6G_DT_UNDERFLOW;
    if (!s->out_file.empty() && (failed || (rc == SPB6G_OK && !(s->t < s->cfg.tend * (1 - 1e-12))))) {
        if (rc == SPB6G_OK && s->cfg.relax) {  // the activation projection before the final profile (:1388)
            State u;
            for (int k = 0; k < NV; k++) u.v[k] = s->U[k];
            launch_relax_activate(s->c, s->st, u);
        }
        const int r = spb6g_write_profile(s, s->out_file.c_str(), s->prec);
        if (r != SPB6G_OK && rc == SPB6G_OK) rc = r;
    }
    return rc;
}

int spb6g_set_output(spb6g_solver* s, const spb6g_output* o) {
    if (!s) return SPB6G_BAD_ARG;
    if (!o || !o->out_file || !o->out_file[0]) {
        s->out_file.clear();
        s->snaps.clear();
        s->snapi = 0;
        s->probe = false;
        return SPB6G_OK;
    }
    if (o->nsnap < 0 || (o->nsnap > 0 && !o->snaps)) return SPB6G_BAD_ARG;
    s->out_file = o->out_file;
    s->snaps.assign(o->snaps, o->snaps + o->nsnap);
    s->snapi = 0;
    while (s->snapi < s->snaps.size() && s->t >= s->snaps[s->snapi] * (1 - 1e-12)) s->snapi++;  // times already passed
    s->probe = o->probe != 0;
    s->probe_x = o->probe_x;
    s->probe_y = o->probe_y;
    s->prec = o->prec > 0 ? o->prec : 16;
    if (s->probe) {  // the first probe line, at the current state (:1306)
        const int r = stage_host_state(s);
        if (r != SPB6G_OK) return r;
        return out::write_probe(s->cfg, s->host_U.data(), s->t, s->probe_x, s->probe_y, s->out_file + ".probe", true);
    }
    return SPB6G_OK;
}

int spb6g_format_profile(const spb6g_config* cfg, const double* U, const char* path, int prec) {
    if (!cfg || !U || !path || prec < 0 || cfg->nx < 1 || cfg->ny < 1) return SPB6G_BAD_ARG;
    return out::write_profile(*cfg, U, path, prec > 0 ? prec : 16);
}

int spb6g_write_profile(spb6g_solver* s, const char* path, int prec) {
    if (!s || !path || prec < 0) return SPB6G_BAD_ARG;
    const int r = stage_host_state(s);
    if (r != SPB6G_OK) return r;
    return out::write_profile(s->cfg, s->host_U.data(), path, prec > 0 ? prec : 16);
}

int spb6g_conserved_totals(spb6g_solver* s, double* M) {
    if (!s || !M) return SPB6G_BAD_ARG;
    const int r = stage_host_state(s);
    if (r != SPB6G_OK) return r;
    out::conserved_totals(s->cfg, s->host_U.data(), M);
    return SPB6G_OK;
}

int spb6g_stats_line(spb6g_solver* s, int case_id, double wall_s, char* buf, size_t len) {
    if (!s || !buf || len == 0) return SPB6G_BAD_ARG;
    double M1[3];
    const int r = spb6g_conserved_totals(s, M1);
    if (r != SPB6G_OK) return r;
    const spb6g_stats& q = s->stats;
    const double* M0 = s->M0;
    // st_cl_fail is never incremented by the reference's IMEX program, so its column is always 0
    std::snprintf(buf, len,
                  "case %d mode 1 order %d rk %d N %d CFL %g | steps %ld (rk1 %ld) rejects %ld floor %ld | stages %ld newton it %ld "
                  "(%.2f/stage) maxres %.2e Tmax %.4g %.4g | closure fails %ld | dM1/M %.2e dM2/M %.2e dE/E %.2e | wall %.2f s",
                  case_id, s->P.order, s->cfg.rk, s->cfg.nx, s->cfg.cfl, (long)q.steps, (long)q.rk1, (long)q.rejects, (long)q.floor_count,
                  (long)q.stages, (long)q.newton_it, q.stages ? (double)q.newton_it / q.stages : 0.0, q.maxres, q.tmax[0], q.tmax[1],
                  0L, (M1[0] - M0[0]) / M0[0], (M1[1] - M0[1]) / M0[1], (M1[2] - M0[2]) / M0[2], wall_s);
    return SPB6G_OK;
}
int spb6g_stage_dump(spb6g_solver* s, double dt, double* Xs, double* a2s, double* ube_x, double* ube_y, double* phi_x,
                     double* phi_y) {
    if (!s || !(dt > 0)) return SPB6G_BAD_ARG;
    const int nx = s->g.nx, ny = s->g.ny, n = s->n;
    double Ae[3][3], Ai[3][3];
    set_tab(s->cfg.rk, Ae, Ai);
    s->dt = dt;
    if (begin_attempt_pressure(s)) return SPB6G_CUDA_ERROR;
    // explicit predictor, then the outputs, then the implicit part
    Ctx& c = s->c;
    for (int k = 0; k < NV; k++) c.Un.v[k] = s->U[k];
    c.Hprev = s->Hs;
    c.nH = 0;
    c.ce[0] = c.ce[1] = c.ci[0] = c.ci[1] = 0.0;
    c.adt = Ai[0][0] * dt; c.tau = c.adt; c.rx = c.tau / s->g.dx; c.ry = c.tau / s->g.dy;
    c.sdt = c.adt;
    c.x0l = nullptr;
    c.Prate = nullptr;  // the dumped stage runs from the plain guess
    c.Prate2 = nullptr;
    c.Prate3 = nullptr;
    c.rate_sc = nullptr;
    c.H = s->Hs;
    if (reset_flags(s)) return SPB6G_CUDA_ERROR;
    launch_flux(c, s->st);
    CK(cudaStreamSynchronize(s->st));
    if (Xs) {
        if (copy_state(s, s->Xs, Xs, nullptr, SPB6G_LAYOUT_AOS)) return SPB6G_CUDA_ERROR;
    }
    if (a2s) CK(cudaMemcpy(a2s, c.a2s, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
    if (ube_x) CK(cudaMemcpy(ube_x, c.ube_x, (size_t)(nx + 1) * ny * sizeof(double), cudaMemcpyDeviceToHost));
    if (ube_y) {
        if (ny > 1) CK(cudaMemcpy(ube_y, c.ube_y, (size_t)nx * (ny + 1) * sizeof(double), cudaMemcpyDeviceToHost));
        else memset(ube_y, 0, (size_t)nx * (ny + 1) * sizeof(double));
    }
    if (phi_x || phi_y) {
        std::vector<double> tx((size_t)(nx + 2) * ny), ty((size_t)nx * (ny + 2));
        CK(cudaMemcpy(tx.data(), c.phis_x, tx.size() * sizeof(double), cudaMemcpyDeviceToHost));
        if (ny > 1) CK(cudaMemcpy(ty.data(), c.phis_y, ty.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                if (phi_x) phi_x[(size_t)j * nx + i] = tx[(size_t)(i + 1) + (size_t)j * (nx + 2)];
                if (phi_y) phi_y[(size_t)j * nx + i] = ny > 1 ? ty[(size_t)i + (size_t)(j + 1) * nx] : 0.0;
            }
    }
    prep_and_shock(s);
    double res;
    spb6g_mlp* warm = s->warm;
    s->warm = nullptr;
    int rc = newton(s, res);
    s->warm = warm;
    if (rc != SPB6G_OK) return rc;
    if (reset_fail(s)) return SPB6G_CUDA_ERROR;
    launch_final(c, s->st);
    if (sync_read(s, false)) return SPB6G_CUDA_ERROR;
    if (s->pin->ns.fail) return SPB6G_NEWTON_FAIL;
    for (int k = 0; k < NV; k++) std::swap(s->U[k], s->Ust[k]);
    c.Ust = State{};
    for (int k = 0; k < NV; k++) c.Ust.v[k] = s->Ust[k];
    s->Pmain = c.P;
    return SPB6G_OK;
}
int spb6g_stage(spb6g_solver* s, int rks, const double* Ae_row, const double* Ai_row, double dt, spb6g_stats* st) {
    if (!s || rks < 0 || rks > 2 || !Ai_row || (rks > 0 && !Ae_row) || !(dt > 0) || !std::isfinite(dt) ||
        !(Ai_row[rks] > 0) || !std::isfinite(Ai_row[rks]))
        return SPB6G_BAD_ARG;
    for (int r = 0; r < rks; r++)
        if (!std::isfinite(Ae_row[r]) || !std::isfinite(Ai_row[r])) return SPB6G_BAD_ARG;
    // a later stage needs the earlier stages of the same attempt
    if (rks > 0 && s->attempt_stage != rks - 1) return SPB6G_BAD_ARG;
    CK(cudaSetDevice(s->cfg.device));
    s->dt = dt;
    if (rks == 0) {  // a new attempt: RelaxationActivation (:1333) and Pst = P (:1335)
        s->attempt_stage = -1;
        if (s->cfg.relax) {
            State u;
            for (int k = 0; k < NV; k++) u.v[k] = s->U[k];
            launch_relax_activate(s->c, s->st, u);
        }
        if (begin_attempt_pressure(s)) return SPB6G_CUDA_ERROR;
    }
    const int rc = run_stage(s, rks, Ae_row, Ai_row, dt);
    s->attempt_stage = rc == SPB6G_OK ? rks : -1;
    if (st) *st = s->stats;
    return rc;
}
int spb6g_stage_accept(spb6g_solver* s, double dt) {
    if (!s || !(dt > 0) || !std::isfinite(dt)) return SPB6G_BAD_ARG;
    if (s->attempt_stage < 0) return SPB6G_BAD_ARG;  // no converged stage to accept
    for (int k = 0; k < NV; k++) {  // u_con = Ust, P = Pst (:1374); t += dt (:1379)
        std::swap(s->U[k], s->Ust[k]);
        s->c.Ust.v[k] = s->Ust[k];
    }
    s->Pmain = s->c.P;
    s->attempt_stage = -1;
    s->t = s->t + dt;
    s->dtprev = dt;
    s->stats.steps++;
    return SPB6G_OK;
}
int spb6g_stage_data(spb6g_solver* s, double* fx, double* fy, double* kw, double* qph) {
    if (!s) return SPB6G_BAD_ARG;
    const Ctx& c = s->c;
    const size_t nfx = (size_t)(s->g.nx + 1) * s->g.ny, nfy = (size_t)s->g.nx * (s->g.ny + 1), n = s->n;
    CK(cudaStreamSynchronize(s->st));
    if (fx) {
        const double* a[4] = {c.fx_ubs, c.fx_kp, c.fx_wl, c.fx_pv};
        for (int k = 0; k < 4; k++) CK(cudaMemcpy(fx + k * nfx, a[k], nfx * sizeof(double), cudaMemcpyDeviceToHost));
    }
    if (fy) {
        const double* a[4] = {c.fy_ubs, c.fy_kp, c.fy_wl, c.fy_pv};
        for (int k = 0; k < 4; k++) {
            if (s->g.ny > 1) CK(cudaMemcpy(fy + k * nfy, a[k], nfy * sizeof(double), cudaMemcpyDeviceToHost));
            else memset(fy + k * nfy, 0, nfy * sizeof(double));
        }
    }
    if (kw) CK(cudaMemcpy(kw, c.kw, n * sizeof(double), cudaMemcpyDeviceToHost));
    if (qph) {
        CK(cudaMemcpy(qph, c.qph0, n * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(qph + n, c.qph1, n * sizeof(double), cudaMemcpyDeviceToHost));
    }
    return SPB6G_OK;
}

static int ensure_warm_buffers(spb6g_solver* s);
int spb6g_set_feature_norm(spb6g_solver* s, const double* norm) {
    if (!s || !norm) return SPB6G_BAD_ARG;
    FeatureNorm nm{};
    for (int f = 0; f < NFIELD; f++) {
        if (!std::isfinite(norm[f]) || !(norm[NFIELD + f] > 0) || !(norm[2 * NFIELD + f] > 0)) return SPB6G_BAD_ARG;
        nm.mean[f] = norm[f];
        nm.istd[f] = 1.0 / norm[NFIELD + f];
        nm.idstd[f] = 1.0 / norm[2 * NFIELD + f];
    }
    if (!(norm[3 * NFIELD] > 0) || !std::isfinite(norm[3 * NFIELD])) return SPB6G_BAD_ARG;
    nm.tscale = norm[3 * NFIELD];
    s->norm = nm;
    // the feature rows and the pressure-rate tracking start here, so that R is current at the
    // first stage that is dumped or warm-started
    cudaSetDevice(s->cfg.device);
    return ensure_warm_buffers(s);
}
static int ensure_warm_buffers(spb6g_solver* s) {
    if (!s->cand_ns) {
        if (cudaMalloc((void**)&s->cand_ns, GRAM_K * sizeof(NewtonScalars)) != cudaSuccess) return SPB6G_CUDA_ERROR;
        s->allocs.push_back(s->cand_ns);
    }
    if (!s->featbuf) {
        if (cudaMalloc(&s->featbuf, (size_t)s->n * 128) != cudaSuccess) return SPB6G_CUDA_ERROR;
        s->allocs.push_back(s->featbuf);
    }
    for (float** b : {&s->ybuf, &s->ytmp}) {
        if (*b) continue;
        if (cudaMalloc((void**)b, (size_t)s->n * sizeof(float)) != cudaSuccess) return SPB6G_CUDA_ERROR;
        s->allocs.push_back(*b);
    }
    for (double** b : {&s->Pstart, &s->Prate, &s->Prate2, &s->Prate3, &s->x0buf, &s->rate_sc, &s->gstore, &s->scstore,
                        &s->gram_part, &s->gram}) {
        if (*b) continue;
        const size_t cnt = b == &s->rate_sc ? 2
                           : b == &s->gstore ? (size_t)(GRAM_K + 1) * s->n
                           : b == &s->scstore ? (size_t)GRAM_K * s->n
                           : b == &s->gram_part ? (size_t)red_blocks(s->n, RED_THREADS) * GRAM_Q
                           : b == &s->gram ? (size_t)GRAM_Q
                                                 : (size_t)s->n;
        if (cudaMalloc((void**)b, cnt * sizeof(double)) != cudaSuccess) return SPB6G_CUDA_ERROR;
        s->allocs.push_back(*b);
        // no rate (and no rate scale) before the first converged stage
        if ((b == &s->Prate || b == &s->Prate2 || b == &s->Prate3 || b == &s->rate_sc) && cudaMemsetAsync(*b, 0, cnt * sizeof(double), s->st) != cudaSuccess)
            return SPB6G_CUDA_ERROR;
    }
    return SPB6G_OK;
}
int spb6g_set_warmstart(spb6g_solver* s, spb6g_mlp* m) {
    if (!s) return SPB6G_BAD_ARG;
    if (m && !(s->norm.tscale > 0)) return SPB6G_BAD_ARG;
    if (m) {
        cudaSetDevice(s->cfg.device);
        const int rc = ensure_warm_buffers(s);
        if (rc) return rc;
    }
    s->warm = m;
    return SPB6G_OK;
}
int spb6g_set_warmstart_mode(spb6g_solver* s, int mode) {
    if (!s || mode < 1 || mode > 63) return SPB6G_BAD_ARG;
    s->warm_mode = mode;
    return SPB6G_OK;
}
int spb6g_set_warmstart_smoothing(spb6g_solver* s, int radius) {
    if (!s || radius < 0 || radius > 64 || radius >= s->g.nx || (s->g.ny > 1 && radius >= s->g.ny)) return SPB6G_BAD_ARG;
    s->warm_smooth = radius;
    return SPB6G_OK;
}
int spb6g_set_dump(spb6g_solver* s, void* X_dev, float* target_dev, int64_t capacity) {
    if (!s || capacity < 0 || (capacity > 0 && (!X_dev || !target_dev))) return SPB6G_BAD_ARG;
    if (capacity > 0 && !(s->norm.tscale > 0)) return SPB6G_BAD_ARG;
    if (capacity > 0) {
        cudaSetDevice(s->cfg.device);
        const int rc = ensure_warm_buffers(s);
        if (rc) return rc;
    }
    s->dumpX = capacity > 0 ? X_dev : nullptr;
    s->dumpT = capacity > 0 ? target_dev : nullptr;
    s->dump_cap = capacity;
    s->dump_count = 0;
    return SPB6G_OK;
}
int spb6g_dump_count(spb6g_solver* s, int64_t* count) {
    if (!s || !count) return SPB6G_BAD_ARG;
    // the rows counted are complete when the call returns (the caller reads them on its own stream)
    cudaSetDevice(s->cfg.device);
    if (cudaStreamSynchronize(s->st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    *count = s->dump_count;
    return SPB6G_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------- batched form
struct spb6g_batch {
    int device = 0;
    std::vector<spb6g_solver*> inst;
    std::vector<BatchInst> host;
    std::vector<int> status;
    BatchInst* dev = nullptr;
    cudaStream_t st = nullptr;
    int threads = 128, tw = 256;
    cudaGraphExec_t graph = nullptr;  // the persistent launches for (graph_steps, graph_threads, graph_tw)
    int graph_steps = -1, graph_threads = 0, graph_tw = 0;
    // block-size plan for graph_threads: grids grouped by block size (class c: block size
    // cls[c], grids order[off[c] .. off[c+1]), longest first); one launch per class
    std::vector<int> cls, off, order;
    int* dorder = nullptr;
    std::vector<cudaStream_t> side;  // one stream per class after the first
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
};

namespace {
// What the batched kernel runs: 1D non-periodic grids, SG / NASG phases, p relaxation
// (instantaneous), per-face Rusanov speed, a fresh Jacobian every Newton iteration, second order,
// FP64.
bool batch_config_ok(const spb6g_config& c) {
    return c.ny == 1 && c.bc[0] != SPB6G_BC_PERIODIC && c.kind[0] == 0 && c.kind[1] == 0 && c.relax == 0 &&
           c.rus_local == 1 && std::isinf(c.mu_rate) && c.unify != 1 && c.jreuse == 0 && c.order != 1 && c.precision == 0;
}
void batch_pack(spb6g_batch* b) {
    for (size_t i = 0; i < b->inst.size(); i++) {
        spb6g_solver* s = b->inst[i];
        BatchInst& B = b->host[i];
        memset(&B, 0, sizeof B);
        B.c = s->c;
        for (int k = 0; k < NV; k++) { B.U[k] = s->U[k]; B.Ust[k] = s->Ust[k]; B.c.Ust.v[k] = s->Ust[k]; }
        B.Hs = s->Hs;
        for (int q = 0; q < 3; q++) {
            B.Pbuf[q] = s->Pbuf[q];
            if (s->Pbuf[q] == s->Pmain) B.pmain = q;
        }
        B.status = SPB6G_OK;
        B.t = s->t; B.dt = s->dt; B.dtprev = s->dtprev; B.startup = s->startup ? 1 : 0;
        const spb6g_config& cf = s->cfg;
        B.cfl = cf.cfl; B.cfl_ac = cf.cfl_ac; B.dtfix = cf.dtfix; B.tend = cf.tend; B.newton_tol = cf.newton_tol;
        B.ramp = cf.ramp; B.acdt = cf.acdt; B.rk = cf.rk; B.newton_iter = cf.newton_iter;
        B.steps = s->stats.steps; B.rejects = s->stats.rejects; B.rk1 = s->stats.rk1; B.stages = s->stats.stages;
        B.newton_it = s->stats.newton_it; B.floor_count = s->stats.floor_count; B.maxres = s->stats.maxres;
        B.tmax[0] = s->stats.tmax[0]; B.tmax[1] = s->stats.tmax[1];
    }
}
void batch_unpack(spb6g_batch* b) {
    for (size_t i = 0; i < b->inst.size(); i++) {
        spb6g_solver* s = b->inst[i];
        const BatchInst& B = b->host[i];
        s->c = B.c;
        for (int k = 0; k < NV; k++) { s->U[k] = B.U[k]; s->Ust[k] = B.Ust[k]; }
        s->Pmain = B.Pbuf[B.pmain];
        s->t = B.t; s->dt = B.dt; s->dtprev = B.dtprev; s->startup = B.startup != 0;
        s->stats.steps = B.steps; s->stats.rejects = B.rejects; s->stats.rk1 = B.rk1; s->stats.stages = B.stages;
        s->stats.newton_it = B.newton_it; s->stats.floor_count = B.floor_count; s->stats.maxres = B.maxres;
        s->stats.tmax[0] = B.tmax[0]; s->stats.tmax[1] = B.tmax[1];
        b->status[i] = B.status;
    }
}
// Block size of every grid: threads in proportion to its cells (a multiple of 32, at least
// 32, at most `threads`), so that every block has about the same cells per thread -- the
// launch lasts as long as its slowest grid.  The cells per thread are the fewest for which
// all blocks are resident at once (their threads within 15/16 of the device's thread slots
// at the kernel's register count), and at least the largest grid's cells over `threads`.
// Grids are grouped by block size, each group longest first; the groups run as concurrent
// launches.
int batch_plan(spb6g_batch* b, int threads, int tw) {
    const int count = (int)b->inst.size();
    std::vector<int64_t> cells(count);
    for (int i = 0; i < count; i++) cells[i] = b->inst[i]->n;
    const int64_t slots = (int64_t)batch_max_blocks(256, tw, b->device) * 256 * 15 / 16;
    std::vector<int> bs(count);
    if (spb6g_batch_block_sizes(cells.data(), count, threads, slots, bs.data(), nullptr) != SPB6G_OK) return SPB6G_UNSUPPORTED;
    b->order.resize(count);
    for (int i = 0; i < count; i++) b->order[i] = i;
    std::stable_sort(b->order.begin(), b->order.end(), [&](int x, int y) {
        return bs[x] != bs[y] ? bs[x] > bs[y] : b->inst[x]->n > b->inst[y]->n;
    });
    b->cls.clear();
    b->off.clear();
    for (int k = 0; k < count; k++)
        if (k == 0 || bs[b->order[k]] != bs[b->order[k - 1]]) {
            b->cls.push_back(bs[b->order[k]]);
            b->off.push_back(k);
        }
    b->off.push_back(count);
    for (int bsz : b->cls)
        if (batch_max_blocks(bsz, tw, b->device) <= 0) return SPB6G_UNSUPPORTED;
    while (b->side.size() + 1 < b->cls.size()) {
        cudaStream_t st = nullptr;
        cudaEvent_t e = nullptr;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        b->side.push_back(st);
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->join.push_back(e);
    }
    if (!b->fork) CK(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    CK(cudaMemcpy(b->dorder, b->order.data(), (size_t)count * sizeof(int), cudaMemcpyHostToDevice));
    return SPB6G_OK;
}
// One persistent launch of nsteps steps per instance (a captured CUDA graph, rebuilt when the
// step count or the launch shape changes), device time in *ms if not NULL.
int batch_run(spb6g_batch* b, int nsteps, int threads, int tw, float* ms) {
    if (!b->graph || b->graph_steps != nsteps || b->graph_threads != threads || b->graph_tw != tw) {
        if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
        b->graph_steps = -1;
        const int prc = batch_plan(b, threads, tw);
        if (prc != SPB6G_OK) return prc;
    }
    batch_pack(b);
    CK(cudaMemcpyAsync(b->dev, b->host.data(), b->host.size() * sizeof(BatchInst), cudaMemcpyHostToDevice, b->st));
    if (!b->graph) {
        cudaGraph_t g = nullptr;
        CK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
        int lrc = 0;
        const int ncls = (int)b->cls.size();
        if (ncls > 1) lrc |= cudaEventRecord(b->fork, b->st) != cudaSuccess;
        for (int c = 1; c < ncls; c++) lrc |= cudaStreamWaitEvent(b->side[c - 1], b->fork, 0) != cudaSuccess;
        for (int c = 0; c < ncls; c++) {
            const int n_c = b->off[c + 1] - b->off[c];
            lrc |= launch_batch(b->dev, b->dorder + b->off[c], n_c, nsteps, b->cls[c], tw, n_c, c ? b->side[c - 1] : b->st) != 0;
        }
        for (int c = 1; c < ncls; c++) {
            lrc |= cudaEventRecord(b->join[c - 1], b->side[c - 1]) != cudaSuccess;
            lrc |= cudaStreamWaitEvent(b->st, b->join[c - 1], 0) != cudaSuccess;
        }
        CK(cudaStreamEndCapture(b->st, &g));
        if (lrc) { cudaGraphDestroy(g); return SPB6G_CUDA_ERROR; }
        CK(cudaGraphInstantiate(&b->graph, g, 0));
        cudaGraphDestroy(g);
        b->graph_steps = nsteps; b->graph_threads = threads; b->graph_tw = tw;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ms) { cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventRecord(e0, b->st); }
    CK(cudaGraphLaunch(b->graph, b->st));
    if (ms) cudaEventRecord(e1, b->st);
    CK(cudaMemcpyAsync(b->host.data(), b->dev, b->host.size() * sizeof(BatchInst), cudaMemcpyDeviceToHost, b->st));
    CK(cudaStreamSynchronize(b->st));
    if (ms) { cudaEventElapsedTime(ms, e0, e1); cudaEventDestroy(e0); cudaEventDestroy(e1); }
    batch_unpack(b);
    for (size_t i = 0; i < b->status.size(); i++)
        if (b->status[i] != SPB6G_OK) return b->status[i];
    return SPB6G_OK;
}

}  // namespace

extern "C" {

int spb6g_batch_block_sizes(const int64_t* cells, int count, int threads, int64_t slots, int* block,
                            int64_t* per_thread_out) {
    if (!cells || !block || count < 1 || threads < 32 || threads > 256 || threads % 32 != 0 || slots < 0)
        return SPB6G_BAD_ARG;
    int64_t nmax = 1;
    for (int i = 0; i < count; i++) {
        if (cells[i] < 1) return SPB6G_BAD_ARG;
        nmax = std::max(nmax, cells[i]);
    }
    auto block_of = [&](int64_t n, int64_t per_thread) {
        const int64_t t = (n + 32 * per_thread - 1) / (32 * per_thread) * 32;
        return (int)std::min<int64_t>(std::max<int64_t>(t, 32), threads);
    };
    int64_t per_thread = (nmax + threads - 1) / threads;
    if (slots > 0)
        for (; per_thread < nmax; per_thread++) {
            int64_t total = 0;
            for (int i = 0; i < count; i++) total += block_of(cells[i], per_thread);
            if (total <= slots) break;
        }
    for (int i = 0; i < count; i++) block[i] = block_of(cells[i], per_thread);
    if (per_thread_out) *per_thread_out = per_thread;
    return SPB6G_OK;
}

int spb6g_batch_create(const spb6g_config* cfgs, int count, spb6g_batch** out) {
    if (!cfgs || !out || count < 1) return SPB6G_BAD_ARG;
    *out = nullptr;
    for (int i = 0; i < count; i++)
        if (!batch_config_ok(cfgs[i]) || cfgs[i].device != cfgs[0].device) return SPB6G_UNSUPPORTED;
    spb6g_batch* b = new spb6g_batch();
    b->device = cfgs[0].device;
    for (int i = 0; i < count; i++) {
        spb6g_solver* s = nullptr;
        const int rc = spb6g_create(&cfgs[i], &s);
        if (rc != SPB6G_OK) { spb6g_batch_destroy(b); return rc; }
        b->inst.push_back(s);
    }
    cudaSetDevice(b->device);
    b->host.resize(count);
    b->status.assign(count, SPB6G_OK);
    if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void**)&b->dev, (size_t)count * sizeof(BatchInst)) != cudaSuccess ||
        cudaMalloc((void**)&b->dorder, (size_t)count * sizeof(int)) != cudaSuccess) {
        spb6g_batch_destroy(b);
        return SPB6G_CUDA_ERROR;
    }
    *out = b;
    return SPB6G_OK;
}
void spb6g_batch_destroy(spb6g_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->dev) cudaFree(b->dev);
    if (b->dorder) cudaFree(b->dorder);
    for (cudaStream_t st : b->side) cudaStreamDestroy(st);
    for (cudaEvent_t e : b->join) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->st) cudaStreamDestroy(b->st);
    for (spb6g_solver* s : b->inst) spb6g_destroy(s);
    delete b;
}
spb6g_solver* spb6g_batch_instance(spb6g_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->inst.size()) return nullptr;
    return b->inst[i];
}
int spb6g_batch_status(spb6g_batch* b, int i) {
    if (!b || i < 0 || i >= (int)b->inst.size()) return SPB6G_BAD_ARG;
    return b->status[i];
}
int spb6g_batch_launches(spb6g_batch* b) {
    if (!b) return SPB6G_BAD_ARG;
    return b->graph && b->graph_threads == b->threads && b->graph_tw == b->tw ? (int)b->cls.size() : 0;
}
int spb6g_batch_set_shape(spb6g_batch* b, int threads, int tile) {
    if (!b || threads < 32 || threads > 256 || threads % 32 != 0 || (tile != 128 && tile != 256)) return SPB6G_BAD_ARG;
    b->threads = threads;
    b->tw = tile;
    return SPB6G_OK;
}
int spb6g_batch_advance(spb6g_batch* b, int nsteps, float* ms) {
    if (!b || nsteps < 1) return SPB6G_BAD_ARG;
    cudaSetDevice(b->device);
    for (spb6g_solver* s : b->inst) CK(cudaStreamSynchronize(s->st));  // uploads and set-up on the instances' streams
    return batch_run(b, nsteps, b->threads, b->tw, ms);
}
// Times `nsteps` steps of every launch shape (threads per instance x flux tile width) from the
// current state, restores the state after each trial, and keeps the fastest shape.
int spb6g_batch_autotune(spb6g_batch* b, int nsteps, int* threads_out, int* tile_out, float* best_ms) {
    if (!b || nsteps < 1) return SPB6G_BAD_ARG;
    cudaSetDevice(b->device);
    for (spb6g_solver* s : b->inst) CK(cudaStreamSynchronize(s->st));
    const size_t n0 = b->inst.size();
    // snapshot: the state arrays, the accepted pressure and the host-side time state
    std::vector<std::vector<double*>> snap(n0);
    std::vector<spb6g_solver> keep;
    keep.reserve(n0);
    for (size_t i = 0; i < n0; i++) {
        spb6g_solver* s = b->inst[i];
        keep.push_back(*s);
        for (int k = 0; k < NV + 1; k++) {
            double* d = nullptr;
            if (cudaMalloc(&d, (size_t)s->n * sizeof(double)) != cudaSuccess) return SPB6G_CUDA_ERROR;
            CK(cudaMemcpy(d, k < NV ? s->U[k] : s->Pmain, (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice));
            snap[i].push_back(d);
        }
    }
    int bt = b->threads, bw = b->tw;
    float bms = INFINITY;
    for (int threads : {64, 96, 128, 256})
        for (int tw : {128, 256}) {
            float ms = 0;
            const int rc = batch_run(b, nsteps, threads, tw, &ms);
            // restore
            for (size_t i = 0; i < n0; i++) {
                spb6g_solver* s = b->inst[i];
                const spb6g_solver& k0 = keep[i];
                s->c = k0.c;
                for (int k = 0; k < NV; k++) { s->U[k] = k0.U[k]; s->Ust[k] = k0.Ust[k]; }
                s->Pmain = k0.Pmain;
                s->t = k0.t; s->dt = k0.dt; s->dtprev = k0.dtprev; s->startup = k0.startup; s->stats = k0.stats;
                for (int k = 0; k < NV + 1; k++)
                    CK(cudaMemcpy(k < NV ? s->U[k] : s->Pmain, snap[i][k], (size_t)s->n * sizeof(double), cudaMemcpyDeviceToDevice));
                b->status[i] = SPB6G_OK;
            }
            if (rc == SPB6G_OK && ms < bms) { bms = ms; bt = threads; bw = tw; }
        }
    for (auto& v : snap)
        for (double* d : v) cudaFree(d);
    b->threads = bt;
    b->tw = bw;
    if (threads_out) *threads_out = bt;
    if (tile_out) *tile_out = bw;
    if (best_ms) *best_ms = bms;
    return isfinite(bms) ? SPB6G_OK : SPB6G_STEP_FAILED;
}

int spb6g_get_stats(spb6g_solver* s, spb6g_stats* st) {
    if (!s || !st) return SPB6G_BAD_ARG;
    *st = s->stats;
    st->t = s->t;
    st->dt = s->dt;
    st->p_ref = s->p_ref;
    return SPB6G_OK;
}
int spb6g_set_time(spb6g_solver* s, double t, double dtprev, int startup) {
    if (!s) return SPB6G_BAD_ARG;
    s->t = t; s->dtprev = dtprev; s->startup = startup != 0;
    return SPB6G_OK;
}
int spb6g_get_time(const spb6g_solver* s, double* t, double* dtprev, int* startup) {
    if (!s) return SPB6G_BAD_ARG;
    if (t) *t = s->t;
    if (dtprev) *dtprev = s->dtprev;
    if (startup) *startup = s->startup ? 1 : 0;
    return SPB6G_OK;
}
int spb6g_timing_enable(spb6g_solver* s, int on) {
    if (!s) return SPB6G_BAD_ARG;
    cudaStreamSynchronize(s->st);
    resolve_timing(s);
    s->timing = on != 0;
    for (int g = 0; g < TG_COUNT; g++) { s->tms[g] = 0; s->tcnt[g] = 0; }
    return SPB6G_OK;
}
int spb6g_timing_get(spb6g_solver* s, double* ms, int64_t* launches, int max_groups, int* n_groups) {
    if (!s) return SPB6G_BAD_ARG;
    cudaStreamSynchronize(s->st);
    resolve_timing(s);
    for (int g = 0; g < TG_COUNT && g < max_groups; g++) {
        if (ms) ms[g] = s->tms[g];
        if (launches) launches[g] = s->tcnt[g];
    }
    if (n_groups) *n_groups = TG_COUNT;
    return SPB6G_OK;
}
int spb6g_region_begin(spb6g_solver* s) {
    if (!s) return SPB6G_BAD_ARG;
    CK(cudaEventRecord(s->region[0], s->st));
    return SPB6G_OK;
}
int spb6g_region_end(spb6g_solver* s, double* ms) {
    if (!s || !ms) return SPB6G_BAD_ARG;
    CK(cudaEventRecord(s->region[1], s->st));
    CK(cudaEventSynchronize(s->region[1]));
    float f = 0;
    CK(cudaEventElapsedTime(&f, s->region[0], s->region[1]));
    *ms = f;
    return SPB6G_OK;
}
int64_t spb6g_kernel_launches(spb6g_solver* s) { return s ? (int64_t)s->nlaunch : -1; }

const char* spb6g_timing_name(int group) { return (group >= 0 && group < TG_COUNT) ? kTimerNames[group] : "?"; }

const char* spb6g_status_string(int status) {
    switch (status) {
        case SPB6G_OK: return "ok";
        case SPB6G_INADMISSIBLE: return "inadmissible state";
        case SPB6G_NEWTON_FAIL: return "Newton failed";
        case SPB6G_LINEAR_FAIL: return "BiCGStab failed";
        case SPB6G_STEP_FAILED: return "step failed after 30 halvings";
        case SPB6G_DT_UNDERFLOW: return "time step underflow";
        case SPB6G_CUDA_ERROR: return "CUDA error";
        case SPB6G_BAD_ARG: return "bad argument";
        case SPB6G_UNSUPPORTED: return "unsupported configuration";
        case SPB6G_NO_DEVICE: return "no CUDA device";
        case SPB6G_TOO_LARGE: return "grid larger than the allocation-free entry point's fixed scratch";
    }
    return "unknown";
}

}  // extern "C"
