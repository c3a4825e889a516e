/* spb6g.h -- C ABI of the B200 SPB 6+1-equation IMEX solver.
 *
 * The reference (src/SPB6_PC_IMEX_omp.cpp + src/spb6_physics_omp.h) has no
 * library interface: its API is main()'s time loop over mutable globals and
 * the stage functions TVDReconstruction / Update / PressureSubsystem / caldt /
 * bound_cond_u.  This header is the boundary a host driver (the reference's
 * main() loop, a cgo / ctypes / JNI binding, or this package's Python layer)
 * links against instead.  Every entry point names the reference code it
 * replaces.  Plain C types only; all functions return an spb6g_status; no
 * exceptions cross the ABI.  One solver handle = one CUDA stream = one host
 * thread at a time; the handle owns its device memory, the caller owns every
 * host buffer.
 *
 * State layout on the host side: SPB6G_LAYOUT_AOS is the reference Grid's
 * interior cells (Grid, :124-143, without the two ghost layers): index
 * ((j * nx + i) * 8 + k); SPB6G_LAYOUT_SOA is k-major: (k * ny + j) * nx + i.
 * Variables k follow the reference order alpha1, m1, m2, rho u, rho v, eps1,
 * eps2, E (src/spb6_physics_omp.h:27-28).
 */
#ifndef SPB6G_H
#define SPB6G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    SPB6G_OK = 0,
    SPB6G_INADMISSIBLE = 1,     /* Update / stage prep found rho <= 0 or sum alpha <= 0 (:272, :929) */
    SPB6G_NEWTON_FAIL = 2,      /* Newton_Solver returned false (:799-904) */
    SPB6G_LINEAR_FAIL = 3,      /* GMRES_Solver (BiCGStab) returned false (:752-794) */
    SPB6G_STEP_FAILED = 4,      /* 30 halvings without success: the reference's "FAILED" exit (:1378) */
    SPB6G_DT_UNDERFLOW = 5,     /* dt <= 1e-12 t_end (:1326) */
    SPB6G_CUDA_ERROR = 6,
    SPB6G_BAD_ARG = 7,
    SPB6G_UNSUPPORTED = 8,
    SPB6G_NO_DEVICE = 9,
    SPB6G_TOO_LARGE = 10        /* grid larger than spb6g_caldt_noalloc's fixed scratch, or an
                                   output buffer too small */
} spb6g_status;

enum { SPB6G_BC_TRANS = 0, SPB6G_BC_WALL = 1, SPB6G_BC_PERIODIC = 2, SPB6G_BC_PRES = 3 };
enum { SPB6G_LAYOUT_AOS = 0, SPB6G_LAYOUT_SOA = 1 };

/* Replaces main()'s globals and test_setup()'s TestSetup
 * (src/SPB6_PC_IMEX_omp.cpp:55-95, src/spb6_physics_omp.h:954-961, :1014).
 * Phases are stiffened gas / NASG: p = (gamma-1)(e - q)/(v - b) - gamma pinf. */
typedef struct {
    int32_t nx, ny;                 /* interior cells; ny = 1 is the 1D solver */
    double x0, x1, y0, y1;          /* domain */
    int32_t bc[4];                  /* left, right, bottom, top: SPB6G_BC_* (BCS, physics :964) */
    double bcu[4];                  /* wall normal velocity (piston), BCU */
    double bcp[4];                  /* outlet pressure, BCP */
    double gamma[2], pinf[2], q[2], qp[2], cv[2], b[2]; /* PH[2], physics :55-56 */
    int32_t rk;                     /* 1 backward Euler, 2 LSDIRK2(2,2,2), 3 SSP2(3,3,2) (RKs, :69) */
    double cfl, cfl_ac;             /* material CFL, start-up acoustic CFL (:71-72) */
    int32_t ramp;                   /* start-up ramp (RAMP, :75) */
    double dtfix;                   /* > 0: fixed step (DTFIX, :77) */
    int32_t rus_local;              /* RUS_LOCAL (:93): 1 per-face max(|u_L|, |u_R|), 0 the grid-wide
                                       maximum over cells and face states (batched form: 1 only) */
    int32_t limiter;                /* LIMITER (physics :969) */
    int32_t acdt;                   /* 1: acoustic CFL every step (caltimestep = Fullydt, :55) */
    double newton_tol;              /* NewtonTol (:79) */
    int32_t newton_iter;            /* NewtonIter (:82) */
    double bicg_tol;                /* GMREStol (:84) */
    int32_t bicg_iter;              /* GMRESiter (:85) */
    int32_t share_mode;             /* SHARE_MODE (physics :436) */
    double tend;                    /* time_stop */
    int32_t device;                 /* CUDA device ordinal */
    int32_t precision;              /* 0: FP64 throughout; 1: precision form -- FP32 reconstruction,
                                       Rusanov fluxes and SpMV, FP64 EOS inversion, relaxation Newton,
                                       BiCGStab reductions and residuals (no counterpart in the reference) */
    int32_t kind[2];                /* 0 SG / NASG; Mie-Grueneisen p = G rho (e - er(rho)) + pr(rho):
                                       1 Cochran-Chan pr = c1 x^e1 - c2 x^e2, x = rho / rr;
                                       2 JWL pr = c1 exp(-e1 rr / rho) + c2 exp(-e2 rr / rho), er - e0
                                       (Phase.kind, physics :51-69); MG phases use only G, rr, c1, c2,
                                       e1, e2, e0 and cv (temperature output) */
    int32_t relax;                  /* RELAX_LEVEL (physics :39): 0 mechanical relaxation; in the interface zone
                                       1 p-pT (instantaneous thermal relaxation), 2 p-pT-pTg and 3 p-pTg
                                       (instantaneous chemical relaxation above the saturation temperature);
                                       SG / NASG phases only (SPB6G_UNSUPPORTED with a Mie-Grueneisen phase);
                                       the rates are mu_rate, theta_rate, nu_rate below */
    int32_t jreuse;                 /* JREUSE (:83): 1 modified Newton -- the FD Jacobian of the stage's first
                                       iteration is kept while each step is undamped and contracts the
                                       residual 4x (batched form: 0 only) */
    int32_t order;                  /* spatial order (order=, :1210): 2 MUSCL reconstruction (the default;
                                       0 reads as 2), 1 the cell values on the faces (NoRecon, :372-375) */
    int32_t reserved[1];
    double mg_G[2], mg_rr[2], mg_c1[2], mg_c2[2], mg_e1[2], mg_e2[2], mg_e0[2];
    double eps_i;                   /* EPS_I (physics :40): interface zone eps_I <= alpha1 <= 1 - eps_I (1e-4) */
    /* Relaxation rates (physics :34-46; mu=, theta=, nu=, relaxform=, unify=, unifyproj=, nulaw=,
     * nucr=, nupc= arguments).  A rate of INFINITY is instantaneous; a finite rate turns the p, pT or
     * pTg closure of a cell into its finite-rate form (closure_mu, closure_theta, closure_nu). */
    double mu_rate;                 /* pressure relaxation rate (INFINITY) */
    double theta_rate;              /* heat exchange rate; < 0: INFINITY for relax >= 1, else 0 (-1) */
    double nu_rate;                 /* mass transfer rate; < 0: INFINITY for relax 2, 3, else 0 (-1) */
    double nu_cr, nu_pc;            /* nu law (physics :36-38): coefficient (1) and pressure (22.064e6) */
    int32_t relax_form;             /* RELAX_FORM: 0 backward Euler over the stage step, 1 exponential (0) */
    int32_t unify;                  /* UNIFY: 1 the instantaneous closures as their rate = inf forms (0) */
    int32_t unify_proj;             /* UNIFY_PROJ: 0 no projection of the step's state at activation (1) */
    int32_t nu_law;                 /* NU_LAW: 1 the mass transfer rate of each cell from nu_law at the
                                       step start (0) */
} spb6g_config;

/* Run statistics: the counters of the reference's stats line (:98-99, :1425). */
typedef struct {
    int64_t steps, rejects, rk1, stages, newton_it, floor_count, bicg_it;
    int64_t learned;                /* stages whose Newton started from the learned guess */
    double t, dt, maxres, p_ref;
    double tmax[2];                 /* max phase temperatures of the stages' final states (st_Tmax :96, :1070) */
    int64_t learned_x0;             /* BiCGStab solves that started from a learned first iterate */
    int64_t extrapolated;           /* stages whose Newton started from the extrapolated pressure */
    int64_t extrapolated2;          /* ... from the second-order extrapolation */
    int64_t combined;               /* ... from the residual-minimising combination (mode bit 8) */
    int64_t refined;                /* stages whose start Jacobi sweeps improved (mode bit 16) */
} spb6g_stats;

typedef struct spb6g_solver spb6g_solver;
typedef struct spb6g_mlp spb6g_mlp;

/* Fills *cfg with the reference defaults (SPB6_PC_IMEX_omp.cpp:55-95, set_SG physics :1014). */
void spb6g_default_config(spb6g_config* cfg);

/* Allocates the device state of one grid (replaces main's Grid/Array allocations :1245-1248). */
int spb6g_create(const spb6g_config* cfg, spb6g_solver** out);
int spb6g_destroy(spb6g_solver* s);

/* Initial / current conservative state of the interior cells (u_initialization :475-492). */
int spb6g_upload_state(spb6g_solver* s, const double* U, int layout);
int spb6g_download_state(spb6g_solver* s, double* U, int layout);

/* P_REF = min pbar and P = pbar - P_REF, the plain Newton guess at t = 0 (:1307-1312). */
int spb6g_init_pressure(spb6g_solver* s);
/* The pressure unknown P - P_REF (PField, :172), nx*ny doubles. */
int spb6g_set_pressure(spb6g_solver* s, const double* P, double p_ref);
int spb6g_get_pressure(spb6g_solver* s, double* P, double* p_ref);

/* The saturation table of cfg's two SG / NASG phases (build_sat, physics :127-153), host only:
 * n, pcrit, vcrit, pmin, then ln p[n] and Tsat[n] -- 4 + 2n doubles, the count in *len.  With
 * out == NULL only *len is set; SPB6G_TOO_LARGE if cap < *len.  Solvers with relax >= 2 build and
 * keep it on the device themselves. */
int spb6g_saturation_table(const spb6g_config* cfg, double* out, int cap, int* len);

/* caldt (:502-514): returns 1 / (a_x/dx + a_y/dy) (INFINITY if the rate is 0). */
int spb6g_caldt(spb6g_solver* s, int acoustic, double* inv_rate);

/* One iteration of main()'s time loop (:1316-1384): step size, ramp, stages,
 * halving on failure, acceptance.  Statistics accumulate in the handle. */
int spb6g_step(spb6g_solver* s);
/* Steps until nsteps steps are taken (nsteps > 0) or t reaches t_end. */
int spb6g_advance(spb6g_solver* s, int nsteps);

/* Stage-level API, the reference's stage functions on the device state:
 * stage 0 of the configured tableau with step dt -- TVDReconstruction + Update
 * (:369, :264) followed by PressureSubsystem (:908) -- leaving the new state in
 * the handle.  Optional outputs (NULL to skip) mirror the stage globals the
 * reference passes between them: X* (AoS), alpha2*, ube_x ((nx+1)*ny),
 * ube_y (nx*(ny+1)), phi_x, phi_y (nx*ny). */
int spb6g_stage_dump(spb6g_solver* s, double dt, double* Xs, double* a2s, double* ube_x, double* ube_y,
                     double* phi_x, double* phi_y);

/* One stage of any tableau on the device state, the three calls of main()'s stage loop
 * (:1341-1366): Qe = U^n + sum_{r<rks} Ae_row[r] dt H_r, Qs = U^n + sum_{r<rks} Ai_row[r] dt H_r,
 * TVDReconstruction + Update (:369, :264) and PressureSubsystem (:908) with adt = Ai_row[rks] dt,
 * then H_rks = (U_s - Qs) / adt (:1360).  U^n is the handle's state, which stages do not change.
 * rks = 0 begins an attempt: RelaxationActivation (:1333, relax > 0) and Pst = P (:1335); stage
 * rks > 0 needs stage rks - 1 of the same attempt to have converged (else SPB6G_BAD_ARG).
 * Ae_row needs rks entries, Ai_row rks + 1.  A failed stage returns its status (the caller halves
 * dt and starts a new attempt at rks = 0); *st (if not NULL) receives the handle's statistics. */
int spb6g_stage(spb6g_solver* s, int rks, const double* Ae_row, const double* Ai_row, double dt, spb6g_stats* st);
/* Accepts the attempt whose last stage converged: u_con = U_s, P = Pst (:1374), and advances the
 * handle's time by dt (t, the last accepted step, the step count; :1379).  SPB6G_BAD_ARG when no
 * stage of the current attempt has converged. */
int spb6g_stage_accept(spb6g_solver* s, double dt);

/* Stage data of the last stage (StageData, :591-608): x-face coefficients ubs, kp, wL, pv
 * (4 blocks of (nx+1)*ny, faces i-1/2 .. nx-1/2), y-face coefficients (4 blocks of nx*(ny+1)),
 * the residual scale K + P_E (nx*ny) and the shock budget Q_1, Q_2 (2 blocks of nx*ny). */
int spb6g_stage_data(spb6g_solver* s, double* fx, double* fy, double* kw, double* qph);

int spb6g_get_stats(spb6g_solver* s, spb6g_stats* st);

/* ---------------------------------------------------------------------------
 * Output of the reference's main(): the 17-column profile (write_profile,
 * :1083-1094: "# x y p u v rho alpha2 Y2 rho1 rho2 c_frozen c_wood T1 T2 p1 p2
 * g1-g2", one line per interior cell, j outer, i inner), snapshots (snap=:
 * the step size is cut to land on each time, physics :972, and the profile is
 * written to <out>_s<k>.dat when t reaches it, :1380), the pressure probe
 * (probe=x,y: "t p Y2 alpha2 T1" of the nearest cell before the first step
 * and after every accepted step to <out>.probe, :1191-1197) and the final
 * profile at t_end or when a step fails (:1326, :1379, :1388).  Cell
 * diagnostics are evaluated on the host in FP64 with the reference's
 * formulas, so a state equal to the reference's prints the same text. */
typedef struct {
    const char* out_file;           /* NULL or "": no files */
    const double* snaps;            /* snapshot times, ascending (snap=) */
    int32_t nsnap;
    int32_t probe;                  /* 1: write the probe file (probe=) */
    double probe_x, probe_y;
    int32_t prec;                   /* significant digits of the profile columns (prec=, 0: 16) */
} spb6g_output;
/* Copies *o; with a probe, writes the probe file's first line at the current state. */
int spb6g_set_output(spb6g_solver* s, const spb6g_output* o);
/* The profile of the current state to `path` (prec 0: 16 digits). */
int spb6g_write_profile(spb6g_solver* s, const char* path, int prec);
/* The same profile of a host state (AoS layout) for the grid and phases of *cfg; host code only,
 * needs no device. */
int spb6g_format_profile(const spb6g_config* cfg, const double* U, const char* path, int prec);
/* Sums of m1, m2 and E over the interior cells (conserved_totals, :1185-1188). */
int spb6g_conserved_totals(spb6g_solver* s, double* M3);
/* The reference's end-of-run line (:1425-1427) for this run: "case <id> mode 1 order 2 rk ...
 * | dM1/M .. dM2/M .. dE/E .. | wall <wall_s> s" (no newline); conservation against the totals
 * at spb6g_init_pressure. */
int spb6g_stats_line(spb6g_solver* s, int case_id, double wall_s, char* buf, size_t len);
/* Simulation time t (settable, e.g. when restarting from a dump). */
int spb6g_set_time(spb6g_solver* s, double t, double dtprev, int startup);
/* The time-loop state spb6g_set_time restores: t, the last accepted step (dtprev) and whether the
 * start-up ramp still runs (startup).  With spb6g_download_state and spb6g_get_pressure it is
 * everything the next step depends on -- a restart point. */
int spb6g_get_time(const spb6g_solver* s, double* t, double* dtprev, int* startup);

/* Per-kernel-group device time (ms, CUDA events on the solver's stream)
 * accumulated since timing was enabled; spb6g_timing_name(g) names group g. */
int spb6g_timing_enable(spb6g_solver* s, int on);
int spb6g_timing_get(spb6g_solver* s, double* ms, int64_t* launches, int max_groups, int* n_groups);
const char* spb6g_timing_name(int group);

/* Device time (ms) between region_begin and region_end, from CUDA events on the
 * solver's stream: everything the handle enqueued in between, host waits included. */
int spb6g_region_begin(spb6g_solver* s);
int spb6g_region_end(spb6g_solver* s, double* ms);
/* Number of kernels the handle has launched since creation. */
int64_t spb6g_kernel_launches(spb6g_solver* s);

/* Allocation-free time-step rate.  No counterpart in the reference: it is for
 * callers that cannot let a library call cudaMalloc -- a host framework that
 * owns all device memory through its own arena or pool, a time-critical loop
 * that cannot afford the device-wide synchronisation cudaMalloc / cudaFree may
 * cause, or a service whose device footprint must not grow after start-up.  Computes what spb6g_caldt computes, 1 / (a_x/dx + a_y/dy),
 * for a state the caller already holds on the device: U_dev is a host array of
 * 8 device pointers, one per conservative variable, each nx*ny interior cells
 * (SoA, cell (i, j) at i + j*nx); cfg supplies the grid and phases.  The only
 * scratch is a file-scope device array sized for SPB6G_NOALLOC_MAX_CELLS cells,
 * held by every GPU that loads the library until the process exits; larger
 * grids return SPB6G_TOO_LARGE.  The call runs on cfg->device (made current
 * for the call; the caller's current device is restored on return), every
 * U_dev[k] must be device or managed memory of that device (SPB6G_BAD_ARG
 * otherwise, found before any launch) and stream must belong to it.  The first
 * call on a device looks up the scratch's device address.  Every call is
 * blocking -- it copies the result to *inv_rate and waits for stream -- so no
 * call, first or later, may be made while a stream is being captured.  All
 * calls share the scratch (its counter is cleared at the start of each call):
 * calls whose GPU work overlaps race.  stream: a cudaStream_t, or NULL for the
 * default stream.  A degenerate domain (x1 <= x0 or y1 <= y0) or a phase kind
 * outside 0..2 is SPB6G_BAD_ARG; a Mie-Grueneisen phase SPB6G_UNSUPPORTED. */
#define SPB6G_NOALLOC_MAX_CELLS (4 * 1024 * 1024)
int spb6g_caldt_noalloc(const spb6g_config* cfg, const double* const* U_dev, int acoustic, void* stream,
                        double* inv_rate);

/* ---------------------------------------------------------------------------
 * Learned warm start (no counterpart in the reference: the reference always
 * starts a stage's Newton from the previous stage's pressure).  A small MLP,
 * 64 inputs (54 used) -> 64 -> 64 -> 64 -> 1 with SiLU, BF16 weights on the
 * tensor cores and FP32 accumulation, FP32 master weights trained with Adam.
 * Inputs are row-major BF16 feature rows of 64 values on the device (16-byte
 * aligned: they are read by TMA); outputs and targets FP32 on the device.  Calls
 * without a stream run on the handle's stream, which is ordered after the legacy
 * default stream only: inputs written on any other stream must be complete
 * before the call.  One handle per device and host thread. */
int spb6g_mlp_create(int device, spb6g_mlp** out);
void spb6g_mlp_destroy(spb6g_mlp* m);
/* Number of FP32 parameters: W1[64][64], b1[64], W2[64][64], b2[64], W3[64][64], b3[64], w4[64], b4. */
int spb6g_mlp_param_count(void);
int spb6g_mlp_set_params(spb6g_mlp* m, const float* params_host);  /* also resets the Adam state */
int spb6g_mlp_get_params(spb6g_mlp* m, float* params_host);
/* y[i] = MLP(X[i]) for n rows; stream NULL: the handle's stream, synchronised. */
int spb6g_mlp_forward(spb6g_mlp* m, const void* X_dev, int n, float* y_dev, void* stream);
/* One pass over the n rows: gradient of mean((y - target)^2) (copied to grad_host if not NULL),
 * loss to *loss_out; with lr > 0 also one Adam step (beta 0.9 / 0.999, eps 1e-8). */
int spb6g_mlp_train_step(spb6g_mlp* m, const void* X_dev, const float* target_dev, int n, float lr, float* loss_out,
                         float* grad_host);
/* The same pass launched on `stream` (NULL: the handle's stream) without waiting or reading
 * anything back, for training loops that keep the device busy. */
int spb6g_mlp_train_async(spb6g_mlp* m, const void* X_dev, const float* target_dev, int n, float lr, void* stream);
/* Sum over the rows of (y - target)^2 of the last pass (waits for `stream`; reports a timed-out
 * tensor-core wait of any earlier call as an error). */
int spb6g_mlp_last_loss(spb6g_mlp* m, void* stream, float* loss_sum);

/* Warm start on the solver (no counterpart in the reference).  The features of a cell are
 * the 3x3 stencils of 7 fields: rho, rho u, rho v, alpha1, E* of the explicit predictor, the
 * stage's starting pressure P - P_REF, and R / sigma, R the pressure rate
 * (P_converged - P_start) / dts of the last converged stage (dts = the stage's time span,
 * (c_s - c_{s-1}) dt from the implicit tableau's row sums; R = 0 before the first stage) and
 * sigma its RMS over the cells -- 63 columns -- and (R - R2) / sigma of the cell itself, R2 the
 * rate of the stage before.  norm: 22 doubles: mean[7], std[7] of the centre values and std[7]
 * of the neighbour differences of the 7 fields, then the target scale (sigma before the first
 * converged stage).  Setting it also starts tracking R. */
int spb6g_set_feature_norm(spb6g_solver* s, const double* norm);
/* m != NULL: every stage predicts its pressure P_start + dts (R + sigma MLP(features)).
 * Mode bits (spb6g_set_warmstart_mode; 15 by default):
 *  1: Newton starts from the guess of smallest residual max-norm among the plain guess (the
 *     previous stage's pressure), the extrapolation P_start + dts R (the network's zero output),
 *     the second-order extrapolation P_start + dts (R + k (R - R2)) (R2 the rate of the stage
 *     before, k from the stages' time spans) and the network's guess;
 *  2: when the network's guess is not the start, the first BiCGStab solve of the stage starts
 *     from x0 = a M^-1 b + c dP, dP the network's step from the start and (a, c) minimising
 *     ||b - A x0||, when that residual is below 0.99 of the plain start's (x0 = M^-1 b,
 *     GMRES_Solver :769), else from M^-1 b;
 *  4: every later solve of the stage takes the last Newton correction as that candidate dP;
 *  8: with bit 1, the start combining the candidates' steps that minimises ||G||_2 of the
 *     residual taken linear in P (from the candidates' residuals) is a candidate too;
 *  16: up to two Jacobi sweeps of the start (the last Jacobian's diagonal, step length by the
 *     same minimisation) when its residual is within 30 tolerances;
 *  32: with bit 8, the older rate change dts (R2 - R3) as a fourth direction.
 * Newton and BiCGStab keep their tolerances, and a warm-started stage always takes at least one
 * Newton step.  NULL: off. */
int spb6g_set_warmstart(spb6g_solver* s, spb6g_mlp* m);
int spb6g_set_warmstart_mode(spb6g_solver* s, int mode);
/* Radius r (0: none, the default; at most 64 and below nx, ny) of a separable box average of the
 * network's output before it forms a guess: the implicit pressure operator amplifies a cell-to-
 * cell error of the guess by about (c tau / h)^2, so only the smooth part of a per-cell prediction
 * can improve a start whose own error is smooth. */
int spb6g_set_warmstart_smoothing(spb6g_solver* s, int radius);
/* Training data: each stage appends n feature rows (64 BF16 each) to X_dev and n
 * targets (R' - R) / sigma to target_dev while capacity allows (R' the stage's converged
 * pressure rate, R the last stage's). */
int spb6g_set_dump(spb6g_solver* s, void* X_dev, float* target_dev, int64_t capacity);
int spb6g_dump_count(spb6g_solver* s, int64_t* count);

/* ---------------------------------------------------------------------------
 * Batched form (no counterpart in the reference): independent 1D grids (ny = 1,
 * non-periodic, so the Thomas path) advanced together by persistent launches -- one
 * thread block per grid runs that grid's whole time loop, one launch per block size,
 * the launches concurrent -- replayed from a captured CUDA graph.  Each grid is an ordinary solver handle
 * (spb6g_batch_instance) for upload, initial pressure, download and statistics. */
typedef struct spb6g_batch spb6g_batch;
int spb6g_batch_create(const spb6g_config* cfgs, int count, spb6g_batch** out);
void spb6g_batch_destroy(spb6g_batch* b);
spb6g_solver* spb6g_batch_instance(spb6g_batch* b, int i);
/* Status of grid i after the last advance (SPB6G_OK, or the error that stopped it). */
int spb6g_batch_status(spb6g_batch* b, int i);
/* Launch shape: block size of the largest grid (a multiple of 32 from 32 to 256) and flux
 * tile width (128, 256).  Every other grid gets a block size in proportion to its cells
 * (rounded up to a multiple of 32, at least 32); grids of one block size form one launch,
 * longest first, and the launches run concurrently. */
int spb6g_batch_set_shape(spb6g_batch* b, int threads, int tile);
/* nsteps time steps of every grid (fewer for a grid that reaches its t_end); device time
 * of the launch in *ms if not NULL.  Returns the first grid's error, if any. */
int spb6g_batch_advance(spb6g_batch* b, int nsteps, float* ms);
/* The block size each grid of a batch gets (host only, no device): threads in proportion to its
 * cells, a multiple of 32 from 32 to `threads` (the largest grid's cap), with the fewest cells
 * per thread for which the blocks' threads fit in `slots` (0: no limit; the batch uses 15/16 of
 * the device's thread slots at the kernel's register count); the cells per thread in
 * *per_thread if not NULL. */
int spb6g_batch_block_sizes(const int64_t* cells, int count, int threads, int64_t slots, int* block,
                            int64_t* per_thread);
/* Kernel launches of one advance under the current shape (one per block size); 0 before the
 * first advance under it, or a negative status. */
int spb6g_batch_launches(spb6g_batch* b);
/* Times nsteps steps with every launch shape (largest block 64, 96, 128, 256 x tile 128, 256)
 * from the current state (restored after each trial) and keeps the fastest. */
int spb6g_batch_autotune(spb6g_batch* b, int nsteps, int* threads, int* tile, float* best_ms);

/* Human-readable status name. */
const char* spb6g_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif
