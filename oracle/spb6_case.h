/* Test infrastructure (oracle side): the binary case / result records shared by
 * the reference harness (oracle/ref_harness.cpp, built into oracle/_ref/) and
 * the C restatement (oracle/spb6_oracle.c).  Nothing in the product includes
 * this file.
 *
 * A case file is one spb6_case record followed by the initial conservative
 * state: nx*ny cells x 8 doubles, interior cells only, row-major (j outer,
 * i inner), variables innermost in the reference order
 * alpha1, m1, m2, rho*u, rho*v, eps1, eps2, E (src/spb6_physics_omp.h:27-28).
 *
 * A result file is one spb6_result record followed by U (same layout) and the
 * pressure unknown P (nx*ny doubles, P - P_REF as in src/SPB6_PC_IMEX_omp.cpp:
 * 1307-1312).  In stage-dump mode it is followed by the explicit predictor
 * X* (nx*ny*8), alpha2* (nx*ny), the x-face velocities ube_x ((nx+1)*ny,
 * faces i-1/2 .. nx-1/2 of interior rows), the y-face velocities ube_y
 * (nx*(ny+1)), and the limiter factors phi_x, phi_y (nx*ny each).
 */
#ifndef SPB6_CASE_H
#define SPB6_CASE_H
#include <stdint.h>

#define SPB6_CASE_MAGIC 0x36425053u /* "SPB6" */
#define SPB6_CASE_VERSION 4

enum { SPB6_MODE_STEPS = 0, SPB6_MODE_TEND = 1, SPB6_MODE_STAGE = 2, SPB6_MODE_SAT = 3 };
enum { SPB6_BC_TRANS = 0, SPB6_BC_WALL = 1, SPB6_BC_PERIODIC = 2, SPB6_BC_PRES = 3 };

typedef struct {
    uint32_t magic;
    int32_t version;
    int32_t nx, ny;
    int32_t bc[4]; /* left, right, bottom, top */
    int32_t rk, ramp, rus_local, limiter, acdt, newton_iter, bicg_iter, share_mode;
    int32_t mode, nsteps;
    int32_t threads;
    int32_t order;     /* spatial order: 1 no reconstruction, else MUSCL (reference harness only) */
    double x0, x1, y0, y1;
    double bcu[4], bcp[4];
    double g[2], pinf[2], q[2], qp[2], cv[2], b[2];
    double cfl, cfl_ac, dtfix, newton_tol, bicg_tol, tend;
    double budget_s;   /* > 0: stop stepping once the timed steps have used this much wall time */
    int32_t warmup;    /* steps run before the timed region (wall_s counts the rest) */
    int32_t inject_qph; /* stage mode, C restatement only: U0 is followed by Q_1, Q_2 (2 x nx*ny) */
    int32_t kind[2];    /* 0 SG / NASG, 1 Cochran-Chan, 2 JWL (reference harness only; the C restatement
                           runs SG / NASG phases) */
    double mg_G[2], mg_rr[2], mg_c1[2], mg_c2[2], mg_e1[2], mg_e2[2], mg_e0[2];
    int32_t relax;        /* RELAX_LEVEL (reference harness only; the C restatement has relax 0) */
    int32_t jreuse;       /* JREUSE (reference harness only; the C restatement has 0) */
    double eps_i;
    /* relaxation rates (reference harness only; the C restatement has the defaults): mu_rate, and
       theta_rate / nu_rate < 0 for the level's default, nu law coefficient and pressure */
    double mu_rate, theta_rate, nu_rate, nu_cr, nu_pc;
    int32_t relax_form, unify, unify_proj, nu_law;
} spb6_case;

typedef struct {
    uint32_t magic;
    int32_t status; /* 0 ok, 1 bad input, 2 solver failure (as the reference's exit code 2) */
    int32_t nx, ny;
    int64_t steps, rejects, rk1, stages, newton_it, floor_count, bicg_it, timed_steps; /* steps inside the timed region (all steps when warmup = 0) */
    double t, dt, maxres, p_ref, wall_s;
    double dM[3];
} spb6_result;

#endif
