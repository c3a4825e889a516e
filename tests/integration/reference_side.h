// Stand-ins for the reference program's globals that the C++ binding in INTEGRATION.md reads,
// with the reference's names and meaning (src/SPB6_PC_IMEX_omp.cpp:55-95, :124-143, :1280-1303;
// src/spb6_physics_omp.h:51-69), filled from a case file instead of the reference's test_setup.
// Test infrastructure: tests/test_integration.py compiles the INTEGRATION.md blocks against it.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

struct PhaseRec { double g, pi, q, qp, cv, b; int kind; double G, rr, c1, c2, e1, e2, e0; };
static PhaseRec PH[2];
static int nxCells, nyCells;
static double x_0, x_1, y_0, y_1;
static int BCS[4];
static double BCU[4], BCP[4];
static int RKs, RAMP, RUS_LOCAL, LIMITER, NewtonIter, GMRESiter, SHARE_MODE, SpaceOrder, JREUSE;
static int RELAX_LEVEL, NU_LAW, RELAX_FORM, UNIFY, UNIFY_PROJ;
static double CFL, CFL_ac, DTFIX, NewtonTol, GMREStol, time_stop, EPS_I, mu_rate, theta_rate, nu_rate, NU_CR, NU_PC;
enum { Materialdt = 0, Fullydt = 1 };
static int caltimestep;
static const int NUM_VARS = 8, ghost_cells = 2;
static const double ramp_factor = 1.2;
inline int IG(int i) { return i + ghost_cells; }

// the conservative state with two ghost layers, AoS like the reference's Grid
struct GridT {
    int nx = 0, ny = 0;
    std::vector<double> v;
    void resize(int x, int y) { nx = x; ny = y; v.assign((size_t)(x + 4) * (y + 4) * NUM_VARS, 0.0); }
    double& operator()(int i, int j, int k) { return v[((size_t)j * (nx + 4) + i) * NUM_VARS + k]; }
};
static GridT u_con;

// main()'s tableaux (set_tab, :1281-1303)
static double Ae[3][3], Ai[3][3];
inline void set_tab(int rk) {
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

// Case file: one "name v0 v1 ..." line per global; state file: the interior cells, AoS, doubles.
inline bool load_case(const char* case_path, const char* state_path) {
    FILE* f = std::fopen(case_path, "r");
    if (!f) return false;
    char name[64];
    auto rd = [&](double* dst, int n) { for (int q = 0; q < n; q++) if (std::fscanf(f, "%lf", &dst[q]) != 1) return false; return true; };
    auto ri = [&](int* dst, int n) { for (int q = 0; q < n; q++) if (std::fscanf(f, "%d", &dst[q]) != 1) return false; return true; };
    bool ok = true;
    while (ok && std::fscanf(f, "%63s", name) == 1) {
        const std::string k = name;
        double d[2];
        int iv[2];
        if (k == "nxCells") ok = ri(&nxCells, 1);
        else if (k == "nyCells") ok = ri(&nyCells, 1);
        else if (k == "domain") { double b[4]; ok = rd(b, 4); x_0 = b[0]; x_1 = b[1]; y_0 = b[2]; y_1 = b[3]; }
        else if (k == "BCS") ok = ri(BCS, 4);
        else if (k == "BCU") ok = rd(BCU, 4);
        else if (k == "BCP") ok = rd(BCP, 4);
        else if (k == "g") { ok = rd(d, 2); PH[0].g = d[0]; PH[1].g = d[1]; }
        else if (k == "pi") { ok = rd(d, 2); PH[0].pi = d[0]; PH[1].pi = d[1]; }
        else if (k == "q") { ok = rd(d, 2); PH[0].q = d[0]; PH[1].q = d[1]; }
        else if (k == "qp") { ok = rd(d, 2); PH[0].qp = d[0]; PH[1].qp = d[1]; }
        else if (k == "cv") { ok = rd(d, 2); PH[0].cv = d[0]; PH[1].cv = d[1]; }
        else if (k == "b") { ok = rd(d, 2); PH[0].b = d[0]; PH[1].b = d[1]; }
        else if (k == "kind") { ok = ri(iv, 2); PH[0].kind = iv[0]; PH[1].kind = iv[1]; }
        else if (k == "mg") {  // G rr c1 c2 e1 e2 e0 of phase 0, then of phase 1
            for (int p = 0; p < 2 && ok; p++) {
                double m[7];
                ok = rd(m, 7);
                PH[p].G = m[0]; PH[p].rr = m[1]; PH[p].c1 = m[2]; PH[p].c2 = m[3]; PH[p].e1 = m[4]; PH[p].e2 = m[5]; PH[p].e0 = m[6];
            }
        }
        else if (k == "RKs") ok = ri(&RKs, 1);
        else if (k == "RAMP") ok = ri(&RAMP, 1);
        else if (k == "RUS_LOCAL") ok = ri(&RUS_LOCAL, 1);
        else if (k == "LIMITER") ok = ri(&LIMITER, 1);
        else if (k == "NewtonIter") ok = ri(&NewtonIter, 1);
        else if (k == "GMRESiter") ok = ri(&GMRESiter, 1);
        else if (k == "SHARE_MODE") ok = ri(&SHARE_MODE, 1);
        else if (k == "SpaceOrder") ok = ri(&SpaceOrder, 1);
        else if (k == "JREUSE") ok = ri(&JREUSE, 1);
        else if (k == "RELAX_LEVEL") ok = ri(&RELAX_LEVEL, 1);
        else if (k == "NU_LAW") ok = ri(&NU_LAW, 1);
        else if (k == "RELAX_FORM") ok = ri(&RELAX_FORM, 1);
        else if (k == "UNIFY") ok = ri(&UNIFY, 1);
        else if (k == "UNIFY_PROJ") ok = ri(&UNIFY_PROJ, 1);
        else if (k == "caltimestep") ok = ri(&caltimestep, 1);
        else if (k == "CFL") ok = rd(&CFL, 1);
        else if (k == "CFL_ac") ok = rd(&CFL_ac, 1);
        else if (k == "DTFIX") ok = rd(&DTFIX, 1);
        else if (k == "NewtonTol") ok = rd(&NewtonTol, 1);
        else if (k == "GMREStol") ok = rd(&GMREStol, 1);
        else if (k == "time_stop") ok = rd(&time_stop, 1);
        else if (k == "EPS_I") ok = rd(&EPS_I, 1);
        else if (k == "mu_rate") ok = rd(&mu_rate, 1);
        else if (k == "theta_rate") ok = rd(&theta_rate, 1);
        else if (k == "nu_rate") ok = rd(&nu_rate, 1);
        else if (k == "NU_CR") ok = rd(&NU_CR, 1);
        else if (k == "NU_PC") ok = rd(&NU_PC, 1);
        else ok = false;
    }
    std::fclose(f);
    if (!ok) return false;
    u_con.resize(nxCells, nyCells);
    FILE* s = std::fopen(state_path, "rb");
    if (!s) return false;
    std::vector<double> in((size_t)nxCells * nyCells * NUM_VARS);
    const bool got = std::fread(in.data(), sizeof(double), in.size(), s) == in.size();
    std::fclose(s);
    if (!got) return false;
    for (int j = 0; j < nyCells; j++)
        for (int i = 0; i < nxCells; i++)
            for (int k = 0; k < NUM_VARS; k++) u_con(IG(i), IG(j), k) = in[((size_t)j * nxCells + i) * NUM_VARS + k];
    return true;
}
