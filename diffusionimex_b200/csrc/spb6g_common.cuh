// Grid geometry, virtual ghost cells and deterministic reductions.
//
// Device arrays hold interior cells only, one FP64 array per variable (SoA),
// cell (i, j) at i + j * nx.  The reference keeps two ghost layers in every
// grid and refills them with bc_apply / bound_cond_array
// (src/spb6_physics_omp.h:982-1013, src/SPB6_PC_IMEX_omp.cpp:516-537) after
// each update; here a ghost read is an index map plus the same transform
// (mirror / wrap / clamp, wall momentum reversal, piston and pressure-outlet
// energies), applied x first and y second exactly as the reference's two
// passes compose at the corners.  The pressure unknown uses the reference's
// M_P map (:709-718): clamp for every non-periodic side.
#pragma once
#include "spb6g_physics.cuh"

namespace spb6g {

struct Geom {
    int nx, ny;
    int bcs[4];  // left, right, bottom, top (BC_TRANS / BC_WALL / BC_PERIODIC / BC_PRES)
    double bcu[4], bcp[4];
    double dx, dy;
};

// Conservative state, SoA.
struct State {
    double* v[NV];
};
struct CState {
    const double* v[NV];
};

SPB6G_DEV bool one_d(const Geom& g) { return g.ny == 1 && g.bcs[2] != BC_PERIODIC; }

// Source column of a (possibly ghost) column i for state/array fills; side = 0/1 when i is a ghost.
SPB6G_DEV int src_x(const Geom& g, int i, int& side) {
    side = -1;
    if (i < 0) {
        side = 0;
        const int b = g.bcs[0];
        return b == BC_PERIODIC ? g.nx + i : (b == BC_WALL ? -1 - i : 0);
    }
    if (i >= g.nx) {
        side = 1;
        const int b = g.bcs[1];
        return b == BC_PERIODIC ? i - g.nx : (b == BC_WALL ? 2 * g.nx - 1 - i : g.nx - 1);
    }
    return i;
}
SPB6G_DEV int src_y(const Geom& g, int j, int& side) {
    side = -1;
    if (one_d(g)) return 0;  // 1D: y ghosts are plain copies (bc_apply :1008-1012)
    if (j < 0) {
        side = 2;
        const int b = g.bcs[2];
        return b == BC_PERIODIC ? g.ny + j : (b == BC_WALL ? -1 - j : 0);
    }
    if (j >= g.ny) {
        side = 3;
        const int b = g.bcs[3];
        return b == BC_PERIODIC ? j - g.ny : (b == BC_WALL ? 2 * g.ny - 1 - j : g.ny - 1);
    }
    return j;
}
// Ghost transform of ghost_fill (bc_apply's lambda, physics :983-992) on a copied cell.
SPB6G_DEV void ghost_transform(const Phys& P, const Geom& g, int side, double* d) {
    const int b = g.bcs[side];
    if (b == BC_PRES) {
        const double a1 = d[IA1], e1 = eps_amp(P, 0, a1, d[IM1], g.bcp[side]), e2 = eps_amp(P, 1, 1 - a1, d[IM2], g.bcp[side]);
        d[IEN] += (e1 + e2) - (d[IE1] + d[IE2]);
        d[IE1] = e1;
        d[IE2] = e2;
        return;
    }
    if (b != BC_WALL) return;
    const int kn = side < 2 ? IMU : IMV;
    const double rho = d[IM1] + d[IM2];
    if (g.bcu[side] == 0.0) { d[kn] = -d[kn]; return; }
    const double s = d[kn];
    const double mn = 2.0 * rho * g.bcu[side] - s;
    d[IEN] += 0.5 * (mn * mn - s * s) / rho;
    d[kn] = mn;
}
// Full 8-variable state at (i, j), i in [-2, nx+1], j in [-2, ny+1].
SPB6G_DEV void load_state(const Phys& P, const Geom& g, const CState& U, int i, int j, double* q) {
    int sx, sy;
    const int si = src_x(g, i, sx), sj = src_y(g, j, sy);
    const size_t c = (size_t)si + (size_t)sj * g.nx;
#pragma unroll
    for (int k = 0; k < NV; k++) q[k] = U.v[k][c];
    if (sx >= 0) ghost_transform(P, g, sx, q);
    if (sy >= 0) ghost_transform(P, g, sy, q);
}
// Array with ghosts filled by bound_cond_array(a, 1, 1): the mapped copy.
SPB6G_DEV double load_arr(const Geom& g, const double* a, int i, int j) {
    int sx, sy;
    const int si = src_x(g, i, sx), sj = src_y(g, j, sy);
    return a[(size_t)si + (size_t)sj * g.nx];
}
// Pressure-unknown index M_P (SPB6_PC_IMEX_omp.cpp:709-718), interior coordinates.
SPB6G_DEV int mp_index(const Geom& g, int i, int j) {
    int I, J;
    const bool xp = g.bcs[0] == BC_PERIODIC, yp = g.bcs[2] == BC_PERIODIC && g.ny > 1;
    if (i < 0) I = xp ? g.nx + i : 0;
    else if (i > g.nx - 1) I = xp ? i - g.nx : g.nx - 1;
    else I = i;
    if (j < 0) J = yp ? g.ny + j : 0;
    else if (j > g.ny - 1) J = yp ? j - g.ny : g.ny - 1;
    else J = j;
    return I + g.nx * J;
}

// ------------------------------------------------------------ reductions
// Every reduction is deterministic: each thread folds its grid-stride
// elements in index order, blocks fold warps in a fixed tree, and the last
// block to finish folds the per-block partials in block order.
constexpr int RED_THREADS = 256;
constexpr int MAXQ = 8;

struct RedSum {
    SPB6G_DEV static double id() { return 0.0; }
    SPB6G_DEV static double op(double a, double b) { return a + b; }
};
// max of non-negative finite values; NaN/inf-free by construction at the call sites
struct RedMax {
    SPB6G_DEV static double id() { return 0.0; }
    SPB6G_DEV static double op(double a, double b) { return SMAX(a, b); }
};
struct RedMin {
    SPB6G_DEV static double id() { return INFINITY; }
    SPB6G_DEV static double op(double a, double b) { return SMIN(a, b); }
};

template <class R>
SPB6G_DEV double warp_fold(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = R::op(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Folds NQ values over the block; result valid in thread 0.
template <class R, int NQ>
SPB6G_DEV void block_fold(double (&v)[NQ], double* sh /* [NQ][32] */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
        double x = warp_fold<R>(v[q]);
        if (lane == 0) sh[q * 32 + wid] = x;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NQ; q++) {
            double x = lane < nw ? sh[q * 32 + lane] : R::id();
            v[q] = warp_fold<R>(x);
        }
    }
    __syncthreads();
}

// Writes this block's partials; returns true in every thread of the last block,
// which then holds the folded totals in `tot` (valid in thread 0).
template <class R, int NQ>
SPB6G_DEV bool grid_fold(double (&v)[NQ], double* partials, unsigned* counter, double (&tot)[NQ]) {
    __shared__ double sh[NQ * 32];
    __shared__ bool last;
    const unsigned nblocks = gridDim.x * gridDim.y, bid = blockIdx.x + blockIdx.y * gridDim.x;
    block_fold<R, NQ>(v, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; q++) partials[(size_t)bid * NQ + q] = v[q];
        __threadfence();
        const unsigned t = atomicAdd(counter, 1u);
        last = (t == nblocks - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double acc[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) acc[q] = R::id();
    for (unsigned b = threadIdx.x; b < nblocks; b += blockDim.x) {
#pragma unroll
        for (int q = 0; q < NQ; q++) acc[q] = R::op(acc[q], __ldcg(partials + (size_t)b * NQ + q));
    }
    block_fold<R, NQ>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < NQ; q++) tot[q] = acc[q];
        *counter = 0u;
    }
    return true;
}

}  // namespace spb6g
