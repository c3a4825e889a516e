// Allocation-free time-step rate (caldt) on caller-owned device buffers.
//
// Some callers cannot let a library call cudaMalloc: a host framework that owns
// every device byte through its own arena or pool, a time-critical loop that
// cannot afford the device-wide synchronisation cudaMalloc / cudaFree may cause,
// or a long-running service whose device footprint must not grow after start-up.  For them this entry point takes
// the state as device pointers the caller already owns and keeps its only
// scratch -- one partial (max |u| + c, max |v| + c) per block, a block counter
// and the two results -- in file-scope __device__ arrays that every GPU loading
// the library holds until the process exits.
//
// Limits and rules:
//   * at most SPB6G_NOALLOC_MAX_CELLS interior cells (one cell per thread,
//     one partial per 256-thread block); larger grids are rejected with
//     SPB6G_TOO_LARGE before any device work;
//   * it runs on cfg->device (made current for the call, the caller's current
//     device restored on return); every U_dev[k] must be device (or managed)
//     memory of that device, checked with cudaPointerGetAttributes before any
//     launch (SPB6G_BAD_ARG otherwise), and `stream` must belong to it;
//   * the first call on a device looks up the device addresses of the scratch
//     arrays (cudaGetSymbolAddress, with that device current);
//   * every call is blocking: it copies the result to the host and waits for
//     `stream`, so no call -- the first or any later one -- may be made while a
//     stream is being captured into a CUDA graph;
//   * every call shares the scratch: the block counter is cleared at the start
//     of each call, and two calls whose work overlaps on the GPU (different
//     streams, or host threads, at the same time) race on it.
#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/spb6g.h"
#include "spb6g_common.cuh"
#include "spb6g_ctx.cuh"

using namespace spb6g;

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_MAX_BLOCKS = SPB6G_NOALLOC_MAX_CELLS / NOALLOC_THREADS;

static __device__ __align__(256) double g_na_partials[NOALLOC_MAX_BLOCKS * 2];
static __device__ __align__(256) unsigned g_na_counter[64];
static __device__ __align__(256) double g_na_result[2];

// Device addresses of the scratch arrays for each device, looked up on first use.
struct NoallocSymbols {
    bool ready = false;
    double* partials = nullptr;
    unsigned* counter = nullptr;
    double* result = nullptr;
};
NoallocSymbols g_syms[64];
std::mutex g_syms_mutex;

// One cell per thread: the maxima of caldt (:502-514) over admissible cells.
__global__ void __launch_bounds__(NOALLOC_THREADS) k_caldt_noalloc(Phys P, int n, CState U, int acoustic,
                                                                   double* partials, unsigned* counter, double* result) {
    double m[2] = {0.0, 0.0};
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) {
        double q[NV];
#pragma unroll
        for (int k = 0; k < NV; k++) q[k] = U.v[k][x];
        Prim w;
        if (prim_of(P, q, w)) {
            const double cs = acoustic ? w.cf : 0.0;
            m[0] = SMAX(0.0, fabs(w.u) + cs);
            m[1] = SMAX(0.0, fabs(w.v) + cs);
        }
    }
    double tot[2];
    if (grid_fold<RedMax, 2>(m, partials, counter, tot) && threadIdx.x == 0) {
        result[0] = tot[0];
        result[1] = tot[1];
    }
}

// Makes `dev` current for the call and puts the caller's device back on every return.
struct DeviceScope {
    int prev = -1;
    bool set(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) return false;
        return prev == dev || cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceScope() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

// True when p is device (or managed) memory of device `dev`.
bool on_device(const void* p, int dev) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

}  // namespace

extern "C" int spb6g_caldt_noalloc(const spb6g_config* cfg, const double* const* U_dev, int acoustic, void* stream,
                                   double* inv_rate) {
    if (!cfg || !U_dev || !inv_rate || cfg->nx < 1 || cfg->ny < 1) return SPB6G_BAD_ARG;
    // the geometry checks of spb6g_create: a degenerate domain has no finite rate
    if (!(cfg->x1 > cfg->x0) || !(cfg->y1 > cfg->y0) || cfg->device < 0) return SPB6G_BAD_ARG;
    for (int k = 0; k < 2; k++)
        if (cfg->kind[k] < 0 || cfg->kind[k] > 2) return SPB6G_BAD_ARG;
    if (cfg->kind[0] != 0 || cfg->kind[1] != 0) return SPB6G_UNSUPPORTED;  // stiffened gas / NASG phases only
    for (int k = 0; k < NV; k++)
        if (!U_dev[k]) return SPB6G_BAD_ARG;
    const long long n = (long long)cfg->nx * cfg->ny;
    if (n > SPB6G_NOALLOC_MAX_CELLS) {
        fprintf(stderr, "spb6g_caldt_noalloc: %lld cells exceed the fixed scratch of %d cells\n", n,
                (int)SPB6G_NOALLOC_MAX_CELLS);
        return SPB6G_TOO_LARGE;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device >= ndev || cfg->device >= 64) {
        cudaGetLastError();
        return SPB6G_NO_DEVICE;
    }
    const int dev = cfg->device;
    DeviceScope scope;
    if (!scope.set(dev)) return SPB6G_NO_DEVICE;
    for (int k = 0; k < NV; k++)
        if (!on_device(U_dev[k], dev)) return SPB6G_BAD_ARG;
    {
        std::lock_guard<std::mutex> lock(g_syms_mutex);
        NoallocSymbols& sy = g_syms[dev];
        if (!sy.ready) {
            if (cudaGetSymbolAddress((void**)&sy.partials, g_na_partials) != cudaSuccess ||
                cudaGetSymbolAddress((void**)&sy.counter, g_na_counter) != cudaSuccess ||
                cudaGetSymbolAddress((void**)&sy.result, g_na_result) != cudaSuccess) {
                cudaGetLastError();
                return SPB6G_CUDA_ERROR;
            }
            sy.ready = true;
        }
    }
    const NoallocSymbols& sy = g_syms[dev];
    cudaStream_t st = (cudaStream_t)stream;
    Phys P;
    phys_from_config(cfg, P);
    CState U;
    for (int k = 0; k < NV; k++) U.v[k] = U_dev[k];
    double host[2];
    const int blocks = (int)((n + NOALLOC_THREADS - 1) / NOALLOC_THREADS);
    if (cudaMemsetAsync(sy.counter, 0, sizeof(unsigned), st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    k_caldt_noalloc<<<blocks, NOALLOC_THREADS, 0, st>>>(P, (int)n, U, acoustic ? 1 : 0, sy.partials, sy.counter, sy.result);
    if (cudaGetLastError() != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (cudaMemcpyAsync(host, sy.result, sizeof host, cudaMemcpyDeviceToHost, st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    const double dx = (cfg->x1 - cfg->x0) / cfg->nx, dy = (cfg->y1 - cfg->y0) / cfg->ny;
    const double rate = host[0] / dx + (cfg->ny > 1 ? host[1] / dy : 0.0);
    *inv_rate = rate > 0 ? 1.0 / rate : INFINITY;
    return SPB6G_OK;
}
