// Learned warm start: a small MLP (54 -> 64 -> 64 -> 64 -> 1, SiLU) on the
// Blackwell tensor cores, BF16 operands with FP32 accumulation in tensor memory.
//
// No counterpart in the reference: the reference starts every stage's Newton
// from the previous stage's pressure.  The network maps a cell's 3x3 stencil of
// (rho, rho u, rho v, alpha1, E*, P_prev) to a predicted pressure change; the
// solver evaluates the residual at the predicted pressure and keeps whichever
// of the two guesses gives the smaller residual norm, and Newton then converges
// to the same tolerance either way.
//
// Kernels (one CTA of 128 threads per SM, one sample per thread, tiles of 128
// samples = the MMA's M):
//   k_mlp_forward  inference: three M=128, N=64, K=64 GEMMs (X W1^T, H1 W2^T,
//                  H2 W3^T) with bias + SiLU between them, last layer a 64-term
//                  FP32 dot product per thread;
//   k_mlp_grad     one training pass over a batch: the same forward, then the
//                  backward GEMMs dH = dZ W (M=128, N=64, K=64) and the weight
//                  gradients dW^T... = dZ^T [H | 1] (M=128 of which 64 rows
//                  used, N=80 = 64 inputs + the bias column, K=128 samples)
//                  accumulated in tensor memory across every tile the CTA
//                  processes; one FP32 partial per CTA;
//   k_mlp_adam     folds the per-CTA partials in CTA order (deterministic) and
//                  applies Adam to the FP32 master weights.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/spb6g.h"
#include "spb6g_tc.cuh"

namespace spb6g {
namespace mlp {

using namespace tc;

constexpr int TILE = 128;  // samples per tile (MMA M)
constexpr int F = 64;      // padded input width and hidden width
constexpr int NB = 80;     // weight-gradient N: 64 inputs, the bias column, zero padding
// parameter offsets (FP32 master copy; W[n][k], n = output, k = input)
constexpr int OW1 = 0, OB1 = 4096, OW2 = 4160, OB2 = 8256, OW3 = 8320, OB3 = 12416, OW4 = 12480, OB4 = 12544;
constexpr int NPARAM = 12545;
constexpr int PSTRIDE = 12608;  // per-CTA partial record: gradients + loss at NPARAM
constexpr long long WAIT_CYCLES = 2000000000LL;  // about one second at 1.9 GHz

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float dsilu(float z) {
    const float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}
__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, float v) {
    *(__nv_bfloat16*)(base + off) = __float2bfloat16_rn(v);
}

// Weights into K-major BF16 operands (and optionally their transposes).
__device__ void load_weight(unsigned char* dst, const float* W, bool transpose) {
    for (int e = threadIdx.x; e < F * F; e += blockDim.x) {
        const int n = e / F, k = e % F;
        if (!transpose) st_bf16(dst, kmajor_off(n, k, F), W[e]);   // row n, column k
        else st_bf16(dst, kmajor_off(k, n, F), W[e]);              // row k, column n
    }
}

struct Sync {
    uint64_t* bar;
    uint32_t phase;
    bool ok;
    // all threads: wait for the last commit, then order TMEM reads after it; the
    // outcome is the same in every thread (a CTA-wide vote), so callers may branch on it
    __device__ bool wait() {
        const bool mine = mbar_wait(bar, phase, WAIT_CYCLES);
        phase ^= 1u;
        ok = !__syncthreads_or(!(ok && mine));
        fence_after();
        return ok;
    }
};
// Operands written by the threads become visible to the tensor cores, and every
// earlier TMEM read of the CTA is complete, before thread 0 issues more MMAs.
__device__ __forceinline__ void publish() {
    tmem_wait_ld();
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
}

// The dynamic shared memory follows the kernel's static shared variables, so its
// base is only 16-byte aligned whatever its declaration says: operands are laid
// out from the next 1024-byte boundary (1 KB of slack is requested), computed at
// run time so that no descriptor relies on an alignment the layout does not give.
__device__ __forceinline__ unsigned char* align_smem(unsigned char* raw) {
    return raw + ((1024u - (smem_u32(raw) & 1023u)) & 1023u);
}

// --------------------------------------------------------------------------- inference
constexpr size_t FWD_SMEM = 3 * 8192 + 2 * 16384 + 1024;

__global__ void __launch_bounds__(TILE, 1) k_mlp_forward(const float* __restrict__ P, const __nv_bfloat16* __restrict__ X, int n,
                                                          float* __restrict__ y, int* err) {
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* sm = align_smem(smraw);
    __shared__ uint64_t bar;
    __shared__ uint32_t tbase;
    __shared__ float bias[3 * F + F + 1];
    unsigned char* W1s = sm;
    unsigned char* W2s = sm + 8192;
    unsigned char* W3s = sm + 16384;
    unsigned char* Xs = sm + 24576;
    unsigned char* Hs = sm + 40960;
    const int t = threadIdx.x;
    load_weight(W1s, P + OW1, false);
    load_weight(W2s, P + OW2, false);
    load_weight(W3s, P + OW3, false);
    for (int e = t; e < F; e += TILE) {
        bias[e] = P[OB1 + e]; bias[F + e] = P[OB2 + e]; bias[2 * F + e] = P[OB3 + e]; bias[3 * F + e] = P[OW4 + e];
    }
    if (t == 0) { bias[4 * F] = P[OB4]; mbar_init(&bar, 1); }
    if (t < 32) tmem_alloc(&tbase, 256);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tb = tbase;
    Sync sy{&bar, 0u, true};
    const uint32_t id64 = idesc_bf16(TILE, F);
    const int ntiles = (n + TILE - 1) / TILE;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long row = (long)tile * TILE + t;
        const bool valid = row < n;
        {   // X row -> operand
            const uint4* src = (const uint4*)(X + row * F);
#pragma unroll
            for (int c = 0; c < F / 8; c++) {
                const uint4 v = valid ? src[c] : make_uint4(0, 0, 0, 0);
                *(uint4*)(Xs + kmajor_off(t, c * 8, F)) = v;
            }
        }
        publish();
        const unsigned char* Ain = Xs;
        float acc = 0.0f;
        for (int layer = 0; layer < 3; layer++) {
            const unsigned char* Wl = layer == 0 ? W1s : (layer == 1 ? W2s : W3s);
            if (t == 0) {
                mma_chain(tb + layer * F, smem_u32(Ain), F, smem_u32(Wl), F, F, id64, 0);
                mma_commit(&bar);
            }
            if (!sy.wait()) break;
            for (int c = 0; c < F; c += 16) {
                float z[16];
                tmem_ld16(tmem_lane_addr(tb, layer * F + c), z);
                tmem_wait_ld();
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const float h = silu(z[q] + bias[layer * F + c + q]);
                    if (layer < 2) st_bf16(Hs, kmajor_off(t, c + q, F), h);
                    else acc += bias[3 * F + c + q] * h;
                }
            }
            if (layer < 2) {
                publish();
                Ain = Hs;
            }
        }
        if (!sy.ok) { if (t == 0) atomicExch(err, 1); break; }
        if (valid) y[row] = acc + bias[4 * F];
        fence_before();
        __syncthreads();
        fence_after();
    }
    fence_before();
    __syncthreads();
    if (t < 32) tmem_free(tb, 256);
}

// --------------------------------------------------------------------------- training pass
// shared memory map (bytes)
constexpr int S_W1 = 0, S_W2 = 8192, S_W3 = 16384, S_W2T = 24576, S_W3T = 32768;
constexpr int S_X = 40960;            // 128 x 64   (layer-1 A)
constexpr int S_XT = S_X + 16384;     // 80 x 128   (dW1 B: features, ones row, zero rows)
constexpr int S_H1 = S_XT + 20480;    // 128 x 64
constexpr int S_H1T = S_H1 + 16384;   // 80 x 128
constexpr int S_H2 = S_H1T + 20480;   // 128 x 64
constexpr int S_H2T = S_H2 + 16384;   // 80 x 128
constexpr int S_DZ = S_H2T + 20480;   // 128 x 64   (dH A)
constexpr int S_DZT = S_DZ + 16384;   // 128 x 128  (dW A: rows n < 64, zero rows 64..127)
constexpr size_t GRAD_SMEM = S_DZT + 32768 + 1024;
// TMEM columns
constexpr int T_Z3 = 128, T_DH = 192,  // Z1, Z2 at 0, 64 (layer * F)
              T_DW1 = 256, T_DW2 = 336, T_DW3 = 416;

__global__ void __launch_bounds__(TILE, 1) k_mlp_grad(const float* __restrict__ P, const __nv_bfloat16* __restrict__ X,
                                                       const float* __restrict__ target, int n, float dscale,
                                                       float* __restrict__ part, int* err) {
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* sm = align_smem(smraw);
    __shared__ uint64_t bar;
    __shared__ uint32_t tbase;
    __shared__ float bias[3 * F + F + 1];
    __shared__ float w4acc[4][F + 1];  // per-warp partial of dL/dw4 (and dL/db4 at F)
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    load_weight(sm + S_W1, P + OW1, false);
    load_weight(sm + S_W2, P + OW2, false);
    load_weight(sm + S_W3, P + OW3, false);
    load_weight(sm + S_W2T, P + OW2, true);
    load_weight(sm + S_W3T, P + OW3, true);
    for (int e = t; e < F; e += TILE) {
        bias[e] = P[OB1 + e]; bias[F + e] = P[OB2 + e]; bias[2 * F + e] = P[OB3 + e]; bias[3 * F + e] = P[OW4 + e];
    }
    for (int e = t; e < 4 * (F + 1); e += TILE) (&w4acc[0][0])[e] = 0.0f;
    // constant parts: zero rows 64..79 of the transposed activations, zero rows 64..127 of dZ^T
    for (int e = t; e < 16 * TILE; e += TILE) {
        const int r = 64 + e / TILE, i = e % TILE;
        st_bf16(sm + S_XT, kmajor_off(r, i, TILE), 0.0f);
        st_bf16(sm + S_H1T, kmajor_off(r, i, TILE), 0.0f);
        st_bf16(sm + S_H2T, kmajor_off(r, i, TILE), 0.0f);
    }
    for (int e = t; e < 64 * TILE; e += TILE) st_bf16(sm + S_DZT, kmajor_off(64 + e / TILE, e % TILE, TILE), 0.0f);
    if (t == 0) { bias[4 * F] = P[OB4]; mbar_init(&bar, 1); }
    if (t < 32) tmem_alloc(&tbase, 512);
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tb = tbase;
    Sync sy{&bar, 0u, true};
    const uint32_t id64 = idesc_bf16(TILE, F), id80 = idesc_bf16(TILE, NB);
    const uint32_t aX = smem_u32(sm + S_X), aXT = smem_u32(sm + S_XT), aH1 = smem_u32(sm + S_H1), aH1T = smem_u32(sm + S_H1T);
    const uint32_t aH2 = smem_u32(sm + S_H2), aH2T = smem_u32(sm + S_H2T), aDZ = smem_u32(sm + S_DZ), aDZT = smem_u32(sm + S_DZT);
    const uint32_t aW1 = smem_u32(sm + S_W1), aW2 = smem_u32(sm + S_W2), aW3 = smem_u32(sm + S_W3);
    const uint32_t aW2T = smem_u32(sm + S_W2T), aW3T = smem_u32(sm + S_W3T);
    float loss = 0.0f;
    int first = 1;
    const int ntiles = (n + TILE - 1) / TILE;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long row = (long)tile * TILE + t;
        const bool valid = row < n;
        {
            const uint4* src = (const uint4*)(X + row * F);
#pragma unroll
            for (int c = 0; c < F / 8; c++) {
                const uint4 v = valid ? src[c] : make_uint4(0, 0, 0, 0);
                *(uint4*)(sm + S_X + kmajor_off(t, c * 8, F)) = v;
                const __nv_bfloat16* e = (const __nv_bfloat16*)&v;
#pragma unroll
                for (int q = 0; q < 8; q++) *(__nv_bfloat16*)(sm + S_XT + kmajor_off(c * 8 + q, t, TILE)) = e[q];
            }
            st_bf16(sm + S_XT, kmajor_off(64, t, TILE), valid ? 1.0f : 0.0f);
        }
        publish();
        // forward
        for (int layer = 0; layer < 3; layer++) {
            if (t == 0) {
                const uint32_t a = layer == 0 ? aX : (layer == 1 ? aH1 : aH2);
                const uint32_t w = layer == 0 ? aW1 : (layer == 1 ? aW2 : aW3);
                mma_chain(tb + layer * F, a, F, w, F, F, id64, 0);
                mma_commit(&bar);
            }
            if (!sy.wait() || layer == 2) break;
            unsigned char* Hn = sm + (layer == 0 ? S_H1 : S_H2);
            unsigned char* HnT = sm + (layer == 0 ? S_H1T : S_H2T);
            for (int c = 0; c < F; c += 16) {
                float z[16];
                tmem_ld16(tmem_lane_addr(tb, layer * F + c), z);
                tmem_wait_ld();
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const float h = valid ? silu(z[q] + bias[layer * F + c + q]) : 0.0f;
                    st_bf16(Hn, kmajor_off(t, c + q, F), h);
                    st_bf16(HnT, kmajor_off(c + q, t, TILE), h);
                }
            }
            st_bf16(HnT, kmajor_off(64, t, TILE), valid ? 1.0f : 0.0f);
            publish();
        }
        if (!sy.ok) break;
        // output layer, loss, dL/dw4, dL/db4, dZ3
        float yv = bias[4 * F];
        for (int c = 0; c < F; c += 16) {
            float z[16];
            tmem_ld16(tmem_lane_addr(tb, T_Z3 + c), z);
            tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) yv += bias[3 * F + c + q] * silu(z[q] + bias[2 * F + c + q]);
        }
        const float r = valid ? yv - target[row] : 0.0f;
        loss += r * r;
        const float dy = 2.0f * r * dscale;
        for (int c = 0; c < F; c += 16) {
            float z[16];
            tmem_ld16(tmem_lane_addr(tb, T_Z3 + c), z);
            tmem_wait_ld();
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const float zz = z[q] + bias[2 * F + c + q];
                float g = dy * silu(zz);  // dL/dw4 term
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
                if (lane == 0) w4acc[warp][c + q] += g;
                const float dz = dy * bias[3 * F + c + q] * dsilu(zz);
                st_bf16(sm + S_DZ, kmajor_off(t, c + q, F), dz);
                st_bf16(sm + S_DZT, kmajor_off(c + q, t, TILE), dz);
            }
        }
        {
            float g = dy;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
            if (lane == 0) w4acc[warp][F] += g;
        }
        publish();
        // dW3 += dZ3^T [H2 | 1];  dH2 = dZ3 W3
        if (t == 0) {
            mma_chain(tb + T_DW3, aDZT, TILE, aH2T, TILE, TILE, id80, !first);
            mma_chain(tb + T_DH, aDZ, F, aW3T, F, F, id64, 0);
            mma_commit(&bar);
        }
        if (!sy.wait()) break;
        for (int layer = 1; layer >= 0; layer--) {
            // dZ_l = dH_l * silu'(Z_l)
            for (int c = 0; c < F; c += 16) {
                float dh[16], z[16];
                tmem_ld16(tmem_lane_addr(tb, T_DH + c), dh);
                tmem_ld16(tmem_lane_addr(tb, layer * F + c), z);
                tmem_wait_ld();
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const float dz = valid ? dh[q] * dsilu(z[q] + bias[layer * F + c + q]) : 0.0f;
                    if (layer == 1) st_bf16(sm + S_DZ, kmajor_off(t, c + q, F), dz);
                    st_bf16(sm + S_DZT, kmajor_off(c + q, t, TILE), dz);
                }
            }
            publish();
            if (t == 0) {
                if (layer == 1) {  // dW2 += dZ2^T [H1 | 1];  dH1 = dZ2 W2
                    mma_chain(tb + T_DW2, aDZT, TILE, aH1T, TILE, TILE, id80, !first);
                    mma_chain(tb + T_DH, aDZ, F, aW2T, F, F, id64, 0);
                } else {           // dW1 += dZ1^T [X | 1]
                    mma_chain(tb + T_DW1, aDZT, TILE, aXT, TILE, TILE, id80, !first);
                }
                mma_commit(&bar);
            }
            if (!sy.wait()) break;
        }
        if (!sy.ok) break;
        first = 0;
    }
    const bool ok = sy.ok;
    if (!ok && t == 0) atomicExch(err, 1);
    // per-CTA partial: rows n < 64 of the dW accumulators (column 64 = bias gradient)
    float* out = part + (size_t)blockIdx.x * PSTRIDE;
    if (t < F) {
        const int offs[3][2] = {{OW1, OB1}, {OW2, OB2}, {OW3, OB3}};
        const int cols[3] = {T_DW1, T_DW2, T_DW3};
        for (int l = 0; l < 3; l++) {
            for (int c = 0; c < NB; c += 16) {
                float v[16];
                if (!first && ok) {
                    tmem_ld16(tmem_lane_addr(tb, cols[l] + c), v);
                    tmem_wait_ld();
                } else {
#pragma unroll
                    for (int q = 0; q < 16; q++) v[q] = 0.0f;
                }
#pragma unroll
                for (int q = 0; q < 16; q++) {
                    const int k = c + q;
                    if (k < F) out[offs[l][0] + t * F + k] = v[q];
                    else if (k == F) out[offs[l][1] + t] = v[q];
                }
            }
        }
    }
    __syncthreads();
    if (t <= F) out[(t < F ? OW4 + t : OB4)] = w4acc[0][t] + w4acc[1][t] + w4acc[2][t] + w4acc[3][t];
    {
        __shared__ float ls[4];
        float l = loss;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
        if (lane == 0) ls[warp] = l;
        __syncthreads();
        if (t == 0) out[NPARAM] = ls[0] + ls[1] + ls[2] + ls[3];
    }
    fence_before();
    __syncthreads();
    if (t < 32) tmem_free(tb, 512);
}

// Folds the CTA partials in CTA order; optionally applies Adam (step >= 1).
__global__ void k_mlp_adam(const float* __restrict__ part, int G, float* __restrict__ grad, float* __restrict__ P,
                           float* __restrict__ m, float* __restrict__ v, long step, float lr, float b1, float b2, float eps,
                           float* loss) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e <= NPARAM; e += gridDim.x * blockDim.x) {
        float g = 0.0f;
        for (int b = 0; b < G; b++) g += part[(size_t)b * PSTRIDE + e];
        if (e == NPARAM) { *loss = g; continue; }
        grad[e] = g;
        if (step < 1) continue;
        const float mm = b1 * m[e] + (1.0f - b1) * g, vv = b2 * v[e] + (1.0f - b2) * g * g;
        m[e] = mm;
        v[e] = vv;
        const float mh = mm / (1.0f - powf(b1, (float)step)), vh = vv / (1.0f - powf(b2, (float)step));
        P[e] -= lr * mh / (sqrtf(vh) + eps);
    }
}

}  // namespace mlp
}  // namespace spb6g

using namespace spb6g::mlp;

struct spb6g_mlp {
    int device = 0;
    int G = 0;
    long step = 0;
    cudaStream_t st = nullptr;
    float *P = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *part = nullptr, *loss = nullptr;
    int* err = nullptr;
};

namespace {
int mlp_prepare(int device) {
    static std::mutex mu;
    static unsigned done = 0;
    std::lock_guard<std::mutex> lk(mu);
    if (device < 32 && (done >> device) & 1u) return 0;
    if (cudaFuncSetAttribute(k_mlp_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GRAD_SMEM) != cudaSuccess)
        return -1;
    if (device < 32) done |= 1u << device;
    return 0;
}
int mlp_check(spb6g_mlp* h) {
    int e = 0;
    if (cudaMemcpyAsync(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (cudaStreamSynchronize(h->st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (e) {
        fprintf(stderr, "spb6g_mlp: a tensor-core wait timed out\n");
        cudaMemsetAsync(h->err, 0, sizeof(int), h->st);
        return SPB6G_CUDA_ERROR;
    }
    return SPB6G_OK;
}
}  // namespace

extern "C" {

int spb6g_mlp_create(int device, spb6g_mlp** out) {
    if (!out) return SPB6G_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) return SPB6G_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return SPB6G_NO_DEVICE;
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) return SPB6G_UNSUPPORTED;
    if (mlp_prepare(device)) return SPB6G_CUDA_ERROR;
    spb6g_mlp* h = new spb6g_mlp();
    h->device = device;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    h->G = sms > 0 ? sms : 148;
    bool ok = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) == cudaSuccess;
    ok = ok && cudaMalloc(&h->P, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->m, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->v, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->grad, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->part, (size_t)h->G * PSTRIDE * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->loss, sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->err, sizeof(int)) == cudaSuccess;
    if (ok) {
        cudaMemsetAsync(h->P, 0, NPARAM * sizeof(float), h->st);
        cudaMemsetAsync(h->m, 0, NPARAM * sizeof(float), h->st);
        cudaMemsetAsync(h->v, 0, NPARAM * sizeof(float), h->st);
        cudaMemsetAsync(h->err, 0, sizeof(int), h->st);
        ok = cudaStreamSynchronize(h->st) == cudaSuccess;
    }
    if (!ok) { spb6g_mlp_destroy(h); return SPB6G_CUDA_ERROR; }
    *out = h;
    return SPB6G_OK;
}

void spb6g_mlp_destroy(spb6g_mlp* h) {
    if (!h) return;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    for (void* p : {(void*)h->P, (void*)h->m, (void*)h->v, (void*)h->grad, (void*)h->part, (void*)h->loss, (void*)h->err})
        if (p) cudaFree(p);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
}

int spb6g_mlp_param_count(void) { return NPARAM; }

int spb6g_mlp_set_params(spb6g_mlp* h, const float* params) {
    if (!h || !params) return SPB6G_BAD_ARG;
    cudaSetDevice(h->device);
    if (cudaMemcpyAsync(h->P, params, NPARAM * sizeof(float), cudaMemcpyHostToDevice, h->st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    cudaMemsetAsync(h->m, 0, NPARAM * sizeof(float), h->st);
    cudaMemsetAsync(h->v, 0, NPARAM * sizeof(float), h->st);
    h->step = 0;
    return cudaStreamSynchronize(h->st) == cudaSuccess ? SPB6G_OK : SPB6G_CUDA_ERROR;
}

int spb6g_mlp_get_params(spb6g_mlp* h, float* params) {
    if (!h || !params) return SPB6G_BAD_ARG;
    cudaSetDevice(h->device);
    if (cudaMemcpyAsync(params, h->P, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, h->st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    return cudaStreamSynchronize(h->st) == cudaSuccess ? SPB6G_OK : SPB6G_CUDA_ERROR;
}

int spb6g_mlp_forward(spb6g_mlp* h, const void* X_dev, int n, float* y_dev, void* stream) {
    if (!h || !X_dev || !y_dev || n < 0) return SPB6G_BAD_ARG;
    if (n == 0) return SPB6G_OK;
    cudaSetDevice(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->st;
    const int ntiles = (n + TILE - 1) / TILE;
    k_mlp_forward<<<ntiles < h->G ? ntiles : h->G, TILE, FWD_SMEM, st>>>(h->P, (const __nv_bfloat16*)X_dev, n, y_dev, h->err);
    if (cudaGetLastError() != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (stream) return SPB6G_OK;
    return mlp_check(h);
}

// One pass over the batch: gradient of mean((y - target)^2); with lr > 0 also an Adam step.
int spb6g_mlp_train_step(spb6g_mlp* h, const void* X_dev, const float* target_dev, int n, float lr, float* loss_out,
                         float* grad_host) {
    if (!h || !X_dev || !target_dev || n <= 0) return SPB6G_BAD_ARG;
    cudaSetDevice(h->device);
    const int ntiles = (n + TILE - 1) / TILE;
    const int G = ntiles < h->G ? ntiles : h->G;
    k_mlp_grad<<<G, TILE, GRAD_SMEM, h->st>>>(h->P, (const __nv_bfloat16*)X_dev, target_dev, n, 1.0f / (float)n, h->part, h->err);
    if (cudaGetLastError() != cudaSuccess) return SPB6G_CUDA_ERROR;
    const long step = lr > 0 ? ++h->step : 0;
    k_mlp_adam<<<(NPARAM + 256) / 256, 256, 0, h->st>>>(h->part, G, h->grad, h->P, h->m, h->v, step, lr, 0.9f, 0.999f, 1e-8f,
                                                         h->loss);
    if (cudaGetLastError() != cudaSuccess) return SPB6G_CUDA_ERROR;
    float l = 0;
    if (cudaMemcpyAsync(&l, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (grad_host && cudaMemcpyAsync(grad_host, h->grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, h->st) != cudaSuccess)
        return SPB6G_CUDA_ERROR;
    const int rc = mlp_check(h);
    if (loss_out) *loss_out = l / (float)n;
    return rc;
}

}  // extern "C"
