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
// Kernels (tiles of 128 samples = the MMA's M; sample i of a tile in TMEM lane i):
//   k_mlp_forward  inference: three M=128, N=64, K=64 GEMMs (X W1^T, H1 W2^T,
//                  H2 W3^T) with bias + SiLU between them, last layer a 64-term
//                  FP32 dot product per sample;
//   k_mlp_grad     one training pass over a batch: the same forward, then the
//                  backward GEMMs dH = dZ W (M=128, N=64, K=64) and the weight
//                  gradients dW^T = [H | 1]^T dZ (M=128: the 64 inputs, the bias
//                  row and zero rows; N=64; K=128 samples) accumulated in tensor
//                  memory across every tile the CTA processes; one FP32 partial
//                  per CTA;
//   k_mlp_adam     folds the per-CTA partials in CTA order (deterministic),
//                  applies Adam to the FP32 master weights and rewrites their
//                  BF16 operand images.
//
// Every operand is a BF16 tile with 128-byte rows (64 values) in the 128-byte
// swizzled layout: the feature rows arrive by TMA straight into it, the
// epilogues write 16-byte vectors into it, and the transposed operands of the
// backward GEMMs are the same tiles read through MN-major descriptors, so no
// transposed copy is ever written.  Feature tiles are double-buffered (the TMA
// load of a later tile runs while the current one is computed), and the CTA's
// warpgroups split the 64 columns of every epilogue between them.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/spb6g.h"
#include "spb6g_tc.cuh"

namespace spb6g {
namespace mlp {

using namespace tc;

constexpr int TILE = 128;         // samples per tile (MMA M)
constexpr int F = 64;             // padded input width and hidden width
constexpr uint32_t TB = 16384;    // bytes of a 128 x 64 BF16 tile
constexpr uint32_t WB = 8192;     // bytes of a 64 x 64 BF16 weight image
// parameter offsets (FP32 master copy; W[n][k], n = output, k = input)
constexpr int OW1 = 0, OB1 = 4096, OW2 = 4160, OB2 = 8256, OW3 = 8320, OB3 = 12416, OW4 = 12480, OB4 = 12544;
constexpr int NPARAM = 12545;
constexpr int PSTRIDE = 12608;  // per-CTA partial record: gradients + loss at NPARAM
constexpr int LSTRIDE = OW2 - OW1;  // distance between the hidden layers' parameter blocks
static_assert(OB1 == OW1 + F * F && OB2 == OB1 + LSTRIDE && OW3 == OW2 + LSTRIDE && OB3 == OB2 + LSTRIDE && OW4 == OB3 + F &&
                  OB4 == OW4 + F && NPARAM == OB4 + 1 && PSTRIDE > NPARAM,
              "parameter layout");
constexpr long long WAIT_CYCLES = 2000000000LL;  // about one second at 1.9 GHz

// SiLU(z) = z s(z) with the logistic function s(z) = 1 / (1 + e^-z) = 1 / (1 + 2^(-z log2 e)),
// evaluated with the approximate base-2 exponential and reciprocal instructions (one
// special-function operation each); SiLU'(z) = s (1 + z (1 - s)).
constexpr float NEG_LOG2E = -1.44269504088896340736f;
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float logistic(float z) { return rcp_approx(1.0f + ex2_approx(z * NEG_LOG2E)); }
__device__ __forceinline__ float dsilu(float z, float s) { return s * __fmaf_rn(z, 1.0f - s, 1.0f); }
__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *(const uint32_t*)&v;
}

// All threads: a CTA-wide vote, so that every thread takes the same branch after a
// bounded wait (one thread's timeout stops the whole CTA).
__device__ __forceinline__ bool vote_ok(bool mine) { return !__syncthreads_or(!mine); }

// Operands written by the threads become visible to the tensor cores, and every
// earlier TMEM read of the CTA is complete, before thread 0 issues more MMAs.
__device__ __forceinline__ void publish() {
    tmem_wait_ld();
    tmem_wait_st();
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

// CW columns of this thread's TMEM lane starting at column `col` (CW a multiple of 16).
template <int CW>
__device__ __forceinline__ void tmem_load(uint32_t tb, int col, float* v) {
#pragma unroll
    for (int c = 0; c < CW; c += 16) tmem_ld16(tmem_lane_addr(tb, col + c), v + c);
}

// Hidden-layer epilogue for CW columns from c0 of sample `row`: zz = z + bias, h = SiLU(zz)
// as BF16 into `tile` (16-byte stores); with DERIV also SiLU'(zz) into d.
template <int CW, bool DERIV>
__device__ __forceinline__ void hidden_epilogue(unsigned char* tile, int row, int c0, const float* z, const float* bias,
                                                float* d) {
#pragma unroll
    for (int c = 0; c < CW; c += 8) {
        const float4 ba = *(const float4*)(bias + c0 + c), bb = *(const float4*)(bias + c0 + c + 4);
        const float b8[8] = {ba.x, ba.y, ba.z, ba.w, bb.x, bb.y, bb.z, bb.w};
        float h[8];
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const float zz = z[c + q] + b8[q], sg = logistic(zz);
            h[q] = zz * sg;
            if (DERIV) d[c + q] = dsilu(zz, sg);
        }
        *(uint4*)(tile + sw128_off(row, c0 + c)) =
            make_uint4(pack_bf16(h[0], h[1]), pack_bf16(h[2], h[3]), pack_bf16(h[4], h[5]), pack_bf16(h[6], h[7]));
    }
}
// CW columns from this thread's registers into its TMEM lane (CW a multiple of 16).
template <int CW>
__device__ __forceinline__ void tmem_store(uint32_t tb, int col, const float* v) {
#pragma unroll
    for (int c = 0; c < CW; c += 16) tmem_st16(tmem_lane_addr(tb, col + c), v + c);
}

// The three hidden layers' weights as BF16 operand images into shared memory, the
// biases (and w4, b4) as FP32.
__device__ __forceinline__ void load_params(unsigned char* wdst, const uint4* __restrict__ Wimg, const float* __restrict__ P,
                                            float* bias) {
    for (int e = threadIdx.x; e < (int)(3 * WB / 16); e += blockDim.x) ((uint4*)wdst)[e] = Wimg[e];
    for (int e = threadIdx.x; e < 4 * F; e += blockDim.x) {
        const int l = e / F, j = e % F;
        bias[e] = l < 3 ? P[OB1 + l * LSTRIDE + j] : P[OW4 + j];
    }
    if (threadIdx.x == 0) bias[4 * F] = P[OB4];
}

// --------------------------------------------------------------------------- inference
constexpr uint32_t F_W = 0, F_X = 3 * WB, F_H = F_X + TB, F_END = F_H + TB;
constexpr size_t FWD_SMEM = F_END + 1024;
constexpr int FWD_NWG = 2;   // warpgroups per CTA
constexpr int FWD_CTAS = 3;  // resident CTAs per SM (each with its own tile chain)

template <int NWG>
__global__ void __launch_bounds__(128 * NWG, FWD_CTAS) k_mlp_forward(const __grid_constant__ CUtensorMap xmap,
                                                                      const float* __restrict__ P, const uint4* __restrict__ Wimg,
                                                                      int n, float* __restrict__ y, int* err) {
    constexpr int CW = F / NWG;
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* sm = align_smem(smraw);
    __shared__ uint64_t barx, barm;
    __shared__ uint32_t tbase;
    __shared__ __align__(16) float bias[4 * F + 4];
    __shared__ float ypart[NWG][TILE];
    const int t = threadIdx.x, row = t & (TILE - 1), g = t >> 7, c0 = g * CW;
    const int ntiles = (n + TILE - 1) / TILE;
    if (t == 0) {
        mbar_init(&barx, 1);
        mbar_init(&barm, 1);
        tma_prefetch_map(&xmap);
    }
    load_params(sm + F_W, Wimg, P, bias);
    if (t < 32) tmem_alloc(&tbase, 64);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    int issued = 0, used = 0;  // TMA loads of feature tiles (thread 0's count)
    if (t == 0 && (int)blockIdx.x < ntiles) {
        mbar_expect_tx(&barx, TB);
        tma_load_2d(sm + F_X, &xmap, 0, blockIdx.x * TILE, &barx);
        issued++;
    }
    const uint32_t tb = tbase, id = idesc_bf16(TILE, F);
    const uint32_t xa = smem_u32(sm + F_X), ha = smem_u32(sm + F_H);
    uint32_t pm = 0;
    bool ok = true;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        ok = vote_ok(mbar_wait(&barx, (uint32_t)it & 1u, WAIT_CYCLES));
        if (!ok) break;
        used++;
        float yp = 0.0f;
        for (int l = 0; l < 3; l++) {
            if (t == 0) {
                const uint32_t a = l == 0 ? xa : ha, w = smem_u32(sm + F_W + l * WB);
#pragma unroll
                for (int s = 0; s < F / 16; s++) mma_bf16(tb, desc_sw128_k(a, s), desc_sw128_k(w, s), id, s > 0);
                mma_commit(&barm);
            }
            ok = vote_ok(mbar_wait(&barm, pm, WAIT_CYCLES));
            pm ^= 1u;
            fence_after();
            if (!ok) break;
            if (l == 0 && t == 0) {  // the feature tile has been consumed: load the next one into it
                const int next = tile + gridDim.x;
                if (next < ntiles) {
                    mbar_expect_tx(&barx, TB);
                    tma_load_2d(sm + F_X, &xmap, 0, next * TILE, &barx);
                    issued++;
                }
            }
            float z[CW];
            tmem_load<CW>(tb, c0, z);
            tmem_wait_ld();
            if (l < 2) {
                hidden_epilogue<CW, false>(sm + F_H, row, c0, z, bias + l * F, nullptr);
                publish();
            } else {
#pragma unroll
                for (int c = 0; c < CW; c += 4) {
                    const float4 b = *(const float4*)(bias + 2 * F + c0 + c), w = *(const float4*)(bias + 3 * F + c0 + c);
                    const float zz[4] = {z[c] + b.x, z[c + 1] + b.y, z[c + 2] + b.z, z[c + 3] + b.w};
                    const float w4[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                    for (int q = 0; q < 4; q++) yp = __fmaf_rn(w4[q], zz[q] * logistic(zz[q]), yp);
                }
            }
        }
        if (!ok) break;
        ypart[g][row] = yp;
        fence_before();
        __syncthreads();  // TMEM reads done before the next tile's MMA; partial sums visible
        fence_after();
        if (g == 0) {
            const long r = (long)tile * TILE + row;
            if (r < n) {
                float s = bias[4 * F];
#pragma unroll
                for (int q = 0; q < NWG; q++) s += ypart[q][row];
                y[r] = s;
            }
        }
    }
    if (t == 0) {
        // only after a timeout can a load still be in flight: wait for it (bounded)
        if (issued > used) mbar_wait(&barx, (uint32_t)used & 1u, WAIT_CYCLES);
        if (!ok) atomicExch(err, 1);
    }
    fence_before();
    __syncthreads();
    if (t < 32) tmem_free(tbase, 64);
}

// --------------------------------------------------------------------------- training pass
// shared memory map (bytes from the 1024-aligned base)
constexpr uint32_t G_W = 0, G_X = 3 * WB, G_H1 = G_X + 2 * TB, G_H2 = G_H1 + TB, G_DZ = G_H2 + TB, G_ONE = G_DZ + TB,
                   G_END = G_ONE + TB;
constexpr size_t GRAD_SMEM = G_END + 1024;
constexpr int GRAD_NWG = 4;
// TMEM columns: Z1, Z2, Z3 (then dH2, dH1), dW1^T, dW2^T, dW3^T
constexpr int T_Z1 = 0, T_Z2 = 64, T_Z3 = 128, T_DW = 192;

// dW_l^T (+)= [A | 1]^T dZ over the tile's 128 samples: A (128 samples x 64) read MN-major
// with the constant block `one` (column 0 = 1, rest 0) as its second 64-wide block, so TMEM
// lane k < 64 gets the weight gradient of input k and lane 64 the bias gradient.
__device__ __forceinline__ void mma_weight_grad(uint32_t tmem, uint32_t a, uint32_t one, uint32_t dz, int accumulate) {
    const uint32_t id = idesc_bf16(TILE, F, 1, 1);
#pragma unroll
    for (int s = 0; s < TILE / 16; s++)
        mma_bf16(tmem, desc_sw128_mn(a, s, one - a), desc_sw128_mn(dz, s, TB), id, (s > 0 || accumulate) ? 1 : 0);
}
// dH = dZ W: A = dZ (K-major over the 64 outputs), B = W read MN-major (its rows are K).
__device__ __forceinline__ void mma_input_grad(uint32_t tmem, uint32_t dz, uint32_t w) {
    const uint32_t id = idesc_bf16(TILE, F, 0, 1);
#pragma unroll
    for (int s = 0; s < F / 16; s++) mma_bf16(tmem, desc_sw128_k(dz, s), desc_sw128_mn(w, s, WB), id, s > 0);
}

template <int NWG>
__global__ void __launch_bounds__(128 * NWG, 1) k_mlp_grad(const __grid_constant__ CUtensorMap xmap, const float* __restrict__ P,
                                                            const uint4* __restrict__ Wimg, const float* __restrict__ target,
                                                            int n, float dscale, float* __restrict__ part, int* err) {
    constexpr int CW = F / NWG;
    extern __shared__ __align__(16) unsigned char smraw[];
    unsigned char* sm = align_smem(smraw);
    __shared__ uint64_t barx[2], barm;
    __shared__ uint32_t tbase;
    __shared__ __align__(16) float bias[4 * F + 4];
    __shared__ float ypart[NWG][TILE];
    __shared__ float red[4 * NWG][CW + 2];
    const int t = threadIdx.x, row = t & (TILE - 1), g = t >> 7, c0 = g * CW, lane = t & 31, warp = t >> 5;
    const int ntiles = (n + TILE - 1) / TILE;
    if (t == 0) {
        mbar_init(&barx[0], 1);
        mbar_init(&barx[1], 1);
        mbar_init(&barm, 1);
        tma_prefetch_map(&xmap);
    }
    load_params(sm + G_W, Wimg, P, bias);
    // the constant block: BF16 1.0 in column 0 of every row, zeros elsewhere
    for (int e = t; e < (int)(TB / 16); e += blockDim.x) {
        const int r = e >> 3, ch = e & 7;
        ((uint4*)(sm + G_ONE))[e] = make_uint4(ch == (r & 7) ? 0x3F80u : 0u, 0u, 0u, 0u);
    }
    if (t < 32) tmem_alloc(&tbase, 512);
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    // TMA loads issued and consumed per feature buffer (thread 0's count; 16 bits each)
    uint32_t issued = 0, used = 0;
    if (t == 0) {
        for (int b = 0; b < 2; b++) {
            const int tile = blockIdx.x + b * gridDim.x;
            if (tile < ntiles) {
                mbar_expect_tx(&barx[b], TB);
                tma_load_2d(sm + G_X + b * TB, &xmap, 0, tile * TILE, &barx[b]);
                issued += 1u << (16 * b);
            }
        }
    }
    const uint32_t tb = tbase, id = idesc_bf16(TILE, F);
    const uint32_t aH1 = smem_u32(sm + G_H1), aH2 = smem_u32(sm + G_H2), aDZ = smem_u32(sm + G_DZ), aONE = smem_u32(sm + G_ONE);
    const uint32_t aW1 = smem_u32(sm + G_W), aW2 = aW1 + WB, aW3 = aW1 + 2 * WB;
    uint32_t pm = 0;
    bool ok = true;
    float acc4[CW];  // this sample's share of dL/dw4, summed over the CTA's tiles
#pragma unroll
    for (int c = 0; c < CW; c++) acc4[c] = 0.0f;
    float loss = 0.0f, accb4 = 0.0f;
    auto mma_wait = [&]() {
        if (t == 0) mma_commit(&barm);
        ok = vote_ok(mbar_wait(&barm, pm, WAIT_CYCLES));
        pm ^= 1u;
        fence_after();
        return ok;
    };
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, it++) {
        const int b = it & 1;
        const long grow = (long)tile * TILE + row;
        const bool valid = grow < n;
        const float tgt = valid ? target[grow] : 0.0f;  // needed after the forward GEMMs
        ok = vote_ok(mbar_wait(&barx[b], (uint32_t)(it >> 1) & 1u, WAIT_CYCLES));
        if (!ok) break;
        used += 1u << (16 * b);
        const uint32_t aX = smem_u32(sm + G_X + b * TB);
        // ---- forward
        if (t == 0)
            for (int s = 0; s < F / 16; s++) mma_bf16(tb + T_Z1, desc_sw128_k(aX, s), desc_sw128_k(aW1, s), id, s > 0);
        if (!mma_wait()) break;
        if (t == 0 && it > 0) {
            // this wait also covered the previous tile's last MMA (dW1, which read the other
            // feature buffer): load the next tile into that buffer
            const int next = tile + gridDim.x;
            if (next < ntiles) {
                mbar_expect_tx(&barx[b ^ 1], TB);
                tma_load_2d(sm + G_X + (b ^ 1) * TB, &xmap, 0, next * TILE, &barx[b ^ 1]);
                issued += 1u << (16 * (b ^ 1));
            }
        }
        {   // H1 = SiLU(Z1 + b1); SiLU' kept in TMEM over Z1 for the backward pass
            float z[CW], d[CW];
            tmem_load<CW>(tb, T_Z1 + c0, z);
            tmem_wait_ld();
            hidden_epilogue<CW, true>(sm + G_H1, row, c0, z, bias, d);
            tmem_store<CW>(tb, T_Z1 + c0, d);
        }
        publish();
        if (t == 0)
            for (int s = 0; s < F / 16; s++) mma_bf16(tb + T_Z2, desc_sw128_k(aH1, s), desc_sw128_k(aW2, s), id, s > 0);
        if (!mma_wait()) break;
        {
            float z[CW], d[CW];
            tmem_load<CW>(tb, T_Z2 + c0, z);
            tmem_wait_ld();
            hidden_epilogue<CW, true>(sm + G_H2, row, c0, z, bias + F, d);
            tmem_store<CW>(tb, T_Z2 + c0, d);
        }
        publish();
        if (t == 0)
            for (int s = 0; s < F / 16; s++) mma_bf16(tb + T_Z3, desc_sw128_k(aH2, s), desc_sw128_k(aW3, s), id, s > 0);
        if (!mma_wait()) break;
        // ---- output layer, loss, dL/dw4, dL/db4, dZ3
        {
            float z[CW], sg[CW];
            tmem_load<CW>(tb, T_Z3 + c0, z);
            tmem_wait_ld();
            float yp = 0.0f;
            float w4[CW];
#pragma unroll
            for (int c = 0; c < CW; c += 4) {
                const float4 b = *(const float4*)(bias + 2 * F + c0 + c), w = *(const float4*)(bias + 3 * F + c0 + c);
                z[c] += b.x; z[c + 1] += b.y; z[c + 2] += b.z; z[c + 3] += b.w;
                w4[c] = w.x; w4[c + 1] = w.y; w4[c + 2] = w.z; w4[c + 3] = w.w;
            }
#pragma unroll
            for (int c = 0; c < CW; c++) {
                sg[c] = logistic(z[c]);
                yp = __fmaf_rn(w4[c], z[c] * sg[c], yp);
            }
            ypart[g][row] = yp;
            __syncthreads();
            float yv = bias[4 * F];
#pragma unroll
            for (int q = 0; q < NWG; q++) yv += ypart[q][row];
            const float r = valid ? yv - tgt : 0.0f;
            const float dy = 2.0f * r * dscale;
            if (g == 0) {
                loss += r * r;
                accb4 += dy;
            }
#pragma unroll
            for (int c = 0; c < CW; c += 8) {
                float d[8];
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int j = c + q;
                    acc4[j] = __fmaf_rn(dy, z[j] * sg[j], acc4[j]);
                    d[q] = dy * w4[j] * dsilu(z[j], sg[j]);
                }
                *(uint4*)(sm + G_DZ + sw128_off(row, c0 + c)) =
                    make_uint4(pack_bf16(d[0], d[1]), pack_bf16(d[2], d[3]), pack_bf16(d[4], d[5]), pack_bf16(d[6], d[7]));
            }
        }
        publish();
        // ---- dW3^T += [H2 | 1]^T dZ3;  dH2 = dZ3 W3 (over Z3, which is no longer needed)
        if (t == 0) {
            mma_weight_grad(tb + T_DW + 2 * F, aH2, aONE, aDZ, it > 0);
            mma_input_grad(tb + T_Z3, aDZ, aW3);
        }
        if (!mma_wait()) break;
        for (int l = 1; l >= 0; l--) {
            {   // dZ_l = dH_l * SiLU'(Z_l) (the derivative stored by the forward epilogue)
                float dh[CW], d[CW];
                tmem_load<CW>(tb, T_Z3 + c0, dh);
                tmem_load<CW>(tb, l * F + c0, d);
                tmem_wait_ld();
#pragma unroll
                for (int c = 0; c < CW; c += 8) {
                    uint32_t pk[4];
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        pk[q] = pack_bf16(dh[c + 2 * q] * d[c + 2 * q], dh[c + 2 * q + 1] * d[c + 2 * q + 1]);
                    *(uint4*)(sm + G_DZ + sw128_off(row, c0 + c)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                }
            }
            publish();
            if (t == 0) {
                if (l == 1) {  // dW2^T += [H1 | 1]^T dZ2;  dH1 = dZ2 W2
                    mma_weight_grad(tb + T_DW + F, aH1, aONE, aDZ, it > 0);
                    mma_input_grad(tb + T_Z3, aDZ, aW2);
                } else {       // dW1^T += [X | 1]^T dZ1 (completion awaited with the next tile's first GEMM)
                    mma_weight_grad(tb + T_DW, aX, aONE, aDZ, it > 0);
                }
            }
            if (l == 1 && !mma_wait()) break;
        }
        if (!ok) break;
    }
    if (ok && it > 0) mma_wait();  // the last dW1 MMAs
    if (t == 0) {
        for (int b = 0; b < 2; b++) {
            const uint32_t ib = (issued >> (16 * b)) & 0xFFFFu, ub = (used >> (16 * b)) & 0xFFFFu;
            if (ib > ub) mbar_wait(&barx[b], ub & 1u, WAIT_CYCLES);
        }
        if (!ok) atomicExch(err, 1);
    }
    // ---- per-CTA partial record
    float* out = part + (size_t)blockIdx.x * PSTRIDE;
    for (int l = 0; l < 3; l++) {
        float v[CW];
        tmem_load<CW>(tb, T_DW + l * F + c0, v);
        tmem_wait_ld();
        if (!ok || it == 0) {
#pragma unroll
            for (int c = 0; c < CW; c++) v[c] = 0.0f;
        }
        if (row < F) {  // lane k = input k: dW_l[n][k] for this warpgroup's outputs n
#pragma unroll
            for (int c = 0; c < CW; c++) out[OW1 + l * LSTRIDE + (c0 + c) * F + row] = v[c];
        } else if (row == F) {  // the bias row
#pragma unroll
            for (int c = 0; c < CW; c++) out[OB1 + l * LSTRIDE + c0 + c] = v[c];
        }
    }
    // dL/dw4 (this warpgroup's columns), dL/db4 and the loss: sums over the CTA's samples in
    // a fixed order (lanes by shuffles, then the warps)
#pragma unroll
    for (int c = 0; c < CW; c++) {
        float v = acc4[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[warp][c] = v;
    }
    {
        float l = loss, bb = accb4;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            l += __shfl_xor_sync(0xffffffffu, l, o);
            bb += __shfl_xor_sync(0xffffffffu, bb, o);
        }
        if (lane == 0) {
            red[warp][CW] = l;
            red[warp][CW + 1] = bb;
        }
    }
    __syncthreads();
    if (row < CW) {  // one thread per column of each warpgroup
        float s = 0.0f;
        for (int w = 0; w < 4; w++) s += red[4 * g + w][row];
        out[OW4 + c0 + row] = ok ? s : 0.0f;
    }
    if (t == 0) {
        float l = 0.0f, bb = 0.0f;
        for (int w = 0; w < 4; w++) {
            l += red[w][CW];
            bb += red[w][CW + 1];
        }
        out[NPARAM] = ok ? l : 0.0f;
        out[OB4] = ok ? bb : 0.0f;
    }
    fence_before();
    __syncthreads();
    if (t < 32) tmem_free(tbase, 512);
}

// BF16 operand image of weight element e of the hidden layers (e < 3 * 4096), or -1.
__device__ __forceinline__ int image_index(int e) {
    const int l = e / LSTRIDE, r = e - l * LSTRIDE;
    if (l > 2 || r >= F * F) return -1;
    return (int)((l * WB + sw128_off(r / F, r % F)) / 2);
}

__global__ void k_mlp_pack(const float* __restrict__ P, __nv_bfloat16* __restrict__ Wimg) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < OW4; e += gridDim.x * blockDim.x) {
        const int i = image_index(e);
        if (i >= 0) Wimg[i] = __float2bfloat16_rn(P[e]);
    }
}

// Folds the CTA partials in a fixed order (slice j of 8 sums CTAs j, j + 8, ..., then the
// slices in order); optionally applies Adam (step >= 1) and rewrites the operand images.
constexpr int ADAM_PARAMS = 32, ADAM_SLICES = 8;
__global__ void __launch_bounds__(ADAM_PARAMS * ADAM_SLICES) k_mlp_adam(const float* __restrict__ part, int G, float* __restrict__ grad,
                                                                       float* __restrict__ P, float* __restrict__ m, float* __restrict__ v,
                                                                       __nv_bfloat16* __restrict__ Wimg, long step, float lr, float b1,
                                                                       float b2, float eps, float* loss) {
    __shared__ float red[ADAM_SLICES][ADAM_PARAMS];
    const int p = threadIdx.x % ADAM_PARAMS, j = threadIdx.x / ADAM_PARAMS;
    const int e = blockIdx.x * ADAM_PARAMS + p;
    float g = 0.0f;
    if (e <= NPARAM)
        for (int b = j; b < G; b += ADAM_SLICES) g += part[(size_t)b * PSTRIDE + e];
    red[j][p] = g;
    __syncthreads();
    if (j != 0 || e > NPARAM) return;
    g = 0.0f;
    for (int q = 0; q < ADAM_SLICES; q++) g += red[q][p];
    if (e == NPARAM) { *loss = g; return; }
    grad[e] = g;
    if (step < 1) return;
    const float mm = b1 * m[e] + (1.0f - b1) * g, vv = b2 * v[e] + (1.0f - b2) * g * g;
    m[e] = mm;
    v[e] = vv;
    const float mh = mm / (1.0f - powf(b1, (float)step)), vh = vv / (1.0f - powf(b2, (float)step));
    const float w = P[e] - lr * mh / (sqrtf(vh) + eps);
    P[e] = w;
    const int i = image_index(e);
    if (i >= 0) Wimg[i] = __float2bfloat16_rn(w);
}

}  // namespace mlp
}  // namespace spb6g

using namespace spb6g::mlp;

struct spb6g_mlp {
    int device = 0;
    int G = 0;       // CTAs of a training pass (one per SM)
    int Gf = 0;      // CTAs of an inference pass (resident CTAs per SM x SMs)
    long step = 0;
    cudaStream_t st = nullptr;
    float *P = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *part = nullptr, *loss = nullptr;
    __nv_bfloat16* Wimg = nullptr;
    int* err = nullptr;
    // feature-row tensor maps of the last calls
    const void* fx = nullptr;
    int fn = -1;
    CUtensorMap fmap;
    const void* gx = nullptr;
    int gn = -1;
    CUtensorMap gmap;
};

namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}
// Rows of 64 BF16 (128 bytes), n rows; 128-row boxes in the 128-byte swizzle; rows past n read as zeros.
int feature_map(CUtensorMap* map, const void* X, int n) {
    const auto enc = encode_fn();
    if (!enc || ((uintptr_t)X & 15u) || n <= 0) return -1;
    const cuuint64_t dims[2] = {(cuuint64_t)F, (cuuint64_t)n};
    const cuuint64_t strides[1] = {(cuuint64_t)F * 2};
    const cuuint32_t box[2] = {(cuuint32_t)F, (cuuint32_t)TILE};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(X), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS
               ? 0
               : -1;
}
int mlp_prepare(int device, int* fwd_per_sm) {
    static std::mutex mu;
    static unsigned done = 0;
    static int per_sm[32] = {0};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 32 && (done >> device) & 1u) {
        *fwd_per_sm = per_sm[device];
        return 0;
    }
    if (cudaFuncSetAttribute(k_mlp_forward<FWD_NWG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)FWD_SMEM) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_forward<FWD_NWG>, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_grad<GRAD_NWG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GRAD_SMEM) != cudaSuccess)
        return -1;
    // the kernel's launch bounds, shared memory and 64 TMEM columns are sized for FWD_CTAS per SM
    const int k = FWD_CTAS;
    if (device < 32) {
        done |= 1u << device;
        per_sm[device] = k;
    }
    *fwd_per_sm = k;
    return 0;
}
int mlp_check(spb6g_mlp* h) {
    int e = 0;
    if (cudaMemcpyAsync(&e, h->err, sizeof(int), cudaMemcpyDeviceToHost, h->st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (cudaStreamSynchronize(h->st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (e) {
        fprintf(stderr, "spb6g_mlp: a tensor-core or TMA wait timed out\n");
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
    if (!encode_fn()) return SPB6G_UNSUPPORTED;
    int per_sm = 0;
    if (mlp_prepare(device, &per_sm)) return SPB6G_CUDA_ERROR;
    spb6g_mlp* h = new spb6g_mlp();
    h->device = device;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    h->G = sms > 0 ? sms : 148;
    h->Gf = h->G * per_sm;
    // a blocking stream: the handle's work orders itself after the caller's work on the
    // legacy default stream (which produces X and the targets in the usual case)
    bool ok = cudaStreamCreate(&h->st) == cudaSuccess;
    ok = ok && cudaMalloc(&h->P, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->m, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->v, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->grad, NPARAM * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->part, (size_t)h->G * PSTRIDE * sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->loss, sizeof(float)) == cudaSuccess;
    ok = ok && cudaMalloc(&h->Wimg, 3 * WB) == cudaSuccess;
    ok = ok && cudaMalloc(&h->err, sizeof(int)) == cudaSuccess;
    if (ok) {
        cudaMemsetAsync(h->P, 0, NPARAM * sizeof(float), h->st);
        cudaMemsetAsync(h->m, 0, NPARAM * sizeof(float), h->st);
        cudaMemsetAsync(h->v, 0, NPARAM * sizeof(float), h->st);
        cudaMemsetAsync(h->Wimg, 0, 3 * WB, h->st);
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
    for (void* p : {(void*)h->P, (void*)h->m, (void*)h->v, (void*)h->grad, (void*)h->part, (void*)h->loss, (void*)h->Wimg,
                    (void*)h->err})
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
    k_mlp_pack<<<(OW4 + 255) / 256, 256, 0, h->st>>>(h->P, h->Wimg);
    if (cudaGetLastError() != cudaSuccess) return SPB6G_CUDA_ERROR;
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
    if (!h || !X_dev || !y_dev || n < 0 || ((uintptr_t)X_dev & 15u)) return SPB6G_BAD_ARG;
    if (n == 0) return SPB6G_OK;
    cudaSetDevice(h->device);
    if (X_dev != h->fx || n != h->fn) {
        if (feature_map(&h->fmap, X_dev, n)) return SPB6G_CUDA_ERROR;
        h->fx = X_dev;
        h->fn = n;
    }
    cudaStream_t st = stream ? (cudaStream_t)stream : h->st;
    const int ntiles = (n + TILE - 1) / TILE;
    const int G = ntiles < h->Gf ? ntiles : h->Gf;
    k_mlp_forward<FWD_NWG><<<G, 128 * FWD_NWG, FWD_SMEM, st>>>(h->fmap, h->P, (const uint4*)h->Wimg, n, y_dev, h->err);
    if (cudaGetLastError() != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (stream) return SPB6G_OK;
    return mlp_check(h);
}

// One pass over the batch on `stream`, nothing read back: gradient of mean((y - target)^2)
// into the handle, with lr > 0 also an Adam step.
static int mlp_train_launch(spb6g_mlp* h, const void* X_dev, const float* target_dev, int n, float lr, cudaStream_t st) {
    if (X_dev != h->gx || n != h->gn) {
        if (feature_map(&h->gmap, X_dev, n)) return SPB6G_CUDA_ERROR;
        h->gx = X_dev;
        h->gn = n;
    }
    const int ntiles = (n + TILE - 1) / TILE;
    const int G = ntiles < h->G ? ntiles : h->G;
    k_mlp_grad<GRAD_NWG><<<G, 128 * GRAD_NWG, GRAD_SMEM, st>>>(h->gmap, h->P, (const uint4*)h->Wimg, target_dev, n, 1.0f / (float)n,
                                                               h->part, h->err);
    if (cudaGetLastError() != cudaSuccess) return SPB6G_CUDA_ERROR;
    const long step = lr > 0 ? ++h->step : 0;
    k_mlp_adam<<<(NPARAM + ADAM_PARAMS) / ADAM_PARAMS, ADAM_PARAMS * ADAM_SLICES, 0, st>>>(
        h->part, G, h->grad, h->P, h->m, h->v, h->Wimg, step, lr, 0.9f, 0.999f, 1e-8f, h->loss);
    return cudaGetLastError() == cudaSuccess ? SPB6G_OK : SPB6G_CUDA_ERROR;
}

int spb6g_mlp_train_async(spb6g_mlp* h, const void* X_dev, const float* target_dev, int n, float lr, void* stream) {
    if (!h || !X_dev || !target_dev || n <= 0 || ((uintptr_t)X_dev & 15u)) return SPB6G_BAD_ARG;
    cudaSetDevice(h->device);
    return mlp_train_launch(h, X_dev, target_dev, n, lr, stream ? (cudaStream_t)stream : h->st);
}

int spb6g_mlp_last_loss(spb6g_mlp* h, void* stream, float* loss_sum) {
    if (!h || !loss_sum) return SPB6G_BAD_ARG;
    cudaSetDevice(h->device);
    cudaStream_t st = stream ? (cudaStream_t)stream : h->st;
    float l = 0;
    if (cudaMemcpyAsync(&l, h->loss, sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    *loss_sum = l;
    return mlp_check(h);
}

// One pass over the batch: gradient of mean((y - target)^2); with lr > 0 also an Adam step.
int spb6g_mlp_train_step(spb6g_mlp* h, const void* X_dev, const float* target_dev, int n, float lr, float* loss_out,
                         float* grad_host) {
    if (!h || !X_dev || !target_dev || n <= 0 || ((uintptr_t)X_dev & 15u)) return SPB6G_BAD_ARG;
    cudaSetDevice(h->device);
    const int lrc = mlp_train_launch(h, X_dev, target_dev, n, lr, h->st);
    if (lrc != SPB6G_OK) return lrc;
    float l = 0;
    if (cudaMemcpyAsync(&l, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->st) != cudaSuccess) return SPB6G_CUDA_ERROR;
    if (grad_host && cudaMemcpyAsync(grad_host, h->grad, NPARAM * sizeof(float), cudaMemcpyDeviceToHost, h->st) != cudaSuccess)
        return SPB6G_CUDA_ERROR;
    const int rc = mlp_check(h);
    if (loss_out) *loss_out = l / (float)n;
    return rc;
}

}  // extern "C"
