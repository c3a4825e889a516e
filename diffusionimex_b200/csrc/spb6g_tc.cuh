// Blackwell tensor-core building blocks (sm_100a): tcgen05 MMA with operands in
// shared memory and the accumulator in tensor memory (TMEM), BF16 inputs,
// FP32 accumulation.
//
// Operand layout ("K-major, no swizzle"): an operand of R rows x K columns of
// BF16 is stored as 8x8 core matrices of 128 contiguous bytes (8 rows of 16
// bytes); core matrices run along K first, then along rows:
//   byte(r, k) = ((r / 8) * (K / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2.
// One MMA consumes a K-slice of 16: its descriptor starts at the slice's first
// core matrix, the two core matrices of the slice are 128 B apart (leading byte
// offset) and consecutive 8-row groups K/8 * 128 B apart (stride byte offset).
//
// D[M x N] (+)= A[M x K] * B[K x N] with A stored as M rows x K and B stored as
// N rows x K (both K-major).  For M = 128 accumulator row i lives in TMEM lane i,
// column j in column base + j; warp w of the CTA reads lanes 32 w .. 32 w + 31.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace spb6g {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) in a K-major operand with K columns.
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int K) {
    return (uint32_t)(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor for the 16-wide K-slice `s` of a K-major
// operand starting at shared address `base` with K columns.
__device__ __forceinline__ uint64_t smem_desc(uint32_t base, int K, int s) {
    const uint32_t start = base + (uint32_t)s * 256u;
    const uint64_t lbo = 128u, sbo = (uint64_t)(K >> 3) * 128u;
    return (uint64_t)((start >> 4) & 0x3FFFu) | (((lbo >> 4) & 0x3FFFu) << 16) | (((sbo >> 4) & 0x3FFFu) << 32) |
           (1ull << 46);  // descriptor version 1 (Blackwell); base offset 0; no swizzle
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 D; A and B K-major unless
// a_mn / b_mn (MN-major: the operand's M or N index runs along its rows).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn = 0, int b_mn = 0) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---- 128-byte swizzled tiles: rows of 64 BF16 (128 bytes); the 16-byte chunk c of
// row r sits at chunk position c ^ (r % 8), the pattern TMA's 128-byte swizzle
// writes (tile base 1024-byte aligned).  One physical tile serves as either operand
// form: K-major (rows = M or N, the 64 columns = K) or MN-major (rows = K, the 64
// columns = M or N).
__host__ __device__ __forceinline__ uint32_t sw128_off(int r, int k) {
    return (uint32_t)(r * 128 + ((((k >> 3) ^ r) & 7) << 4) + (k & 7) * 2);
}
// K-major descriptor of the 16-wide K-slice `s`: the slice starts 32 bytes further
// into each 128-byte row (the swizzle is applied by the hardware on the address),
// 8-row groups 1024 bytes apart; the leading offset is unused (set to 16 bytes).
__device__ __forceinline__ uint64_t desc_sw128_k(uint32_t base, int s) {
    const uint32_t start = base + (uint32_t)s * 32u;
    return (uint64_t)((start >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}
// MN-major descriptor of the 16-wide K-slice `s` (16 rows = two 8-row groups of
// 1024 bytes); `atom_stride` = byte distance to the next 64-wide block along M/N.
__device__ __forceinline__ uint64_t desc_sw128_mn(uint32_t base, int s, uint32_t atom_stride) {
    const uint32_t start = base + (uint32_t)s * 2048u;
    return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((atom_stride >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) | (2ull << 61);
}

// ---- TMA (no multicast) and transaction-count mbarriers
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Tile {x, y} of a 2D tensor map into shared memory; completion counted on `bar`.
__device__ __forceinline__ void tma_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)tmap), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_prefetch_map(const void* tmap) {
    asm volatile("prefetch.tensormap [%0];" ::"l"((uint64_t)tmap) : "memory");
}

// One MMA (issued by a single thread): D = A * B (+ D when accumulate).
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, int accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// D = A[M x K] * B, K a multiple of 16: K/16 MMAs.
__device__ __forceinline__ void mma_chain(uint32_t tmem_d, uint32_t a_base, int Ka, uint32_t b_base, int Kb, int K, uint32_t idesc,
                                          int accumulate) {
    for (int s = 0; s < K / 16; s++)
        mma_bf16(tmem_d, smem_desc(a_base, Ka, s), smem_desc(b_base, Kb, s), idesc, (s > 0 || accumulate) ? 1 : 0);
}
// Arrives on the mbarrier once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor cores.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Waits for the phase of parity `phase` to complete; gives up after about
// `limit` clock cycles and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, long long limit) {
    const uint32_t a = smem_u32(bar);
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) return false;
    }
}

// TMEM allocation (one full warp; `ncols` a power of two >= 32); the base address is written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}
// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr)
        : "memory");
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
// 16 consecutive FP32 columns into this thread's TMEM lane.
__device__ __forceinline__ void tmem_st16(uint32_t addr, const float* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(addr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
        "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
        "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
// TMEM address of column `col` for the lanes of this thread's warp.
__device__ __forceinline__ uint32_t tmem_lane_addr(uint32_t base, int col) {
    return base + ((uint32_t)((threadIdx.x >> 5) & 3) * 32u << 16) + (uint32_t)col;
}

}  // namespace tc
}  // namespace spb6g
