// 5th-generation tensor core (tcgen05) building blocks for sm_100a, written
// against the PTX ISA: TMEM allocation, shared-memory matrix descriptors,
// instruction descriptors for kind::f16 (BF16 x BF16 -> FP32), MMA issue,
// completion through an mbarrier, and accumulator loads from TMEM.
//
// Operand layout: both operands K-major, no swizzle ("interleaved" canonical
// layout). A tile of R rows x K columns of 16-bit values is stored as 8x8 core
// matrices of 128 contiguous bytes (row r of a core matrix at r * 16 bytes);
// core matrix (row group g, k group j) starts at (j * R/8 + g) * 128 bytes. In
// descriptor terms: stride between row groups (SBO) = 128 B, stride between k
// groups (LBO) = R/8 * 128 B; one MMA consumes K = 16 (two k groups) and the
// next K step starts 2 * LBO further.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace pbf {
namespace tc {

// byte offset of element (row, k) in the canonical K-major layout of an R-row tile
__device__ __forceinline__ uint32_t kmajor_offset(int row, int k, int R) {
    return (uint32_t)((((k >> 3) * (R >> 3) + (row >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1));
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared memory matrix descriptor (64 bit): start >> 4 [0,14), LBO >> 4 [16,30),
// SBO >> 4 [32,46), fixed version 1 at [46,48), base offset 0, layout 0 (no swizzle).
__device__ __forceinline__ uint64_t smem_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((start >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;
}

// Instruction descriptor, kind::f16: D f32 (bits 4-5 = 1), A bf16 (bits 7-9 = 1),
// B bf16 (bits 10-12 = 1), A and B K-major (bits 15, 16 = 0), N >> 3 at bits
// 17-22, M >> 4 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---- TMEM -------------------------------------------------------------------
// Executed by one whole warp; writes the TMEM base address to *slot (smem).
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// generic-proxy smem writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// ---- MMA ----------------------------------------------------------------------
// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// Arrives once on the mbarrier when every MMA this thread issued has completed.
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(mbar))
                 : "memory");
}

// ---- mbarrier -------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity`; false when the limit expired.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, long long limit = (1ll << 24)) {
    for (long long i = 0; i < limit; ++i)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

// ---- accumulator loads ------------------------------------------------------------
// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: warp w of
// a warpgroup reads lanes 32w .. 32w+31).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// TMEM address of (lane, column) relative to a base returned by tmem_alloc
__device__ __forceinline__ uint32_t tmem_addr(uint32_t base, int lane, int col) {
    return base + ((uint32_t)lane << 16) + (uint32_t)col;
}

// Issues D[128 x N] = A[128 x K] * B[N x K]^T (both K-major canonical tiles in
// smem) as K/16 MMAs; `accumulate` applies to the first one.
__device__ __forceinline__ void gemm_issue(uint32_t d_tmem, const void* sA, const void* sB, int N, int K,
                                           uint32_t accumulate) {
    const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
    const uint32_t lbo_a = (128 / 8) * 128, lbo_b = (uint32_t)(N / 8) * 128;
    const uint32_t idesc = idesc_bf16_f32(128, N);
    for (int ks = 0; ks < K / 16; ++ks) {
        const uint64_t da = smem_desc(a0 + ks * 2 * lbo_a, lbo_a, 128);
        const uint64_t db = smem_desc(b0 + ks * 2 * lbo_b, lbo_b, 128);
        mma_bf16(d_tmem, da, db, idesc, (ks > 0 || accumulate) ? 1u : 0u);
    }
}

}  // namespace tc
}  // namespace pbf
