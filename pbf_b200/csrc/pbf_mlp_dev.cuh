// Device-side building blocks of the warm-start network shared by the
// network's own kernels (pbf_mlp.cu) and the fused feature + inference pass
// (pbf_pairs.cu): the GELU activation, staging of BF16 operands in the
// tensor core's canonical K-major layout, and the bounded waits on the
// tensor-core barrier.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pbf_device.cuh"
#include "pbf_packed.cuh"
#include "pbf_tc.cuh"

namespace pbf {

using namespace tc;

// ---------------------------------------------------------------------------
// activation
// ---------------------------------------------------------------------------
constexpr float GELU_C = 0.7978845608028654f;  // sqrt(2 / pi)
constexpr float GELU_A = 0.044715f;

// hardware tanh (one MUFU operation, about 2^-11 relative error: below the BF16
// rounding the activations go through anyway)
__device__ __forceinline__ float tanh_fast(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// GELU, tanh form: 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))
__device__ __forceinline__ float gelu(float z) {
    const float u = GELU_C * (z + GELU_A * z * z * z);
    return 0.5f * z * (1.0f + tanh_fast(u));
}

// GELU of two values with packed FP32 arithmetic (same expression order)
__device__ __forceinline__ float2 gelu2(float2 z) {
    const float2 z3 = vmul(vmul(vmul(bc<float2>(GELU_A), z), z), z);
    const float2 u = vmul(bc<float2>(GELU_C), vadd(z, z3));
    const float2 t = make_float2(tanh_fast(u.x), tanh_fast(u.y));
    return vmul(vmul(bc<float2>(0.5f), z), vadd(bc<float2>(1.0f), t));
}

__device__ __forceinline__ float gelu_grad(float z) {
    const float u = GELU_C * (z + GELU_A * z * z * z);
    const float t = tanh_fast(u);
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * GELU_C * (1.0f + 3.0f * GELU_A * z * z);
}

// ---------------------------------------------------------------------------
// shared-memory staging
// ---------------------------------------------------------------------------
// W [rows][K] row-major BF16 in global -> canonical K-major tile of `rows` rows
__device__ __forceinline__ void stage_weight(uint8_t* s, const uint16_t* __restrict__ W, int rows, int K) {
    for (int idx = threadIdx.x; idx < rows * (K / 8); idx += blockDim.x) {
        const int r = idx / (K / 8), j = idx % (K / 8);
        const uint4 v = *reinterpret_cast<const uint4*>(W + (size_t)r * K + 8 * j);
        *reinterpret_cast<uint4*>(s + kmajor_offset(r, 8 * j, rows)) = v;
    }
}

// W [64][K] row-major -> canonical K-major tile of its transpose W^T [K rows][64]
__device__ __forceinline__ void stage_weight_t(uint8_t* s, const uint16_t* __restrict__ W, int K) {
    for (int idx = threadIdx.x; idx < 64 * K; idx += blockDim.x) {
        const int n = idx / K, k = idx % K;
        *reinterpret_cast<uint16_t*>(s + kmajor_offset(k, n, K)) = W[(size_t)n * K + k];
    }
}

__device__ __forceinline__ uint16_t bf16_bits(float f) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(f));
}

__device__ __forceinline__ float bf16_val(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }

// write 64 values of row `row` into a canonical K-major [128 x 64] tile
__device__ __forceinline__ void put_row64(uint8_t* s, int row, const float (&v)[16], int c0) {
    uint32_t pk[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const __nv_bfloat162 b2 = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);  // one packed conversion
        pk[i] = *reinterpret_cast<const uint32_t*>(&b2);
    }
    *reinterpret_cast<uint4*>(s + kmajor_offset(row, c0, 128)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
    *reinterpret_cast<uint4*>(s + kmajor_offset(row, c0 + 8, 128)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
}

// Waits for the tensor core. The outcome is made uniform over the CTA (every
// thread leaves the tile loop together). On an expired wait the error bit is
// set and a second bounded wait gives MMAs still in flight time to finish
// before the caller frees TMEM.
constexpr long long MBAR_WAIT_LIMIT = 1ll << 24;  // polls of one bounded wait

__device__ __forceinline__ bool wait_mma(uint64_t* mbar, uint32_t& phase, int* err,
                                         long long limit = MBAR_WAIT_LIMIT) {
    bool ok = mbar_wait(mbar, phase, limit);
    if (!ok) {
        if ((threadIdx.x & 31) == 0) atomicOr(err, DEVERR_MLP_TIMEOUT);
        mbar_wait(mbar, phase, limit);
    }
    phase ^= 1u;
    ok = __syncthreads_and(ok) != 0;
    fence_after_sync();
    return ok;
}

__device__ __forceinline__ void sync_for_mma() {
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
}

}  // namespace pbf
