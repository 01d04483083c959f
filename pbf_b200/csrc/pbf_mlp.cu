// Learned lambda warm start: per-particle MLP 12 -> 64 -> 64 -> 64 -> 1 (GELU),
// BF16 weights, FP32 accumulation, on the 5th-generation tensor cores (tcgen05,
// accumulators in TMEM). No reference counterpart.
//
// Every tensor-core kernel runs 128 threads per CTA: thread t owns row t of a
// 128-row tile, which is TMEM lane t of the accumulator, so each epilogue
// (bias, GELU, its derivative, the output layer) is per-thread register work
// on one particle after a tcgen05.ld of that thread's lane.
#include <algorithm>

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pbf_device.cuh"
#include "pbf_mlp.h"
#include "pbf_packed.cuh"
#include "pbf_tc.cuh"
#include "pbf_mlp_dev.cuh"

namespace pbf {

using namespace tc;

constexpr int TILE = 128;
constexpr int TMEM_COLS = 256;      // tile GEMM and backward (at most 2 CTAs per SM by smem)
constexpr int TMEM_COLS_FWD = 128;  // forward: layers 1 and 3 share columns [0, 64), so 4 CTAs fit an SM

// ---------------------------------------------------------------------------
// Tile GEMM (exported for tests): D[128 x N] = A[128 x K] * B[N x K]^T.
// ---------------------------------------------------------------------------
constexpr int TC_GEMM_SMEM_MIN = 96 * 1024;

__global__ void __launch_bounds__(128, 1) k_tc_gemm(const __nv_bfloat16* __restrict__ A,
                                                    const __nv_bfloat16* __restrict__ B, float* __restrict__ D,
                                                    int N, int K, int* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    uint8_t* sA = smem;
    uint8_t* sB = smem + ((128 * K * 2 + 1023) & ~1023);
    if (warp == 0) tmem_alloc(&tmem_slot, TMEM_COLS);
    if (t == 0) mbar_init(&mbar, 1);
    for (int j = 0; j < K / 8; ++j) {
        const uint4 v = *reinterpret_cast<const uint4*>(A + (size_t)t * K + 8 * j);
        *reinterpret_cast<uint4*>(sA + kmajor_offset(t, 8 * j, 128)) = v;
    }
    for (int r = t; r < N; r += 128)
        for (int j = 0; j < K / 8; ++j) {
            const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)r * K + 8 * j);
            *reinterpret_cast<uint4*>(sB + kmajor_offset(r, 8 * j, N)) = v;
        }
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = tmem_slot;
    if (t == 0) {
        gemm_issue(tbase, sA, sB, N, K, 0);
        commit(&mbar);
    }
    bool ok = mbar_wait(&mbar, 0);
    if (!ok) {
        if (lane == 0) atomicOr(err, DEVERR_MLP_TIMEOUT);
        ok = mbar_wait(&mbar, 0);  // a second bounded wait for MMAs in flight before TMEM is freed
    }
    fence_after_sync();
    if (ok) {
        for (int c = 0; c < N / 16; ++c) {
            float v[16];
            tmem_ld16(tmem_addr(tbase, 32 * warp, 16 * c), v);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; ++i) D[(size_t)t * N + 16 * c + i] = v[i];
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, TMEM_COLS);
}

int tc_gemm_bf16(const void* A, const void* B, float* D, int N, int K, int* err, cudaStream_t st) {
    const int smem = (128 * K * 2 + 1023) / 1024 * 1024 + N * K * 2;
    const int bytes = smem < TC_GEMM_SMEM_MIN ? TC_GEMM_SMEM_MIN : smem;
    cudaError_t e = cudaFuncSetAttribute(k_tc_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return -1;
    k_tc_gemm<<<1, 128, bytes, st>>>((const __nv_bfloat16*)A, (const __nv_bfloat16*)B, D, N, K, err);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// ---------------------------------------------------------------------------
// Forward pass over 128-row tiles (persistent CTAs). TRAIN additionally saves
// what the backward pass needs and computes the output-layer gradients.
// ---------------------------------------------------------------------------
// Per-slot gradient partials of the training forward pass: loss, db4, dw4[64].
constexpr int FWD_PART = 66;

// out[i] = sum over parts p = 0, 1, ... of part[p * stride + i], in that order
// (deterministic: the gradients are the same bits on every run)
__global__ void k_sum_parts(const float* __restrict__ part, int nparts, int stride, int count,
                            float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float s = 0.0f;
    for (int q = 0; q < nparts; ++q) s += part[(size_t)q * stride + i];
    out[i] = s;
}

struct FwdIO {
    const uint16_t* w;   // bf16 weights
    const float* b;      // biases and constants
    const float* feat;   // raw features [n][12]
    int n;
    // inference outputs
    float* out;
    float4* q;
    float* lam_acc;
    float clamp;  // trust-region factor around q.w (0: none)
    int floor;    // 1: lambda0 at least as strong as q.w (same sign, magnitude >= |q.w|)
    // training
    const float* target;  // [n]
    float inv_batch;
    uint16_t *x16, *h1, *h2, *g1, *g2, *dz3;  // [n][16] and [n][64] bf16
    float* part;  // per tile and warp: loss, db4, dw4[64] (FWD_PART floats; summed by k_sum_parts)
    int* err;
    // failure injection (the bounded-wait test only): no MMA is issued or
    // committed, so every wait on the barrier runs out after wait_limit polls
    int no_commit = 0;
    long long wait_limit = MBAR_WAIT_LIMIT;
};

constexpr int FWD_SW1 = 0;                              // [64 x 16]   2 KB
constexpr int FWD_SW2 = FWD_SW1 + 64 * 16 * 2;          // [64 x 64]   8 KB
constexpr int FWD_SW3 = FWD_SW2 + 64 * 64 * 2;          // [64 x 64]   8 KB
constexpr int FWD_SX = FWD_SW3 + 64 * 64 * 2;           // [128 x 16]  4 KB
constexpr int FWD_SH1 = FWD_SX + 128 * 16 * 2;          // [128 x 64] 16 KB
constexpr int FWD_SH2 = FWD_SH1 + 128 * 64 * 2;         // [128 x 64] 16 KB
constexpr int FWD_SH3F = FWD_SH2 + 128 * 64 * 2;        // [128 x 64] fp32 32 KB (training)
constexpr int FWD_SMEM_INFER = FWD_SH3F;
constexpr int FWD_SMEM_TRAIN = FWD_SH3F + 128 * 64 * 4;

template <bool TRAIN>
__global__ void __launch_bounds__(128, 1) k_mlp_fwd(FwdIO io) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ float sb[MLP_NUM_BIASES];
    __shared__ float sw4[64];
    const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
    if (warp == 0) tmem_alloc(&tmem_slot, TMEM_COLS_FWD);
    if (t == 0) mbar_init(&mbar, 1);
    stage_weight(smem + FWD_SW1, io.w + W1_OFF, 64, 16);
    stage_weight(smem + FWD_SW2, io.w + W2_OFF, 64, 64);
    stage_weight(smem + FWD_SW3, io.w + W3_OFF, 64, 64);
    for (int i = t; i < MLP_NUM_BIASES; i += 128) sb[i] = io.b[i];
    if (t < 64) sw4[t] = bf16_val(io.w[W4_OFF + t]);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = tmem_slot;
    const uint32_t lane_base = tmem_addr(tbase, 32 * warp, 0);
    uint32_t phase = 0;
    bool alive = true;
    const int ntiles = (io.n + TILE - 1) / TILE;
    for (int tile = blockIdx.x; tile < ntiles && alive; tile += gridDim.x) {
        const int row = tile * TILE + t;
        const bool valid = row < io.n;
        // normalised features -> bf16 A tile [128 x 16]
        {
            float xf[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) xf[k] = 0.0f;
            if (valid) {
#pragma unroll
                for (int k = 0; k < MLP_IN; ++k)
                    xf[k] = (io.feat[(size_t)row * MLP_IN + k] - sb[FMEAN_OFF + k]) * sb[FISTD_OFF + k];
            }
            uint32_t pk[8];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                pk[i] = (uint32_t)bf16_bits(xf[2 * i]) | ((uint32_t)bf16_bits(xf[2 * i + 1]) << 16);
            *reinterpret_cast<uint4*>(smem + FWD_SX + kmajor_offset(t, 0, 128)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            *reinterpret_cast<uint4*>(smem + FWD_SX + kmajor_offset(t, 8, 128)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            if (TRAIN && valid) {
                uint4* dst = reinterpret_cast<uint4*>(io.x16 + (size_t)row * 16);
                dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            }
        }
        // ---- layer 1: TMEM cols [0, 64)
        sync_for_mma();
        if (t == 0 && !io.no_commit) {
            gemm_issue(tbase, smem + FWD_SX, smem + FWD_SW1, 64, 16, 0);
            commit(&mbar);
        }
        if (!wait_mma(&mbar, phase, io.err, io.wait_limit)) { alive = false; break; }
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            float v[16];
            tmem_ld16(lane_base + 16 * c, v);
            tmem_wait_ld();
            float g[16];
#pragma unroll
            for (int i = 0; i < 16; i += 2) {
                const float2 z = vadd(make_float2(v[i], v[i + 1]), make_float2(sb[B1_OFF + 16 * c + i], sb[B1_OFF + 16 * c + i + 1]));
                g[i] = TRAIN ? gelu_grad(z.x) : 0.0f;
                g[i + 1] = TRAIN ? gelu_grad(z.y) : 0.0f;
                const float2 hh = gelu2(z);
                v[i] = hh.x;
                v[i + 1] = hh.y;
            }
            put_row64(smem + FWD_SH1, t, v, 16 * c);
            if (TRAIN && valid) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    io.h1[(size_t)row * 64 + 16 * c + i] = bf16_bits(v[i]);
                    io.g1[(size_t)row * 64 + 16 * c + i] = bf16_bits(g[i]);
                }
            }
        }
        // ---- layer 2: TMEM cols [64, 128)
        sync_for_mma();
        if (t == 0 && !io.no_commit) {
            gemm_issue(tbase + 64, smem + FWD_SH1, smem + FWD_SW2, 64, 64, 0);
            commit(&mbar);
        }
        if (!wait_mma(&mbar, phase, io.err, io.wait_limit)) { alive = false; break; }
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            float v[16];
            tmem_ld16(lane_base + 64 + 16 * c, v);
            tmem_wait_ld();
            float g[16];
#pragma unroll
            for (int i = 0; i < 16; i += 2) {
                const float2 z = vadd(make_float2(v[i], v[i + 1]), make_float2(sb[B2_OFF + 16 * c + i], sb[B2_OFF + 16 * c + i + 1]));
                g[i] = TRAIN ? gelu_grad(z.x) : 0.0f;
                g[i + 1] = TRAIN ? gelu_grad(z.y) : 0.0f;
                const float2 hh = gelu2(z);
                v[i] = hh.x;
                v[i + 1] = hh.y;
            }
            put_row64(smem + FWD_SH2, t, v, 16 * c);
            if (TRAIN && valid) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    io.h2[(size_t)row * 64 + 16 * c + i] = bf16_bits(v[i]);
                    io.g2[(size_t)row * 64 + 16 * c + i] = bf16_bits(g[i]);
                }
            }
        }
        // ---- layer 3: TMEM cols [0, 64) again (layer 1's values were consumed
        // before layer 2 was issued), then the output layer on CUDA cores
        sync_for_mma();
        if (t == 0 && !io.no_commit) {
            gemm_issue(tbase, smem + FWD_SH2, smem + FWD_SW3, 64, 64, 0);
            commit(&mbar);
        }
        if (!wait_mma(&mbar, phase, io.err, io.wait_limit)) { alive = false; break; }
        float y = sb[B4_OFF];
        float* h3f = reinterpret_cast<float*>(smem + FWD_SH3F) + t * 64;
#pragma unroll 1
        for (int c = 0; c < 4; ++c) {
            float v[16];
            tmem_ld16(lane_base + 16 * c, v);
            tmem_wait_ld();
            float hs[16];
#pragma unroll
            for (int i = 0; i < 16; i += 2) {
                const float2 hh = gelu2(vadd(make_float2(v[i], v[i + 1]),
                                             make_float2(sb[B3_OFF + 16 * c + i], sb[B3_OFF + 16 * c + i + 1])));
                hs[i] = hh.x;
                hs[i + 1] = hh.y;
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float z = v[i] + sb[B3_OFF + 16 * c + i];
                const float h = hs[i];
                y = __fmaf_rn(h, sw4[16 * c + i], y);
                if (TRAIN) {
                    h3f[16 * c + i] = h;
                    // the derivative is stored in dz3 for now and scaled once dy is known
                    if (valid) io.dz3[(size_t)row * 64 + 16 * c + i] = bf16_bits(gelu_grad(z));
                }
            }
        }
        if (!TRAIN) {
            if (valid) {
                float lam0 = y * sb[OSCALE_OFF];
                if (io.q && io.clamp > 0.0f) {
                    // trust region around the plain lambda of the same pass (q.w):
                    // same sign, at most clamp times its magnitude
                    const float lp = reinterpret_cast<const float*>(io.q)[4 * (size_t)row + 3];
                    const float a = io.clamp * lp;
                    const float f0 = io.floor ? lp : 0.0f;  // the weak end of the interval
                    lam0 = fminf(fmaxf(lam0, fminf(a, f0)), fmaxf(a, f0));
                }
                if (io.out) io.out[row] = lam0;
                if (io.q) reinterpret_cast<float*>(io.q)[4 * (size_t)row + 3] = lam0;
                if (io.lam_acc) io.lam_acc[row] = lam0;
            }
        } else {
            // loss = mean (y - target/scale)^2 ; dy = 2 (y - t) / B
            const float r = valid ? (y - io.target[row] / sb[OSCALE_OFF]) : 0.0f;
            const float dy = 2.0f * r * io.inv_batch;
            float l = r * r * io.inv_batch, db = dy;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                l += __shfl_xor_sync(0xffffffffu, l, o);
                db += __shfl_xor_sync(0xffffffffu, db, o);
            }
            // this warp's sums go to its own slot; k_sum_parts adds the slots in a
            // fixed order, so the gradients do not depend on the blocks' timing
            float* slot = io.part + ((size_t)tile * 4 + warp) * FWD_PART;
            if (lane == 0) {
                slot[0] = l;
                slot[1] = db;
            }
            for (int nn = 0; nn < 64; ++nn) {
                float gwn = dy * h3f[nn];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) gwn += __shfl_xor_sync(0xffffffffu, gwn, o);
                if (lane == 0) slot[2 + nn] = gwn;
                if (valid) {
                    const size_t at = (size_t)row * 64 + nn;
                    io.dz3[at] = bf16_bits(dy * sw4[nn] * bf16_val(io.dz3[at]));
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, TMEM_COLS_FWD);
}

// ---------------------------------------------------------------------------
// Backward through one hidden layer (Kin inputs, 64 outputs) for 128-row tiles:
//   dW[64 x Kin] += dZ^T H   and db += column sums of dZ  (one MMA: a ones row is
//                                                           appended to H^T)
//   dH = dZ W, dZ_prev = dH * gelu'(Z_prev)                 (second MMA, if any)
// ---------------------------------------------------------------------------
struct BwdIO {
    const uint16_t* dz;     // [n][64]
    const uint16_t* h;      // [n][Kin] layer input (bf16)
    const uint16_t* w;      // W [64][Kin]
    const uint16_t* gprev;  // [n][Kin] gelu' of the layer input, null for the first layer
    uint16_t* dz_prev;      // [n][Kin] out, null for the first layer
    float* part;            // per tile: dW [64][Kin] then db [64] (summed by k_sum_parts)
    int n;
    int* err;
};

template <int KIN>
__global__ void __launch_bounds__(128, 1) k_mlp_bwd(BwdIO io) {
    constexpr int NB = KIN + 16;  // H^T rows plus the ones row (padded to a multiple of 16)
    // TMEM: dW | db in columns [0, NB), dH in [128, 128 + KIN). The first layer
    // (KIN = 16) has no dH and needs 128 columns; its smaller footprint lets 3
    // CTAs share an SM, and 3 x 128 columns stay within the SM's 512.
    constexpr uint32_t TCOLS = KIN == 16 ? 128 : 256;
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t* sDZ = smem;                       // [128 x 64]  A of dH = dZ W
    uint8_t* sDZT = sDZ + 128 * 64 * 2;        // [128 x 128] A of dW (rows 64.. zero)
    uint8_t* sHT = sDZT + 128 * 128 * 2;       // [NB x 128]  B of dW
    uint8_t* sWT = sHT + NB * 128 * 2;         // [KIN x 64]  B of dH
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    const int t = threadIdx.x, warp = t >> 5;
    const bool with_dh = io.dz_prev != nullptr && TCOLS >= 128 + KIN;
    if (warp == 0) tmem_alloc(&tmem_slot, TCOLS);
    if (t == 0) mbar_init(&mbar, 1);
    if (with_dh) stage_weight_t(sWT, io.w, KIN);
    // rows 64..127 of dZ^T stay zero
    for (int i = t; i < 64 * 128 / 8; i += 128) {
        const int r = 64 + i / 16, j = i % 16;
        *reinterpret_cast<uint4*>(sDZT + kmajor_offset(r, 8 * j, 128)) = make_uint4(0, 0, 0, 0);
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = tmem_slot;
    const uint32_t lane_base = tmem_addr(tbase, 32 * warp, 0);
    uint32_t phase = 0;
    const int ntiles = (io.n + TILE - 1) / TILE;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int m = t;
        const int row = tile * TILE + m;
        const bool valid = row < io.n;
        // dZ row m -> sDZ row m and column m of sDZT
        for (int j = 0; j < 8; ++j) {
            uint4 v = make_uint4(0, 0, 0, 0);
            if (valid) v = *reinterpret_cast<const uint4*>(io.dz + (size_t)row * 64 + 8 * j);
            *reinterpret_cast<uint4*>(sDZ + kmajor_offset(m, 8 * j, 128)) = v;
            const uint16_t* e = reinterpret_cast<const uint16_t*>(&v);
#pragma unroll
            for (int i = 0; i < 8; ++i) *reinterpret_cast<uint16_t*>(sDZT + kmajor_offset(8 * j + i, m, 128)) = e[i];
        }
        // H row m -> column m of sHT, then the ones row and zero padding
        for (int k = 0; k < KIN; ++k)
            *reinterpret_cast<uint16_t*>(sHT + kmajor_offset(k, m, NB)) = valid ? io.h[(size_t)row * KIN + k] : 0;
        for (int k = KIN; k < NB; ++k)
            *reinterpret_cast<uint16_t*>(sHT + kmajor_offset(k, m, NB)) = (k == KIN && valid) ? 0x3F80 : 0;
        sync_for_mma();
        if (t == 0) {
            gemm_issue(tbase, sDZT, sHT, NB, 128, 0);  // dW | db in TMEM cols [0, NB)
            if (with_dh) gemm_issue(tbase + 128, sDZ, sWT, KIN, 64, 0);  // dH in cols [128, 128 + KIN)
            commit(&mbar);
        }
        if (!wait_mma(&mbar, phase, io.err)) break;
        if (warp < 2) {  // rows 0..63 of the dW product: output unit m, into this tile's slot
            float* slot = io.part + (size_t)tile * (64 * KIN + 64);
#pragma unroll 1
            for (int c = 0; c < NB / 16; ++c) {
                float v[16];
                tmem_ld16(lane_base + 16 * c, v);
                tmem_wait_ld();
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int k = 16 * c + i;
                    if (k < KIN) slot[m * KIN + k] = v[i];
                    else if (k == KIN) slot[64 * KIN + m] = v[i];
                }
            }
        }
        if (with_dh) {
#pragma unroll 1
            for (int c = 0; c < KIN / 16; ++c) {
                float v[16];
                tmem_ld16(lane_base + 128 + 16 * c, v);
                tmem_wait_ld();
                if (valid) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const size_t at = (size_t)row * KIN + 16 * c + i;
                        io.dz_prev[at] = bf16_bits(v[i] * bf16_val(io.gprev[at]));
                    }
                }
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, TCOLS);
}

// ---------------------------------------------------------------------------
// Adam on the FP32 master parameters; refreshes the BF16 weights
// ---------------------------------------------------------------------------
__global__ void k_adam(float* p, float* m, float* v, const float* g, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2, uint16_t* p16) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float upd = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    const float pi = p[i] - upd;
    p[i] = pi;
    if (p16) p16[i] = bf16_bits(pi);
}

__global__ void k_to_bf16(const float* p, uint16_t* q, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) q[i] = bf16_bits(p[i]);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}

int mlp_infer(const uint16_t* w_bf16, const float* b, const float* feat, int n, float* out, float4* q, float* lam_acc,
              float clamp, int floor, int* err, cudaStream_t st) {
    if (n <= 0) return 0;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_mlp_fwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM_INFER) !=
            cudaSuccess)
            return -1;
        attr = true;
    }
    FwdIO io{};
    io.w = w_bf16;
    io.b = b;
    io.feat = feat;
    io.n = n;
    io.out = out;
    io.q = q;
    io.lam_acc = lam_acc;
    io.clamp = clamp;
    io.floor = floor;
    io.err = err;
    // four CTAs per SM (54 KB of shared memory and 128 TMEM columns each) overlap
    // one another's tensor-core waits
    const int tiles = (n + TILE - 1) / TILE;
    const int grid = tiles < 4 * sm_count() ? tiles : 4 * sm_count();
    k_mlp_fwd<false><<<grid, 128, FWD_SMEM_INFER, st>>>(io);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int mlp_infer_uncommitted(const uint16_t* w_bf16, const float* b, const float* feat, int n, float* out,
                          long long wait_limit, int* err, cudaStream_t st) {
    if (n <= 0) return 0;
    if (cudaFuncSetAttribute(k_mlp_fwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM_INFER) !=
        cudaSuccess)
        return -1;
    FwdIO io{};
    io.w = w_bf16;
    io.b = b;
    io.feat = feat;
    io.n = n;
    io.out = out;
    io.err = err;
    io.no_commit = 1;
    io.wait_limit = wait_limit;
    const int tiles = (n + TILE - 1) / TILE;
    k_mlp_fwd<false><<<tiles, 128, FWD_SMEM_INFER, st>>>(io);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

struct MlpTrainer {
    int cap = 0;
    float *w32 = nullptr, *b32 = nullptr, *mw = nullptr, *vw = nullptr, *mb = nullptr, *vb = nullptr;
    float *gw = nullptr, *gb = nullptr, *loss = nullptr;
    float* part = nullptr;  // gradient partials per tile (and warp), summed in a fixed order
    int* err = nullptr;
    uint16_t *w16 = nullptr, *x16 = nullptr, *h1 = nullptr, *h2 = nullptr, *g1 = nullptr, *g2 = nullptr,
             *dz3 = nullptr, *dz2 = nullptr, *dz1 = nullptr;
    int step = 0;
};

MlpTrainer* mlp_trainer_create(int max_batch, const float* w32, const float* b32) {
    MlpTrainer* t = new MlpTrainer();
    t->cap = max_batch;
    bool ok = true;
    auto A = [&](void** p, size_t bytes) {
        if (ok && cudaMalloc(p, bytes) != cudaSuccess) ok = false;
        if (ok) cudaMemset(*p, 0, bytes);
    };
    A((void**)&t->w32, sizeof(float) * MLP_NUM_WEIGHTS);
    A((void**)&t->b32, sizeof(float) * MLP_NUM_BIASES);
    A((void**)&t->mw, sizeof(float) * MLP_NUM_WEIGHTS);
    A((void**)&t->vw, sizeof(float) * MLP_NUM_WEIGHTS);
    A((void**)&t->mb, sizeof(float) * MLP_NUM_BIASES);
    A((void**)&t->vb, sizeof(float) * MLP_NUM_BIASES);
    A((void**)&t->gw, sizeof(float) * MLP_NUM_WEIGHTS);
    A((void**)&t->gb, sizeof(float) * MLP_NUM_BIASES);
    A((void**)&t->loss, sizeof(float));
    A((void**)&t->err, sizeof(int));
    A((void**)&t->w16, sizeof(uint16_t) * MLP_NUM_WEIGHTS);
    const size_t cap = (size_t)max_batch;
    A((void**)&t->x16, sizeof(uint16_t) * cap * 16);
    A((void**)&t->h1, sizeof(uint16_t) * cap * 64);
    A((void**)&t->h2, sizeof(uint16_t) * cap * 64);
    A((void**)&t->g1, sizeof(uint16_t) * cap * 64);
    A((void**)&t->g2, sizeof(uint16_t) * cap * 64);
    A((void**)&t->dz3, sizeof(uint16_t) * cap * 64);
    A((void**)&t->dz2, sizeof(uint16_t) * cap * 64);
    A((void**)&t->dz1, sizeof(uint16_t) * cap * 64);
    const size_t tiles = (cap + TILE - 1) / TILE;
    A((void**)&t->part, sizeof(float) * tiles * std::max<size_t>(64 * 64 + 64, 4 * FWD_PART));
    if (!ok) {
        mlp_trainer_destroy(t);
        return nullptr;
    }
    cudaMemcpy(t->w32, w32, sizeof(float) * MLP_NUM_WEIGHTS, cudaMemcpyHostToDevice);
    cudaMemcpy(t->b32, b32, sizeof(float) * MLP_NUM_BIASES, cudaMemcpyHostToDevice);
    k_to_bf16<<<(MLP_NUM_WEIGHTS + 255) / 256, 256>>>(t->w32, t->w16, MLP_NUM_WEIGHTS);
    if (cudaDeviceSynchronize() != cudaSuccess) {
        mlp_trainer_destroy(t);
        return nullptr;
    }
    return t;
}

void mlp_trainer_destroy(MlpTrainer* t) {
    if (!t) return;
    void* ps[] = {t->w32, t->b32, t->mw, t->vw, t->mb, t->vb, t->gw, t->gb, t->loss, t->err, t->w16,
                  t->x16, t->h1, t->h2, t->g1, t->g2, t->dz3, t->dz2, t->dz1, t->part};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete t;
}

int mlp_gradients(MlpTrainer* t, const float* feat, const float* target, int B, cudaStream_t st) {
    if (B <= 0 || B > t->cap) return -1;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_mlp_fwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM_TRAIN) !=
                cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_bwd<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 128 * 64 * 2 + 128 * 128 * 2 + 80 * 128 * 2 + 64 * 64 * 2) != cudaSuccess ||
            cudaFuncSetAttribute(k_mlp_bwd<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 128 * 64 * 2 + 128 * 128 * 2 + 32 * 128 * 2 + 16 * 64 * 2) != cudaSuccess)
            return -1;
        attr = true;
    }
    cudaMemsetAsync(t->gw, 0, sizeof(float) * MLP_NUM_WEIGHTS, st);
    cudaMemsetAsync(t->gb, 0, sizeof(float) * MLP_NUM_BIASES, st);
    cudaMemsetAsync(t->loss, 0, sizeof(float), st);
    const int tiles = (B + TILE - 1) / TILE;
    const int grid = tiles < sm_count() ? tiles : sm_count();
    FwdIO f{};
    f.w = t->w16;
    f.b = t->b32;
    f.feat = feat;
    f.n = B;
    f.target = target;
    f.inv_batch = 1.0f / (float)B;
    f.x16 = t->x16;
    f.h1 = t->h1;
    f.h2 = t->h2;
    f.g1 = t->g1;
    f.g2 = t->g2;
    f.dz3 = t->dz3;
    f.part = t->part;
    f.err = t->err;
    k_mlp_fwd<true><<<grid, 128, FWD_SMEM_TRAIN, st>>>(f);
    // the output layer's sums: loss, db4, dw4 (each its own sum over the slots)
    k_sum_parts<<<1, 64, 0, st>>>(t->part, tiles * 4, FWD_PART, 1, t->loss);
    k_sum_parts<<<1, 64, 0, st>>>(t->part + 1, tiles * 4, FWD_PART, 1, t->gb + B4_OFF);
    k_sum_parts<<<1, 64, 0, st>>>(t->part + 2, tiles * 4, FWD_PART, 64, t->gw + W4_OFF);
    // hidden layers: dW then db of each, from its per-tile slots
    auto layer_sums = [&](int kin, float* gw, float* gb) {
        const int stride = 64 * kin + 64;
        k_sum_parts<<<(64 * kin + 255) / 256, 256, 0, st>>>(t->part, tiles, stride, 64 * kin, gw);
        k_sum_parts<<<1, 64, 0, st>>>(t->part + 64 * kin, tiles, stride, 64, gb);
    };
    BwdIO b3{t->dz3, t->h2, t->w16 + W3_OFF, t->g2, t->dz2, t->part, B, t->err};
    k_mlp_bwd<64><<<grid, 128, 128 * 64 * 2 + 128 * 128 * 2 + 80 * 128 * 2 + 64 * 64 * 2, st>>>(b3);
    layer_sums(64, t->gw + W3_OFF, t->gb + B3_OFF);
    BwdIO b2{t->dz2, t->h1, t->w16 + W2_OFF, t->g1, t->dz1, t->part, B, t->err};
    k_mlp_bwd<64><<<grid, 128, 128 * 64 * 2 + 128 * 128 * 2 + 80 * 128 * 2 + 64 * 64 * 2, st>>>(b2);
    layer_sums(64, t->gw + W2_OFF, t->gb + B2_OFF);
    BwdIO b1{t->dz1, t->x16, t->w16 + W1_OFF, nullptr, nullptr, t->part, B, t->err};
    k_mlp_bwd<16><<<grid, 128, 128 * 64 * 2 + 128 * 128 * 2 + 32 * 128 * 2 + 16 * 64 * 2, st>>>(b1);
    layer_sums(16, t->gw + W1_OFF, t->gb + B1_OFF);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int mlp_adam(MlpTrainer* t, float lr, float beta1, float beta2, float eps, cudaStream_t st) {
    t->step += 1;
    const float c1 = 1.0f - powf(beta1, (float)t->step), c2 = 1.0f - powf(beta2, (float)t->step);
    k_adam<<<(MLP_NUM_WEIGHTS + 255) / 256, 256, 0, st>>>(t->w32, t->mw, t->vw, t->gw, MLP_NUM_WEIGHTS, lr, beta1,
                                                           beta2, eps, c1, c2, t->w16);
    k_adam<<<1, 256, 0, st>>>(t->b32, t->mb, t->vb, t->gb, MLP_NUM_TRAINED_BIASES, lr, beta1, beta2, eps, c1, c2,
                              nullptr);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int mlp_read(MlpTrainer* t, float* w32, float* b32, float* gw, float* gb, float* loss, int* err) {
    cudaDeviceSynchronize();
    if (w32) cudaMemcpy(w32, t->w32, sizeof(float) * MLP_NUM_WEIGHTS, cudaMemcpyDeviceToHost);
    if (b32) cudaMemcpy(b32, t->b32, sizeof(float) * MLP_NUM_BIASES, cudaMemcpyDeviceToHost);
    if (gw) cudaMemcpy(gw, t->gw, sizeof(float) * MLP_NUM_WEIGHTS, cudaMemcpyDeviceToHost);
    if (gb) cudaMemcpy(gb, t->gb, sizeof(float) * MLP_NUM_BIASES, cudaMemcpyDeviceToHost);
    if (loss) cudaMemcpy(loss, t->loss, sizeof(float), cudaMemcpyDeviceToHost);
    if (err) cudaMemcpy(err, t->err, sizeof(int), cudaMemcpyDeviceToHost);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

const uint16_t* mlp_weights_bf16(MlpTrainer* t) { return t->w16; }
const float* mlp_biases(MlpTrainer* t) { return t->b32; }

}  // namespace pbf
