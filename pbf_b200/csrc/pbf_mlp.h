// Learned lambda warm start: host-side interface of pbf_mlp.cu.
//
// Network: 12 features -> 64 -> 64 -> 64 -> 1, GELU (tanh form) after each
// hidden layer, BF16 weights, FP32 accumulation. Parameter arrays:
//   weights (BF16 for the kernels, FP32 masters in the trainer), row-major [out][in]:
//     W1 [64][16] (inputs 12..15 are zero padding), W2 [64][64], W3 [64][64], w4 [64]
//   biases and constants (FP32):
//     b1[64], b2[64], b3[64], b4, feature mean[16], feature 1/std[16], output scale
// lambda0 = (w4 . h3 + b4) * output scale, with the features normalised as
// (f - mean) * (1/std) before the first layer.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pbf {

constexpr int MLP_IN = 12;
constexpr int MLP_K1 = 16;
constexpr int MLP_H = 64;
constexpr int W1_OFF = 0;
constexpr int W2_OFF = W1_OFF + MLP_H * MLP_K1;
constexpr int W3_OFF = W2_OFF + MLP_H * MLP_H;
constexpr int W4_OFF = W3_OFF + MLP_H * MLP_H;
constexpr int MLP_NUM_WEIGHTS = W4_OFF + MLP_H;  // 9280
constexpr int B1_OFF = 0;
constexpr int B2_OFF = 64;
constexpr int B3_OFF = 128;
constexpr int B4_OFF = 192;
constexpr int FMEAN_OFF = 193;
constexpr int FISTD_OFF = 209;
constexpr int OSCALE_OFF = 225;
constexpr int MLP_NUM_BIASES = 226;
constexpr int MLP_NUM_TRAINED_BIASES = 193;  // b1, b2, b3, b4

// Tile GEMM on the tensor cores, D[128 x N] = A[128 x K] * B[N x K]^T
// (BF16 row-major inputs, FP32 row-major output); N, K multiples of 16, <= 256.
int tc_gemm_bf16(const void* A, const void* B, float* D, int N, int K, int* err, cudaStream_t st);

// Inference: lambda0 for `n` rows of raw features feat[n][12]. Writes lambda0 to
// out (if not null), to q[k].w (if not null) and to lam_acc (if not null). With q
// and clamp > 0, lambda0 is kept to the sign of the plain lambda in q[k].w and
// to at most clamp times its magnitude (and, with floor, to at least its
// magnitude).
int mlp_infer(const uint16_t* w_bf16, const float* b, const float* feat, int n, float* out, float4* q,
              float* lam_acc, float clamp, int floor, int* err, cudaStream_t st);
// failure injection (tests): the same kernel with no MMA committed to its
// barrier, each wait limited to wait_limit polls
int mlp_infer_uncommitted(const uint16_t* w_bf16, const float* b, const float* feat, int n, float* out,
                          long long wait_limit, int* err, cudaStream_t st);

struct MlpTrainer;
MlpTrainer* mlp_trainer_create(int max_batch, const float* w32, const float* b32);
void mlp_trainer_destroy(MlpTrainer* t);
// Gradients of the mean squared error of (network output) vs target / output
// scale over a batch; accumulates into the trainer's gradient buffers (cleared first).
int mlp_gradients(MlpTrainer* t, const float* feat, const float* target, int B, cudaStream_t st);
// One Adam step with the current gradients.
int mlp_adam(MlpTrainer* t, float lr, float beta1, float beta2, float eps, cudaStream_t st);
int mlp_read(MlpTrainer* t, float* w32, float* b32, float* gw, float* gb, float* loss, int* err);
const uint16_t* mlp_weights_bf16(MlpTrainer* t);
const float* mlp_biases(MlpTrainer* t);

}  // namespace pbf
