// Host-side launchers of the substep kernels (pbf_kernels.cu; the neighbour-sum
// passes launch_lambda, launch_dp, launch_features, launch_curl and launch_vort
// are in pbf_pairs.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "pbf_device.cuh"

struct pbf_solver;  // the solver handle of include/pbf.h

namespace pbf {

void launch_hash(const KParams& p, bool predict_on, const float4* x, const float4* v, int* cell, int* ticket, int* cnt,
                 int* err, cudaStream_t st);
size_t scan_status_bytes(int m);
void launch_scan(int* cnt, int* out, int m, void* status_ws, int* err, cudaStream_t st);
// same scan, input left unchanged
void launch_scan_const(const int* in, int* out, int m, void* status_ws, int* err, cudaStream_t st);
// failure injection (tests): tile silent_tile publishes no status and the
// look-back gives up after spin_limit polls (input left unchanged)
void launch_scan_silent_tile(const int* in, int* out, int m, void* status_ws, int* err, int silent_tile,
                             long long spin_limit, cudaStream_t st);
void launch_scatter(int n, const int* cell, const int* ticket, const int* cell_start, int* tmp, int* err,
                    cudaStream_t st);
void launch_reorder(const KParams& p, bool predict_on, const float4* x, const float4* v, const int* perm,
                    const int* cell, const int* cell_start, const int* tmp, float4* xp, float4* vp, float4* xold,
                    int* perm_out, int* cell_sorted, const float* lam_in, float* lam_out, int* err, cudaStream_t st);
void launch_neighbors(const KParams& p, const float4* x, const int* cell_start, int* nbr, int* ncnt, cudaStream_t st);
void launch_lambda(const KParams& p, bool debug, const float4* x, const int* nbr, const int* ncnt, float4* xl,
                   float* rho, const IterCtl& ctl, cudaStream_t st);
void launch_dp(const KParams& p, bool debug, const float4* xl, const int* nbr, const int* ncnt, const float4* xold,
               float4* xout, float4* vout, float4* dp, const IterCtl& ctl, cudaStream_t st);
void launch_features(const KParams& p, const float4* x, const float4* v, const int* nbr, const int* ncnt,
                     const float* lam_prev, float4* xl, float* feat, float* lam_acc, cudaStream_t st);
// The first lambda pass of a warm-started substep fused with the network on the
// tensor cores: writes xl = (x, lambda0), lam_acc = lam0 = lambda0 (feat only
// when not null). Returns nonzero when the launch could not be configured.
int launch_features_warm(const KParams& p, const float4* x, const float4* v, const int* nbr, const int* ncnt,
                         const float* lam_prev, float4* xl, float* feat, float* lam_acc, const uint16_t* w,
                         const float* b, float* lam0, float clamp, int floor, int* err, cudaStream_t st);
void launch_gather_rows(const int* slots, int count, int n, const float* feat, const float* lam_acc, float* out_feat,
                        float* out_target, int* err, cudaStream_t st);
void launch_count_fallback(const int* iters, int first, int configured, int* fallback, long long* total,
                           cudaStream_t st);
void launch_loop_ctl(cudaGraphConditionalHandle h, int* loop_k, const int* done, int first, int max_it,
                     cudaStream_t st);
void launch_velocity(const KParams& p, const float4* x, const float4* xold, float4* v, cudaStream_t st);
// Curl: omega = (w, |w|) and vw = (v, |w|) per particle.
void launch_curl(const KParams& p, const float4* x, const float4* v, const int* nbr, const int* ncnt, float4* omega,
                 float4* vw, cudaStream_t st);
// Vorticity + XSPH from vw = (v, |w|) and omega; also writes the final state
// (xout = x, vout = v + dv, perm_out = perm_in) and the next substep's grid hash
// of that state: cell key and ticket per slot, counts added to hist (which the
// scan left zero).
void launch_vort(const KParams& p, bool debug, const float4* x, const float4* vw, const float4* omega, const int* nbr,
                 const int* ncnt, float4* xout, float4* vout, const int* perm_in, int* perm_out, float4* vort,
                 float4* visc, int* cell, int* ticket, int* hist, int* err, cudaStream_t st);
void launch_density_error(const KParams& p, const float4* x, const int* nbr, const int* ncnt,
                          unsigned long long* max_bits, double* sum, const int* skip, cudaStream_t st);
void launch_from_aos(int n, const float* pos, const float* vel, float4* x, float4* v, int* perm, int* err,
                     cudaStream_t st);
void launch_to_aos(int n, const float4* a, const int* perm, float* out, int* err, cudaStream_t st);
void launch_copy4(int n, const float4* a, float4* b, cudaStream_t st);
void launch_sorted_state(int n, const float4* x, const float4* v, const int* perm, const int* cell_sorted,
                         const int* cell_start, float* pos, float* vel, int* ids, int* key, int* rank,
                         cudaStream_t st);

// FP32 fused multiply-add throughput of the current device, scalar and packed
// (f32x2), in TFLOP/s; synchronises the device. 0 on success.
int measure_fp32_peak(double* scalar_tflops, double* packed_tflops);

// Records the message returned by pbf_last_error() for this thread; returns code.
int set_last_error(int code, const char* msg);

// Current positions of a solver (float4, slot order) for the renderer (pbf_capi.cu).
int solver_positions(::pbf_solver* s, const float4** x, int* n);

}  // namespace pbf
