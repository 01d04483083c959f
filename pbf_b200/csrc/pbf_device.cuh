// Device-side arithmetic of one PBF substep (sm_100a).
//
// The library is compiled with -fmad=false: a multiply followed by an add is
// never fused by the compiler, and every fused multiply-add below is an explicit
// __fmaf_rn at a documented place. Square roots and divisions are the IEEE
// round-to-nearest forms. Together these make each per-particle result a fixed
// sequence of IEEE operations that a CPU evaluation of the same sequence
// reproduces bit for bit.
//
// Formulas follow the reference CUDA kernels (kernels/cudaPBFSolver.cuh:99-181,
// kernels/cudaPBFSolver.cu:4-239); the departures in evaluation order are:
//   * poly6: (h^2-r^2)^3 by two multiplies instead of powf(.,3) (cuh:102)
//   * spiky gradient: one reciprocal square root y = pbf_rsqrt(|r|^2), |r| = |r|^2 y
//     for the cutoff, h - |r| = fma(-|r|^2, y, h), s = c (h-|r|)^2 y, then s * r,
//     instead of powf(.,2) and normalize (cuh:106-109)
//   * the dp pair weight (lambda_i + lambda_j) + s_corr as one fused multiply-add,
//     fma(-k (W/W(dq))^n, scorr_scale, lambda_i + lambda_j) (cu:193-195)
//   * the curl's cross product with one fused multiply-add per component,
//     fma(a_y, b_z, -(a_z b_y)) and its rotations (cu:211)
//   * s_corr exponent: repeated multiplication for integer n in [1,8] (cuh:143)
//   * |r|^2 and every neighbour sum use fused multiply-adds in a fixed order
//   * the wall-jitter hash evaluates sine with pbf_det_sin (double precision)
//     instead of sinf (cuh:117), so that a CPU evaluation reproduces it.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pbf {

// Flags (mirrors include/pbf.h PBF_FLAG_*)
enum : unsigned {
    FLAG_CLAMP_C = 1u,        // unilateral density constraint: C = max(C, 0)
    FLAG_XSPH_RHO = 2u,       // XSPH weight c / rho0
    FLAG_WALL_DENSITY = 4u,   // walls carry the density of a fluid half-space (wall_term)
};

// Error bits written by kernels into the device status word.
enum : int {
    DEVERR_SCAN_TIMEOUT = 1,    // decoupled look-back gave up waiting for a predecessor
    DEVERR_BAD_INDEX = 2,       // a neighbour or slot index fell outside [0, n)
    DEVERR_NONFINITE = 4,       // a non-finite position appeared
    DEVERR_MLP_TIMEOUT = 8,     // tensor-core pipeline gave up waiting on an mbarrier
};

// One scene of a batch: its uniform grid, wall box and obstacle, and where its
// cell keys and particle slots lie in the batch-wide arrays. Keys of scene s are
// cell_base .. cell_base + ncells, the last one being the scene's out-of-grid
// bin, so a single scan over all keys keeps every scene's particles contiguous.
struct SceneView {
    float gmin[3];
    float bmin[3], bmax[3];
    float sphere[4];
    int dims[3];
    int cell_base;  // first key of the scene
    int ncells;     // real cells; key cell_base + ncells is the out-of-grid bin
    int pbase;      // first particle slot of the scene
    int pcount;
};

struct KParams {
    // kernel constants, all computed on the host (pbf_capi.cu: make_kparams)
    float h, h2, cell, inv_cell, poly6_c, spiky_c, inv_wdq, nk, scorr_scale, n_exp;
    float rho0, rho0sq, eps, dt, jit, rmin, visc_c, vort_eps;
    float g[3];
    SceneView sc0;              // the scene when there is one
    const SceneView* scenes;    // device table when nscenes > 1
    const int* sid;             // per slot: scene index (slots never leave their scene)
    int nscenes;
    int nkeys;      // cell keys over all scenes (cells + one out-of-grid bin per scene)
    int radius;     // stencil radius in cells: ceil(1 / cell_scale)
    int n;          // particles
    int block;      // threads per block of the neighbour passes
    int lanes;      // pair lanes per particle of the neighbour passes (1, 2, 4, 8)
    int max_nbr;    // neighbour cap (reference MAX_NEIGHBOR = 63)
    int stride;     // neighbour list stride (slot-major layout: nbr[q * stride + k])
    int cell_order; // 0 ascending, 1 descending within a cell
    int n_int;      // s_corr exponent when a small integer, else 0
    int persistent; // neighbour passes: resident blocks striding over the tiles of slots
    unsigned flags;
    double poly6_c64;  // exact poly6 constant for the FP64 density reduction
    // wall density: n_wall (rest number density), 1/h, 315/(256 h), Horner coefficients
    float wall_n, inv_h, wall_kd, wc3, wc5, wc7, wc9;
};

// Device-resident control of one substep's Jacobi loop (adaptive iteration
// counts). The lambda pass of iteration k measures the one-sided density error
// of the positions it sees into slot k; the dp pass of iteration k ends the loop
// when that error is within tol. done == nullptr: fixed iteration count.
struct IterCtl {
    int* done;
    unsigned long long* max_bits;  // per-slot max error as ordered double bits (slot k: after k corrections)
    double* sum;                   // per-slot sum of errors
    int* iters;                    // corrections applied
    int* conv_slot;                // slot whose error met the tolerance
    double tol;
    int slot;                      // this pass's slot; plus *loop_k when loop_k is set
    int min_slot;                  // the loop may end at slots >= min_slot
    const int* loop_k;             // pass counter of a device-side loop (graph while node), or null
    float* lam_acc;                // when set, the lambda pass adds its lambda here (the
                                   // substep's total lambda: warm-start feature and target)
    __device__ __forceinline__ int cur_slot() const { return loop_k ? slot + *loop_k : slot; }
};

// ---- deterministic sine ------------------------------------------------------
// Quadrant reduction by a two-part Cody-Waite split of pi/2 (first 33 bits, then
// the rounded remainder), Taylor series of sin and cos on [-pi/4, pi/4] in Horner
// form, IEEE double throughout, one rounding to float. Accurate to well under one
// float ulp for |a| < 1e6.
__device__ __forceinline__ float pbf_det_sin(float a) {
    const double x = (double)a;
    const double P1 = 1.5707963267341256;
    const double P2 = 6.077100506506192e-11;
    const double q = floor(x * 0.6366197723675814 + 0.5);
    const double r = (x - q * P1) - q * P2;
    const double r2 = r * r;
    const double s = r + r * r2 * (-1.0 / 6.0 + r2 * (1.0 / 120.0 + r2 * (-1.0 / 5040.0 +
                     r2 * (1.0 / 362880.0 + r2 * (-1.0 / 39916800.0 + r2 * (1.0 / 6227020800.0 +
                     r2 * (-1.0 / 1307674368000.0)))))));
    const double c = 1.0 + r2 * (-0.5 + r2 * (1.0 / 24.0 + r2 * (-1.0 / 720.0 +
                     r2 * (1.0 / 40320.0 + r2 * (-1.0 / 3628800.0 + r2 * (1.0 / 479001600.0 +
                     r2 * (-1.0 / 87178291200.0 + r2 * (1.0 / 20922789888000.0))))))));
    const long long qi = (long long)q;
    double res;
    switch ((int)(qi & 3)) {
        case 0: res = s; break;
        case 1: res = c; break;
        case 2: res = -s; break;
        default: res = -c; break;
    }
    return (float)res;
}

struct f3 {
    float x, y, z;
};

__device__ __forceinline__ f3 make3(const float4& a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ f3 sub3(const f3& a, const f3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
// |r|^2 = fma(z, z, fma(y, y, x*x))
__device__ __forceinline__ float dot_fma(const f3& a, const f3& b) {
    return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, a.x * b.x));
}
__device__ __forceinline__ f3 cross3(const f3& a, const f3& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Wpoly6 (cuh:99-103): zero when r2 > h^2, else c * ((t*t)*t), t = h^2 - r2
__device__ __forceinline__ float w_poly6(const KParams& p, float r2) {
    if (r2 > p.h2) return 0.0f;
    const float t = p.h2 - r2;
    return p.poly6_c * ((t * t) * t);
}

// 1/sqrt(x) for normal x > 0: the published bit-level first estimate
// 0x5f3759df - (bits(x) >> 1) (C. Lomont, "Fast Inverse Square Root", 2003),
// then three Newton steps y <- y (3/2 - (x/2) y^2), each with one fused
// multiply-add. Within 2 ulp of the exact value (tests check it against double
// precision); a fixed sequence of integer and IEEE float operations, so a CPU
// evaluation of the same steps reproduces it bit for bit. It replaces an IEEE
// square root and an IEEE division per neighbour pair.
__device__ __forceinline__ float pbf_rsqrt(float x) {
    const float hx = 0.5f * x;
    float y = __int_as_float(0x5f3759df - (__float_as_int(x) >> 1));
#pragma unroll
    for (int i = 0; i < 3; ++i) y = y * __fmaf_rn(-hx, y * y, 1.5f);
    return y;
}

// WspikyGrad (cuh:105-110): zero when |r| > h or |r| < rmin, else ((c*d)*d)/|r| * r
// with d = h - |r|. |r|^2 is clamped to 1e-30 first so that coincident particles
// give |r| ~ 0 (cut by rmin) instead of an infinite estimate. (The pair passes in
// pbf_pairs.cu evaluate the same steps, two pairs per instruction.)
__device__ __forceinline__ f3 grad_spiky(const KParams& p, const f3& r, float r2) {
    const float y = pbf_rsqrt(fmaxf(r2, 1e-30f));
    const float rl = r2 * y;
    if (rl > p.h || rl < p.rmin) return {0.0f, 0.0f, 0.0f};
    const float d = __fmaf_rn(-r2, y, p.h);
    const float s = ((p.spiky_c * d) * d) * y;
    return {s * r.x, s * r.y, s * r.z};
}

// randomOffset (cuh:112-119) with pbf_det_sin in place of sinf
__device__ __forceinline__ float random_offset(float u, float v) {
    const float a = u * 12.9898f;
    const float b = v * 78.233f;
    const float arg = 2.0f * (a + b);
    const float m = pbf_det_sin(arg) * 43758.5453f;
    return fabsf(m - (float)(int)m);
}

// Static sphere obstacle (no reference counterpart): a point inside the sphere is
// moved radially onto its surface.
__device__ __forceinline__ void sphere_project(const SceneView& sc, f3& q) {
    const float R = sc.sphere[3];
    const f3 d = {q.x - sc.sphere[0], q.y - sc.sphere[1], q.z - sc.sphere[2]};
    const float d2 = dot_fma(d, d);
    if (d2 >= R * R || d2 <= 0.0f) return;
    const float s = __fdiv_rn(R, __fsqrt_rn(d2));
    q = {sc.sphere[0] + d.x * s, sc.sphere[1] + d.y * s, sc.sphere[2] + d.z * s};
}

// The scene of slot k (slots never leave their scene's range).
__device__ __forceinline__ SceneView scene_of(const KParams& p, int k) {
    if (p.nscenes == 1) return p.sc0;
    return p.scenes[p.sid[k]];
}

// BoundParticle (cuh:121-140), including the reference's y-max branch that hashes (y, z)
__device__ __forceinline__ void bound_particle(const KParams& p, const SceneView& sc, f3& q) {
    if (q.x < sc.bmin[0]) q.x = sc.bmin[0] + p.jit * random_offset(q.y, q.z);
    if (q.x > sc.bmax[0]) q.x = sc.bmax[0] - p.jit * random_offset(q.y, q.z);
    if (q.y < sc.bmin[1]) q.y = sc.bmin[1] + p.jit * random_offset(q.x, q.z);
    if (q.y > sc.bmax[1]) q.y = sc.bmax[1] - p.jit * random_offset(q.y, q.z);
    if (q.z < sc.bmin[2]) q.z = sc.bmin[2] + p.jit * random_offset(q.x, q.y);
    if (q.z > sc.bmax[2]) q.z = sc.bmax[2] - p.jit * random_offset(q.x, q.y);
    if (sc.sphere[3] > 0.0f) sphere_project(sc, q);
}

// Wall density (no reference counterpart; stable mode). Each face of the boundary
// box is backed by fluid at rest number density n_wall filling the half-space
// beyond it. For a particle at distance d < h from a face, that half-space adds
//   rho_w = n_wall F(s),  F(s) = 1/2 - (315/256) (s - 4/3 s^3 + 6/5 s^5 - 4/7 s^7 + 1/9 s^9),  s = d/h
// (the poly6 mass beyond a plane, integrated in closed form), and its gradient
// along the face normal, d rho_w / dd = -n_wall (315/(256 h)) (1 - s^2)^4.
// The lambda pass adds rho_w and the gradient to rho_i and to grad_i C_i; the dp
// pass adds lambda_i * grad rho_w / rho0.
__device__ __forceinline__ float wall_face(const KParams& p, float d, float& dfdd) {
    d = fmaxf(d, 0.0f);
    const float s = d * p.inv_h;
    const float s2 = s * s;
    float t = __fmaf_rn(s2, p.wc9, p.wc7);
    t = __fmaf_rn(s2, t, p.wc5);
    t = __fmaf_rn(s2, t, p.wc3);
    t = __fmaf_rn(s2, t, 1.0f);
    const float F = 0.5f - 1.23046875f * (s * t);
    const float om = 1.0f - s2;
    const float om2 = om * om;
    dfdd = -p.wall_kd * (om2 * om2);
    return F;
}

__device__ __forceinline__ float wall_term(const KParams& p, const SceneView& sc, const f3& q, f3& g) {
    float rho = 0.0f;
    g = {0.0f, 0.0f, 0.0f};
    const float qa[3] = {q.x, q.y, q.z};
    float ga[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float dlo = qa[a] - sc.bmin[a];
        if (dlo < p.h) {
            float dfdd;
            const float F = wall_face(p, dlo, dfdd);
            rho = rho + p.wall_n * F;
            ga[a] = ga[a] + p.wall_n * dfdd;
        }
        const float dhi = sc.bmax[a] - qa[a];
        if (dhi < p.h) {
            float dfdd;
            const float F = wall_face(p, dhi, dfdd);
            rho = rho + p.wall_n * F;
            ga[a] = ga[a] - p.wall_n * dfdd;
        }
    }
    g = {ga[0], ga[1], ga[2]};
    return rho;
}

// updateParticles (cu:4-13): v += dt g; x += dt v; bound. Each update is one
// fused multiply-add, fma(dt, g, v) and fma(dt, v, x): the single rounding the
// reference's own build gives these two lines (nvcc contracts a product that
// feeds an add by default). With two roundings, a predicted position could sit
// one ulp from the reference's, which flips the neighbour-list membership of
// pairs at exactly h, and such a pair then acts for every Jacobi iteration once
// the corrections bring it within h.
__device__ __forceinline__ void predict(const KParams& p, const SceneView& sc, f3& x, f3& v) {
    v = {__fmaf_rn(p.dt, p.g[0], v.x), __fmaf_rn(p.dt, p.g[1], v.y), __fmaf_rn(p.dt, p.g[2], v.z)};
    x = {__fmaf_rn(p.dt, v.x, x.x), __fmaf_rn(p.dt, v.y, x.y), __fmaf_rn(p.dt, v.z, x.z)};
    bound_particle(p, sc, x);
}

// Run-aggregated histogram of one warp's cell keys (every lane of the warp
// calls it; key < 0: no particle). Slots are in cell order from the previous
// substep, so equal keys come in runs: one atomic per run. Returns the lane's
// ticket, an arrival order within its cell (the reorder makes the order stable).
__device__ __forceinline__ int warp_histogram(int key, int* cnt) {
    const int lane = threadIdx.x & 31;
    const int prev = __shfl_up_sync(0xffffffffu, key, 1);
    const unsigned starts = __ballot_sync(0xffffffffu, lane == 0 || prev != key);
    const unsigned upto = starts & (0xffffffffu >> (31 - lane));  // run starts at or below this lane
    const int leader = 31 - __clz(upto);
    const unsigned above = starts & ~(0xffffffffu >> (31 - lane));
    const int end = above ? __ffs(above) - 1 : 32;  // first run start above this lane
    int base = 0;
    if (key >= 0 && lane == leader) base = atomicAdd(&cnt[key], end - leader);
    return __shfl_sync(0xffffffffu, base, leader) + (lane - leader);
}

// computeDimID (cuh:156-160): truncation toward zero
__device__ __forceinline__ void cell_dims(const KParams& p, const SceneView& sc, const f3& x, int d[3]) {
    d[0] = (int)((x.x - sc.gmin[0]) * p.inv_cell);
    d[1] = (int)((x.y - sc.gmin[1]) * p.inv_cell);
    d[2] = (int)((x.z - sc.gmin[2]) * p.inv_cell);
}

// computeGid (cuh:172-181) offset by the scene's first key; out-of-grid particles
// go to the scene's out-of-grid bin
__device__ __forceinline__ int cell_key(const KParams& p, const SceneView& sc, const f3& x) {
    int d[3];
    cell_dims(p, sc, x, d);
    if (d[0] < 0 || d[0] >= sc.dims[0] || d[1] < 0 || d[1] >= sc.dims[1] || d[2] < 0 || d[2] >= sc.dims[2])
        return sc.cell_base + sc.ncells;
    return sc.cell_base + d[0] + d[1] * sc.dims[0] + d[2] * sc.dims[0] * sc.dims[1];
}

}  // namespace pbf
