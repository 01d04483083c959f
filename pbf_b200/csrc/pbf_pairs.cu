// Neighbour-sum passes of the PBF substep for sm_100a: density and lambda (with
// the warm-start features in the first pass of a substep), the position
// correction, curl, and vorticity confinement + XSPH.
//
// Reference kernels replaced (kernels/cudaPBFSolver.cu): calculateLambda
// :156-180, calculateOffset :182-199, updatePosition :15-22, calculateCurl
// :201-215, calculateVorticityAndViscosity :217-239, applyVorticityAndViscosity
// :24-29.
//
// Pair lanes. A particle's neighbour list is split over P = L * V lanes: L
// consecutive threads of a warp (a team), each evaluating V = 1 or 2 pairs per
// instruction. With V = 2 the pair arithmetic runs on the sm_100 packed FP32
// operations (add/mul/fma.rn.f32x2), each component of which is the scalar
// IEEE operation, so one instruction evaluates two pairs and the
// per-pair results are the scalar ones bit for bit. Lane p = V t + v (thread t,
// component v) takes list entries p, p + P, p + 2P, ... in list order; the lane
// sums are combined by an xor butterfly over distances 1, 2, 4 (first the two
// components of a thread, then across the team by shuffles), which gives
// ((s0 + s1) + (s2 + s3)) + ... on every lane. pair_lanes = P selects
// (L, V): 1 = (1, 1), 2 = (1, 2), 4 = (2, 2), 8 = (4, 2).
//
// A padding component (an entry past the end of the list) contributes +0 to
// every sum, which leaves the sum unchanged: no accumulator is ever -0 (they
// start at +0, and in round-to-nearest x + (-x) = +0 and +0 + (-0) = +0).
#include "pbf_kernels.h"
#include "pbf_mlp.h"
#include "pbf_mlp_dev.cuh"
#include "pbf_packed.cuh"

#include <algorithm>
#include <type_traits>

namespace pbf {

// bit v set: component v greater than / less than s
__device__ __forceinline__ unsigned gt_mask(float a, float s) { return a > s ? 1u : 0u; }
__device__ __forceinline__ unsigned gt_mask(float2 a, float s) { return (a.x > s ? 1u : 0u) | (a.y > s ? 2u : 0u); }
__device__ __forceinline__ unsigned lt_mask(float a, float s) { return a < s ? 1u : 0u; }
__device__ __forceinline__ unsigned lt_mask(float2 a, float s) { return (a.x < s ? 1u : 0u) | (a.y < s ? 2u : 0u); }
// components whose bit in keep is clear become +0
__device__ __forceinline__ float keep_only(float a, unsigned keep) { return (keep & 1u) ? a : 0.0f; }
__device__ __forceinline__ float2 keep_only(float2 a, unsigned keep) {
    return make_float2((keep & 1u) ? a.x : 0.0f, (keep & 2u) ? a.y : 0.0f);
}
// the first butterfly step: the two lanes of a thread
__device__ __forceinline__ float fold(float a) { return a; }
__device__ __forceinline__ float fold(float2 a) { return a.x + a.y; }

// Negated pbf_rsqrt (pbf_device.cuh) on each component, without a negation:
// the steps y <- y fma(-x/2, y^2, 3/2) take -x/2 as the product (-0.5) x, and the
// last step multiplies by fma(x/2, y^2, -3/2) = -fma(-x/2, y^2, 3/2) (round to
// nearest is symmetric in sign), which yields exactly -pbf_rsqrt(x).
__device__ __forceinline__ unsigned rsqrt_seed(float x) { return 0x5f3759df - (__float_as_int(x) >> 1); }
__device__ __forceinline__ float rsqrt_seed_v(float x) { return __int_as_float(rsqrt_seed(x)); }
__device__ __forceinline__ float2 rsqrt_seed_v(float2 x) {
    return make_float2(__int_as_float(rsqrt_seed(x.x)), __int_as_float(rsqrt_seed(x.y)));
}
template <typename T> __device__ __forceinline__ T vrsqrt_neg(T x) {
    const T hx = vmul(bc<T>(0.5f), x);
    const T nhx = vmul(bc<T>(-0.5f), x);
    T y = rsqrt_seed_v(x);
#pragma unroll
    for (int i = 0; i < 2; ++i) y = vmul(y, vfma(nhx, vmul(y, y), bc<T>(1.5f)));
    return vmul(y, vfma(hx, vmul(y, y), bc<T>(-1.5f)));
}

template <typename T> struct T3 {
    T x, y, z;
};
template <typename T> __device__ __forceinline__ T3<T> add3(const T3<T>& a, const T3<T>& b) {
    return {vadd(a.x, b.x), vadd(a.y, b.y), vadd(a.z, b.z)};
}
template <typename T> __device__ __forceinline__ T3<T> zero3() { return {bc<T>(0.0f), bc<T>(0.0f), bc<T>(0.0f)}; }
__device__ __forceinline__ f3 fold3(const T3<float>& a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ f3 fold3(const T3<float2>& a) { return {fold(a.x), fold(a.y), fold(a.z)}; }
// The curl's cross product, one fused multiply-add per component:
// (fma(a_y, b_z, -(a_z b_y)), fma(a_z, b_x, -(a_x b_z)), fma(a_x, b_y, -(a_y b_x))).
// (A packed multiply whose only use is an add may be fused by the code generator,
// so every product that meets an addition in these passes is an explicit fma.)
// -(a b) is taken as (a b) (-1), which is the same value, signed zeros included.
template <typename T> __device__ __forceinline__ T3<T> cross3v(const T3<T>& a, const T3<T>& b) {
    const T m1 = bc<T>(-1.0f);
    return {vfma(a.y, b.z, vmul(vmul(a.z, b.y), m1)), vfma(a.z, b.x, vmul(vmul(a.x, b.z), m1)),
            vfma(a.x, b.y, vmul(vmul(a.y, b.x), m1))};
}

// xyz (or .w) of V gathered float4s as one packet
__device__ __forceinline__ T3<float> pack3(const float4 (&a)[1]) { return {a[0].x, a[0].y, a[0].z}; }
__device__ __forceinline__ T3<float2> pack3(const float4 (&a)[2]) {
    return {make_float2(a[0].x, a[1].x), make_float2(a[0].y, a[1].y), make_float2(a[0].z, a[1].z)};
}
__device__ __forceinline__ float packw(const float4 (&a)[1]) { return a[0].w; }
__device__ __forceinline__ float2 packw(const float4 (&a)[2]) { return make_float2(a[0].w, a[1].w); }

template <int V> using vec_t = typename std::conditional<V == 1, float, float2>::type;

// r = x_k - x_j, |r|^2 = fma(z, z, fma(y, y, x*x)), Wpoly6 (when NEED_W) and the
// spiky gradient of V pairs, exactly as w_poly6 / grad_spiky (pbf_device.cuh)
// evaluate one pair; components outside `valid` give w = +0 and g = +0 or -0.
// Every difference a - b is fma(b, -1, a), which rounds the same exact value
// once (signed zeros included), and the rsqrt comes negated (ny = -y), so no
// operand needs a negation of its own: h - |r| = fma(|r|^2, ny, h), |r| > h is
// |r|^2 ny < -h, and ((c d) d) y = ((-c d) d) ny. The poly6 cutoff |r|^2 > h^2
// is max(h^2 - |r|^2, +0) (the difference is negative exactly when the same
// rounded |r|^2 exceeds h^2, and c (+0)^3 = +0). A padding entry is the particle
// itself (r = +0, |r| below rmin), which the gradient's cutoff already drops;
// only its density weight needs `valid`.
template <typename T, bool NEED_W>
__device__ __forceinline__ void pair_terms(const KParams& p, const f3& xk, const T3<T>& xj, unsigned valid, T3<T>& r,
                                           T& w, T3<T>& g) {
    const T m1 = bc<T>(-1.0f);
    r = {vfma(xj.x, m1, bc<T>(xk.x)), vfma(xj.y, m1, bc<T>(xk.y)), vfma(xj.z, m1, bc<T>(xk.z))};
    const T r2 = vfma(r.z, r.z, vfma(r.y, r.y, vmul(r.x, r.x)));
    if (NEED_W) {
        const T t = vmax(vfma(r2, m1, bc<T>(p.h2)), 0.0f);
        w = keep_only(vmul(bc<T>(p.poly6_c), vmul(vmul(t, t), t)), valid);
    }
    const T ny = vrsqrt_neg(vmax(r2, 1e-30f));
    const T nrl = vmul(r2, ny);               // -|r| for the cutoff
    const T d = vfma(r2, ny, bc<T>(p.h));      // h - |r|
    const T s = vmul(vmul(vmul(bc<T>(-p.spiky_c), d), d), ny);
    const unsigned keep = ~(lt_mask(nrl, -p.h) | gt_mask(nrl, -p.rmin));
    // the mask on the magnitude: a dropped pair gives a gradient of +0 or -0,
    // which leaves every sum it enters unchanged (no accumulator is ever -0)
    const T sk = keep_only(s, keep);
    g = {vmul(sk, r.x), vmul(sk, r.y), vmul(sk, r.z)};
}

// The dp pair weight (lambda_i + lambda_j) + s_corr (cu:193-195, Scorr cuh:142-144)
// as fma(-k (W / W(dq))^n, scorr_scale, lambda_i + lambda_j).
__device__ __forceinline__ float vpow(float q, const KParams& p) { return powf(q, p.n_exp); }
__device__ __forceinline__ float2 vpow(float2 q, const KParams& p) {
    return make_float2(powf(q.x, p.n_exp), powf(q.y, p.n_exp));
}
template <typename T> __device__ __forceinline__ T dp_weight(const KParams& p, float li, T lj, T w) {
    const T q = vmul(w, bc<T>(p.inv_wdq));
    T pw;
    if (p.n_int == 4) {  // the usual n = 4 without a loop: ((q q) q) q
        pw = vmul(vmul(vmul(q, q), q), q);
    } else if (p.n_int > 0) {
        pw = q;
        for (int i = 1; i < p.n_int; ++i) pw = vmul(pw, q);
    } else {
        pw = vpow(q, p);
    }
    return vfma(vmul(bc<T>(p.nk), pw), bc<T>(p.scorr_scale), vadd(bc<T>(li), lj));
}

// ---- teams -------------------------------------------------------------------
template <int L> struct Team {
    int k;          // particle slot
    int t;          // thread within the team
    unsigned mask;  // the team's lanes within the warp
};

// blockDim.x is a multiple of 32, so a team never straddles a warp. vb is the
// virtual block: blockIdx.x for one block per tile of slots, or one of the tiles
// a persistent block strides over.
template <int L> __device__ __forceinline__ Team<L> team_of(int vb) {
    Team<L> m;
    const long long g = (long long)vb * blockDim.x + threadIdx.x;
    m.k = (int)(g / L);
    m.t = (int)(threadIdx.x & (L - 1));
    const int lane = threadIdx.x & 31;
    m.mask = L >= 32 ? 0xffffffffu : (((1u << L) - 1u) << (lane & ~(L - 1)));
    return m;
}

// the butterfly across the team (distances 1, 2 between threads)
template <int L> __device__ __forceinline__ float team_sum(float v, unsigned mask) {
#pragma unroll
    for (int o = 1; o < L; o <<= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}
template <int L> __device__ __forceinline__ f3 team_sum3(f3 v, unsigned mask) {
    return {team_sum<L>(v.x, mask), team_sum<L>(v.y, mask), team_sum<L>(v.z, mask)};
}

// Entries q0 + u P + v (u < B, v < V) of slot k's list; slot k itself past the
// end (its data is then masked). All index loads of a batch are issued before
// the gathers that depend on them.
template <int V, int P, int B>
__device__ __forceinline__ void load_idx(const KParams& p, const int* __restrict__ nbr, int k, int q0, int cnt,
                                         int (&jj)[B][V]) {
#pragma unroll
    for (int u = 0; u < B; ++u)
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int q = q0 + u * P + v;
            jj[u][v] = q < cnt ? nbr[(size_t)q * p.stride + k] : k;
        }
}

// bit v: entry q + v exists (the callers have q < cnt, so bit 0 is always set)
template <int V> __device__ __forceinline__ unsigned valid_bits(int q, int cnt) {
    return V == 1 ? 1u : (q + 1 < cnt ? 3u : 1u);
}

// Block-wide max and sum of a per-thread error, folded into one slot with a
// single pair of atomics per block (max as ordered double bits, value >= 0).
__device__ __forceinline__ void block_error_reduce(float e, unsigned long long* max_bits, double* sum) {
    __shared__ float s_max[32];
    __shared__ float s_sum[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float m = e, s = e;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if (lane == 0) { s_max[warp] = m; s_sum[warp] = s; }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double dsum = 0.0;
        for (int w = 0; w < nw; ++w) { m = fmaxf(m, s_max[w]); dsum += (double)s_sum[w]; }
        atomicMax(max_bits, (unsigned long long)__double_as_longlong((double)m));
        atomicAdd(sum, dsum);
    }
    __syncthreads();  // a persistent block's next tile writes s_max / s_sum again
}

// Neighbour entries per thread and batch: four in every pass (V entries per
// packed instruction, 4 / V instructions' worth of gathers issued together).
template <int V> __host__ __device__ constexpr int batches() { return 4 / V; }

// ---------------------------------------------------------------------------
// a9: density, constraint and lambda (calculateLambda cu:156-180), with the
// one-sided density error of the positions it sees
// ---------------------------------------------------------------------------
// Lambda of slot k from its combined fluid density and gradient sums: the wall
// term, the constraint and the denominator. rhos gains the wall term; err is
// the one-sided error of the fluid density alone.
__device__ __forceinline__ float lambda_tail(const KParams& p, int k, const f3& xk, float& rhos, float gms, f3 g3,
                                             float& err) {
    err = fmaxf(__fdiv_rn(rhos, p.rho0) - 1.0f, 0.0f);
    if (p.flags & FLAG_WALL_DENSITY) {
        f3 gw;
        rhos = rhos + wall_term(p, scene_of(p, k), xk, gw);
        g3 = {g3.x + gw.x, g3.y + gw.y, g3.z + gw.z};
    }
    float C = __fdiv_rn(rhos, p.rho0) - 1.0f;
    if (p.flags & FLAG_CLAMP_C) C = fmaxf(C, 0.0f);
    gms = __fmaf_rn(g3.x, g3.x, gms);
    gms = __fmaf_rn(g3.y, g3.y, gms);
    gms = __fmaf_rn(g3.z, g3.z, gms);
    gms = __fdiv_rn(gms, p.rho0sq);
    return __fdiv_rn(-C, gms + p.eps);
}

template <bool DEBUG, int L, int V>
__device__ __forceinline__ void lambda_tile(const KParams& p, int vb, const float4* __restrict__ x,
                                            const int* __restrict__ nbr, const int* __restrict__ ncnt,
                                            float4* __restrict__ xl, float* __restrict__ rho_out, const IterCtl& ctl) {
    using T = vec_t<V>;
    constexpr int P = L * V, B = batches<V>();
    const Team<L> tm = team_of<L>(vb);
    const int k = tm.k;
    float err = 0.0f;
    if (k < p.n) {
        const f3 xk = make3(x[k]);
        const int cnt = ncnt[k];
        T rho = bc<T>(0.0f), gm = bc<T>(0.0f);
        T3<T> gs = zero3<T>();
        int jj[B][V];
        load_idx<V, P, B>(p, nbr, k, V * tm.t, cnt, jj);
        for (int q0 = V * tm.t; q0 < cnt; q0 += P * B) {
            float4 xj[B][V];
#pragma unroll
            for (int u = 0; u < B; ++u)
#pragma unroll
                for (int v = 0; v < V; ++v) xj[u][v] = x[jj[u][v]];
            // the next batch's indices load while this batch computes
            load_idx<V, P, B>(p, nbr, k, q0 + P * B, cnt, jj);
#pragma unroll
            for (int u = 0; u < B; ++u) {
                const int q = q0 + u * P;
                if (q >= cnt) break;
                T3<T> r, g;
                T w;
                pair_terms<T, true>(p, xk, pack3(xj[u]), valid_bits<V>(q, cnt), r, w, g);
                rho = vadd(rho, w);
                gs = add3(gs, g);
                gm = vfma(g.x, g.x, gm);
                gm = vfma(g.y, g.y, gm);
                gm = vfma(g.z, g.z, gm);
            }
        }
        float rhos = team_sum<L>(fold(rho), tm.mask);
        const float gms = team_sum<L>(fold(gm), tm.mask);
        const f3 g3 = team_sum3<L>(fold3(gs), tm.mask);
        if (tm.t == 0) {
            const float lam = lambda_tail(p, k, xk, rhos, gms, g3, err);
            xl[k] = make_float4(xk.x, xk.y, xk.z, lam);
            if (ctl.lam_acc) ctl.lam_acc[k] += lam;
            if (DEBUG) rho_out[k] = rhos;
        }
    }
    if (ctl.max_bits) {
        const int sl = ctl.cur_slot();
        block_error_reduce(err, ctl.max_bits + sl, ctl.sum + sl);
    }
}

// nvb tiles of blockDim.x slots' teams; the grid strides over them (a grid of
// nvb blocks is the ordinary one-block-per-tile launch)
template <bool DEBUG, int L, int V>
__global__ void __launch_bounds__(256, V == 1 ? 6 : 4) k_lambda(KParams p, int nvb, const float4* __restrict__ x,
                                                                const int* __restrict__ nbr,
                                                                const int* __restrict__ ncnt, float4* __restrict__ xl,
                                                                float* __restrict__ rho_out, IterCtl ctl) {
    if (ctl.done && *ctl.done) return;
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) lambda_tile<DEBUG, L, V>(p, vb, x, nbr, ncnt, xl, rho_out, ctl);
}

// ---------------------------------------------------------------------------
// a17: warm-start features (no reference counterpart), computed in the first
// lambda pass of a substep together with that pass's lambda (the same
// arithmetic as k_lambda, so recording features changes no result):
//   0 neighbour count / cap          1 fluid density / rho0
//   2 previous substep's total lambda
//   3 sum |grad C|^2 (the lambda denominator without eps)
//   4 velocity divergence sum (v_j - v_i) . grad W / rho0 (predicted velocities)
//   5-7 distance to the nearer wall per axis / h, clamped to [0, 4]
//   8 neighbours closer than h/2, / cap
//   9 |sum of (x_i - x_j)| / (h max(count, 1))  (offset of the neighbourhood)
//   10 |sum grad W| h / rho0
//   11 sum |v_j - v_i|^2 (dt / h)^2 / max(count, 1)
// None depends on the grid's cell size. lam_acc starts the substep's total lambda
// at this pass's lambda.
// ---------------------------------------------------------------------------
// One team's particle: writes xl[k] = (x, plain lambda), lam_acc[k] = lambda
// and, when feat is not null, the 12 features; returns true on the team's first
// thread (with the features in f and the plain lambda in lam) when k < n.
template <int L, int V>
__device__ __forceinline__ bool features_one(const KParams& p, const Team<L>& tm, const float4* __restrict__ x,
                                             const float4* __restrict__ v, const int* __restrict__ nbr,
                                             const int* __restrict__ ncnt, const float* __restrict__ lam_prev,
                                             float4* __restrict__ xl, float* __restrict__ feat,
                                             float* __restrict__ lam_acc, float (&f)[12], float& lam) {
    using T = vec_t<V>;
    constexpr int P = L * V, B = batches<V>();
    const int k = tm.k;
    if (k >= p.n) return false;  // uniform over the team
    const f3 xk = make3(x[k]);
    const f3 vk = make3(v[k]);
    const int cnt = ncnt[k];
    T rho = bc<T>(0.0f), gm = bc<T>(0.0f), div = bc<T>(0.0f), close = bc<T>(0.0f), dv2 = bc<T>(0.0f);
    T3<T> gs = zero3<T>(), rs = zero3<T>();
    const float q2 = 0.25f * p.h2;
    int jj[B][V];
    load_idx<V, P, B>(p, nbr, k, V * tm.t, cnt, jj);
    for (int q0 = V * tm.t; q0 < cnt; q0 += P * B) {
        float4 xj[B][V], vj[B][V];
#pragma unroll
        for (int u = 0; u < B; ++u)
#pragma unroll
            for (int c = 0; c < V; ++c) {
                xj[u][c] = x[jj[u][c]];
                vj[u][c] = v[jj[u][c]];
            }
        // the next batch's indices load while this batch computes
        load_idx<V, P, B>(p, nbr, k, q0 + P * B, cnt, jj);
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const int q = q0 + u * P;
            if (q >= cnt) break;
            const unsigned valid = valid_bits<V>(q, cnt);
            T3<T> r, g;
            T w;
            pair_terms<T, true>(p, xk, pack3(xj[u]), valid, r, w, g);
            rho = vadd(rho, w);
            gs = add3(gs, g);
            gm = vfma(g.x, g.x, gm);
            gm = vfma(g.y, g.y, gm);
            gm = vfma(g.z, g.z, gm);
            const T3<T> vv = pack3(vj[u]);
            const T3<T> vji = {vsub(vv.x, bc<T>(vk.x)), vsub(vv.y, bc<T>(vk.y)), vsub(vv.z, bc<T>(vk.z))};
            div = vfma(vji.x, g.x, div);
            div = vfma(vji.y, g.y, div);
            div = vfma(vji.z, g.z, div);
            const T r2 = vfma(r.z, r.z, vfma(r.y, r.y, vmul(r.x, r.x)));
            close = vadd(close, keep_only(bc<T>(1.0f), valid & lt_mask(r2, q2)));
            rs = add3(rs, T3<T>{keep_only(r.x, valid), keep_only(r.y, valid), keep_only(r.z, valid)});
            dv2 = vadd(dv2, keep_only(vfma(vji.z, vji.z, vfma(vji.y, vji.y, vmul(vji.x, vji.x))), valid));
        }
    }
    float rhos = team_sum<L>(fold(rho), tm.mask);
    float gms = team_sum<L>(fold(gm), tm.mask);
    f3 g3 = team_sum3<L>(fold3(gs), tm.mask);
    const float divs = team_sum<L>(fold(div), tm.mask);
    const float closes = team_sum<L>(fold(close), tm.mask);
    const f3 r3 = team_sum3<L>(fold3(rs), tm.mask);
    const float dv2s = team_sum<L>(fold(dv2), tm.mask);
    if (tm.t != 0) return false;
    const SceneView sc = scene_of(p, k);
    const float rho_fluid = rhos;
    const float gsl = __fsqrt_rn(dot_fma(g3, g3));
    if (p.flags & FLAG_WALL_DENSITY) {
        f3 gw;
        rhos = rhos + wall_term(p, sc, xk, gw);
        g3 = {g3.x + gw.x, g3.y + gw.y, g3.z + gw.z};
    }
    float C = __fdiv_rn(rhos, p.rho0) - 1.0f;
    if (p.flags & FLAG_CLAMP_C) C = fmaxf(C, 0.0f);
    gms = __fmaf_rn(g3.x, g3.x, gms);
    gms = __fmaf_rn(g3.y, g3.y, gms);
    gms = __fmaf_rn(g3.z, g3.z, gms);
    gms = __fdiv_rn(gms, p.rho0sq);
    lam = __fdiv_rn(-C, gms + p.eps);
    xl[k] = make_float4(xk.x, xk.y, xk.z, lam);
    lam_acc[k] = lam;

    const float inv_cnt = 1.0f / (float)max(cnt, 1);
    f[0] = (float)cnt / (float)p.max_nbr;
    f[1] = rho_fluid / p.rho0;
    f[2] = lam_prev[k];
    f[3] = gms;
    f[4] = divs / p.rho0;
    const float qa[3] = {xk.x, xk.y, xk.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float dw = fminf(qa[a] - sc.bmin[a], sc.bmax[a] - qa[a]) * p.inv_h;
        f[5 + a] = fminf(fmaxf(dw, 0.0f), 4.0f);
    }
    f[8] = closes / (float)p.max_nbr;
    f[9] = __fsqrt_rn(dot_fma(r3, r3)) * p.inv_h * inv_cnt;
    f[10] = gsl * p.h / p.rho0;
    const float dth = p.dt * p.inv_h;
    f[11] = dv2s * (dth * dth) * inv_cnt;
    if (feat) {
#pragma unroll
        for (int i = 0; i < 12; ++i) feat[(size_t)k * 12 + i] = f[i];
    }
    return true;
}

template <int L, int V>
__global__ void __launch_bounds__(256) k_features(KParams p, int nvb, const float4* __restrict__ x,
                                                  const float4* __restrict__ v, const int* __restrict__ nbr,
                                                  const int* __restrict__ ncnt, const float* __restrict__ lam_prev,
                                                  float4* __restrict__ xl, float* __restrict__ feat,
                                                  float* __restrict__ lam_acc) {
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
        float f[12], lam;
        features_one<L, V>(p, team_of<L>(vb), x, v, nbr, ncnt, lam_prev, xl, feat, lam_acc, f, lam);
    }
}

// ---------------------------------------------------------------------------
// a17, fused: the first lambda pass of a warm-started substep with the network
// in the same kernel. Each block computes its particles' features and plain
// lambda as k_features does; the team leaders write their normalised features
// as BF16 straight into the tensor core's A tile in shared memory (K-major,
// never to HBM), and the block evaluates 12 -> 64 -> 64 -> 64 on the tensor
// cores (one 128-row MMA per tile of rows and layer, issued by one thread,
// accumulated in TMEM, 64 columns per tile) with the GELU epilogues on the CUDA
// cores, then the output layer and the trust region. Thread t runs the
// epilogue of row t: a warp reads its quarter of the TMEM lanes, and the warps
// of the second half of a 256-thread block the second tile's columns. While
// one block waits on its MMAs the SM runs the other resident blocks' gathers.
// The arithmetic is k_mlp_fwd's (same operands, MMA shapes and epilogue), so
// lambda0 is the unfused path's bit for bit.
// ---------------------------------------------------------------------------
struct WarmIO {
    const uint16_t* w;  // BF16 weights (W1 [64][16], W2, W3 [64][64], w4 [64])
    const float* b;     // biases and constants (normalisation, output scale)
    float* lam0;        // lambda0 per slot
    float clamp;        // trust region around the plain lambda (0: none)
    int floor;          // 1: lambda0 at least as strong as the plain lambda
    int* err;           // PBF_DEVERR_MLP_TIMEOUT on an expired tensor-core wait
};

constexpr int FW_SW1 = 0;                     // W1 [64 x 16]  2 KB
constexpr int FW_SW2 = FW_SW1 + 64 * 16 * 2;  // W2 [64 x 64]  8 KB
constexpr int FW_SW3 = FW_SW2 + 64 * 64 * 2;  // W3 [64 x 64]  8 KB
constexpr int FW_SX = FW_SW3 + 64 * 64 * 2;   // X: per tile [128 x 16] BF16, 4 KB; then H: per tile [128 x 64], 16 KB
constexpr int FW_X_TILE = 128 * 16 * 2;
constexpr int FW_H_TILE = 128 * 64 * 2;
__host__ __device__ constexpr int warm_smem_bytes(int tiles) { return FW_SX + tiles * (FW_X_TILE + FW_H_TILE); }

template <int L, int V>
__global__ void __launch_bounds__(256, 3) k_features_warm(KParams p, int nvb, const float4* __restrict__ x,
                                                          const float4* __restrict__ v, const int* __restrict__ nbr,
                                                          const int* __restrict__ ncnt,
                                                          const float* __restrict__ lam_prev,
                                                          float4* __restrict__ xl, float* __restrict__ feat,
                                                          float* __restrict__ lam_acc, WarmIO io) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ uint64_t mbar;
    __shared__ uint32_t tmem_slot;
    __shared__ float sb[MLP_NUM_BIASES];
    __shared__ float sw4[64];
    __shared__ float s_lam[256];
    const int t = threadIdx.x, warp = t >> 5;
    const int R = blockDim.x / L;            // particles per tile of slots: rows
    const int tiles = (R + 127) >> 7;        // 128-row MMA tiles
    const uint32_t cols = tiles > 1 ? 128u : 64u;
    uint8_t* sX = smem + FW_SX;
    uint8_t* sH = sX + tiles * FW_X_TILE;
    if (warp == 0) tmem_alloc(&tmem_slot, cols);
    if (t == 0) mbar_init(&mbar, 1);
    stage_weight(smem + FW_SW1, io.w + W1_OFF, 64, 16);
    stage_weight(smem + FW_SW2, io.w + W2_OFF, 64, 64);
    stage_weight(smem + FW_SW3, io.w + W3_OFF, 64, 64);
    for (int i = t; i < MLP_NUM_BIASES; i += blockDim.x) sb[i] = io.b[i];
    if (t < 64) sw4[t] = bf16_val(io.w[W4_OFF + t]);
    // rows of the last tile past R stay zero
    for (int i = t; i < tiles * FW_X_TILE / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(sX)[i] = make_uint4(0u, 0u, 0u, 0u);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = tmem_slot;
    const bool ep_warp = (warp >> 2) < tiles;  // this warp's TMEM quarter holds rows of a tile
    const uint32_t lane_base = tmem_addr(tbase, 32 * (warp & 3), 64 * (warp >> 2));
    uint8_t* my_h = sH + (warp >> 2) * FW_H_TILE;
    uint32_t phase = 0;
    bool alive = true;
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
        const Team<L> tm = team_of<L>(vb);
        float f[12], lam = 0.0f;
        const bool have = features_one<L, V>(p, tm, x, v, nbr, ncnt, lam_prev, xl, feat, lam_acc, f, lam);
        if (tm.t == 0) {
            const int row = t / L;
            float xf[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) xf[i] = 0.0f;
            if (have) {
#pragma unroll
                for (int i = 0; i < MLP_IN; ++i) xf[i] = (f[i] - sb[FMEAN_OFF + i]) * sb[FISTD_OFF + i];
            }
            uint32_t pk[8];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                pk[i] = (uint32_t)bf16_bits(xf[2 * i]) | ((uint32_t)bf16_bits(xf[2 * i + 1]) << 16);
            uint8_t* xt = sX + (row >> 7) * FW_X_TILE;
            *reinterpret_cast<uint4*>(xt + kmajor_offset(row & 127, 0, 128)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            *reinterpret_cast<uint4*>(xt + kmajor_offset(row & 127, 8, 128)) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            s_lam[row] = lam;
        }
        if (!alive) continue;  // an expired wait: no more tensor-core work (the error bit is set)
        // three hidden layers; layer l reads X (l = 0) or H and writes H (l < 2)
        float y = sb[B4_OFF];
        // row t's plain lambda, read after the first barrier (its team leader
        // wrote it) and before the second (after which that leader may write
        // the next tile's)
        float lam_plain = 0.0f;
#pragma unroll 1
        for (int l = 0; l < 3; ++l) {
            sync_for_mma();
            if (l == 0 && t < R) lam_plain = s_lam[t];
            if (t == 0) {
                for (int j = 0; j < tiles; ++j) {
                    if (l == 0) gemm_issue(tbase + 64 * j, sX + j * FW_X_TILE, smem + FW_SW1, 64, 16, 0);
                    else gemm_issue(tbase + 64 * j, sH + j * FW_H_TILE, smem + (l == 1 ? FW_SW2 : FW_SW3), 64, 64, 0);
                }
                commit(&mbar);
            }
            if (!wait_mma(&mbar, phase, io.err)) {
                alive = false;
                break;
            }
            if (ep_warp) {
                const float* bias = sb + (l == 0 ? B1_OFF : l == 1 ? B2_OFF : B3_OFF);
#pragma unroll 1
                for (int c = 0; c < 4; ++c) {
                    float vv[16];
                    tmem_ld16(lane_base + 16 * c, vv);
                    tmem_wait_ld();
#pragma unroll
                    for (int i = 0; i < 16; i += 2) {
                        const float2 hh =
                            gelu2(vadd(make_float2(vv[i], vv[i + 1]),
                                       make_float2(bias[16 * c + i], bias[16 * c + i + 1])));
                        vv[i] = hh.x;
                        vv[i + 1] = hh.y;
                    }
                    if (l < 2) {
                        put_row64(my_h, t & 127, vv, 16 * c);
                    } else {
#pragma unroll
                        for (int i = 0; i < 16; ++i) y = __fmaf_rn(vv[i], sw4[16 * c + i], y);
                    }
                }
            }
        }
        if (!alive) continue;
        const int k = vb * R + t;
        if (t < R && k < p.n) {
            float l0 = y * sb[OSCALE_OFF];
            if (io.clamp > 0.0f) {
                // trust region around the plain lambda of this pass: same sign,
                // at most clamp times its magnitude
                const float a = io.clamp * lam_plain;
                const float f0 = io.floor ? lam_plain : 0.0f;  // the weak end of the interval
                l0 = fminf(fmaxf(l0, fminf(a, f0)), fmaxf(a, f0));
            }
            reinterpret_cast<float*>(xl)[4 * (size_t)k + 3] = l0;
            lam_acc[k] = l0;
            io.lam0[k] = l0;
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tbase, cols);
}

// ---------------------------------------------------------------------------
// a10 + a11: position correction with tensile s_corr, then x += dp, wall clamp,
// and on the last iteration v = (x - x_old) / dt
// (calculateOffset cu:182-199, updatePosition cu:15-22)
// ---------------------------------------------------------------------------
template <bool DEBUG, int L, int V>
__device__ __forceinline__ void dp_tile(const KParams& p, int vb, const float4* __restrict__ xl,
                                        const int* __restrict__ nbr, const int* __restrict__ ncnt,
                                        const float4* __restrict__ xold, float4* __restrict__ xout,
                                        float4* __restrict__ vout, float4* __restrict__ dp_out);

template <bool DEBUG, int L, int V>
__global__ void __launch_bounds__(256, V == 1 ? 6 : 4) k_dp(KParams p, int nvb, const float4* __restrict__ xl,
                                                            const int* __restrict__ nbr, const int* __restrict__ ncnt,
                                                            const float4* __restrict__ xold, float4* __restrict__ xout,
                                                            float4* __restrict__ vout, float4* __restrict__ dp_out,
                                                            IterCtl ctl) {
    if (ctl.done) {
        if (*ctl.done) return;
        // the lambda pass just measured the positions this pass would correct;
        // when they are within tolerance the loop ends here
        const int sl = ctl.cur_slot();
        if (sl >= ctl.min_slot && __longlong_as_double((long long)ctl.max_bits[sl]) <= ctl.tol) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                *ctl.done = 1;
                *ctl.conv_slot = sl;
            }
            return;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(ctl.iters, 1);
    }
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x)
        dp_tile<DEBUG, L, V>(p, vb, xl, nbr, ncnt, xold, xout, vout, dp_out);
}

template <bool DEBUG, int L, int V>
__device__ __forceinline__ void dp_tile(const KParams& p, int vb, const float4* __restrict__ xl,
                                        const int* __restrict__ nbr, const int* __restrict__ ncnt,
                                        const float4* __restrict__ xold, float4* __restrict__ xout,
                                        float4* __restrict__ vout, float4* __restrict__ dp_out) {
    using T = vec_t<V>;
    constexpr int P = L * V, B = batches<V>();
    const Team<L> tm = team_of<L>(vb);
    const int k = tm.k;
    if (k >= p.n) return;  // uniform over the team
    const float4 xk4 = xl[k];
    const f3 xk = make3(xk4);
    const float lk = xk4.w;
    const int cnt = ncnt[k];
    T3<T> a = zero3<T>();
    // index prefetch one batch ahead (packed form only: the scalar form has no
    // registers left for it within 40)
    constexpr bool PF = V == 2;
    int jj[B][V];
    if (PF) load_idx<V, P, B>(p, nbr, k, V * tm.t, cnt, jj);
    for (int q0 = V * tm.t; q0 < cnt; q0 += P * B) {
        if (!PF) load_idx<V, P, B>(p, nbr, k, q0, cnt, jj);
        float4 xj[B][V];
#pragma unroll
        for (int u = 0; u < B; ++u)
#pragma unroll
            for (int c = 0; c < V; ++c) xj[u][c] = xl[jj[u][c]];
        if (PF) load_idx<V, P, B>(p, nbr, k, q0 + P * B, cnt, jj);
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const int q = q0 + u * P;
            if (q >= cnt) break;
            T3<T> r, g;
            T w;
            pair_terms<T, true>(p, xk, pack3(xj[u]), valid_bits<V>(q, cnt), r, w, g);
            const T s = dp_weight(p, lk, packw(xj[u]), w);
            a = {vfma(s, g.x, a.x), vfma(s, g.y, a.y), vfma(s, g.z, a.z)};
        }
    }
    f3 as = team_sum3<L>(fold3(a), tm.mask);
    if (tm.t != 0) return;
    if (p.flags & FLAG_WALL_DENSITY) {
        f3 gw;
        wall_term(p, scene_of(p, k), xk, gw);
        as.x = __fmaf_rn(lk, gw.x, as.x);
        as.y = __fmaf_rn(lk, gw.y, as.y);
        as.z = __fmaf_rn(lk, gw.z, as.z);
    }
    const f3 dp = {__fdiv_rn(as.x, p.rho0), __fdiv_rn(as.y, p.rho0), __fdiv_rn(as.z, p.rho0)};
    f3 xn = {xk.x + dp.x, xk.y + dp.y, xk.z + dp.z};
    bound_particle(p, scene_of(p, k), xn);
    xout[k] = make_float4(xn.x, xn.y, xn.z, 0.0f);
    if (vout) {
        const float4 xo = xold[k];
        vout[k] = make_float4(__fdiv_rn(xn.x - xo.x, p.dt), __fdiv_rn(xn.y - xo.y, p.dt),
                              __fdiv_rn(xn.z - xo.z, p.dt), 0.0f);
    }
    if (DEBUG) dp_out[k] = make_float4(dp.x, dp.y, dp.z, 0.0f);
}

// ---------------------------------------------------------------------------
// a12: vorticity (calculateCurl cu:201-215): w_i = sum (v_j - v_i) x gradW(x_i - x_j);
// writes (w_i, |w_i|) and (v_i, |w_i|): the vorticity pass then gathers two
// float4s per neighbour (x_j and v_j with |w_j|) instead of three
// ---------------------------------------------------------------------------
template <int L, int V>
__device__ __forceinline__ void curl_tile(const KParams& p, int vb, const float4* __restrict__ x,
                                          const float4* __restrict__ v, const int* __restrict__ nbr,
                                          const int* __restrict__ ncnt, float4* __restrict__ omega,
                                          float4* __restrict__ vw) {
    using T = vec_t<V>;
    constexpr int P = L * V, B = batches<V>();
    const Team<L> tm = team_of<L>(vb);
    const int k = tm.k;
    if (k >= p.n) return;  // uniform over the team
    const f3 xk = make3(x[k]);
    const f3 vk = make3(v[k]);
    const int cnt = ncnt[k];
    T3<T> wsum = zero3<T>();
    int jj[B][V];
    load_idx<V, P, B>(p, nbr, k, V * tm.t, cnt, jj);
    for (int q0 = V * tm.t; q0 < cnt; q0 += P * B) {
        float4 xj[B][V], vj[B][V];
#pragma unroll
        for (int u = 0; u < B; ++u)
#pragma unroll
            for (int c = 0; c < V; ++c) {
                xj[u][c] = x[jj[u][c]];
                vj[u][c] = v[jj[u][c]];
            }
        // the next batch's indices load while this batch computes
        load_idx<V, P, B>(p, nbr, k, q0 + P * B, cnt, jj);
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const int q = q0 + u * P;
            if (q >= cnt) break;
            T3<T> r, g;
            T w;
            pair_terms<T, false>(p, xk, pack3(xj[u]), valid_bits<V>(q, cnt), r, w, g);
            const T3<T> vv = pack3(vj[u]);
            const T3<T> vji = {vsub(vv.x, bc<T>(vk.x)), vsub(vv.y, bc<T>(vk.y)), vsub(vv.z, bc<T>(vk.z))};
            wsum = add3(wsum, cross3v(vji, g));
        }
    }
    const f3 w3 = team_sum3<L>(fold3(wsum), tm.mask);
    if (tm.t == 0) {
        const float wl = __fsqrt_rn(dot_fma(w3, w3));
        omega[k] = make_float4(w3.x, w3.y, w3.z, wl);
        vw[k] = make_float4(vk.x, vk.y, vk.z, wl);
    }
}

template <int L, int V>
__global__ void __launch_bounds__(256) k_curl(KParams p, int nvb, const float4* __restrict__ x,
                                              const float4* __restrict__ v, const int* __restrict__ nbr,
                                              const int* __restrict__ ncnt, float4* __restrict__ omega,
                                              float4* __restrict__ vw) {
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) curl_tile<L, V>(p, vb, x, v, nbr, ncnt, omega, vw);
}

// ---------------------------------------------------------------------------
// a13: vorticity confinement and XSPH, applied to v
// (calculateVorticityAndViscosity cu:217-239, applyVorticityAndViscosity cu:24-29);
// also writes the substep's final state (x, v, perm) for the next substep, and
// with the final x and v in registers does the next substep's grid hash (a1 +
// a2: prediction, wall clamp, cell key and its histogram), which therefore needs
// no pass of its own.
// ---------------------------------------------------------------------------
// One particle (team tm); returns its next cell key on the team's first thread
// and -1 on the others.
template <bool DEBUG, int L, int V>
__device__ __forceinline__ int vort_one(const KParams& p, const Team<L>& tm, int k, const float4* __restrict__ x,
                                        const float4* __restrict__ vw, const float4* __restrict__ omega,
                                        const int* __restrict__ nbr, const int* __restrict__ ncnt,
                                        float4* __restrict__ xout, float4* __restrict__ vout,
                                        const int* __restrict__ perm_in, int* __restrict__ perm_out,
                                        float4* __restrict__ vort_out, float4* __restrict__ visc_out,
                                        int* __restrict__ err) {
    using T = vec_t<V>;
    constexpr int P = L * V, B = batches<V>();  // two 16-byte gathers per entry
    const f3 xk = make3(x[k]);
    const f3 vk = make3(vw[k]);
    const int cnt = ncnt[k];
    T3<T> pv = zero3<T>(), eta = zero3<T>();
    // (no index prefetch here: the three gathers per entry leave no registers
    // for it within 64)
    for (int q0 = V * tm.t; q0 < cnt; q0 += P * B) {
        int jj[B][V];
        load_idx<V, P, B>(p, nbr, k, q0, cnt, jj);
        float4 xj[B][V], vj[B][V];
#pragma unroll
        for (int u = 0; u < B; ++u)
#pragma unroll
            for (int c = 0; c < V; ++c) {
                xj[u][c] = x[jj[u][c]];
                vj[u][c] = vw[jj[u][c]];
            }
#pragma unroll
        for (int u = 0; u < B; ++u) {
            const int q = q0 + u * P;
            if (q >= cnt) break;
            T3<T> r, g;
            T w;
            pair_terms<T, true>(p, xk, pack3(xj[u]), valid_bits<V>(q, cnt), r, w, g);
            const T3<T> vv = pack3(vj[u]);
            const T3<T> vji = {vsub(vv.x, bc<T>(vk.x)), vsub(vv.y, bc<T>(vk.y)), vsub(vv.z, bc<T>(vk.z))};
            pv = {vfma(vji.x, w, pv.x), vfma(vji.y, w, pv.y), vfma(vji.z, w, pv.z)};
            const T wl = packw(vj[u]);  // |w_j| (k_curl)
            eta = {vfma(wl, g.x, eta.x), vfma(wl, g.y, eta.y), vfma(wl, g.z, eta.z)};
        }
    }
    const f3 pvs = team_sum3<L>(fold3(pv), tm.mask);
    f3 etas = team_sum3<L>(fold3(eta), tm.mask);
    if (tm.t != 0) return -1;
    const float el = __fsqrt_rn(dot_fma(etas, etas));
    if ((double)el > 1e-3) etas = {__fdiv_rn(etas.x, el), __fdiv_rn(etas.y, el), __fdiv_rn(etas.z, el)};
    const f3 cr = cross3(etas, make3(omega[k]));
    const f3 fv = {p.vort_eps * cr.x, p.vort_eps * cr.y, p.vort_eps * cr.z};
    const f3 vs = {p.visc_c * pvs.x, p.visc_c * pvs.y, p.visc_c * pvs.z};
    const f3 t = {p.dt * fv.x + vs.x, p.dt * fv.y + vs.y, p.dt * fv.z + vs.z};
    f3 vn = {vk.x + t.x, vk.y + t.y, vk.z + t.z};
    xout[k] = make_float4(xk.x, xk.y, xk.z, 0.0f);
    vout[k] = make_float4(vn.x, vn.y, vn.z, 0.0f);
    perm_out[k] = perm_in[k];
    if (DEBUG) {
        vort_out[k] = make_float4(fv.x, fv.y, fv.z, 0.0f);
        visc_out[k] = make_float4(vs.x, vs.y, vs.z, 0.0f);
    }
    // the next substep's prediction and cell key (as k_hash computes them from
    // the state just written)
    const SceneView sc = scene_of(p, k);
    f3 xq = xk;
    predict(p, sc, xq, vn);
    if (!(isfinite(xq.x) && isfinite(xq.y) && isfinite(xq.z))) atomicOr(err, DEVERR_NONFINITE);
    return cell_key(p, sc, xq);
}

template <bool DEBUG, int L, int V>
__global__ void __launch_bounds__(256, 4) k_vort(KParams p, int nvb, const float4* __restrict__ x,
                                              const float4* __restrict__ vw, const float4* __restrict__ omega,
                                              const int* __restrict__ nbr, const int* __restrict__ ncnt,
                                              float4* __restrict__ xout, float4* __restrict__ vout,
                                              const int* __restrict__ perm_in, int* __restrict__ perm_out,
                                              float4* __restrict__ vort_out, float4* __restrict__ visc_out,
                                              int* __restrict__ cell, int* __restrict__ ticket, int* __restrict__ hist,
                                              int* __restrict__ err) {
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x) {
        const Team<L> tm = team_of<L>(vb);
        const int k = tm.k;
        int key = -1;
        if (k < p.n)  // uniform over the team
            key = vort_one<DEBUG, L, V>(p, tm, k, x, vw, omega, nbr, ncnt, xout, vout, perm_in, perm_out, vort_out,
                                        visc_out, err);
        // the next substep's histogram (every lane of the warp takes part)
        const int tk = warp_histogram(key, hist);
        if (key >= 0) {
            cell[k] = key;
            ticket[k] = tk;
        }
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// blocks for n particles with L threads each
static inline int team_blocks(int n, int L, int bs) { return (int)(((long long)n * L + bs - 1) / bs); }

// Grid of a neighbour pass over nvb tiles: nvb blocks, or with p.persistent the
// blocks that are resident at once (SMs x blocks per SM at this block size), each
// striding over the tiles.
template <typename K> static int pass_grid(const KParams& p, K kernel, int nvb) {
    if (!p.persistent) return nvb;
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 1;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, p.block, 0) != cudaSuccess || per_sm <= 0)
        per_sm = 1;
    const long long g = (long long)per_sm * sms;
    return (int)(g < nvb ? g : nvb);
}

// Calls f with (L, V) of pair_lanes as compile-time constants.
template <int A, int B> struct LV {
    static constexpr int L = A, V = B;
};
template <typename F> void with_lanes(int lanes, F&& f) {
    switch (lanes) {
        case 1: f(LV<1, 1>{}); break;
        case 4: f(LV<2, 2>{}); break;
        case 8: f(LV<4, 2>{}); break;
        default: f(LV<1, 2>{}); break;
    }
}

void launch_lambda(const KParams& p, bool debug, const float4* x, const int* nbr, const int* ncnt, float4* xl,
                   float* rho, const IterCtl& ctl, cudaStream_t st) {
    with_lanes(p.lanes, [&](auto c) {
        constexpr int L = decltype(c)::L, V = decltype(c)::V;
        const int b = team_blocks(p.n, L, p.block);
        if (debug) k_lambda<true, L, V><<<pass_grid(p, k_lambda<true, L, V>, b), p.block, 0, st>>>(p, b, x, nbr, ncnt, xl, rho, ctl);
        else k_lambda<false, L, V><<<pass_grid(p, k_lambda<false, L, V>, b), p.block, 0, st>>>(p, b, x, nbr, ncnt, xl, rho, ctl);
    });
}

void launch_dp(const KParams& p, bool debug, const float4* xl, const int* nbr, const int* ncnt, const float4* xold,
               float4* xout, float4* vout, float4* dp, const IterCtl& ctl, cudaStream_t st) {
    with_lanes(p.lanes, [&](auto c) {
        constexpr int L = decltype(c)::L, V = decltype(c)::V;
        const int b = team_blocks(p.n, L, p.block);
        if (debug)
            k_dp<true, L, V><<<pass_grid(p, k_dp<true, L, V>, b), p.block, 0, st>>>(p, b, xl, nbr, ncnt, xold, xout,
                                                                                     vout, dp, ctl);
        else
            k_dp<false, L, V><<<pass_grid(p, k_dp<false, L, V>, b), p.block, 0, st>>>(p, b, xl, nbr, ncnt, xold, xout,
                                                                                       vout, dp, ctl);
    });
}

void launch_features(const KParams& p, const float4* x, const float4* v, const int* nbr, const int* ncnt,
                     const float* lam_prev, float4* xl, float* feat, float* lam_acc, cudaStream_t st) {
    with_lanes(p.lanes, [&](auto c) {
        constexpr int L = decltype(c)::L, V = decltype(c)::V;
        const int b = team_blocks(p.n, L, p.block);
        k_features<L, V><<<pass_grid(p, k_features<L, V>, b), p.block, 0, st>>>(p, b, x, v, nbr, ncnt, lam_prev, xl,
                                                                                 feat, lam_acc);
    });
}

int launch_features_warm(const KParams& p, const float4* x, const float4* v, const int* nbr, const int* ncnt,
                         const float* lam_prev, float4* xl, float* feat, float* lam_acc, const uint16_t* w,
                         const float* b, float* lam0, float clamp, int floor, int* err, cudaStream_t st) {
    int rc = 0;
    with_lanes(p.lanes, [&](auto c) {
        constexpr int L = decltype(c)::L, V = decltype(c)::V;
        const int rows = p.block / L;
        const int smem = warm_smem_bytes((rows + 127) / 128);
        if (cudaFuncSetAttribute(k_features_warm<L, V>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
            cudaSuccess) {
            rc = -1;
            return;
        }
        const int nvb = team_blocks(p.n, L, p.block);
        int grid = nvb;
        if (p.persistent) {
            int dev = 0, sms = 1, per_sm = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_features_warm<L, V>, p.block, smem) !=
                    cudaSuccess || per_sm <= 0)
                per_sm = 1;
            grid = (int)std::min<long long>((long long)per_sm * sms, nvb);
        }
        const WarmIO io{w, b, lam0, clamp, floor, err};
        k_features_warm<L, V><<<grid, p.block, smem, st>>>(p, nvb, x, v, nbr, ncnt, lam_prev, xl, feat, lam_acc, io);
    });
    return rc;
}

void launch_curl(const KParams& p, const float4* x, const float4* v, const int* nbr, const int* ncnt, float4* omega,
                 float4* vw, cudaStream_t st) {
    with_lanes(p.lanes, [&](auto c) {
        constexpr int L = decltype(c)::L, V = decltype(c)::V;
        const int b = team_blocks(p.n, L, p.block);
        k_curl<L, V><<<pass_grid(p, k_curl<L, V>, b), p.block, 0, st>>>(p, b, x, v, nbr, ncnt, omega, vw);
    });
}

void launch_vort(const KParams& p, bool debug, const float4* x, const float4* vw, const float4* omega, const int* nbr,
                 const int* ncnt, float4* xout, float4* vout, const int* perm_in, int* perm_out, float4* vort,
                 float4* visc, int* cell, int* ticket, int* hist, int* err, cudaStream_t st) {
    with_lanes(p.lanes, [&](auto c) {
        constexpr int L = decltype(c)::L, V = decltype(c)::V;
        const int b = team_blocks(p.n, L, p.block);
        if (debug)
            k_vort<true, L, V><<<pass_grid(p, k_vort<true, L, V>, b), p.block, 0, st>>>(
                p, b, x, vw, omega, nbr, ncnt, xout, vout, perm_in, perm_out, vort, visc, cell, ticket, hist, err);
        else
            k_vort<false, L, V><<<pass_grid(p, k_vort<false, L, V>, b), p.block, 0, st>>>(
                p, b, x, vw, omega, nbr, ncnt, xout, vout, perm_in, perm_out, vort, visc, cell, ticket, hist, err);
    });
}

}  // namespace pbf
