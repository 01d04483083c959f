// TEST INFRASTRUCTURE ONLY. Nothing in the shipped library links or calls this
// file; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg
// load it, and only as the checker.
//
// CPU restatement of one Position Based Fluids substep as the reference
// implements it, templated on the arithmetic type (float for FP32 parity,
// double for the FP64 density-error oracle).
//
// Two reference formulations exist and differ in physics; both are restated:
//   formulation 0 (GPU)  kernels/cudaPBFSolver.cu:4-239, kernels/cudaPBFSolver.cuh:99-181,
//                        launch order kernels/cudaPBF.cu:50-115
//   formulation 1 (CPU)  src/solver.cpp:3-156, include/solver.h:49-199
// and two arithmetic modes:
//   arith 0 (reference)  the reference's own expressions (powf / std::pow, sinf,
//                        the reference's mixed float/double constants)
//   arith 1 (product)    the evaluation order the CUDA library uses (explicit fused
//                        multiply-adds at fixed places, cubes by multiplication, a
//                        double-precision sine); every place where it departs from
//                        arith 0 is marked "product:" below.
// Parity is pinned by comparing formulation 1 / arith 0 against the reference CPU
// solver compiled from its own sources, formulation 0 / arith 0 against the
// reference CUDA kernels, and formulation 0 / arith 1 against the CUDA library.
//
// Build: g++ -O2 -ffp-contract=off -fno-fast-math -shared -fPIC (oracle/Makefile).
// -ffp-contract=off matters: every fused multiply-add must be an explicit fma().
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

extern "C" {

// Mirrors the parameter block of the CUDA library (include/pbf.h) in plain form.
typedef struct oracle_params {
    // SolverParameter fields (include/solverBase.h:16-40)
    float h, restRho, epsilon, k, n, deltaq, c, dt, vort_eps;
    int iterations;
    // extensions
    float gravity[3];     // GPU reference hard-codes (0,-49,0), CPU (0,-9.8,0)
    float grid_min[3];    // gridSpace.pMin (grid origin)
    int dims[3];          // grid cells per axis (reference: 64^3 macros)
    float bmin[3], bmax[3];  // boundary box
    float wall_jitter;    // RANDOM_OFFSET_COEFF (GPU 0.01) / delta (CPU 0.02)
    float grad_rmin;      // spiky-gradient lower cutoff (0.01 in both references)
    int max_nbr;          // MAX_NEIGHBOR (63)
    int formulation;      // 0 GPU, 1 CPU
    int arith;            // 0 reference, 1 product
    int cell_order;       // 0 ascending slot order within a cell, 1 descending
    int reorder;          // 1: keep particle arrays permuted into cell order
    int flags;            // stable-mode bits (ORACLE_* below)
    float scorr_scale;    // multiplies s_corr (1 = reference)
    float sphere[4];      // static sphere obstacle centre xyz, radius (radius<=0: none)
    double wall_jitter_d; // the GPU reference's RANDOM_OFFSET_COEFF is the double literal 0.01
    float cell_scale;     // grid cell edge = h * cell_scale (reference: 1)
    int lanes;            // product: pair lanes per particle (1, 2, 4 or 8; <= 1: one lane)
} oracle_params;

enum {
    ORACLE_CLAMP_C = 1,      // unilateral density constraint C = max(C, 0)
    ORACLE_XSPH_RHO = 2,     // XSPH weight c/rho0 instead of c
    ORACLE_WALL_DENSITY = 4, // boundary faces carry the density of a fluid half-space
};

// Field ids shared with the Python wrapper (oracle/oracle.py).
enum {
    F_X = 0, F_V, F_XOLD, F_XPRED, F_LAMBDA, F_RHO, F_DP, F_CURL, F_VORT, F_VISC,
    F_CELL, F_CNT, F_START, F_END, F_SORTED, F_NCNT, F_NBR, F_PERM, F_DPMAG,
    F_COUNT
};

}  // extern "C"

namespace {

constexpr double kRefInvPi = 0.31830988618;  // INVPI, include/solverBase.h:4

// ---- deterministic sine (product arithmetic) ---------------------------------
// Own implementation from the mathematics: round-to-nearest quadrant reduction
// by a two-part Cody-Waite split of pi/2 (first 33 bits, then the remainder
// rounded to double), then Taylor series of sin and cos on [-pi/4, pi/4] in
// Horner form, all in IEEE double without contraction, rounded once to float.
// The CUDA library evaluates the same expression sequence, so both sides agree
// bit for bit.
float det_sin(float a) {
    const double x = (double)a;
    const double P1 = 1.5707963267341256;
    const double P2 = 6.077100506506192e-11;
    const double q = std::floor(x * 0.6366197723675814 + 0.5);
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

// product: reciprocal square root for normal x > 0 from the published bit-level
// estimate 0x5f3759df - (bits >> 1) (C. Lomont, "Fast Inverse Square Root",
// 2003) and three Newton steps y <- y (3/2 - (x/2) y^2), one fused multiply-add
// each; the CUDA library evaluates the same steps (pbf_rsqrt).
float soft_rsqrt(float x) {
    const float hx = 0.5f * x;
    int32_t bits;
    std::memcpy(&bits, &x, 4);
    bits = 0x5f3759df - (bits >> 1);
    float y;
    std::memcpy(&y, &bits, 4);
    for (int i = 0; i < 3; ++i) y = y * std::fma(-hx, y * y, 1.5f);
    return y;
}

template <typename T> struct V3 {
    T x, y, z;
};
template <typename T> inline V3<T> sub(const V3<T>& a, const V3<T>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename T> inline V3<T> add(const V3<T>& a, const V3<T>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }

// product: the CUDA library splits a particle's neighbour list over L pair lanes
// (lane t takes entries t, t+L, t+2L, ... in list order) and combines the lane
// sums by an xor butterfly over distances 1, 2, 4, i.e. ((a0+a1)+(a2+a3))+... .
constexpr int kMaxLanes = 8;
template <typename T> inline T combine_lanes(T* a, int L) {
    for (int o = 1; o < L; o <<= 1)
        for (int t = 0; t < L; t += 2 * o) a[t] = a[t] + a[t + o];
    return a[0];
}
template <typename T> inline V3<T> combine_lanes(V3<T>* a, int L) {
    for (int o = 1; o < L; o <<= 1)
        for (int t = 0; t < L; t += 2 * o) a[t] = add(a[t], a[t + o]);
    return a[0];
}
// glm compute_dot and the reference Vec3 dot: (x*x + y*y) + z*z
template <typename T> inline T dot_ref(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// product: fma(z,z, fma(y,y, x*x))
template <typename T> inline T dot_fma(const V3<T>& a, const V3<T>& b) {
    return std::fma(a.z, b.z, std::fma(a.y, b.y, a.x * b.x));
}
template <typename T> inline V3<T> cross(const V3<T>& a, const V3<T>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// product (the curl's pair term): one fused multiply-add per component
template <typename T> inline V3<T> cross_fma(const V3<T>& a, const V3<T>& b) {
    return {std::fma(a.y, b.z, -(a.z * b.y)), std::fma(a.z, b.x, -(a.x * b.z)), std::fma(a.x, b.y, -(a.y * b.x))};
}

template <typename T> struct Consts {
    T h, h2, invH, poly6_c, spiky_c, wdq, inv_wdq, nk, rho0, rho0sq, eps, dt, jit, rmin, visc_c, vort_eps;
    T wall_n, inv_h, wall_kd, wc3, wc5, wc7, wc9;  // wall density (see wall_term)
    int n_int;  // integer exponent of s_corr, 0 when not a small integer
};

template <typename T> class Solver {
public:
    oracle_params p;
    int n;
    int ncells;
    Consts<T> k;
    std::vector<V3<T>> x, v, xold, xpred, dp, curl, vort, visc;
    std::vector<T> lambda, rho, dpmag;
    std::vector<int> perm, cell, cnt, start, end, sorted, ncnt, nbr;
    bool is_double = sizeof(T) == 8;

    Solver(const oracle_params& prm, int n_, const float* pos, const float* vel) : p(prm), n(n_) {
        ncells = p.dims[0] * p.dims[1] * p.dims[2];
        x.resize(n); v.resize(n); xold.resize(n); xpred.resize(n); dp.resize(n);
        curl.resize(n); vort.resize(n); visc.resize(n);
        lambda.assign(n, 0); rho.assign(n, 0); dpmag.assign(n, 0);
        perm.resize(n); cell.assign(n, -1); cnt.assign(ncells, 0); start.assign(ncells, 0);
        end.assign(ncells, 0); sorted.assign(n, 0); ncnt.assign(n, 0);
        nbr.assign((size_t)n * p.max_nbr, -1);
        for (int i = 0; i < n; ++i) {
            x[i] = {(T)pos[3 * i], (T)pos[3 * i + 1], (T)pos[3 * i + 2]};
            v[i] = {(T)vel[3 * i], (T)vel[3 * i + 1], (T)vel[3 * i + 2]};
            perm[i] = i;
        }
        make_consts();
    }

    void make_consts() {
        const float hf = p.h;
        k.h = (T)hf;
        k.h2 = (T)(hf * hf);
        // GPU: float invH = 1.0f / h (cu:35); CPU: float invH = 1.0 / h (src/solver.cpp:5)
        k.invH = (p.formulation == 1 && p.arith == 0 && !is_double) ? (T)(float)(1.0 / (double)hf)
                                                                    : (T)(1.0f / (hf * p.cell_scale));
        k.rho0 = (T)p.restRho;
        k.rho0sq = (T)(p.restRho * p.restRho);
        k.eps = (T)p.epsilon;
        k.dt = (T)p.dt;
        k.jit = (T)p.wall_jitter;
        k.rmin = (T)p.grad_rmin;
        k.vort_eps = (T)p.vort_eps;
        k.visc_c = (T)((p.flags & ORACLE_XSPH_RHO) ? (float)((double)p.c / (double)p.restRho) : p.c);
        k.n_int = 0;
        if (p.n >= 1.0f && p.n <= 8.0f && p.n == std::floor(p.n)) k.n_int = (int)p.n;
        if (is_double) {
            // FP64 oracle: exact constants
            const double h = hf;
            k.poly6_c = (T)(315.0 / (64.0 * M_PI * std::pow(h, 9)));
            k.spiky_c = (T)(-45.0 / (M_PI * std::pow(h, 6)));
        } else if (p.arith == 1) {
            // product: constants in double from the reference's truncated 1/pi, rounded once
            k.poly6_c = (T)(float)(315.0 * kRefInvPi / (64.0 * std::pow((double)hf, 9)));
            k.spiky_c = (T)(float)(-45.0 * kRefInvPi / std::pow((double)hf, 6));
        } else if (p.formulation == 0) {
            // kernels/cudaPBFSolver.cuh:101,108: float powf inside a double expression
            k.poly6_c = (T)(float)(315.0f * kRefInvPi / (double)(64.0f * powf(hf, 9)));
            k.spiky_c = (T)(float)(-45.0f * kRefInvPi / (double)powf(hf, 6));
        } else {
            // include/solver.h:51,58: std::pow(float,int) is double
            const float invPi = 0.31830988618f;
            k.poly6_c = (T)(float)(315.0f * invPi / (64.0f * std::pow(hf, 9)));
            k.spiky_c = (T)(float)(-45.0f * invPi / std::pow(hf, 6));
        }
        {
            const float h2f = hf * hf, pc = (float)k.poly6_c;
            const float h3 = (h2f * h2f) * h2f;
            k.wall_n = (T)(p.restRho + pc * h3);
            k.inv_h = (T)(1.0f / hf);
            k.wall_kd = (T)(float)(315.0 / (256.0 * (double)hf));
            k.wc3 = (T)(float)(-4.0 / 3.0);
            k.wc5 = (T)(float)(6.0 / 5.0);
            k.wc7 = (T)(float)(-4.0 / 7.0);
            k.wc9 = (T)(float)(1.0 / 9.0);
        }
        V3<T> rq{(T)p.deltaq, 0, 0};
        k.wdq = W6(rq);
        k.inv_wdq = (T)1 / k.wdq;
        k.nk = -(T)p.k;
    }

    // ---- SPH kernels ----------------------------------------------------------
    // Wpoly6: kernels/cudaPBFSolver.cuh:99-103 (GPU), include/solver.h:49-53 (CPU)
    T W6(const V3<T>& r) const {
        if (is_double) {
            const T r2 = dot_ref(r, r);
            if (r2 > k.h2) return 0;
            const T t = k.h2 - r2;
            return k.poly6_c * t * t * t;
        }
        if (p.arith == 1) {  // product: r2 by fma chain, cube by multiplication
            const T r2 = dot_fma(r, r);
            if (r2 > k.h2) return 0;
            const T t = k.h2 - r2;
            return k.poly6_c * ((t * t) * t);
        }
        if (p.formulation == 0) {
            const float r2 = (float)dot_ref(r, r);
            if (r2 > (float)k.h2) return 0;
            return (T)((float)k.poly6_c * powf((float)k.h2 - r2, 3));
        }
        // CPU: cutoff on |r| (glm::length), body in double via std::pow(float,int)
        const float len = std::sqrt((float)dot_ref(r, r));
        if (len > (float)k.h) return 0;
        const float t = (float)k.h2 - (float)dot_ref(r, r);
        return (T)(float)((double)(float)k.poly6_c * std::pow(t, 3));
    }

    // WspikyGrad: kernels/cudaPBFSolver.cuh:105-110 (GPU), delWspiky include/solver.h:55-60 (CPU)
    V3<T> gradW(const V3<T>& r) const {
        if (is_double) {
            const T r2 = dot_ref(r, r);
            const T rl = std::sqrt(r2);
            if (rl > k.h || rl < k.rmin) return {0, 0, 0};
            const T d = k.h - rl;
            const T s = ((k.spiky_c * d) * d) / rl;
            return {s * r.x, s * r.y, s * r.z};
        }
        if (p.arith == 1) {
            // product: y = rsqrt(|r|^2) by soft_rsqrt, |r| = |r|^2 y for the cutoff,
            // h - |r| = fma(-|r|^2, y, h), s = c (h-|r|)^2 y
            const float r2 = (float)dot_fma(r, r);
            const float y = soft_rsqrt(std::max(r2, 1e-30f));
            const float rl = r2 * y;
            if (rl > (float)k.h || rl < (float)k.rmin) return {0, 0, 0};
            const float d = std::fma(-r2, y, (float)k.h);
            const float s = (((float)k.spiky_c * d) * d) * y;
            return {(T)(s * (float)r.x), (T)(s * (float)r.y), (T)(s * (float)r.z)};
        }
        const float rl = std::sqrt((float)dot_ref(r, r));
        if (rl > (float)k.h || rl < (float)k.rmin) return {0, 0, 0};
        if (p.formulation == 0) {
            const float s = (float)k.spiky_c * powf((float)k.h - rl, 2);
            return {(T)(s * ((float)r.x / rl)), (T)(s * ((float)r.y / rl)), (T)(s * ((float)r.z / rl))};
        }
        const float s = (float)k.spiky_c * (float)std::pow((float)k.h - rl, 2);
        const float inv = 1.0f / rl;  // glm::normalize = v * inversesqrt(dot(v,v))
        return {(T)(s * ((float)r.x * inv)), (T)(s * ((float)r.y * inv)), (T)(s * ((float)r.z * inv))};
    }

    // Scorr: kernels/cudaPBFSolver.cuh:142-144 (GPU), include/solver.h:138-140 (CPU)
    T scorr(T w) const {
        if (is_double) return k.nk * std::pow(w / k.wdq, (T)p.n) * (T)p.scorr_scale;
        if (p.arith == 1) {
            const T q = w * k.inv_wdq;
            T pw;
            if (k.n_int > 0) {
                pw = q;
                for (int i = 1; i < k.n_int; ++i) pw = pw * q;
            } else {
                pw = (T)powf((float)q, p.n);
            }
            return (k.nk * pw) * (T)p.scorr_scale;
        }
        if (p.formulation == 0) return (T)(-p.k * powf((float)w / (float)k.wdq, p.n) * p.scorr_scale);
        return (T)(-p.k * std::pow((float)w / (float)k.wdq, p.n) * p.scorr_scale);
    }

    // product: the dp pair weight (lambda_i + lambda_j) + Scorr as one fused multiply-add
    T dp_weight(T li, T lj, T w) const {
        const T q = w * k.inv_wdq;
        T pw;
        if (k.n_int > 0) {
            pw = q;
            for (int i = 1; i < k.n_int; ++i) pw = pw * q;
        } else {
            pw = (T)powf((float)q, p.n);
        }
        return std::fma(k.nk * pw, (T)p.scorr_scale, li + lj);
    }

    // randomOffset: kernels/cudaPBFSolver.cuh:112-119 (GPU), include/solver.h:62-69 (CPU)
    T random_offset(T u, T w) const {
        if (p.arith == 1 || is_double) {
            const float a = (float)u * 12.9898f;
            const float b = (float)w * 78.233f;
            const float arg = 2.0f * (a + b);
            const float m = det_sin(arg) * 43758.5453f;
            return (T)std::fabs(m - (float)(int)m);
        }
        if (p.formulation == 0) {
            const float m = sinf(2.0f * ((float)u * 12.9898f + (float)w * 78.233f)) * 43758.5453f;
            return (T)fabsf(m - (float)(int)m);
        }
        // glm::dot(uv, vec2(12.9898, 78.233) * 2.0f); std::sin(float); * double literal
        const float c0 = 12.9898f * 2.0f, c1 = 78.233f * 2.0f;
        const float d = (float)u * c0 + (float)w * c1;
        const float m = (float)((double)std::sin(d) * 43758.5453);
        return (T)std::fabs(m - (float)(int)m);
    }

    T wall_pos(T wall, T ro, bool plus) const {
        if (p.arith == 1 || is_double) {
            const T t = k.jit * ro;
            return plus ? wall + t : wall - t;
        }
        if (p.formulation == 1) {  // include/solver.h:120: float delta * float offset
            const float t = p.wall_jitter * (float)ro;
            return (T)(plus ? (float)wall + t : (float)wall - t);
        }
        // cuh:123: float + (double literal * float), evaluated in double, stored as float
        const double t = p.wall_jitter_d * (double)(float)ro;
        return (T)(float)(plus ? (double)(float)wall + t : (double)(float)wall - t);
    }

    // BoundParticle: kernels/cudaPBFSolver.cuh:121-140 (GPU; y-max uses (y,z)),
    // include/solver.h:113-137 (CPU; y-max uses (x,z))
    void bound(V3<T>& q) const {
        const T bx0 = p.bmin[0], by0 = p.bmin[1], bz0 = p.bmin[2];
        const T bx1 = p.bmax[0], by1 = p.bmax[1], bz1 = p.bmax[2];
        if (q.x < bx0) q.x = wall_pos(bx0, random_offset(q.y, q.z), true);
        if (q.x > bx1) q.x = wall_pos(bx1, random_offset(q.y, q.z), false);
        if (q.y < by0) q.y = wall_pos(by0, random_offset(q.x, q.z), true);
        if (q.y > by1) q.y = wall_pos(by1, p.formulation == 0 ? random_offset(q.y, q.z) : random_offset(q.x, q.z), false);
        if (q.z < bz0) q.z = wall_pos(bz0, random_offset(q.x, q.y), true);
        if (q.z > bz1) q.z = wall_pos(bz1, random_offset(q.x, q.y), false);
        if (p.sphere[3] > 0) sphere_project(q);
    }

    // Static sphere obstacle (no reference counterpart): a point inside the sphere
    // is moved radially onto its surface. Same expression sequence as the CUDA library.
    void sphere_project(V3<T>& q) const {
        const T cx = p.sphere[0], cy = p.sphere[1], cz = p.sphere[2], R = p.sphere[3];
        const V3<T> d{q.x - cx, q.y - cy, q.z - cz};
        const T d2 = is_double ? dot_ref(d, d) : dot_fma(d, d);
        if (d2 >= R * R || d2 <= (T)0) return;
        const T s = R / std::sqrt(d2);
        q = {cx + d.x * s, cy + d.y * s, cz + d.z * s};
    }

    // Wall density (no reference counterpart): each boundary face is backed by a
    // fluid half-space at rest number density wall_n; at distance d < h it adds
    // wall_n F(d/h) to rho and wall_n dF/dd along the face normal to grad rho,
    // F(s) = 1/2 - 315/256 (s - 4/3 s^3 + 6/5 s^5 - 4/7 s^7 + s^9/9),
    // dF/dd = -315/(256 h) (1 - s^2)^4. Same expression sequence as the CUDA library.
    T wall_face(T d, T& dfdd) const {
        d = std::max(d, (T)0);
        const T s = d * k.inv_h;
        const T s2 = s * s;
        T t = std::fma(s2, k.wc9, k.wc7);
        t = std::fma(s2, t, k.wc5);
        t = std::fma(s2, t, k.wc3);
        t = std::fma(s2, t, (T)1);
        const T F = (T)0.5 - (T)1.23046875 * (s * t);
        const T om = (T)1 - s2;
        const T om2 = om * om;
        dfdd = -k.wall_kd * (om2 * om2);
        return F;
    }
    T wall_term(const V3<T>& q, V3<T>& g) const {
        T rho = 0;
        const T qa[3] = {q.x, q.y, q.z};
        T ga[3] = {0, 0, 0};
        for (int a = 0; a < 3; ++a) {
            const T dlo = qa[a] - (T)p.bmin[a];
            if (dlo < k.h) {
                T dfdd;
                const T F = wall_face(dlo, dfdd);
                rho = rho + k.wall_n * F;
                ga[a] = ga[a] + k.wall_n * dfdd;
            }
            const T dhi = (T)p.bmax[a] - qa[a];
            if (dhi < k.h) {
                T dfdd;
                const T F = wall_face(dhi, dfdd);
                rho = rho + k.wall_n * F;
                ga[a] = ga[a] - k.wall_n * dfdd;
            }
        }
        g = {ga[0], ga[1], ga[2]};
        return rho;
    }

    void dims_of(const V3<T>& q, int dim[3]) const {
        // computeDimID: kernels/cudaPBFSolver.cuh:156-160; int() truncates toward zero
        dim[0] = (int)((q.x - (T)p.grid_min[0]) * k.invH);
        dim[1] = (int)((q.y - (T)p.grid_min[1]) * k.invH);
        dim[2] = (int)((q.z - (T)p.grid_min[2]) * k.invH);
    }
    bool out_of_range(const int d[3]) const {
        return d[0] < 0 || d[0] >= p.dims[0] || d[1] < 0 || d[1] >= p.dims[1] || d[2] < 0 || d[2] >= p.dims[2];
    }
    int gid(const int d[3]) const {
        if (out_of_range(d)) return -1;
        return d[0] + d[1] * p.dims[0] + d[2] * p.dims[0] * p.dims[1];
    }

    // ---- one substep ----------------------------------------------------------
    void predict() {
        // updateParticles kernels/cudaPBFSolver.cu:4-13; CPU src/solver.cpp:63-69.
        // GPU formulation: v += dt g and x += dt v each round once, as fused
        // multiply-adds (nvcc contracts these lines of the reference by default;
        // the library evaluates the same fma). CPU formulation: a product and a
        // sum (g++ without -mfma does not contract).
        const V3<T> g{(T)p.gravity[0], (T)p.gravity[1], (T)p.gravity[2]};
        for (int i = 0; i < n; ++i) {
            xold[i] = x[i];
            if (p.formulation == 0) {
                v[i] = {std::fma(k.dt, g.x, v[i].x), std::fma(k.dt, g.y, v[i].y), std::fma(k.dt, g.z, v[i].z)};
                x[i] = {std::fma(k.dt, v[i].x, x[i].x), std::fma(k.dt, v[i].y, x[i].y), std::fma(k.dt, v[i].z, x[i].z)};
            } else {
                v[i] = {v[i].x + k.dt * g.x, v[i].y + k.dt * g.y, v[i].z + k.dt * g.z};
                x[i] = {x[i].x + k.dt * v[i].x, x[i].y + k.dt * v[i].y, x[i].z + k.dt * v[i].z};
            }
            bound(x[i]);
            xpred[i] = x[i];
        }
    }

    void build_grid() {
        // calculateParticlesGid cu:31-40, calculatePrefixSum/addBlockSum cu:42-96,
        // setGrid cu:99-111, countingSort cu:112-122; CPU src/solver.cpp:5-29
        std::fill(cnt.begin(), cnt.end(), 0);
        for (int i = 0; i < n; ++i) {
            int d[3];
            dims_of(x[i], d);
            cell[i] = gid(d);
            if (cell[i] >= 0) cnt[cell[i]]++;
        }
        int acc = 0;
        for (int c = 0; c < ncells; ++c) {
            start[c] = acc;
            acc += cnt[c];
            end[c] = acc;
        }
        const int inside = acc;
        // stable scatter, ascending or descending slot order within a cell
        std::vector<int> fill(ncells, 0);
        if (p.cell_order == 0) {
            for (int i = 0; i < n; ++i)
                if (cell[i] >= 0) sorted[start[cell[i]] + fill[cell[i]]++] = i;
        } else {
            for (int i = n - 1; i >= 0; --i)
                if (cell[i] >= 0) sorted[start[cell[i]] + fill[cell[i]]++] = i;
        }
        int tail = inside;
        for (int i = 0; i < n; ++i)
            if (cell[i] < 0) sorted[tail++] = i;
        if (p.reorder) {
            auto permute3 = [&](std::vector<V3<T>>& a) {
                std::vector<V3<T>> b(n);
                for (int s = 0; s < n; ++s) b[s] = a[sorted[s]];
                a.swap(b);
            };
            permute3(x); permute3(v); permute3(xold); permute3(xpred);
            std::vector<int> pb(n), cb(n);
            for (int s = 0; s < n; ++s) { pb[s] = perm[sorted[s]]; cb[s] = cell[sorted[s]]; }
            perm.swap(pb); cell.swap(cb);
            for (int s = 0; s < n; ++s) sorted[s] = s;
        }
    }

    void append(int i, int j, int& cntv) {
        const V3<T> r = sub(x[i], x[j]);
        T r2;
        if (p.formulation == 1 && !(p.arith == 1 || is_double)) r2 = r.x * r.x + r.y * r.y + r.z * r.z;
        else if (p.arith == 1 && !is_double) r2 = dot_fma(r, r);
        else r2 = dot_ref(r, r);
        if (r2 <= k.h2) nbr[(size_t)i * p.max_nbr + cntv++] = j;
    }

    void build_neighbors() {
        // buildNeighborhood cu:124-154 (x-fastest stencil); CPU src/solver.cpp:31-57 (x outer, z inner)
        const int cap = p.max_nbr;
        for (int i = 0; i < n; ++i) {
            int c = 0;
            int d[3];
            dims_of(x[i], d);
            if (p.formulation == 0) {
                // dz-major, dy, dx fastest (j % 3, j / 3 % 3, j / 9 for R = 1); cells
                // smaller than h widen the stencil to R = ceil(1 / cell_scale)
                const int R = p.cell_scale >= 1.0f ? 1 : (int)std::ceil(1.0 / (double)p.cell_scale);
                for (int dz = -R; dz <= R && c < cap; ++dz)
                    for (int dy = -R; dy <= R && c < cap; ++dy)
                        for (int dx = -R; dx <= R && c < cap; ++dx) {
                            int nd[3] = {d[0] + dx, d[1] + dy, d[2] + dz};
                            const int g = gid(nd);
                            if (g < 0) continue;
                            for (int s = start[g]; s < end[g] && c < cap; ++s) {
                                const int jj = sorted[s];
                                if (jj != i) append(i, jj, c);
                            }
                        }
            } else {
                for (int ox = -1; ox <= 1 && c < cap; ++ox)
                    for (int oy = -1; oy <= 1 && c < cap; ++oy)
                        for (int oz = -1; oz <= 1 && c < cap; ++oz) {
                            int nd[3] = {d[0] + ox, d[1] + oy, d[2] + oz};
                            const int g = gid(nd);
                            if (g < 0) continue;
                            for (int s = start[g]; s < end[g] && c < cap; ++s) {
                                const int jj = sorted[s];
                                if (jj != i) append(i, jj, c);
                            }
                        }
            }
            ncnt[i] = c;
        }
    }

    const int* nb(int i) const { return &nbr[(size_t)i * p.max_nbr]; }

    // pair lanes of the product arithmetic (reference arithmetic: one sequential sum)
    int lanes() const {
        if (!(p.arith == 1 && !is_double) || p.lanes <= 1) return 1;
        return std::min(p.lanes, kMaxLanes);
    }

    T err_max = 0;  // max one-sided density error seen by the last compute_lambda

    void compute_lambda() {
        // calculateLambda cu:156-180; CPU src/solver.cpp:78-95
        const int L = lanes();
        err_max = 0;
        for (int i = 0; i < n; ++i) {
            T rl[kMaxLanes], gml[kMaxLanes];
            V3<T> gsl[kMaxLanes];
            for (int t = 0; t < L; ++t) {
                T r = 0, gm = 0;
                V3<T> gs{0, 0, 0};
                for (int q = t; q < ncnt[i]; q += L) {
                    const int j = nb(i)[q];
                    const V3<T> d = sub(x[i], x[j]);
                    r += W6(d);
                    const V3<T> g = gradW(d);
                    gs = {gs.x + g.x, gs.y + g.y, gs.z + g.z};
                    if (p.arith == 1 && !is_double) {
                        gm = std::fma(g.x, g.x, gm);
                        gm = std::fma(g.y, g.y, gm);
                        gm = std::fma(g.z, g.z, gm);
                    } else {
                        gm += dot_ref(g, g);
                    }
                }
                rl[t] = r; gml[t] = gm; gsl[t] = gs;
            }
            T r = combine_lanes(rl, L), gm = combine_lanes(gml, L);
            V3<T> gs = combine_lanes(gsl, L);
            // one-sided error of the fluid density (before any wall term)
            err_max = std::max(err_max, std::max(r / k.rho0 - (T)1, (T)0));
            if (p.flags & ORACLE_WALL_DENSITY) {
                V3<T> gw;
                r = r + wall_term(x[i], gw);
                gs = {gs.x + gw.x, gs.y + gw.y, gs.z + gw.z};
            }
            T C = r / k.rho0 - (T)1;
            if (p.flags & ORACLE_CLAMP_C) C = std::max(C, (T)0);
            if (p.arith == 1 && !is_double) {
                gm = std::fma(gs.x, gs.x, gm);
                gm = std::fma(gs.y, gs.y, gm);
                gm = std::fma(gs.z, gs.z, gm);
                gm = gm / k.rho0sq;
            } else if (p.formulation == 0 || is_double) {
                gm += dot_ref(gs, gs);
                gm /= k.rho0sq;
            } else {
                gm += dot_ref(gs, gs);
                gm = (T)(float)((double)gm * (1.0 / (double)(p.restRho * p.restRho)));
            }
            rho[i] = r;
            lambda[i] = -C / (gm + k.eps);
        }
    }

    void compute_dp() {
        // calculateOffset cu:182-199; CPU src/solver.cpp:97-108
        const int L = lanes();
        for (int i = 0; i < n; ++i) {
            V3<T> al[kMaxLanes];
            T mag = 0;
            for (int t = 0; t < L; ++t) {
                V3<T> a{0, 0, 0};
                for (int q = t; q < ncnt[i]; q += L) {
                    const int j = nb(i)[q];
                    const V3<T> d = sub(x[i], x[j]);
                    const T w = W6(d);
                    const V3<T> g = gradW(d);
                    // product: fma(-k (W/W(dq))^n, scorr_scale, lambda_i + lambda_j)
                    const T s = (p.arith == 1 && !is_double) ? dp_weight(lambda[i], lambda[j], w)
                                                             : (lambda[i] + lambda[j]) + scorr(w);
                    if (p.arith == 1 && !is_double) {
                        a.x = std::fma(s, g.x, a.x);
                        a.y = std::fma(s, g.y, a.y);
                        a.z = std::fma(s, g.z, a.z);
                    } else {
                        a = {a.x + s * g.x, a.y + s * g.y, a.z + s * g.z};
                    }
                    mag += std::fabs(s) * (std::fabs(g.x) + std::fabs(g.y) + std::fabs(g.z));
                }
                al[t] = a;
            }
            V3<T> a = combine_lanes(al, L);
            if (p.flags & ORACLE_WALL_DENSITY) {
                V3<T> gw;
                wall_term(x[i], gw);
                a.x = std::fma(lambda[i], gw.x, a.x);
                a.y = std::fma(lambda[i], gw.y, a.y);
                a.z = std::fma(lambda[i], gw.z, a.z);
            }
            dp[i] = {a.x / k.rho0, a.y / k.rho0, a.z / k.rho0};
            dpmag[i] = mag / k.rho0;
        }
    }

    void update_positions(bool last) {
        // updatePosition cu:15-22; CPU src/solver.cpp:110-115
        for (int i = 0; i < n; ++i) {
            x[i] = {x[i].x + dp[i].x, x[i].y + dp[i].y, x[i].z + dp[i].z};
            bound(x[i]);
            if (p.formulation == 0 && (last || p.arith == 0))
                v[i] = {(x[i].x - xold[i].x) / k.dt, (x[i].y - xold[i].y) / k.dt, (x[i].z - xold[i].z) / k.dt};
        }
    }

    void vorticity_viscosity() {
        // calculateCurl cu:201-215, calculateVorticityAndViscosity cu:217-239,
        // applyVorticityAndViscosity cu:24-29; CPU src/solver.cpp:117-155
        if (p.formulation == 1) {
            const T invDt = (T)(1.0f / p.dt);
            for (int i = 0; i < n; ++i)
                v[i] = {(x[i].x - xold[i].x) * invDt, (x[i].y - xold[i].y) * invDt, (x[i].z - xold[i].z) * invDt};
        }
        const bool pa = p.arith == 1 && !is_double;
        const int L = lanes();
        for (int i = 0; i < n; ++i) {
            V3<T> wl[kMaxLanes];
            for (int t = 0; t < L; ++t) {
                V3<T> w{0, 0, 0};
                for (int q = t; q < ncnt[i]; q += L) {
                    const int j = nb(i)[q];
                    // GPU: (v_j - v_i) x gradW ; CPU: (v_i - v_j) x gradW
                    const V3<T> vij = p.formulation == 0 ? sub(v[j], v[i]) : sub(v[i], v[j]);
                    const V3<T> g = gradW(sub(x[i], x[j]));
                    const V3<T> c = pa ? cross_fma(vij, g) : cross(vij, g);
                    w = {w.x + c.x, w.y + c.y, w.z + c.z};
                }
                wl[t] = w;
            }
            curl[i] = combine_lanes(wl, L);
        }
        for (int i = 0; i < n; ++i) {
            V3<T> pvl[kMaxLanes], etal[kMaxLanes];
            for (int t = 0; t < L; ++t) {
                V3<T> pv{0, 0, 0}, eta{0, 0, 0};
                for (int q = t; q < ncnt[i]; q += L) {
                    const int j = nb(i)[q];
                    const V3<T> d = sub(x[i], x[j]);
                    const T w = W6(d);
                    if (pa) {
                        const V3<T> vji = sub(v[j], v[i]);
                        pv.x = std::fma(vji.x, w, pv.x);
                        pv.y = std::fma(vji.y, w, pv.y);
                        pv.z = std::fma(vji.z, w, pv.z);
                        const T wl = std::sqrt(dot_fma(curl[j], curl[j]));
                        const V3<T> g = gradW(d);
                        eta.x = std::fma(wl, g.x, eta.x);
                        eta.y = std::fma(wl, g.y, eta.y);
                        eta.z = std::fma(wl, g.z, eta.z);
                    } else {
                        const V3<T> vij = sub(v[i], v[j]);
                        pv = {pv.x - vij.x * w, pv.y - vij.y * w, pv.z - vij.z * w};
                        if (p.formulation == 0) {
                            const T wl = std::sqrt(dot_ref(curl[j], curl[j]));
                            const V3<T> g = gradW(d);
                            eta = {eta.x + wl * g.x, eta.y + wl * g.y, eta.z + wl * g.z};
                        } else {
                            const T s = std::sqrt(dot_ref(curl[j], curl[j])) * w;  // glm vec3 += scalar
                            eta = {eta.x + s, eta.y + s, eta.z + s};
                        }
                    }
                }
                pvl[t] = pv; etal[t] = eta;
            }
            const V3<T> pv = combine_lanes(pvl, L);
            V3<T> eta = combine_lanes(etal, L);
            const T el = std::sqrt(pa ? dot_fma(eta, eta) : dot_ref(eta, eta));
            if (p.formulation == 0) {
                if ((double)el > 1e-3) eta = {eta.x / el, eta.y / el, eta.z / el};
            } else {
                if (!((double)el > -1e-3 && (double)el < 1e-3)) {  // equalZero, include/solver.h:25
                    const T inv = (T)1 / el;
                    eta = {eta.x * inv, eta.y * inv, eta.z * inv};
                }
            }
            const V3<T> cr = cross(eta, curl[i]);
            const T ve = p.formulation == 0 ? k.vort_eps : (T)0.5f;
            vort[i] = {ve * cr.x, ve * cr.y, ve * cr.z};
            visc[i] = {k.visc_c * pv.x, k.visc_c * pv.y, k.visc_c * pv.z};
        }
        for (int i = 0; i < n; ++i) {
            const V3<T> t{k.dt * vort[i].x + visc[i].x, k.dt * vort[i].y + visc[i].y, k.dt * vort[i].z + visc[i].z};
            v[i] = {v[i].x + t.x, v[i].y + t.y, v[i].z + t.z};
        }
    }

    void substep() {
        predict();
        build_grid();
        build_neighbors();
        for (int it = 0; it < p.iterations; ++it) {
            compute_lambda();
            compute_dp();
            update_positions(it == p.iterations - 1);
        }
        vorticity_viscosity();
    }

    // The CUDA library's adaptive substep (no reference counterpart): Jacobi
    // corrections until the max one-sided density error measured by the lambda
    // pass is <= tol, at least min_it and at most max_it corrections; the
    // velocity then comes from the total displacement. Returns the corrections.
    int substep_adaptive(double tol, int min_it, int max_it) {
        predict();
        build_grid();
        build_neighbors();
        int it = 0;
        for (; it < max_it; ++it) {
            compute_lambda();
            if (it >= min_it && (double)err_max <= tol) break;
            compute_dp();
            update_positions(false);
        }
        for (int i = 0; i < n; ++i)
            v[i] = {(x[i].x - xold[i].x) / k.dt, (x[i].y - xold[i].y) / k.dt, (x[i].z - xold[i].z) / k.dt};
        vorticity_viscosity();
        return it;
    }
};

struct Handle {
    int prec;
    Solver<float>* f = nullptr;
    Solver<double>* d = nullptr;
};

template <typename T> int get_field(Solver<T>& s, int field, double* outd, int* outi) {
    const int n = s.n;
    auto put3 = [&](const std::vector<V3<T>>& a) {
        for (int i = 0; i < n; ++i) {
            outd[3 * i] = (double)a[i].x; outd[3 * i + 1] = (double)a[i].y; outd[3 * i + 2] = (double)a[i].z;
        }
        return 0;
    };
    auto put1 = [&](const std::vector<T>& a) {
        for (int i = 0; i < n; ++i) outd[i] = (double)a[i];
        return 0;
    };
    auto puti = [&](const std::vector<int>& a) {
        std::memcpy(outi, a.data(), a.size() * sizeof(int));
        return 0;
    };
    switch (field) {
        case F_X: return put3(s.x);
        case F_V: return put3(s.v);
        case F_XOLD: return put3(s.xold);
        case F_XPRED: return put3(s.xpred);
        case F_LAMBDA: return put1(s.lambda);
        case F_RHO: return put1(s.rho);
        case F_DP: return put3(s.dp);
        case F_CURL: return put3(s.curl);
        case F_VORT: return put3(s.vort);
        case F_VISC: return put3(s.visc);
        case F_DPMAG: return put1(s.dpmag);
        case F_CELL: return puti(s.cell);
        case F_CNT: return puti(s.cnt);
        case F_START: return puti(s.start);
        case F_END: return puti(s.end);
        case F_SORTED: return puti(s.sorted);
        case F_NCNT: return puti(s.ncnt);
        case F_NBR:  // slots past each particle's count are reported as -1
            for (int i = 0; i < n; ++i)
                for (int q = 0; q < s.p.max_nbr; ++q)
                    outi[(size_t)i * s.p.max_nbr + q] = q < s.ncnt[i] ? s.nbr[(size_t)i * s.p.max_nbr + q] : -1;
            return 0;
        case F_PERM: return puti(s.perm);
        default: return -1;
    }
}

}  // namespace

extern "C" {

void* oracle_create(const oracle_params* p, int precision, int n, const float* pos, const float* vel) {
    if (!p || n < 0 || p->dims[0] <= 0 || p->dims[1] <= 0 || p->dims[2] <= 0 || p->max_nbr <= 0) return nullptr;
    Handle* h = new Handle();
    h->prec = precision;
    if (precision == 64) h->d = new Solver<double>(*p, n, pos, vel);
    else h->f = new Solver<float>(*p, n, pos, vel);
    return h;
}

// New parameter values for the following substeps (the library's
// pbf_set_parameter): the grid (dims, cell scale) and neighbour cap must stay.
int oracle_set_params(void* hv, const oracle_params* p) {
    Handle* h = (Handle*)hv;
    if (!h || !p) return -1;
    auto apply = [&](auto* sv) {
        if (p->dims[0] != sv->p.dims[0] || p->dims[1] != sv->p.dims[1] || p->dims[2] != sv->p.dims[2] ||
            p->max_nbr != sv->p.max_nbr)
            return -1;
        sv->p = *p;
        sv->make_consts();
        return 0;
    };
    return h->f ? apply(h->f) : apply(h->d);
}

int oracle_substep(void* hv) {
    Handle* h = (Handle*)hv;
    if (!h) return -1;
    if (h->f) h->f->substep(); else h->d->substep();
    return 0;
}

int oracle_substep_adaptive(void* hv, double tol, int min_it, int max_it) {
    Handle* h = (Handle*)hv;
    if (!h) return -1;
    return h->f ? h->f->substep_adaptive(tol, min_it, max_it) : h->d->substep_adaptive(tol, min_it, max_it);
}

// Runs only the grid build (hash, count, scan, sort) and neighbour search on the
// current positions, without prediction: the stage test of buildNeiborhood.
int oracle_build_only(void* hv) {
    Handle* h = (Handle*)hv;
    if (!h) return -1;
    if (h->f) { h->f->build_grid(); h->f->build_neighbors(); }
    else { h->d->build_grid(); h->d->build_neighbors(); }
    return 0;
}

int oracle_get(void* hv, int field, double* outd, int* outi) {
    Handle* h = (Handle*)hv;
    if (!h) return -1;
    return h->f ? get_field(*h->f, field, outd, outi) : get_field(*h->d, field, outd, outi);
}

int oracle_ncells(void* hv) {
    Handle* h = (Handle*)hv;
    return h->f ? h->f->ncells : h->d->ncells;
}

void oracle_destroy(void* hv) {
    Handle* h = (Handle*)hv;
    if (!h) return;
    delete h->f;
    delete h->d;
    delete h;
}

float oracle_det_sin(float a) { return det_sin(a); }
float oracle_rsqrt(float x) { return soft_rsqrt(x); }

// FP64 density-error oracle: rho_i = sum_{j != i, |r|<=h} W6(r) with the exact
// poly6 constant, over every pair (no neighbour cap), from the given positions.
// Writes the one-sided error max(rho_i/rho0 - 1, 0) per particle when err is not
// null, and returns max and mean over particles.
int oracle_density_error(int n, const float* pos, float h, float rho0, double* out_max, double* out_mean,
                         double* err) {
    if (n <= 0) { *out_max = 0; *out_mean = 0; return 0; }
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], (double)pos[3 * i + a]);
            hi[a] = std::max(hi[a], (double)pos[3 * i + a]);
        }
    const double hd = h;
    int dims[3];
    for (int a = 0; a < 3; ++a) dims[a] = std::max(1, (int)std::floor((hi[a] - lo[a]) / hd) + 1);
    const long long nc = (long long)dims[0] * dims[1] * dims[2];
    std::vector<int> cs(nc + 1, 0), ids(n), cid(n);
    auto cellof = [&](int i, int d[3]) {
        for (int a = 0; a < 3; ++a) d[a] = std::min(dims[a] - 1, (int)std::floor(((double)pos[3 * i + a] - lo[a]) / hd));
    };
    for (int i = 0; i < n; ++i) {
        int d[3];
        cellof(i, d);
        cid[i] = d[0] + dims[0] * (d[1] + dims[1] * d[2]);
        cs[cid[i] + 1]++;
    }
    for (long long c = 0; c < nc; ++c) cs[c + 1] += cs[c];
    std::vector<int> fill(cs.begin(), cs.end() - 1);
    for (int i = 0; i < n; ++i) ids[fill[cid[i]]++] = i;
    const double c6 = 315.0 / (64.0 * M_PI * std::pow(hd, 9));
    const double h2 = hd * hd;
    double mx = 0, sum = 0;
    for (int i = 0; i < n; ++i) {
        int d[3];
        cellof(i, d);
        double rho = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int x = d[0] + dx, y = d[1] + dy, z = d[2] + dz;
                    if (x < 0 || y < 0 || z < 0 || x >= dims[0] || y >= dims[1] || z >= dims[2]) continue;
                    const long long c = x + (long long)dims[0] * (y + (long long)dims[1] * z);
                    for (int s = cs[c]; s < cs[c + 1]; ++s) {
                        const int j = ids[s];
                        if (j == i) continue;
                        const double rx = (double)pos[3 * i] - pos[3 * j];
                        const double ry = (double)pos[3 * i + 1] - pos[3 * j + 1];
                        const double rz = (double)pos[3 * i + 2] - pos[3 * j + 2];
                        const double r2 = rx * rx + ry * ry + rz * rz;
                        if (r2 > h2) continue;
                        const double t = h2 - r2;
                        rho += c6 * t * t * t;
                    }
                }
        const double e = std::max(rho / (double)rho0 - 1.0, 0.0);
        if (err) err[i] = e;
        mx = std::max(mx, e);
        sum += e;
    }
    *out_max = mx;
    *out_mean = sum / n;
    return 0;
}

}  // extern "C"
