// PBF substep kernels for sm_100a.
//
// Data layout in HBM (all particle arrays in cell-sorted slot order, float4 with
// xyz in .x/.y/.z so that a neighbour gather is one 16-byte load):
//   x, v, x_old        float4[n]
//   xl                 float4[n]  positions with lambda in .w (output of the lambda pass)
//   perm               int[n]     slot -> original particle id
//   cell, ticket, tmp  int[n]     hash key, arrival ticket, unsorted cell fill
//   cell_start         int[ncells + 2]: start of each cell, then the out-of-grid bin, then n
//   nbr                int[max_nbr][stride]  slot-major neighbour list (coalesced per slot)
//   ncnt               int[n]
//
// Reference kernels replaced (kernels/cudaPBFSolver.cu): updateParticles :4-13,
// calculateParticlesGid :31-40, calculatePrefixSum :42-89, addBlockSum :91-96,
// setGrid :99-111, countingSort :112-122, buildNeighborhood :124-154,
// calculateLambda :156-180, calculateOffset :182-199, updatePosition :15-22,
// calculateCurl :201-215, calculateVorticityAndViscosity :217-239,
// applyVorticityAndViscosity :24-29.
#include "pbf_kernels.h"

#include <type_traits>

namespace pbf {

// ---------------------------------------------------------------------------
// a1 + a2: predict, bound, hash, histogram (one arrival ticket per particle)
// ---------------------------------------------------------------------------
template <bool PREDICT>
__global__ void __launch_bounds__(256) k_hash(KParams p, const float4* __restrict__ x, const float4* __restrict__ v,
                                              int* __restrict__ cell, int* __restrict__ ticket, int* __restrict__ cnt,
                                              int* __restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    int key = -1;
    if (i < p.n) {
        const SceneView sc = scene_of(p, i);
        f3 xi = make3(x[i]);
        if (PREDICT) {
            f3 vi = make3(v[i]);
            predict(p, sc, xi, vi);
        }
        if (!(isfinite(xi.x) && isfinite(xi.y) && isfinite(xi.z))) atomicOr(err, DEVERR_NONFINITE);
        key = cell_key(p, sc, xi);
    }
    // warp-aggregated histogram: one atomic per distinct cell in the warp
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(peers) - 1;
    const int rank = __popc(peers & ((1u << lane) - 1u));
    int base = 0;
    if (key >= 0 && lane == leader) base = atomicAdd(&cnt[key], __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (i < p.n) {
        cell[i] = key;
        ticket[i] = base + rank;
    }
}

// ---------------------------------------------------------------------------
// a3 + a4: exclusive scan of the cell counts with decoupled look-back; writes
// cell_start[0..m) and cell_start[m] = total, and clears the counts for the next
// substep. Status words: (flag << 32) | value, flag 1 = tile aggregate,
// 2 = inclusive prefix. Tiles are numbered in launch order by an atomic ticket,
// so every predecessor is already running and the wait always ends; the wait is
// bounded anyway and reports DEVERR_SCAN_TIMEOUT.
// ---------------------------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr long long SCAN_SPIN_LIMIT = 1ll << 22;

__device__ __forceinline__ void st_release_u64(unsigned long long* a, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(a), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* a) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a) : "memory");
    return v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan(int* __restrict__ cnt, int* __restrict__ out, int m,
                                                       unsigned long long* __restrict__ status,
                                                       int* __restrict__ tile_counter, int* __restrict__ err,
                                                       int clear) {
    __shared__ int s_tile;
    __shared__ int s_warp[SCAN_THREADS / 32];
    __shared__ int s_excl, s_tot;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) s_tile = atomicAdd(tile_counter, 1);
    __syncthreads();
    const int tile = s_tile;

    // Warp w owns elements [tile * TILE + w * 512, +512) in 16 rounds of 32
    // consecutive elements (one coalesced 128-byte access per round); each round
    // is scanned across the warp and carried into the next.
    const long long wbase = (long long)tile * SCAN_TILE + (long long)warp * (32 * SCAN_ITEMS);
    int item[SCAN_ITEMS];
#pragma unroll
    for (int q = 0; q < SCAN_ITEMS; ++q) {
        const long long idx = wbase + q * 32 + lane;
        item[q] = idx < m ? cnt[idx] : 0;
    }
    int carry = 0;  // warp-exclusive offset of round q
#pragma unroll
    for (int q = 0; q < SCAN_ITEMS; ++q) {
        int incl = item[q];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int excl_q = carry + incl - item[q];
        carry += __shfl_sync(0xffffffffu, incl, 31);
        item[q] = excl_q;  // now the exclusive prefix within the warp's range
    }
    if (lane == 0) s_warp[warp] = carry;  // the warp's total
    __syncthreads();
    if (warp == 0) {
        int w = lane < SCAN_THREADS / 32 ? s_warp[lane] : 0;
        int wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        if (lane < SCAN_THREADS / 32) s_warp[lane] = wi - w;  // exclusive warp offsets
        const int total = __shfl_sync(0xffffffffu, wi, SCAN_THREADS / 32 - 1);
        // decoupled look-back
        int excl = 0;
        if (tile == 0) {
            if (lane == 0) st_release_u64(&status[0], (2ull << 32) | (unsigned)total);
        } else {
            if (lane == 0) st_release_u64(&status[tile], (1ull << 32) | (unsigned)total);
            int pos = tile - 1;  // highest tile not yet folded in
            bool done = false;
            while (!done) {
                const int look = pos - lane;
                unsigned long long s = 0;
                if (look >= 0) {
                    long long spins = 0;
                    s = ld_acquire_u64(&status[look]);
                    while ((s >> 32) == 0ull) {
                        if (++spins > SCAN_SPIN_LIMIT) {
                            atomicOr(err, DEVERR_SCAN_TIMEOUT);
                            s = 2ull << 32;  // give up: treat as prefix 0 so the tile finishes
                            break;
                        }
                        __nanosleep(64);
                        s = ld_acquire_u64(&status[look]);
                    }
                } else {
                    s = 2ull << 32;  // before tile 0: an empty prefix
                }
                const unsigned flag = (unsigned)(s >> 32);
                const int val = (int)(unsigned)(s & 0xffffffffu);
                const unsigned prefix_mask = __ballot_sync(0xffffffffu, flag == 2u);
                const int stop = prefix_mask ? __ffs(prefix_mask) - 1 : 31;
                int contrib = lane <= stop ? val : 0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, o);
                excl += contrib;
                if (prefix_mask) done = true;
                else pos -= 32;
            }
            if (lane == 0) st_release_u64(&status[tile], (2ull << 32) | (unsigned)(excl + total));
        }
        if (lane == 0) {
            s_excl = excl;
            s_tot = total;
        }
    }
    __syncthreads();
    const int off = s_excl + s_warp[warp];
#pragma unroll
    for (int q = 0; q < SCAN_ITEMS; ++q) {
        const long long idx = wbase + q * 32 + lane;
        if (idx < m) {
            out[idx] = off + item[q];
            if (clear) cnt[idx] = 0;
        }
    }
    if (tile == (int)(((long long)m - 1) / SCAN_TILE) && threadIdx.x == SCAN_THREADS - 1) {
        // the last tile writes the grand total at out[m] (its inclusive prefix)
        out[m] = s_excl + s_tot;
    }
}

// ---------------------------------------------------------------------------
// a5: scatter by ticket (unordered within a cell), then a stable rank within the
// cell and the reorder of the particle state into slot order (a6).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_scatter(int n, const int* __restrict__ cell, const int* __restrict__ ticket,
                                                 const int* __restrict__ cell_start, int* __restrict__ tmp,
                                                 int* __restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int dst = cell_start[cell[i]] + ticket[i];
    if (dst < 0 || dst >= n) {  // counts and tickets disagree: report, never write out of bounds
        atomicOr(err, DEVERR_BAD_INDEX);
        return;
    }
    tmp[dst] = i;
}

template <bool PREDICT>
__global__ void __launch_bounds__(256) k_reorder(KParams p, const float4* __restrict__ x, const float4* __restrict__ v,
                                                 const int* __restrict__ perm, const int* __restrict__ cell,
                                                 const int* __restrict__ cell_start, const int* __restrict__ tmp,
                                                 float4* __restrict__ xp, float4* __restrict__ vp,
                                                 float4* __restrict__ xold, int* __restrict__ perm_out,
                                                 int* __restrict__ cell_sorted, const float* __restrict__ lam_in,
                                                 float* __restrict__ lam_out, int* __restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= p.n) return;
    const int c = cell[i];
    const int s = cell_start[c], e = min(cell_start[c + 1], p.n);
    if (s < 0 || s >= e) {
        atomicOr(err, DEVERR_BAD_INDEX);
        return;
    }
    const SceneView sc = scene_of(p, i);
    const bool desc = p.cell_order == 1 && c != sc.cell_base + sc.ncells;  // out-of-grid bin stays ascending
    int q = 0;
    for (int k = s; k < e; ++k) {
        const int o = tmp[k];
        q += desc ? (o > i) : (o < i);
    }
    const int dst = s + q;  // < e <= n
    const float4 x4 = x[i];
    f3 xi = make3(x4);
    f3 vi = make3(v[i]);
    if (PREDICT) predict(p, sc, xi, vi);
    xp[dst] = make_float4(xi.x, xi.y, xi.z, 0.0f);
    vp[dst] = make_float4(vi.x, vi.y, vi.z, 0.0f);
    xold[dst] = make_float4(x4.x, x4.y, x4.z, 0.0f);
    perm_out[dst] = perm[i];
    cell_sorted[dst] = c;
    if (lam_out) lam_out[dst] = lam_in[i];
}

// ---------------------------------------------------------------------------
// Pair lanes. L consecutive threads of a warp (a team) share one particle of the
// neighbour sums: lane t takes list entries t, t+L, t+2L, ... in order and the L
// partial sums are combined by an xor butterfly over distances 1, 2, 4:
// ((p0 + p1) + (p2 + p3)) + ..., the same value on every lane of the team (IEEE
// addition is commutative). A team shortens each thread's dependent index ->
// position gather chain L-fold and puts L times as many threads in flight, at
// the price of the team's shuffles and of the per-particle epilogue running on
// one lane of L. (The neighbour search stays one thread per particle: with teams
// it issued 2.8x the instructions for the same lists.)
// ---------------------------------------------------------------------------
template <int L> struct Team {
    int k;          // particle slot
    int t;          // lane within the team
    unsigned mask;  // the team's lanes within the warp
};

// blockDim.x is a multiple of 32, so a team never straddles a warp
template <int L> __device__ __forceinline__ Team<L> team_of() {
    Team<L> m;
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    m.k = (int)(g / L);
    m.t = (int)(threadIdx.x & (L - 1));
    const int lane = threadIdx.x & 31;
    m.mask = L >= 32 ? 0xffffffffu : (((1u << L) - 1u) << (lane & ~(L - 1)));
    return m;
}

template <int L> __device__ __forceinline__ float team_sum(float v, unsigned mask) {
#pragma unroll
    for (int o = 1; o < L; o <<= 1) v += __shfl_xor_sync(mask, v, o);
    return v;
}

template <int L> __device__ __forceinline__ f3 team_sum3(f3 v, unsigned mask) {
    return {team_sum<L>(v.x, mask), team_sum<L>(v.y, mask), team_sum<L>(v.z, mask)};
}

// ---------------------------------------------------------------------------
// a7: 27-cell neighbour search (a (2R+1)^3 stencil when cells are smaller than
// h). The stencil is visited dz-major, dy, then the dx cells of a row, which are
// one contiguous slot range because keys are x-fastest; within a cell, slot
// order. For R = 1 this is the reference order (buildNeighborhood cu:133-136)
// applied to the sorted slots.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_neighbors(KParams p, const float4* __restrict__ x,
                                                   const int* __restrict__ cell_start, int* __restrict__ nbr,
                                                   int* __restrict__ ncnt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.n) return;
    const SceneView sc = scene_of(p, k);
    const f3 xk = make3(x[k]);
    int d[3];
    cell_dims(p, sc, xk, d);
    const int nx = sc.dims[0], ny = sc.dims[1], nz = sc.dims[2];
    const int R = p.radius;
    const int x0 = max(d[0] - R, 0), x1 = min(d[0] + R, nx - 1);
    int c = 0;
    const int cap = p.max_nbr;
    if (x0 <= x1) {
        for (int dz = -R; dz <= R && c < cap; ++dz) {
            const int z = d[2] + dz;
            if (z < 0 || z >= nz) continue;
            for (int dy = -R; dy <= R && c < cap; ++dy) {
                const int y = d[1] + dy;
                if (y < 0 || y >= ny) continue;
                const int row = sc.cell_base + y * nx + z * nx * ny;
                const int s = cell_start[row + x0], e = cell_start[row + x1 + 1];
                for (int j = s; j < e && c < cap; ++j) {
                    if (j == k) continue;
                    const f3 r = sub3(xk, make3(x[j]));
                    if (dot_fma(r, r) <= p.h2) {
                        nbr[(size_t)c * p.stride + k] = j;
                        ++c;
                    }
                }
            }
        }
    }
    ncnt[k] = c;
}

// ---------------------------------------------------------------------------
// a9: density, constraint and lambda (calculateLambda cu:156-180)
// ---------------------------------------------------------------------------
// Neighbour gathers are issued NB at a time: NB list loads (coalesced, slot-major
// list), then NB 16-byte position loads, so a thread keeps several memory
// requests in flight instead of one dependent index->position chain per pair.
constexpr int NB = 4;

// Entries q0, q0 + L, ..., q0 + (B-1) L of slot k's list (slot k itself past the end).
template <int L, int B>
__device__ __forceinline__ void load_idx(const KParams& p, const int* __restrict__ nbr, int k, int q0, int cnt,
                                         int (&jj)[B]) {
#pragma unroll
    for (int u = 0; u < B; ++u) {
        const int q = q0 + u * L;
        jj[u] = q < cnt ? nbr[(size_t)q * p.stride + k] : k;
    }
}

template <int L, typename V>
__device__ __forceinline__ void gather_batch(const KParams& p, const int* __restrict__ nbr, const V* __restrict__ src,
                                             int k, int q0, int cnt, V (&out)[NB]) {
    int jj[NB];
    load_idx<L, NB>(p, nbr, k, q0, cnt, jj);
#pragma unroll
    for (int u = 0; u < NB; ++u) out[u] = src[jj[u]];
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
}

template <bool DEBUG, int L>
// 6 resident blocks per SM: 40 registers without spills (7 spills)
__global__ void __launch_bounds__(256, 6) k_lambda(KParams p, const float4* __restrict__ x, const int* __restrict__ nbr,
                                                const int* __restrict__ ncnt, float4* __restrict__ xl,
                                                float* __restrict__ rho_out, IterCtl ctl) {
    if (ctl.done && *ctl.done) return;
    const Team<L> tm = team_of<L>();
    const int k = tm.k;
    float err = 0.0f;
    if (k < p.n) {
        const f3 xk = make3(x[k]);
        const int cnt = ncnt[k];
        float rho = 0.0f, gm = 0.0f;
        f3 gs = {0.0f, 0.0f, 0.0f};
        // batches of NB of this lane's entries: all index loads, then all position
        // loads, then the pairs in list order
        for (int q0 = tm.t; q0 < cnt; q0 += L * NB) {
            float4 xj[NB];
            gather_batch<L>(p, nbr, x, k, q0, cnt, xj);
#pragma unroll
            for (int u = 0; u < NB; ++u) {
                if (q0 + u * L >= cnt) break;
                const f3 r = sub3(xk, make3(xj[u]));
                const float r2 = dot_fma(r, r);
                rho = rho + w_poly6(p, r2);
                const f3 g = grad_spiky(p, r, r2);
                gs = {gs.x + g.x, gs.y + g.y, gs.z + g.z};
                gm = __fmaf_rn(g.x, g.x, gm);
                gm = __fmaf_rn(g.y, g.y, gm);
                gm = __fmaf_rn(g.z, g.z, gm);
            }
        }
        rho = team_sum<L>(rho, tm.mask);
        gm = team_sum<L>(gm, tm.mask);
        gs = team_sum3<L>(gs, tm.mask);
        if (tm.t == 0) {
            // one-sided error of the fluid density at these positions (no wall term)
            err = fmaxf(__fdiv_rn(rho, p.rho0) - 1.0f, 0.0f);
            if (p.flags & FLAG_WALL_DENSITY) {
                f3 gw;
                rho = rho + wall_term(p, scene_of(p, k), xk, gw);
                gs = {gs.x + gw.x, gs.y + gw.y, gs.z + gw.z};
            }
            float C = __fdiv_rn(rho, p.rho0) - 1.0f;
            if (p.flags & FLAG_CLAMP_C) C = fmaxf(C, 0.0f);
            gm = __fmaf_rn(gs.x, gs.x, gm);
            gm = __fmaf_rn(gs.y, gs.y, gm);
            gm = __fmaf_rn(gs.z, gs.z, gm);
            gm = __fdiv_rn(gm, p.rho0sq);
            const float lam = __fdiv_rn(-C, gm + p.eps);
            xl[k] = make_float4(xk.x, xk.y, xk.z, lam);
            if (ctl.lam_acc) ctl.lam_acc[k] += lam;
            if (DEBUG) rho_out[k] = rho;
        }
    }
    if (ctl.max_bits) block_error_reduce(err, ctl.max_bits, ctl.sum);
}

// ---------------------------------------------------------------------------
// a17: warm-start features (no reference counterpart), computed in the first
// lambda pass of a substep together with that pass's lambda (the same
// arithmetic as k_lambda, so recording features changes no result):
//   0 neighbour count / cap         1 fluid density / rho0
//   2 previous substep's total lambda
//   3 sum |grad C|^2 (the lambda denominator without eps)
//   4 velocity divergence sum (v_j - v_i) . grad W / rho0 (predicted velocities)
//   5-7 distance to the nearer wall per axis / h, clamped to [0, 4]
//   8-11 occupancy of the 27 cells around the particle's cell: own cell, mean,
//        fraction non-empty, maximum
// lam_acc starts the substep's total lambda at this pass's lambda.
// ---------------------------------------------------------------------------
template <int L>
__global__ void __launch_bounds__(256) k_features(KParams p, const float4* __restrict__ x,
                                                  const float4* __restrict__ v, const int* __restrict__ nbr,
                                                  const int* __restrict__ ncnt, const int* __restrict__ cell_start,
                                                  const float* __restrict__ lam_prev, float4* __restrict__ xl,
                                                  float* __restrict__ feat, float* __restrict__ lam_acc) {
    const Team<L> tm = team_of<L>();
    const int k = tm.k;
    if (k >= p.n) return;  // uniform over the team
    const f3 xk = make3(x[k]);
    const f3 vk = make3(v[k]);
    const int cnt = ncnt[k];
    float rho = 0.0f, gm = 0.0f, div = 0.0f;
    f3 gs = {0.0f, 0.0f, 0.0f};
    for (int q0 = tm.t; q0 < cnt; q0 += L * NB) {
        int jj[NB];
        load_idx<L, NB>(p, nbr, k, q0, cnt, jj);
        float4 xj[NB], vj[NB];
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            xj[u] = x[jj[u]];
            vj[u] = v[jj[u]];
        }
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            if (q0 + u * L >= cnt) break;
            const f3 r = sub3(xk, make3(xj[u]));
            const float r2 = dot_fma(r, r);
            rho = rho + w_poly6(p, r2);
            const f3 g = grad_spiky(p, r, r2);
            gs = {gs.x + g.x, gs.y + g.y, gs.z + g.z};
            gm = __fmaf_rn(g.x, g.x, gm);
            gm = __fmaf_rn(g.y, g.y, gm);
            gm = __fmaf_rn(g.z, g.z, gm);
            const f3 vji = sub3(make3(vj[u]), vk);
            div = __fmaf_rn(vji.x, g.x, div);
            div = __fmaf_rn(vji.y, g.y, div);
            div = __fmaf_rn(vji.z, g.z, div);
        }
    }
    rho = team_sum<L>(rho, tm.mask);
    gm = team_sum<L>(gm, tm.mask);
    gs = team_sum3<L>(gs, tm.mask);
    div = team_sum<L>(div, tm.mask);
    if (tm.t != 0) return;
    const SceneView sc = scene_of(p, k);
    const float rho_fluid = rho;
    if (p.flags & FLAG_WALL_DENSITY) {
        f3 gw;
        rho = rho + wall_term(p, sc, xk, gw);
        gs = {gs.x + gw.x, gs.y + gw.y, gs.z + gw.z};
    }
    float C = __fdiv_rn(rho, p.rho0) - 1.0f;
    if (p.flags & FLAG_CLAMP_C) C = fmaxf(C, 0.0f);
    gm = __fmaf_rn(gs.x, gs.x, gm);
    gm = __fmaf_rn(gs.y, gs.y, gm);
    gm = __fmaf_rn(gs.z, gs.z, gm);
    gm = __fdiv_rn(gm, p.rho0sq);
    const float lam = __fdiv_rn(-C, gm + p.eps);
    xl[k] = make_float4(xk.x, xk.y, xk.z, lam);
    lam_acc[k] = lam;

    float f[12];
    f[0] = (float)cnt / (float)p.max_nbr;
    f[1] = rho_fluid / p.rho0;
    f[2] = lam_prev[k];
    f[3] = gm;
    f[4] = div / p.rho0;
    const float qa[3] = {xk.x, xk.y, xk.z};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float dw = fminf(qa[a] - sc.bmin[a], sc.bmax[a] - qa[a]) * p.inv_h;
        f[5 + a] = fminf(fmaxf(dw, 0.0f), 4.0f);
    }
    int d[3];
    cell_dims(p, sc, xk, d);
    int own = 0, tot = 0, nonempty = 0, mx = 0;
    // nine rows of three x-adjacent cells; a row's counts are differences of
    // consecutive cell starts (keys are x-fastest)
    const int x0 = max(d[0] - 1, 0), x1 = min(d[0] + 1, sc.dims[0] - 1);
    if (x0 <= x1) {
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy) {
                const int cy = d[1] + dy, cz = d[2] + dz;
                if (cy < 0 || cz < 0 || cy >= sc.dims[1] || cz >= sc.dims[2]) continue;
                const int row = sc.cell_base + cy * sc.dims[0] + cz * sc.dims[0] * sc.dims[1];
                int prev = cell_start[row + x0];
                for (int cx = x0; cx <= x1; ++cx) {
                    const int next = cell_start[row + cx + 1];
                    const int occ = next - prev;
                    prev = next;
                    if (cx == d[0] && dy == 0 && dz == 0) own = occ;
                    tot += occ;
                    nonempty += occ > 0;
                    mx = max(mx, occ);
                }
            }
    }
    f[8] = (float)own;
    f[9] = (float)tot / 27.0f;
    f[10] = (float)nonempty / 27.0f;
    f[11] = (float)mx;
#pragma unroll
    for (int i = 0; i < 12; ++i) feat[(size_t)k * 12 + i] = f[i];
}

// Copies features and total lambda of the given slots (training rows).
__global__ void k_gather_rows(const int* __restrict__ slots, int count, int n, const float* __restrict__ feat,
                              const float* __restrict__ lam_acc, float* __restrict__ out_feat,
                              float* __restrict__ out_target, int* __restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int s = slots[i];
    if (s < 0 || s >= n) {
        atomicOr(err, DEVERR_BAD_INDEX);
        return;
    }
#pragma unroll
    for (int c = 0; c < 12; ++c) out_feat[(size_t)i * 12 + c] = feat[(size_t)s * 12 + c];
    out_target[i] = lam_acc[s];
}

// Adds the substep's corrections to the running total and counts the substep as
// a fallback when the adaptive loop needed more than the configured count.
__global__ void k_count_fallback(const int* __restrict__ iters, int first, int configured, int* __restrict__ fallback,
                                 long long* __restrict__ total) {
    const int used = first + *iters;
    if (used > configured) *fallback += 1;
    *total += used;
}

// ---------------------------------------------------------------------------
// a10 + a11: position correction with tensile s_corr, then x += dp, wall clamp,
// and on the last iteration v = (x - x_old) / dt
// (calculateOffset cu:182-199, updatePosition cu:15-22)
// ---------------------------------------------------------------------------
template <bool DEBUG, int L>
__global__ void __launch_bounds__(256, 6) k_dp(KParams p, const float4* __restrict__ xl, const int* __restrict__ nbr,
                                            const int* __restrict__ ncnt, const float4* __restrict__ xold,
                                            float4* __restrict__ xout, float4* __restrict__ vout,
                                            float4* __restrict__ dp_out, IterCtl ctl) {
    if (ctl.done) {
        if (*ctl.done) return;
        // the lambda pass just measured the positions this pass would correct;
        // when they are within tolerance the loop ends here
        if (ctl.may_stop && __longlong_as_double((long long)*ctl.max_bits) <= ctl.tol) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                *ctl.done = 1;
                *ctl.conv_slot = ctl.slot;
            }
            return;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(ctl.iters, 1);
    }
    const Team<L> tm = team_of<L>();
    const int k = tm.k;
    if (k >= p.n) return;  // uniform over the team
    const float4 xk4 = xl[k];
    const f3 xk = make3(xk4);
    const float lk = xk4.w;
    const int cnt = ncnt[k];
    f3 a = {0.0f, 0.0f, 0.0f};
    for (int q0 = tm.t; q0 < cnt; q0 += L * NB) {
        float4 xj[NB];
        gather_batch<L>(p, nbr, xl, k, q0, cnt, xj);
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            if (q0 + u * L >= cnt) break;
            const float4 xj4 = xj[u];
            const f3 r = sub3(xk, make3(xj4));
            const float r2 = dot_fma(r, r);
            const float w = w_poly6(p, r2);
            const f3 g = grad_spiky(p, r, r2);
            const float s = (lk + xj4.w) + s_corr(p, w);
            a.x = __fmaf_rn(s, g.x, a.x);
            a.y = __fmaf_rn(s, g.y, a.y);
            a.z = __fmaf_rn(s, g.z, a.z);
        }
    }
    a = team_sum3<L>(a, tm.mask);
    if (tm.t != 0) return;
    if (p.flags & FLAG_WALL_DENSITY) {
        f3 gw;
        wall_term(p, scene_of(p, k), xk, gw);
        a.x = __fmaf_rn(lk, gw.x, a.x);
        a.y = __fmaf_rn(lk, gw.y, a.y);
        a.z = __fmaf_rn(lk, gw.z, a.z);
    }
    const f3 dp = {__fdiv_rn(a.x, p.rho0), __fdiv_rn(a.y, p.rho0), __fdiv_rn(a.z, p.rho0)};
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

// v = (x - x_old) / dt as its own pass (adaptive iteration counts)
__global__ void __launch_bounds__(256) k_velocity(KParams p, const float4* __restrict__ x,
                                                  const float4* __restrict__ xold, float4* __restrict__ v) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.n) return;
    const float4 xn = x[k], xo = xold[k];
    v[k] = make_float4(__fdiv_rn(xn.x - xo.x, p.dt), __fdiv_rn(xn.y - xo.y, p.dt), __fdiv_rn(xn.z - xo.z, p.dt), 0.0f);
}

// ---------------------------------------------------------------------------
// a12: vorticity (calculateCurl cu:201-215): w_i = sum (v_j - v_i) x gradW(x_i - x_j)
// ---------------------------------------------------------------------------
template <int L>
__global__ void __launch_bounds__(256) k_curl(KParams p, const float4* __restrict__ x, const float4* __restrict__ v,
                                              const int* __restrict__ nbr, const int* __restrict__ ncnt,
                                              float4* __restrict__ omega) {
    const Team<L> tm = team_of<L>();
    const int k = tm.k;
    if (k >= p.n) return;  // uniform over the team
    const f3 xk = make3(x[k]);
    const f3 vk = make3(v[k]);
    const int cnt = ncnt[k];
    f3 w = {0.0f, 0.0f, 0.0f};
    for (int q0 = tm.t; q0 < cnt; q0 += L * NB) {
        int jj[NB];
        load_idx<L, NB>(p, nbr, k, q0, cnt, jj);
        float4 xj[NB], vj[NB];
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            xj[u] = x[jj[u]];
            vj[u] = v[jj[u]];
        }
#pragma unroll
        for (int u = 0; u < NB; ++u) {
            if (q0 + u * L >= cnt) break;
            const f3 r = sub3(xk, make3(xj[u]));
            const f3 g = grad_spiky(p, r, dot_fma(r, r));
            const f3 c = cross3(sub3(make3(vj[u]), vk), g);
            w = {w.x + c.x, w.y + c.y, w.z + c.z};
        }
    }
    w = team_sum3<L>(w, tm.mask);
    // |w| in .w: the vorticity pass needs |w_j| for every pair
    if (tm.t == 0) omega[k] = make_float4(w.x, w.y, w.z, __fsqrt_rn(dot_fma(w, w)));
}

// ---------------------------------------------------------------------------
// a13: vorticity confinement and XSPH, applied to v
// (calculateVorticityAndViscosity cu:217-239, applyVorticityAndViscosity cu:24-29)
// ---------------------------------------------------------------------------
template <bool DEBUG, int L>
__global__ void __launch_bounds__(256) k_vort(KParams p, const float4* __restrict__ x, const float4* __restrict__ v,
                                              const float4* __restrict__ omega, const int* __restrict__ nbr,
                                              const int* __restrict__ ncnt, float4* __restrict__ vout,
                                              const int* __restrict__ perm_in, int* __restrict__ perm_out,
                                              float4* __restrict__ vort_out, float4* __restrict__ visc_out) {
    const Team<L> tm = team_of<L>();
    const int k = tm.k;
    if (k >= p.n) return;  // uniform over the team
    const f3 xk = make3(x[k]);
    const f3 vk = make3(v[k]);
    const int cnt = ncnt[k];
    f3 pv = {0.0f, 0.0f, 0.0f}, eta = {0.0f, 0.0f, 0.0f};
    constexpr int NBV = 2;  // entries per batch: three 16-byte gathers each
    for (int q0 = tm.t; q0 < cnt; q0 += L * NBV) {
        int jj[NBV];
        load_idx<L, NBV>(p, nbr, k, q0, cnt, jj);
        float4 xj[NBV], vj[NBV], oj4[NBV];
#pragma unroll
        for (int u = 0; u < NBV; ++u) {
            xj[u] = x[jj[u]];
            vj[u] = v[jj[u]];
            oj4[u] = omega[jj[u]];
        }
#pragma unroll
        for (int u = 0; u < NBV; ++u) {
            if (q0 + u * L >= cnt) break;
            const f3 r = sub3(xk, make3(xj[u]));
            const float r2 = dot_fma(r, r);
            const float w = w_poly6(p, r2);
            const f3 vji = sub3(make3(vj[u]), vk);
            pv.x = __fmaf_rn(vji.x, w, pv.x);
            pv.y = __fmaf_rn(vji.y, w, pv.y);
            pv.z = __fmaf_rn(vji.z, w, pv.z);
            const float wl = oj4[u].w;  // |w_j| (k_curl)
            const f3 g = grad_spiky(p, r, r2);
            eta.x = __fmaf_rn(wl, g.x, eta.x);
            eta.y = __fmaf_rn(wl, g.y, eta.y);
            eta.z = __fmaf_rn(wl, g.z, eta.z);
        }
    }
    pv = team_sum3<L>(pv, tm.mask);
    eta = team_sum3<L>(eta, tm.mask);
    if (tm.t != 0) return;
    const float el = __fsqrt_rn(dot_fma(eta, eta));
    if ((double)el > 1e-3) eta = {__fdiv_rn(eta.x, el), __fdiv_rn(eta.y, el), __fdiv_rn(eta.z, el)};
    const f3 cr = cross3(eta, make3(omega[k]));
    const f3 fv = {p.vort_eps * cr.x, p.vort_eps * cr.y, p.vort_eps * cr.z};
    const f3 vs = {p.visc_c * pv.x, p.visc_c * pv.y, p.visc_c * pv.z};
    const f3 t = {p.dt * fv.x + vs.x, p.dt * fv.y + vs.y, p.dt * fv.z + vs.z};
    vout[k] = make_float4(vk.x + t.x, vk.y + t.y, vk.z + t.z, 0.0f);
    perm_out[k] = perm_in[k];
    if (DEBUG) {
        vort_out[k] = make_float4(fv.x, fv.y, fv.z, 0.0f);
        visc_out[k] = make_float4(vs.x, vs.y, vs.z, 0.0f);
    }
}

// ---------------------------------------------------------------------------
// a18: one-sided density error over the neighbour list, accumulated in FP64:
// e_k = max(rho_k / rho0 - 1, 0); writes max (as ordered bits) and sum.
// When tol >= 0 it also raises *done once max <= tol (adaptive iterations).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_density_error(KParams p, const float4* __restrict__ x,
                                                       const int* __restrict__ nbr, const int* __restrict__ ncnt,
                                                       unsigned long long* __restrict__ max_bits,
                                                       double* __restrict__ sum, const int* __restrict__ skip) {
    if (skip && *skip) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (k < p.n) {
        const float4 xk = x[k];
        const int cnt = ncnt[k];
        double rho = 0.0;
        const double h2 = (double)p.h * (double)p.h;
        for (int q = 0; q < cnt; ++q) {
            const int j = nbr[(size_t)q * p.stride + k];
            const float4 xj = x[j];
            const double rx = (double)xk.x - (double)xj.x, ry = (double)xk.y - (double)xj.y,
                         rz = (double)xk.z - (double)xj.z;
            const double r2 = rx * rx + ry * ry + rz * rz;
            if (r2 <= h2) {
                const double t = h2 - r2;
                rho += p.poly6_c64 * t * t * t;
            }
        }
        e = fmax(rho / (double)p.rho0 - 1.0, 0.0);
    }
    __shared__ double s_max[8], s_sum[8];
    double m = e, s = e;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { s_max[warp] = m; s_sum[warp] = s; }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int w = 1; w < nw; ++w) { m = fmax(m, s_max[w]); s += s_sum[w]; }
        atomicMax(max_bits, (unsigned long long)__double_as_longlong(m));  // m >= 0: bits order as values
        atomicAdd(sum, s);
    }
}

// ---------------------------------------------------------------------------
// layout kernels
// ---------------------------------------------------------------------------
__global__ void k_from_aos(int n, const float* __restrict__ pos, const float* __restrict__ vel, float4* __restrict__ x,
                           float4* __restrict__ v, int* __restrict__ perm, int* __restrict__ err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const float vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
    if (!(isfinite(px) && isfinite(py) && isfinite(pz) && isfinite(vx) && isfinite(vy) && isfinite(vz)))
        atomicOr(err, DEVERR_NONFINITE);
    x[i] = make_float4(px, py, pz, 0.0f);
    v[i] = make_float4(vx, vy, vz, 0.0f);
    perm[i] = i;
}

// slot order -> original order, AoS xyz
__global__ void k_to_aos(int n, const float4* __restrict__ a, const int* __restrict__ perm, float* __restrict__ out,
                         int* __restrict__ err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = perm[k];
    if (o < 0 || o >= n) {
        atomicOr(err, DEVERR_BAD_INDEX);
        return;
    }
    const float4 q = a[k];
    out[3 * o] = q.x;
    out[3 * o + 1] = q.y;
    out[3 * o + 2] = q.z;
}

__global__ void k_copy4(int n, const float4* __restrict__ a, float4* __restrict__ b) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) b[k] = a[k];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline int blocks_for(int n, int bs) { return (n + bs - 1) / bs; }
// blocks for n particles with L threads each
static inline int team_blocks(int n, int L, int bs) { return (int)(((long long)n * L + bs - 1) / bs); }

// Calls f with the pair-lane count as a compile-time constant.
template <typename F> void with_lanes(int lanes, F&& f) {
    switch (lanes) {
        case 1: f(std::integral_constant<int, 1>{}); break;
        case 8: f(std::integral_constant<int, 8>{}); break;
        case 4: f(std::integral_constant<int, 4>{}); break;
        default: f(std::integral_constant<int, 2>{}); break;
    }
}

void launch_hash(const KParams& p, bool predict_on, const float4* x, const float4* v, int* cell, int* ticket, int* cnt,
                 int* err, cudaStream_t st) {
    const int b = blocks_for(p.n, 256);
    if (predict_on) k_hash<true><<<b, 256, 0, st>>>(p, x, v, cell, ticket, cnt, err);
    else k_hash<false><<<b, 256, 0, st>>>(p, x, v, cell, ticket, cnt, err);
}

size_t scan_status_bytes(int m) {
    const int tiles = (m + SCAN_TILE - 1) / SCAN_TILE;
    return (size_t)tiles * sizeof(unsigned long long) + 16;
}

void launch_scan(int* cnt, int* out, int m, void* status_ws, int* err, cudaStream_t st) {
    const int tiles = (m + SCAN_TILE - 1) / SCAN_TILE;
    unsigned long long* status = (unsigned long long*)status_ws;
    int* counter = (int*)(status + tiles);
    cudaMemsetAsync(status_ws, 0, scan_status_bytes(m), st);
    k_scan<<<tiles, SCAN_THREADS, 0, st>>>(cnt, out, m, status, counter, err, 1);
}

void launch_scan_const(const int* in, int* out, int m, void* status_ws, int* err, cudaStream_t st) {
    const int tiles = (m + SCAN_TILE - 1) / SCAN_TILE;
    unsigned long long* status = (unsigned long long*)status_ws;
    int* counter = (int*)(status + tiles);
    cudaMemsetAsync(status_ws, 0, scan_status_bytes(m), st);
    k_scan<<<tiles, SCAN_THREADS, 0, st>>>(const_cast<int*>(in), out, m, status, counter, err, 0);
}

void launch_scatter(int n, const int* cell, const int* ticket, const int* cell_start, int* tmp, int* err,
                    cudaStream_t st) {
    k_scatter<<<blocks_for(n, 256), 256, 0, st>>>(n, cell, ticket, cell_start, tmp, err);
}

void launch_reorder(const KParams& p, bool predict_on, const float4* x, const float4* v, const int* perm,
                    const int* cell, const int* cell_start, const int* tmp, float4* xp, float4* vp, float4* xold,
                    int* perm_out, int* cell_sorted, const float* lam_in, float* lam_out, int* err, cudaStream_t st) {
    const int b = blocks_for(p.n, 256);
    if (predict_on)
        k_reorder<true><<<b, 256, 0, st>>>(p, x, v, perm, cell, cell_start, tmp, xp, vp, xold, perm_out, cell_sorted,
                                           lam_in, lam_out, err);
    else
        k_reorder<false><<<b, 256, 0, st>>>(p, x, v, perm, cell, cell_start, tmp, xp, vp, xold, perm_out, cell_sorted,
                                            lam_in, lam_out, err);
}

void launch_neighbors(const KParams& p, const float4* x, const int* cell_start, int* nbr, int* ncnt, cudaStream_t st) {
    k_neighbors<<<blocks_for(p.n, p.block), p.block, 0, st>>>(p, x, cell_start, nbr, ncnt);
}

void launch_lambda(const KParams& p, bool debug, const float4* x, const int* nbr, const int* ncnt, float4* xl,
                   float* rho, const IterCtl& ctl, cudaStream_t st) {
    with_lanes(p.lanes, [&](auto lc) {
        constexpr int L = decltype(lc)::value;
        const int b = team_blocks(p.n, L, p.block);
        if (debug) k_lambda<true, L><<<b, p.block, 0, st>>>(p, x, nbr, ncnt, xl, rho, ctl);
        else k_lambda<false, L><<<b, p.block, 0, st>>>(p, x, nbr, ncnt, xl, rho, ctl);
    });
}

void launch_dp(const KParams& p, bool debug, const float4* xl, const int* nbr, const int* ncnt, const float4* xold,
               float4* xout, float4* vout, float4* dp, const IterCtl& ctl, cudaStream_t st) {
    with_lanes(p.lanes, [&](auto lc) {
        constexpr int L = decltype(lc)::value;
        const int b = team_blocks(p.n, L, p.block);
        if (debug) k_dp<true, L><<<b, p.block, 0, st>>>(p, xl, nbr, ncnt, xold, xout, vout, dp, ctl);
        else k_dp<false, L><<<b, p.block, 0, st>>>(p, xl, nbr, ncnt, xold, xout, vout, dp, ctl);
    });
}

void launch_features(const KParams& p, const float4* x, const float4* v, const int* nbr, const int* ncnt,
                     const int* cell_start, const float* lam_prev, float4* xl, float* feat, float* lam_acc,
                     cudaStream_t st) {
    with_lanes(p.lanes, [&](auto lc) {
        constexpr int L = decltype(lc)::value;
        k_features<L><<<team_blocks(p.n, L, p.block), p.block, 0, st>>>(p, x, v, nbr, ncnt, cell_start, lam_prev,
                                                                         xl, feat, lam_acc);
    });
}

void launch_gather_rows(const int* slots, int count, int n, const float* feat, const float* lam_acc, float* out_feat,
                        float* out_target, int* err, cudaStream_t st) {
    if (count > 0)
        k_gather_rows<<<blocks_for(count, 256), 256, 0, st>>>(slots, count, n, feat, lam_acc, out_feat, out_target,
                                                               err);
}

void launch_count_fallback(const int* iters, int first, int configured, int* fallback, long long* total,
                           cudaStream_t st) {
    k_count_fallback<<<1, 1, 0, st>>>(iters, first, configured, fallback, total);
}

void launch_velocity(const KParams& p, const float4* x, const float4* xold, float4* v, cudaStream_t st) {
    k_velocity<<<blocks_for(p.n, 256), 256, 0, st>>>(p, x, xold, v);
}

void launch_curl(const KParams& p, const float4* x, const float4* v, const int* nbr, const int* ncnt, float4* omega,
                 cudaStream_t st) {
    with_lanes(p.lanes, [&](auto lc) {
        constexpr int L = decltype(lc)::value;
        k_curl<L><<<team_blocks(p.n, L, p.block), p.block, 0, st>>>(p, x, v, nbr, ncnt, omega);
    });
}

void launch_vort(const KParams& p, bool debug, const float4* x, const float4* v, const float4* omega, const int* nbr,
                 const int* ncnt, float4* vout, const int* perm_in, int* perm_out, float4* vort, float4* visc,
                 cudaStream_t st) {
    with_lanes(p.lanes, [&](auto lc) {
        constexpr int L = decltype(lc)::value;
        const int b = team_blocks(p.n, L, p.block);
        if (debug)
            k_vort<true, L><<<b, p.block, 0, st>>>(p, x, v, omega, nbr, ncnt, vout, perm_in, perm_out, vort, visc);
        else
            k_vort<false, L><<<b, p.block, 0, st>>>(p, x, v, omega, nbr, ncnt, vout, perm_in, perm_out, vort, visc);
    });
}

void launch_density_error(const KParams& p, const float4* x, const int* nbr, const int* ncnt,
                          unsigned long long* max_bits, double* sum, const int* skip, cudaStream_t st) {
    k_density_error<<<blocks_for(p.n, 256), 256, 0, st>>>(p, x, nbr, ncnt, max_bits, sum, skip);
}

void launch_from_aos(int n, const float* pos, const float* vel, float4* x, float4* v, int* perm, int* err,
                     cudaStream_t st) {
    k_from_aos<<<blocks_for(n, 256), 256, 0, st>>>(n, pos, vel, x, v, perm, err);
}

void launch_to_aos(int n, const float4* a, const int* perm, float* out, int* err, cudaStream_t st) {
    k_to_aos<<<blocks_for(n, 256), 256, 0, st>>>(n, a, perm, out, err);
}

void launch_copy4(int n, const float4* a, float4* b, cudaStream_t st) {
    k_copy4<<<blocks_for(n, 256), 256, 0, st>>>(n, a, b);
}

}  // namespace pbf
