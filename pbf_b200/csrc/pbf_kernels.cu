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
// setGrid :99-111, countingSort :112-122, buildNeighborhood :124-154; the
// neighbour-sum passes (lambda, dp, curl, vorticity) are in pbf_pairs.cu.
#include <algorithm>

#include "pbf_kernels.h"
#include "pbf_packed.cuh"

namespace pbf {

// ---------------------------------------------------------------------------
// a1 + a2: predict, bound, hash, histogram (one arrival ticket per particle)
// ---------------------------------------------------------------------------
template <bool PREDICT, int U>
__global__ void __launch_bounds__(256, 8) k_hash(KParams p, const float4* __restrict__ x, const float4* __restrict__ v,
                                              int* __restrict__ cell, int* __restrict__ ticket, int* __restrict__ cnt,
                                              int* __restrict__ err) {
    // Each warp takes U rounds of 32 consecutive slots; the loads, and then the
    // histogram atomics, of all rounds are in flight together.
    const int lane = threadIdx.x & 31;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int key[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const long long i = (w * U + u) * 32 + lane;
        key[u] = -1;
        if (i < p.n) {
            const SceneView sc = scene_of(p, (int)i);
            f3 xi = make3(x[i]);
            if (PREDICT) {
                f3 vi = make3(v[i]);
                predict(p, sc, xi, vi);
            }
            if (!(isfinite(xi.x) && isfinite(xi.y) && isfinite(xi.z))) atomicOr(err, DEVERR_NONFINITE);
            key[u] = cell_key(p, sc, xi);
        }
    }
    // Run-aggregated histogram: slots are in cell order from the previous substep,
    // so equal keys come in runs; one atomic per run of equal keys in the warp.
    // (The ticket is only an arrival order; k_reorder makes the order stable.)
    int base[U], leader[U], rank[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int prev = __shfl_up_sync(0xffffffffu, key[u], 1);
        const unsigned starts = __ballot_sync(0xffffffffu, lane == 0 || prev != key[u]);
        const unsigned upto = starts & (0xffffffffu >> (31 - lane));  // run starts at or below this lane
        leader[u] = 31 - __clz(upto);
        const unsigned above = starts & ~(0xffffffffu >> (31 - lane));
        const int end = above ? __ffs(above) - 1 : 32;  // first run start above this lane
        rank[u] = lane - leader[u];
        base[u] = 0;
        if (key[u] >= 0 && lane == leader[u]) base[u] = atomicAdd(&cnt[key[u]], end - leader[u]);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const int b = __shfl_sync(0xffffffffu, base[u], leader[u]);
        const long long i = (w * U + u) * 32 + lane;
        if (i < p.n) {
            cell[i] = key[u];
            ticket[i] = b + rank[u];
        }
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
constexpr long long SCAN_SPIN_LIMIT = 1ll << 22;
// Counts per thread: 32 (tiles of 8,192), or 64 (tiles of 16,384) above 2^22
// counts, where half as many tiles shorten the look-back chains.
constexpr int SCAN_LARGE_MIN = (1 << 22) + 1;
__host__ __device__ constexpr int scan_items(int m) { return m >= SCAN_LARGE_MIN ? 64 : 32; }

__device__ __forceinline__ void st_release_u64(unsigned long long* a, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(a), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* a) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(a) : "memory");
    return v;
}

// VEC: cnt and out are 16-byte aligned; each lane moves four consecutive counts
// per access (int4), four rounds of 128 per warp instead of sixteen of 32.
// silent_tile >= 0 (the failure-injection test only): that tile publishes no
// status, so its successors' look-back waits run out after spin_limit polls.
template <bool VEC, int SCAN_ITEMS>
__global__ void __launch_bounds__(SCAN_THREADS) k_scan(int* __restrict__ cnt, int* __restrict__ out, int m,
                                                       unsigned long long* __restrict__ status,
                                                       int* __restrict__ tile_counter, int* __restrict__ err,
                                                       int clear, int silent_tile, long long spin_limit) {
    constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
    __shared__ int s_tile;
    __shared__ int s_warp[SCAN_THREADS / 32];
    __shared__ int s_excl, s_tot;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) s_tile = atomicAdd(tile_counter, 1);
    __syncthreads();
    const int tile = s_tile;

    // Warp w owns elements [tile * TILE + w * 32 ITEMS, + 32 ITEMS) in rounds of consecutive
    // elements (coalesced: 32 counts per round, or 128 as int4 when VEC); each
    // round is scanned across the warp and carried into the next.
    const long long wbase = (long long)tile * SCAN_TILE + (long long)warp * (32 * SCAN_ITEMS);
    int item[SCAN_ITEMS];
    int carry = 0;  // warp-exclusive offset of the round
    if (VEC) {
#pragma unroll
        for (int r = 0; r < SCAN_ITEMS / 4; ++r) {
            const long long i0 = wbase + r * 128 + lane * 4;
            if (i0 + 3 < m) {
                const int4 q = *reinterpret_cast<const int4*>(cnt + i0);
                item[4 * r] = q.x; item[4 * r + 1] = q.y; item[4 * r + 2] = q.z; item[4 * r + 3] = q.w;
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e) item[4 * r + e] = i0 + e < m ? cnt[i0 + e] : 0;
            }
        }
#pragma unroll
        for (int r = 0; r < SCAN_ITEMS / 4; ++r) {
            const int a0 = item[4 * r], a1 = a0 + item[4 * r + 1], a2 = a1 + item[4 * r + 2];
            const int tot = a2 + item[4 * r + 3];
            int incl = tot;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int ex = carry + incl - tot;
            carry += __shfl_sync(0xffffffffu, incl, 31);
            item[4 * r] = ex;  // exclusive prefixes within the warp's range
            item[4 * r + 1] = ex + a0;
            item[4 * r + 2] = ex + a1;
            item[4 * r + 3] = ex + a2;
        }
    } else {
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS; ++q) {
            const long long idx = wbase + q * 32 + lane;
            item[q] = idx < m ? cnt[idx] : 0;
        }
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
        const bool publish = tile != silent_tile;
        if (tile == 0) {
            if (lane == 0 && publish) st_release_u64(&status[0], (2ull << 32) | (unsigned)total);
        } else {
            if (lane == 0 && publish) st_release_u64(&status[tile], (1ull << 32) | (unsigned)total);
            int pos = tile - 1;  // highest tile not yet folded in
            bool done = false;
            while (!done) {
                const int look = pos - lane;
                unsigned long long s = 0;
                if (look >= 0) {
                    long long spins = 0;
                    s = ld_acquire_u64(&status[look]);
                    while ((s >> 32) == 0ull) {
                        if (++spins > spin_limit) {
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
            if (lane == 0 && publish) st_release_u64(&status[tile], (2ull << 32) | (unsigned)(excl + total));
        }
        if (lane == 0) {
            s_excl = excl;
            s_tot = total;
        }
    }
    __syncthreads();
    const int off = s_excl + s_warp[warp];
    if (VEC) {
#pragma unroll
        for (int r = 0; r < SCAN_ITEMS / 4; ++r) {
            const long long i0 = wbase + r * 128 + lane * 4;
            if (i0 + 3 < m) {
                *reinterpret_cast<int4*>(out + i0) =
                    make_int4(off + item[4 * r], off + item[4 * r + 1], off + item[4 * r + 2], off + item[4 * r + 3]);
                if (clear) *reinterpret_cast<int4*>(cnt + i0) = make_int4(0, 0, 0, 0);
            } else {
#pragma unroll
                for (int e = 0; e < 4; ++e)
                    if (i0 + e < m) {
                        out[i0 + e] = off + item[4 * r + e];
                        if (clear) cnt[i0 + e] = 0;
                    }
            }
        }
    } else {
#pragma unroll
        for (int q = 0; q < SCAN_ITEMS; ++q) {
            const long long idx = wbase + q * 32 + lane;
            if (idx < m) {
                out[idx] = off + item[q];
                if (clear) cnt[idx] = 0;
            }
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
// Each thread takes U slots 256 apart within its block's tile of 256 U (the
// loads of all U in flight together).
template <int U>
__global__ void __launch_bounds__(256) k_scatter(int n, const int* __restrict__ cell, const int* __restrict__ ticket,
                                                 const int* __restrict__ cell_start, int* __restrict__ tmp,
                                                 int* __restrict__ err) {
    const long long i0 = (long long)blockIdx.x * blockDim.x * U + threadIdx.x;
    int c[U], t[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const long long i = i0 + (long long)u * blockDim.x;
        c[u] = i < n ? cell[i] : 0;
        t[u] = i < n ? ticket[i] : 0;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
        const long long i = i0 + (long long)u * blockDim.x;
        if (i >= n) break;
        const int dst = cell_start[c[u]] + t[u];
        if (dst < 0 || dst >= n) {  // counts and tickets disagree: report, never write out of bounds
            atomicOr(err, DEVERR_BAD_INDEX);
            continue;
        }
        tmp[dst] = (int)i;
    }
}

template <bool PREDICT>
__global__ void __launch_bounds__(256, 8) k_reorder(KParams p, const float4* __restrict__ x, const float4* __restrict__ v,
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
// a7: 27-cell neighbour search (a (2R+1)^3 stencil when cells are smaller than
// h). The stencil is visited dz-major, dy, then the dx cells of a row, which are
// one contiguous slot range because keys are x-fastest; within a cell, slot
// order. For R = 1 this is the reference order (buildNeighborhood cu:133-136)
// applied to the sorted slots. Rows and row ends that lie farther than h from the
// particle are skipped: a row (dy, dz) is visited only where the distance from the
// particle to its y and z slabs leaves room within h, and only over the x cells
// within the remaining half-width. The clipping is conservative (a margin of
// 1e-3 h plus 1e-6 of the coordinates, far above float rounding), so every
// candidate it drops fails the r^2 <= h^2 test and the lists do not change.
// ---------------------------------------------------------------------------
// Stencil radius RR as a constant (1: cells of h, 2: cells of h/2; 0: any radius,
// read from p.radius). For RR > 0 the row ranges of a plane of cells are loaded
// together and candidates are fetched two at a time (a clipped row of cells of
// h/2 holds a few, and wider batches leave more of their slots empty), so a
// thread waits on a few independent loads at once instead of one chain per row
// and per candidate.
template <int RR>
__device__ __forceinline__ void neighbors_one(const KParams& p, int k, const float4* __restrict__ x,
                                              const int* __restrict__ cell_start, int* __restrict__ nbr,
                                              int* __restrict__ ncnt) {
    if (k >= p.n) return;
    const SceneView sc = scene_of(p, k);
    const f3 xk = make3(x[k]);
    int d[3];
    cell_dims(p, sc, xk, d);
    const int nx = sc.dims[0], ny = sc.dims[1], nz = sc.dims[2];
    const int R = RR > 0 ? RR : p.radius;
    const int x0 = max(d[0] - R, 0), x1 = min(d[0] + R, nx - 1);
    int c = 0;
    const int cap = p.max_nbr;
    const float m = p.h * 1e-3f + 1e-6f * (fabsf(xk.x) + fabsf(xk.y) + fabsf(xk.z));
    const float hm2 = (p.h + m) * (p.h + m);
    // squared distance from the particle to the y slab of stencil row dy (less
    // the margin), +inf for a row outside the grid
    auto row_ey2 = [&](int dy) {
        const int y = d[1] + dy;
        if (y < 0 || y >= ny) return INFINITY;
        const float gy = dy > 0 ? (sc.gmin[1] + (float)y * p.cell) - xk.y
                                : xk.y - (sc.gmin[1] + (float)(y + 1) * p.cell);
        const float ey = dy == 0 ? 0.0f : fmaxf(gy - m, 0.0f);
        return ey * ey;
    };
    // slot range [s, e) of the stencil row in cell row y of plane z, clipped to
    // the sphere (rem = (h + m)^2 - ez^2 - ey^2); empty when farther than h
    auto row_clip = [&](int y, int z, float rem, int& s, int& e) {
        s = 0;
        e = 0;
        if (!(rem >= 0.0f)) return;
        // the half-width only bounds the candidates (the margin m of at least
        // 1e-3 h is far above the approximate root's relative error of 2^-22)
        float w;
        asm("sqrt.approx.f32 %0, %1;" : "=f"(w) : "f"(rem));
        w += m;
        const int xa = max(x0, (int)floorf((xk.x - w - sc.gmin[0]) * p.inv_cell));
        const int xb = min(x1, (int)floorf((xk.x + w - sc.gmin[0]) * p.inv_cell));
        if (xa > xb) return;
        const int row = sc.cell_base + y * nx + z * nx * ny;
        s = cell_start[row + xa];
        e = cell_start[row + xb + 1];
    };
    // candidates [s, e) in slot order, NB positions in flight; |r|^2 of two
    // candidates per packed instruction (the same IEEE operations as dot_fma;
    // x_k - x_j as fma(x_j, -1, x_k), the same single rounding of the difference)
    constexpr int NB = 2;  // candidates per batch (even; rows of cells of h/2 hold a few)
    auto scan_row = [&](int s, int e) {
        for (int j0 = s; j0 < e && c < cap; j0 += NB) {
            float4 xj[NB];
#pragma unroll
            for (int u = 0; u < NB; ++u) xj[u] = x[min(j0 + u, e - 1)];
            float r2[NB];
#pragma unroll
            for (int u = 0; u < NB; u += 2) {
                const float2 m1 = bc<float2>(-1.0f);
                const float2 rx = vfma(make_float2(xj[u].x, xj[u + 1].x), m1, bc<float2>(xk.x));
                const float2 ry = vfma(make_float2(xj[u].y, xj[u + 1].y), m1, bc<float2>(xk.y));
                const float2 rz = vfma(make_float2(xj[u].z, xj[u + 1].z), m1, bc<float2>(xk.z));
                const float2 d2 = vfma(rz, rz, vfma(ry, ry, vmul(rx, rx)));
                r2[u] = d2.x;
                r2[u + 1] = d2.y;
            }
#pragma unroll
            for (int u = 0; u < NB; ++u) {
                const int j = j0 + u;
                if (j >= e || c >= cap) break;
                if (j == k) continue;
                if (r2[u] <= p.h2) {
                    nbr[(size_t)c * p.stride + k] = j;
                    ++c;
                }
            }
        }
    };
    if (x0 <= x1) {
        // the rows' y distances are the same in every plane
        constexpr int W = RR > 0 ? 2 * RR + 1 : 1;
        float ey2[W];
        if (RR > 0) {
#pragma unroll
            for (int i = 0; i < W; ++i) ey2[i] = row_ey2(i - RR);
        }
        for (int dz = -R; dz <= R && c < cap; ++dz) {
            const int z = d[2] + dz;
            if (z < 0 || z >= nz) continue;
            // distance from the particle to the z slab of this plane of cells
            const float gz = dz > 0 ? (sc.gmin[2] + (float)z * p.cell) - xk.z
                                    : xk.z - (sc.gmin[2] + (float)(z + 1) * p.cell);
            const float ez = dz == 0 ? 0.0f : fmaxf(gz - m, 0.0f);
            if (ez * ez > hm2) continue;
            const float hz = hm2 - ez * ez;
            if (RR > 0) {
                int s[W], e[W];
#pragma unroll
                for (int i = 0; i < W; ++i) row_clip(d[1] + i - RR, z, hz - ey2[i], s[i], e[i]);
#pragma unroll
                for (int i = 0; i < W; ++i) scan_row(s[i], e[i]);
            } else {
                for (int dy = -R; dy <= R && c < cap; ++dy) {
                    int s, e;
                    row_clip(d[1] + dy, z, hz - row_ey2(dy), s, e);
                    scan_row(s, e);
                }
            }
        }
    }
    ncnt[k] = c;
}

// nvb tiles of blockDim.x slots; the grid strides over them (a grid of nvb
// blocks is the ordinary one-block-per-tile launch)
template <int RR>
__global__ void __launch_bounds__(256) k_neighbors(KParams p, int nvb, const float4* __restrict__ x,
                                                   const int* __restrict__ cell_start, int* __restrict__ nbr,
                                                   int* __restrict__ ncnt) {
    for (int vb = blockIdx.x; vb < nvb; vb += gridDim.x)
        neighbors_one<RR>(p, vb * blockDim.x + threadIdx.x, x, cell_start, nbr, ncnt);
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

// Control of the device-side correction loop (a graph while node whose body is
// one lambda pass and one delta-p pass, then this kernel): counts the pass and
// keeps the loop running while the error is above tolerance and slots are left.
__global__ void k_loop_ctl(cudaGraphConditionalHandle h, int* __restrict__ loop_k, const int* __restrict__ done,
                           int first, int max_it) {
    const int k = *loop_k + 1;
    *loop_k = k;
    cudaGraphSetConditional(h, (*done == 0 && first + k < max_it) ? 1u : 0u);
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

// The state in slot order: AoS x and v, the loaded index of each slot, the key
// of the cell the slot was sorted into and its rank within that cell (any
// output may be null).
__global__ void k_sorted_state(int n, const float4* __restrict__ x, const float4* __restrict__ v,
                               const int* __restrict__ perm, const int* __restrict__ cell_sorted,
                               const int* __restrict__ cell_start, float* __restrict__ pos, float* __restrict__ vel,
                               int* __restrict__ ids, int* __restrict__ key, int* __restrict__ rank) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    if (pos) {
        const float4 q = x[k];
        pos[3 * k] = q.x;
        pos[3 * k + 1] = q.y;
        pos[3 * k + 2] = q.z;
    }
    if (vel) {
        const float4 q = v[k];
        vel[3 * k] = q.x;
        vel[3 * k + 1] = q.y;
        vel[3 * k + 2] = q.z;
    }
    if (ids) ids[k] = perm[k];
    const int c = cell_sorted[k];
    if (key) key[k] = c;
    if (rank) rank[k] = k - cell_start[c];
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
// FP32 throughput probe: every thread runs 8 independent chains of fused
// multiply-adds (scalar FFMA, or packed fma.rn.f32x2 with two lanes each), long
// enough that launch and tail are negligible. The result is stored only under a
// condition the chains never meet, so nothing is optimised away and nothing is
// written. FLOPs = 2 per multiply-add lane.
// ---------------------------------------------------------------------------
template <bool PACKED>
__global__ void __launch_bounds__(256) k_fma_peak(int iters, float seed, float* __restrict__ sink) {
    const float b = 0.999999f, c = 1e-7f;
    if (PACKED) {
        float2 a[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = make_float2(seed + (float)(threadIdx.x + i), seed - (float)i);
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = vfma(a[i], bc<float2>(b), bc<float2>(c));
        }
        float t = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; ++i) t += a[i].x + a[i].y;
        if (t == -1.0f) sink[threadIdx.x] = t;
    } else {
        float a[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) a[i] = seed + (float)(threadIdx.x + i);
        for (int it = 0; it < iters; ++it) {
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = __fmaf_rn(a[i], b, c);
        }
        float t = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; ++i) t += a[i];
        if (t == -1.0f) sink[threadIdx.x] = t;
    }
}

// Best of three timed launches of each form (CUDA events), after a warm-up launch.
int measure_fp32_peak(double* scalar_tflops, double* packed_tflops) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return -1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float* sink = nullptr;
    if (cudaMalloc(&sink, 256 * sizeof(float)) != cudaSuccess) return -1;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    double best[2] = {0.0, 0.0};
    for (int form = 0; form < 2; ++form) {
        const double lanes = form ? 2.0 : 1.0;
        const double flops = 2.0 * 8.0 * lanes * iters * (double)blocks * threads;
        for (int rep = 0; rep < 4; ++rep) {
            cudaEventRecord(a, 0);
            if (form) k_fma_peak<true><<<blocks, threads>>>(iters, 1.0f, sink);
            else k_fma_peak<false><<<blocks, threads>>>(iters, 1.0f, sink);
            cudaEventRecord(b, 0);
            cudaEventSynchronize(b);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, a, b);
            if (rep > 0 && ms > 0.0f) best[form] = std::max(best[form], flops / (ms * 1e-3) / 1e12);
        }
    }
    const cudaError_t e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (e != cudaSuccess) return -1;
    *scalar_tflops = best[0];
    *packed_tflops = best[1];
    return 0;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static inline int blocks_for(int n, int bs) { return (n + bs - 1) / bs; }
static inline bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }
void launch_hash(const KParams& p, bool predict_on, const float4* x, const float4* v, int* cell, int* ticket, int* cnt,
                 int* err, cudaStream_t st) {
    // four rounds per warp once there are enough particles to fill the device
    // with them (about 1 M); below that, one round keeps more blocks resident
    if (p.n >= (1 << 20)) {
        const int b = blocks_for(p.n, 256 * 4);
        if (predict_on) k_hash<true, 4><<<b, 256, 0, st>>>(p, x, v, cell, ticket, cnt, err);
        else k_hash<false, 4><<<b, 256, 0, st>>>(p, x, v, cell, ticket, cnt, err);
    } else {
        const int b = blocks_for(p.n, 256);
        if (predict_on) k_hash<true, 1><<<b, 256, 0, st>>>(p, x, v, cell, ticket, cnt, err);
        else k_hash<false, 1><<<b, 256, 0, st>>>(p, x, v, cell, ticket, cnt, err);
    }
}

// tile count in 64-bit arithmetic (m + tile - 1 would overflow an int near INT_MAX)
static int scan_tiles(int m) {
    const long long tile = (long long)SCAN_THREADS * scan_items(m);
    return (int)(((long long)m + tile - 1) / tile);
}

size_t scan_status_bytes(int m) { return (size_t)scan_tiles(m) * sizeof(unsigned long long) + 16; }

template <bool VEC>
static void launch_scan_kernel(int* cnt, int* out, int m, unsigned long long* status, int* counter, int* err,
                               int clear, cudaStream_t st, int silent_tile = -1,
                               long long spin_limit = SCAN_SPIN_LIMIT) {
    const int tiles = scan_tiles(m);
    if (scan_items(m) == 64)
        k_scan<VEC, 64><<<tiles, SCAN_THREADS, 0, st>>>(cnt, out, m, status, counter, err, clear, silent_tile,
                                                         spin_limit);
    else
        k_scan<VEC, 32><<<tiles, SCAN_THREADS, 0, st>>>(cnt, out, m, status, counter, err, clear, silent_tile,
                                                         spin_limit);
}

void launch_scan(int* cnt, int* out, int m, void* status_ws, int* err, cudaStream_t st) {
    unsigned long long* status = (unsigned long long*)status_ws;
    int* counter = (int*)(status + scan_tiles(m));
    cudaMemsetAsync(status_ws, 0, scan_status_bytes(m), st);
    if (aligned16(cnt) && aligned16(out)) launch_scan_kernel<true>(cnt, out, m, status, counter, err, 1, st);
    else launch_scan_kernel<false>(cnt, out, m, status, counter, err, 1, st);
}

void launch_scan_const(const int* in, int* out, int m, void* status_ws, int* err, cudaStream_t st) {
    unsigned long long* status = (unsigned long long*)status_ws;
    int* counter = (int*)(status + scan_tiles(m));
    cudaMemsetAsync(status_ws, 0, scan_status_bytes(m), st);
    if (aligned16(in) && aligned16(out)) launch_scan_kernel<true>(const_cast<int*>(in), out, m, status, counter, err, 0, st);
    else launch_scan_kernel<false>(const_cast<int*>(in), out, m, status, counter, err, 0, st);
}

void launch_scan_silent_tile(const int* in, int* out, int m, void* status_ws, int* err, int silent_tile,
                             long long spin_limit, cudaStream_t st) {
    unsigned long long* status = (unsigned long long*)status_ws;
    int* counter = (int*)(status + scan_tiles(m));
    cudaMemsetAsync(status_ws, 0, scan_status_bytes(m), st);
    launch_scan_kernel<false>(const_cast<int*>(in), out, m, status, counter, err, 0, st, silent_tile, spin_limit);
}

void launch_scatter(int n, const int* cell, const int* ticket, const int* cell_start, int* tmp, int* err,
                    cudaStream_t st) {
    if (n >= (1 << 20)) k_scatter<4><<<blocks_for(n, 256 * 4), 256, 0, st>>>(n, cell, ticket, cell_start, tmp, err);
    else k_scatter<1><<<blocks_for(n, 256), 256, 0, st>>>(n, cell, ticket, cell_start, tmp, err);
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

// Grid over nvb tiles: nvb blocks, or with p.persistent the blocks resident at
// once (SMs x blocks per SM), each striding over the tiles.
template <typename K> static int resident_grid(const KParams& p, K kernel, int nvb) {
    if (!p.persistent) return nvb;
    int dev = 0, sms = 1, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, p.block, 0) != cudaSuccess || per_sm <= 0)
        per_sm = 1;
    const long long g = (long long)per_sm * (sms > 0 ? sms : 1);
    return (int)(g < nvb ? g : nvb);
}

void launch_neighbors(const KParams& p, const float4* x, const int* cell_start, int* nbr, int* ncnt, cudaStream_t st) {
    const int b = blocks_for(p.n, p.block);
    if (p.radius == 1) k_neighbors<1><<<resident_grid(p, k_neighbors<1>, b), p.block, 0, st>>>(p, b, x, cell_start, nbr, ncnt);
    else if (p.radius == 2) k_neighbors<2><<<resident_grid(p, k_neighbors<2>, b), p.block, 0, st>>>(p, b, x, cell_start, nbr, ncnt);
    else k_neighbors<0><<<resident_grid(p, k_neighbors<0>, b), p.block, 0, st>>>(p, b, x, cell_start, nbr, ncnt);
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

void launch_loop_ctl(cudaGraphConditionalHandle h, int* loop_k, const int* done, int first, int max_it,
                     cudaStream_t st) {
    k_loop_ctl<<<1, 1, 0, st>>>(h, loop_k, done, first, max_it);
}

void launch_velocity(const KParams& p, const float4* x, const float4* xold, float4* v, cudaStream_t st) {
    k_velocity<<<blocks_for(p.n, 256), 256, 0, st>>>(p, x, xold, v);
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

void launch_sorted_state(int n, const float4* x, const float4* v, const int* perm, const int* cell_sorted,
                         const int* cell_start, float* pos, float* vel, int* ids, int* key, int* rank,
                         cudaStream_t st) {
    k_sorted_state<<<blocks_for(n, 256), 256, 0, st>>>(n, x, v, perm, cell_sorted, cell_start, pos, vel, ids, key,
                                                       rank);
}

void launch_copy4(int n, const float4* a, float4* b, cudaStream_t st) {
    k_copy4<<<blocks_for(n, 256), 256, 0, st>>>(n, a, b);
}

}  // namespace pbf
