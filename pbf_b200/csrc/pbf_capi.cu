// C ABI of the solver step (include/pbf.h): handle, device buffers, the captured
// substep graph, and the status/stats plumbing.
//
// Host sequence replaced: kernels/cudaPBF.cu:50-115 (about 22 launch +
// cudaDeviceSynchronize round trips and two leaked host arrays per substep).
// Here one substep is a CUDA graph captured once per handle and replayed.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/pbf.h"
#include "pbf_kernels.h"
#include "pbf_mlp.h"

using namespace pbf;

namespace {

// NVTX range over a scope: every public call that enqueues work is one range,
// and while a substep graph is captured each phase is a range named after it
// (header-only NVTX: without a profiler attached a push/pop is a no-op call).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

}  // namespace

int pbf::set_last_error(int code, const char* msg) {
    g_err = msg ? msg : "";
    return code;
}

namespace {

#define CK(call)                                                                              \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess) return fail(PBF_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// Error slots: slot k holds the density error measured after k corrections
// (adaptive mode); slot kMaxIter + 1 holds a measurement after the loop.
constexpr int kMaxIter = 64;
constexpr int kSlots = kMaxIter + 2;

struct DevStats {
    unsigned long long max_bits[kSlots];
    double sum[kSlots];
    int done;
    int iters;
    int conv_slot;
    int loop_k;  // passes of the device-side correction loop
    // not reset per substep:
    int err;
    int fallback;
    long long total_iters;  // adaptive: corrections applied since upload
};

// Profiling stages (pbf_stage_times)
enum Stage { ST_HASH, ST_SCAN, ST_SCATTER, ST_REORDER, ST_NEIGHBORS, ST_LAMBDA, ST_DP, ST_VELOCITY, ST_CURL,
             ST_VORT, ST_COPY, ST_MEASURE, ST_MLP, ST_COUNT };

struct StageEvents {
    int stage;
    cudaEvent_t a, b;
};

}  // namespace

// Double-buffered staging of pbf_step_host: host copies run on their own
// streams, ordered against the solver's stream by events.
struct HostPipe {
    cudaStream_t h2d = nullptr, d2h = nullptr;
    float* in[2] = {nullptr, nullptr};   // pos, vel: float[6n]
    float* out[2] = {nullptr, nullptr};  // positions: float[3n]
    cudaEvent_t in_ready[2] = {}, in_free[2] = {}, out_ready[2] = {}, out_free[2] = {};
    long long calls = 0;
};

struct pbf_solver {
    pbf_solver_parameter para{};
    pbf_ext_params ext{};
    float grid_space[6]{}, boundary[6]{};
    KParams kp{};
    int n = 0, ncells = 0, nkeys = 0, stride = 0;  // ncells: real cells of scene 0
    int capacity = 0;                              // particles the buffers hold (n <= capacity)
    std::vector<SceneView> scenes_h;
    SceneView* scenes_d = nullptr;  // scene table (batches)
    int* sid = nullptr;             // per slot: scene index (batches)
    // device state (slot order)
    float4 *Sx = nullptr, *Sv = nullptr, *Px = nullptr, *Pv = nullptr, *Pxold = nullptr, *Q = nullptr,
           *omega = nullptr, *vw = nullptr;  // vw: v with |omega| in .w (curl -> vorticity)
    float4 *xpred_dbg = nullptr, *dp_dbg = nullptr, *vort_dbg = nullptr, *visc_dbg = nullptr;
    float* rho_dbg = nullptr;
    int *Sperm = nullptr, *Pperm = nullptr, *cell = nullptr, *ticket = nullptr, *tmp = nullptr,
        *cell_sorted = nullptr, *ncnt = nullptr, *nbr = nullptr, *cnt = nullptr, *cell_start = nullptr,
        *hash_dbg = nullptr;
    // total lambda of the substep (slot order), its copy permuted into the next
    // substep's order, the last warm-start lambda0, and the 12 warm-start features
    float *lam_acc = nullptr, *lam_prev_sorted = nullptr, *lam0 = nullptr, *feat = nullptr;
    void* scan_ws = nullptr;
    DevStats* dstats = nullptr;
    float* staging = nullptr;  // AoS float[3n] x2 for upload/download
    float* bound_pos = nullptr;
    uint16_t* mlp_w = nullptr;  // installed warm-start weights (BF16) and biases/constants
    float* mlp_b = nullptr;
    int first_corrections = 0;  // corrections before the Jacobi loop (1 with features)
    // graph
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap_stream = nullptr;
    cudaStream_t body_stream = nullptr;  // captures the body of the device-side correction loop
    cudaStream_t last_stream = nullptr;
    std::vector<StageEvents> prof;  // event pairs captured around each launch (ext.profile)
    int kernel_nodes = 0;
    int loop_kernel_nodes = 0;  // kernels of one pass of the device-side correction loop
    bool uploaded = false;
    long long substeps = 0, total_iters = 0, fallbacks = 0;
    HostPipe* hp = nullptr;  // pbf_step_host staging, created on first use
};

namespace {

bool finite6(const float* b) {
    for (int i = 0; i < 6; ++i)
        if (!std::isfinite(b[i])) return false;
    return true;
}

// Host-side constants of the product arithmetic (pbf_device.cuh). Every value is
// a fixed IEEE expression so that a CPU evaluation reproduces it.
KParams make_kparams(const pbf_solver& s) {
    KParams k{};
    const pbf_solver_parameter& p = s.para;
    const pbf_ext_params& e = s.ext;
    const double inv_pi_ref = 0.31830988618;  // INVPI, include/solverBase.h:4
    k.h = p.h;
    k.h2 = p.h * p.h;
    const float cs = p.h * e.cell_scale;
    k.cell = cs;
    k.inv_cell = 1.0f / cs;
    k.poly6_c = (float)(315.0 * inv_pi_ref / (64.0 * std::pow((double)p.h, 9)));
    k.spiky_c = (float)(-45.0 * inv_pi_ref / std::pow((double)p.h, 6));
    const float r2 = p.deltaq * p.deltaq;
    float wdq = 0.0f;
    if (!(r2 > k.h2)) {
        const float t = k.h2 - r2;
        wdq = k.poly6_c * ((t * t) * t);
    }
    k.inv_wdq = 1.0f / wdq;
    k.nk = -p.k;
    k.scorr_scale = e.scorr_scale;
    k.n_exp = p.n;
    k.n_int = (p.n >= 1.0f && p.n <= 8.0f && p.n == std::floor(p.n)) ? (int)p.n : 0;
    k.rho0 = p.restRho;
    k.rho0sq = p.restRho * p.restRho;
    k.eps = p.epsilon;
    k.dt = p.dt;
    k.jit = e.wall_jitter;
    k.rmin = e.grad_rmin;
    k.visc_c = (e.flags & PBF_FLAG_XSPH_RHO) ? (float)((double)p.c / (double)p.restRho) : p.c;
    k.vort_eps = p.vorticityConfinementEpilon;
    for (int a = 0; a < 3; ++a) k.g[a] = e.gravity[a];
    k.sc0 = s.scenes_h[0];
    k.scenes = s.scenes_d;
    k.sid = s.sid;
    k.nscenes = (int)s.scenes_h.size();
    k.nkeys = s.nkeys;
    k.radius = e.cell_scale >= 1.0f ? 1 : (int)std::ceil(1.0 / (double)e.cell_scale);
    k.n = s.n;
    k.block = e.block_size > 0 ? e.block_size : 256;
    k.lanes = e.pair_lanes > 0 ? e.pair_lanes : 2;
    k.persistent = e.persistent;
    k.max_nbr = e.max_neighbors;
    k.stride = s.stride;
    k.cell_order = e.cell_order;
    k.flags = e.flags;
    k.poly6_c64 = 315.0 / (64.0 * M_PI * std::pow((double)p.h, 9));
    // wall density: rest number density = rho0 plus the self term W(0) that the
    // reference's density sum leaves out
    const float h3 = (k.h2 * k.h2) * k.h2;
    k.wall_n = p.restRho + k.poly6_c * h3;
    k.inv_h = 1.0f / p.h;
    k.wall_kd = (float)(315.0 / (256.0 * (double)p.h));
    k.wc3 = (float)(-4.0 / 3.0);
    k.wc5 = (float)(6.0 / 5.0);
    k.wc7 = (float)(-4.0 / 7.0);
    k.wc9 = (float)(1.0 / 9.0);
    return k;
}

// Host-side fault injection for tests (pbf_debug_fail_staging_alloc): when
// positive, the device allocation of pbf_step_host's staging with this 1-based
// number fails as if the device were out of memory.
std::atomic<int> g_fail_staging_alloc{0};

cudaError_t staging_malloc(void** p, size_t bytes) {
    if (g_fail_staging_alloc.load() > 0 && g_fail_staging_alloc.fetch_sub(1) == 1) return cudaErrorMemoryAllocation;
    return cudaMalloc(p, bytes);
}

// Frees whatever part of a HostPipe exists (null members are skipped).
void free_host_pipe(HostPipe* hp) {
    if (!hp) return;
    for (int b = 0; b < 2; ++b) {
        if (hp->in[b]) cudaFree(hp->in[b]);
        if (hp->out[b]) cudaFree(hp->out[b]);
        for (cudaEvent_t e : {hp->in_ready[b], hp->in_free[b], hp->out_ready[b], hp->out_free[b]})
            if (e) cudaEventDestroy(e);
    }
    if (hp->h2d) cudaStreamDestroy(hp->h2d);
    if (hp->d2h) cudaStreamDestroy(hp->d2h);
    delete hp;
}

template <typename T> int dalloc(T** p, size_t count) {
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) return fail(PBF_ERR_ALLOC, "cudaMalloc(%zu bytes): %s", count * sizeof(T), cudaGetErrorString(e));
    return PBF_OK;
}

void free_all(pbf_solver* s) {
    void* ptrs[] = {s->Sx, s->Sv, s->Px, s->Pv, s->Pxold, s->Q, s->omega, s->vw, s->xpred_dbg, s->dp_dbg, s->vort_dbg,
                    s->visc_dbg, s->rho_dbg, s->Sperm, s->Pperm, s->cell, s->ticket, s->tmp, s->cell_sorted,
                    s->ncnt, s->nbr, s->cnt, s->cell_start, s->hash_dbg, s->lam_acc, s->lam_prev_sorted, s->lam0,
                    s->feat, s->scan_ws, s->dstats, s->staging, s->scenes_d, s->sid, s->mlp_w, s->mlp_b};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
    free_host_pipe(s->hp);
    s->hp = nullptr;
    if (s->body_stream) cudaStreamDestroy(s->body_stream);
    for (auto& e : s->prof) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    s->prof.clear();
}

int validate_scene(const pbf_scene_desc& d, int idx) {
    if (!finite6(d.grid_space) || !finite6(d.boundary))
        return fail(PBF_ERR_INVALID, "scene %d: non-finite grid space or boundary", idx);
    for (int a = 0; a < 3; ++a) {
        if (d.grid_dims[a] <= 0) return fail(PBF_ERR_INVALID, "scene %d: grid_dims must be positive", idx);
        if (d.boundary[a] > d.boundary[3 + a]) return fail(PBF_ERR_INVALID, "scene %d: boundary pMin > pMax", idx);
    }
    for (int a = 0; a < 4; ++a)
        if (!std::isfinite(d.sphere[a])) return fail(PBF_ERR_INVALID, "scene %d: non-finite sphere", idx);
    const long long cells = (long long)d.grid_dims[0] * d.grid_dims[1] * d.grid_dims[2];
    if (cells > (1ll << 30)) return fail(PBF_ERR_INVALID, "scene %d: grid has too many cells (%lld)", idx, cells);
    if (d.nparticles <= 0) return fail(PBF_ERR_INVALID, "scene %d: nparticles must be positive", idx);
    return PBF_OK;
}

int validate(const pbf_solver_parameter* p, const float* gs, const float* bd, const pbf_ext_params* e) {
    if (!p || !gs || !bd || !e) return fail(PBF_ERR_INVALID, "null argument");
    if (p->nParticles <= 0) return fail(PBF_ERR_INVALID, "nParticles must be positive (got %d)", p->nParticles);
    const float f[] = {p->h, p->restRho, p->epsilon, p->k, p->n, p->deltaq, p->c, p->dt, p->vorticityConfinementEpilon};
    for (float v : f)
        if (!std::isfinite(v)) return fail(PBF_ERR_INVALID, "non-finite SolverParameter field");
    if (!(p->h > 0.0f)) return fail(PBF_ERR_INVALID, "h must be positive");
    if (!(p->restRho > 0.0f)) return fail(PBF_ERR_INVALID, "restRho must be positive");
    if (!(p->dt > 0.0f)) return fail(PBF_ERR_INVALID, "dt must be positive");
    if (!(p->deltaq >= 0.0f && p->deltaq < p->h)) return fail(PBF_ERR_INVALID, "deltaq must lie in [0, h)");
    if (p->iterations < 0 || p->iterations > 64) return fail(PBF_ERR_INVALID, "iterations must lie in [0, 64]");
    if (!finite6(gs) || !finite6(bd)) return fail(PBF_ERR_INVALID, "non-finite grid space or boundary");
    for (int a = 0; a < 3; ++a) {
        if (e->grid_dims[a] <= 0) return fail(PBF_ERR_INVALID, "grid_dims must be positive");
        if (bd[a] > bd[3 + a]) return fail(PBF_ERR_INVALID, "boundary pMin > pMax");
    }
    const long long cells = (long long)e->grid_dims[0] * e->grid_dims[1] * e->grid_dims[2];
    if (cells > (1ll << 30)) return fail(PBF_ERR_INVALID, "grid has too many cells (%lld)", cells);
    if (!(e->cell_scale >= 0.25f) || !std::isfinite(e->cell_scale))
        return fail(PBF_ERR_INVALID, "cell_scale must be >= 0.25");
    if (e->max_neighbors < 1 || e->max_neighbors > 127) return fail(PBF_ERR_INVALID, "max_neighbors must lie in [1, 127]");
    if (e->cell_order != 0 && e->cell_order != 1) return fail(PBF_ERR_INVALID, "cell_order must be 0 or 1");
    if (e->block_size != 0 && e->block_size != 64 && e->block_size != 128 && e->block_size != 256)
        return fail(PBF_ERR_INVALID, "block_size must be 0, 64, 128 or 256");
    if (e->max_iterations < 1 || e->max_iterations > 64) return fail(PBF_ERR_INVALID, "max_iterations must lie in [1, 64]");
    if (e->adaptive && p->iterations > e->max_iterations)
        return fail(PBF_ERR_INVALID, "iterations exceeds max_iterations");
    if (!std::isfinite(e->density_tol) || e->density_tol < 0) return fail(PBF_ERR_INVALID, "density_tol must be >= 0");
    if (!std::isfinite(e->warm_clamp) || e->warm_clamp < 0) return fail(PBF_ERR_INVALID, "warm_clamp must be >= 0");
    if (e->pair_lanes != 0 && e->pair_lanes != 1 && e->pair_lanes != 2 && e->pair_lanes != 4 && e->pair_lanes != 8)
        return fail(PBF_ERR_INVALID, "pair_lanes must be 0, 1, 2, 4 or 8");
    if (e->persistent != 0 && e->persistent != 1) return fail(PBF_ERR_INVALID, "persistent must be 0 or 1");
    if (e->warm_unfused != 0 && e->warm_unfused != 1) return fail(PBF_ERR_INVALID, "warm_unfused must be 0 or 1");
    if (e->warm_floor != 0 && e->warm_floor != 1) return fail(PBF_ERR_INVALID, "warm_floor must be 0 or 1");
    if (e->warm_floor && e->warm_clamp > 0.0f && e->warm_clamp < 1.0f)
        return fail(PBF_ERR_INVALID, "warm_floor needs warm_clamp >= 1 (or 0)");
    return PBF_OK;
}

// Wraps each launch in a pair of timing events when ext.profile is set; the
// events are captured into the graph and read back by pbf_stage_times.
const char* const kStageNames[ST_COUNT] = {"hash", "scan", "scatter", "reorder", "neighbours", "lambda", "dp",
                                            "velocity", "curl", "vorticity", "copy", "density error",
                                            "warm-start mlp"};

struct Prof {
    pbf_solver* s;
    cudaStream_t st;
    bool on;
    template <typename F> void operator()(int stage, F&& f) {
        NvtxRange range(kStageNames[stage]);
        if (!on) {
            f();
            return;
        }
        StageEvents e{stage, nullptr, nullptr};
        cudaEventCreate(&e.a);
        cudaEventCreate(&e.b);
        // external record nodes: the events are recorded by every graph replay
        cudaEventRecordWithFlags(e.a, st, cudaEventRecordExternal);
        f();
        cudaEventRecordWithFlags(e.b, st, cudaEventRecordExternal);
        s->prof.push_back(e);
    }
};

int count_kernel_nodes(cudaGraph_t g, int* out) {
    size_t nn = 0;
    CK(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    CK(cudaGraphGetNodes(g, nodes.data(), &nn));
    int k = 0;
    for (auto nd : nodes) {
        // this runtime cannot name the type of a conditional node under newer
        // drivers (it returns cudaErrorUnknown); such a node is not a kernel
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess) {
            if (t == cudaGraphNodeTypeKernel) ++k;
        } else {
            cudaGetLastError();
        }
    }
    *out = k;
    return PBF_OK;
}

// Appends to the capture on `st` the adaptive correction loop as a graph while
// node. Each pass runs one correction (lambda, then delta-p, which ends the loop
// instead when the lambda pass measured an error within tolerance) and the
// loop-control kernel; passes run for slots first, first + 1, ... < max_it.
// A converged substep therefore launches no further kernels.
int capture_correction_loop(pbf_solver* s, cudaStream_t st, int first, int min_it, int max_it, float* acc, bool dbg) {
    const KParams& kp = s->kp;
    DevStats* ds = s->dstats;
    cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* dp = nullptr;
    size_t nd = 0;
    CK(cudaStreamGetCaptureInfo(st, &status, nullptr, &g, &dp, &nd));
    if (status != cudaStreamCaptureStatusActive) return fail(PBF_ERR_CUDA, "correction loop: stream is not capturing");
    const std::vector<cudaGraphNode_t> deps(dp, dp + nd);
    cudaGraphConditionalHandle h;
    CK(cudaGraphConditionalHandleCreate(&h, g, first < max_it ? 1u : 0u, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CK(cudaGraphAddNode(&node, g, deps.data(), deps.size(), &np));
    CK(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t body = np.conditional.phGraph_out[0];
    cudaStream_t bs = s->body_stream;
    CK(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    const IterCtl c{&ds->done, ds->max_bits, ds->sum, &ds->iters, &ds->conv_slot, (double)s->ext.density_tol,
                    first, min_it, &ds->loop_k, acc};
    launch_lambda(kp, dbg, s->Px, s->nbr, s->ncnt, s->Q, s->rho_dbg, c, bs);
    launch_dp(kp, dbg, s->Q, s->nbr, s->ncnt, s->Pxold, s->Px, nullptr, s->dp_dbg, c, bs);
    launch_loop_ctl(h, &ds->loop_k, &ds->done, first, max_it, bs);
    cudaGraph_t out = nullptr;
    CK(cudaStreamEndCapture(bs, &out));
    return count_kernel_nodes(body, &s->loop_kernel_nodes);
}

// Enqueue one substep on `st` (captured into the graph).
int enqueue_substep(pbf_solver* s, cudaStream_t st) {
    const KParams& kp = s->kp;
    const bool dbg = s->ext.debug != 0;
    const int n = s->n;
    int* err = &s->dstats->err;
    DevStats* ds = s->dstats;
    Prof P{s, st, s->ext.profile != 0};
    // (the grid hash of this substep's predicted positions -- cell keys, tickets
    // and counts -- was done by the previous substep's vorticity pass, or by the
    // upload or grid build that set the state)
    if (dbg) cudaMemcpyAsync(s->hash_dbg, s->cell, sizeof(int) * n, cudaMemcpyDeviceToDevice, st);
    P(ST_SCAN, [&] { launch_scan(s->cnt, s->cell_start, s->nkeys, s->scan_ws, err, st); });
    P(ST_SCATTER, [&] { launch_scatter(n, s->cell, s->ticket, s->cell_start, s->tmp, err, st); });
    // the substep's total lambda is tracked when features are computed (warm
    // start, or recording features for training)
    const bool warm = s->ext.warm_start && s->mlp_w;
    const bool feats = warm || s->ext.record_features;
    P(ST_REORDER, [&] {
        launch_reorder(kp, true, s->Sx, s->Sv, s->Sperm, s->cell, s->cell_start, s->tmp, s->Px, s->Pv, s->Pxold,
                       s->Pperm, s->cell_sorted, feats ? s->lam_acc : nullptr, feats ? s->lam_prev_sorted : nullptr,
                       err, st);
    });
    if (dbg) launch_copy4(n, s->Px, s->xpred_dbg, st);
    P(ST_NEIGHBORS, [&] { launch_neighbors(kp, s->Px, s->cell_start, s->nbr, s->ncnt, st); });

    cudaMemsetAsync(ds, 0, offsetof(DevStats, err), st);  // per-substep slots; keeps the error bits
    const int iters = s->para.iterations;
    float* acc = feats ? s->lam_acc : nullptr;
    // First correction with features: the feature pass computes the plain lambda
    // (and the 12 features); with a warm start the MLP replaces it by lambda0.
    int first = 0;
    if (feats && iters > 0) {
        if (warm && !s->ext.warm_unfused) {
            // features, plain lambda and the network in one pass (the features stay
            // on chip; they reach s->feat only when recorded for training)
            int rc = 0;
            P(ST_LAMBDA, [&] {
                rc = launch_features_warm(kp, s->Px, s->Pv, s->nbr, s->ncnt, s->lam_prev_sorted, s->Q,
                                          s->ext.record_features ? s->feat : nullptr, s->lam_acc, s->mlp_w, s->mlp_b,
                                          s->lam0, s->ext.warm_clamp, s->ext.warm_floor, err, st);
            });
            if (rc) return fail(PBF_ERR_CUDA, "fused warm-start pass: launch configuration failed");
        } else {
            P(ST_LAMBDA, [&] {
                launch_features(kp, s->Px, s->Pv, s->nbr, s->ncnt, s->lam_prev_sorted, s->Q, s->feat, s->lam_acc, st);
            });
            if (warm)
                P(ST_MLP, [&] {
                    mlp_infer(s->mlp_w, s->mlp_b, s->feat, n, s->lam0, s->Q, s->lam_acc, s->ext.warm_clamp,
                              s->ext.warm_floor, err, st);
                });
        }
        const bool last = !s->ext.adaptive && iters == 1;
        P(ST_DP, [&] {
            launch_dp(kp, dbg, s->Q, s->nbr, s->ncnt, s->Pxold, s->Px, last ? s->Pv : nullptr, s->dp_dbg, IterCtl{},
                      st);
        });
        first = 1;
    }
    s->first_corrections = first;
    if (!s->ext.adaptive) {
        for (int it = first; it < iters; ++it) {
            const bool last = it == iters - 1;
            IterCtl c{};
            c.lam_acc = acc;
            P(ST_LAMBDA, [&] { launch_lambda(kp, dbg, s->Px, s->nbr, s->ncnt, s->Q, s->rho_dbg, c, st); });
            P(ST_DP, [&] {
                launch_dp(kp, dbg, s->Q, s->nbr, s->ncnt, s->Pxold, s->Px, last ? s->Pv : nullptr, s->dp_dbg,
                          IterCtl{}, st);
            });
        }
        if (s->ext.measure_error)
            P(ST_MEASURE, [&] {
                launch_density_error(kp, s->Px, s->nbr, s->ncnt, &ds->max_bits[kSlots - 1], &ds->sum[kSlots - 1],
                                     nullptr, st);
            });
    } else {
        // Iterate until the max density error is within tolerance (slot k holds
        // the error after k corrections), at least the configured count and at
        // most max_iterations. Corrections beyond the configured count are the
        // plain-iteration fallback.
        const int min_it = std::max(iters, 1);
        const int max_it = s->ext.max_iterations;
        if (!P.on) {
            const int rc = capture_correction_loop(s, st, first, min_it, max_it, acc, dbg);
            if (rc) return rc;
        } else {
            // Profiled (event records cannot sit in a loop body): the graph holds
            // max_iterations iterations; once converged the rest return at once.
            for (int it = first; it < max_it; ++it) {
                const IterCtl c{&ds->done, ds->max_bits, ds->sum, &ds->iters, &ds->conv_slot,
                                (double)s->ext.density_tol, it, min_it, nullptr, acc};
                P(ST_LAMBDA, [&] { launch_lambda(kp, dbg, s->Px, s->nbr, s->ncnt, s->Q, s->rho_dbg, c, st); });
                P(ST_DP, [&] {
                    launch_dp(kp, dbg, s->Q, s->nbr, s->ncnt, s->Pxold, s->Px, nullptr, s->dp_dbg, c, st);
                });
            }
        }
        // error after the last correction, for substeps that reached the cap
        P(ST_MEASURE, [&] {
            launch_density_error(kp, s->Px, s->nbr, s->ncnt, &ds->max_bits[max_it], &ds->sum[max_it], &ds->done, st);
        });
        launch_count_fallback(&ds->iters, first, iters, &ds->fallback, &ds->total_iters, st);
        P(ST_VELOCITY, [&] { launch_velocity(kp, s->Px, s->Pxold, s->Pv, st); });
    }
    P(ST_CURL, [&] { launch_curl(kp, s->Px, s->Pv, s->nbr, s->ncnt, s->omega, s->vw, st); });
    P(ST_VORT, [&] {
        launch_vort(kp, dbg, s->Px, s->vw, s->omega, s->nbr, s->ncnt, s->Sx, s->Sv, s->Pperm, s->Sperm,
                    s->vort_dbg, s->visc_dbg, s->cell, s->ticket, s->cnt, err, st);
    });
    return PBF_OK;
}

int build_graph(pbf_solver* s) {
    NvtxRange range("capture substep graph");
    if (s->exec) {
        cudaGraphExecDestroy(s->exec);
        s->exec = nullptr;
    }
    if (s->graph) {
        cudaGraphDestroy(s->graph);
        s->graph = nullptr;
    }
    for (auto& e : s->prof) {
        cudaEventDestroy(e.a);
        cudaEventDestroy(e.b);
    }
    s->prof.clear();
    s->loop_kernel_nodes = 0;
    CK(cudaStreamBeginCapture(s->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_substep(s, s->cap_stream);
    cudaError_t e = cudaStreamEndCapture(s->cap_stream, &s->graph);
    if (rc) {
        if (s->graph) cudaGraphDestroy(s->graph);
        s->graph = nullptr;
        return rc;
    }
    if (e != cudaSuccess) return fail(PBF_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    CK(cudaGraphInstantiate(&s->exec, s->graph, 0));
    int top = 0;
    const int rc2 = count_kernel_nodes(s->graph, &top);
    if (rc2) return rc2;
    s->kernel_nodes = top + s->loop_kernel_nodes;
    return PBF_OK;
}

// Allocates a solver over `nscenes` validated scene descriptions (defined below).
int create_common(const pbf_solver_parameter* para, int nscenes, const pbf_scene_desc* descs,
                  const pbf_ext_params* ext, pbf_solver** out);

}  // namespace

extern "C" {

int pbf_abi_version(void) { return PBF_ABI_VERSION; }

size_t pbf_struct_size(int which) {
    switch (which) {
        case 0: return sizeof(pbf_solver_parameter);
        case 1: return sizeof(pbf_ext_params);
        case 2: return sizeof(pbf_stats);
        case 3: return sizeof(pbf_camera);
        default: return 0;
    }
}

const char* pbf_last_error(void) { return g_err.c_str(); }

void pbf_ext_params_default(pbf_ext_params* e) {
    if (!e) return;
    std::memset(e, 0, sizeof *e);
    e->gravity[0] = 0.0f;
    e->gravity[1] = -49.0f;
    e->gravity[2] = 0.0f;
    e->grid_dims[0] = e->grid_dims[1] = e->grid_dims[2] = 64;
    e->cell_scale = 1.0f;
    e->wall_jitter = 0.01f;
    e->grad_rmin = 0.01f;
    e->max_neighbors = 63;
    e->cell_order = 0;
    e->flags = 0;
    e->scorr_scale = 1.0f;
    e->density_tol = 0.01f;
    e->max_iterations = 16;
    e->warm_clamp = 4.0f;
    e->pair_lanes = 2;
}

int pbf_create(const pbf_solver_parameter* para, const float grid_space[6], const float boundary[6],
               const pbf_ext_params* ext, pbf_solver** out) {
    if (!out) return fail(PBF_ERR_INVALID, "null output handle");
    *out = nullptr;
    pbf_ext_params def;
    if (!ext) {
        pbf_ext_params_default(&def);
        ext = &def;
    }
    int rc = validate(para, grid_space, boundary, ext);
    if (rc) return rc;
    pbf_scene_desc d{};
    std::memcpy(d.grid_space, grid_space, sizeof d.grid_space);
    std::memcpy(d.boundary, boundary, sizeof d.boundary);
    for (int a = 0; a < 3; ++a) d.grid_dims[a] = ext->grid_dims[a];
    for (int a = 0; a < 4; ++a) d.sphere[a] = ext->sphere[a];
    d.nparticles = para->nParticles;
    return create_common(para, 1, &d, ext, out);
}

int pbf_create_batch(const pbf_solver_parameter* para, int nscenes, const pbf_scene_desc* scenes,
                     const pbf_ext_params* ext, pbf_solver** out) {
    if (!out) return fail(PBF_ERR_INVALID, "null output handle");
    *out = nullptr;
    if (!para || !scenes || nscenes <= 0) return fail(PBF_ERR_INVALID, "need a parameter block and >= 1 scene");
    pbf_ext_params def;
    if (!ext) {
        pbf_ext_params_default(&def);
        ext = &def;
    }
    long long total = 0;
    for (int i = 0; i < nscenes; ++i) {
        int rc = validate_scene(scenes[i], i);
        if (rc) return rc;
        total += scenes[i].nparticles;
    }
    if (total != para->nParticles)
        return fail(PBF_ERR_INVALID, "nParticles (%d) differs from the scenes' total (%lld)", para->nParticles, total);
    int rc = validate(para, scenes[0].grid_space, scenes[0].boundary, ext);
    if (rc) return rc;
    return create_common(para, nscenes, scenes, ext, out);
}

int pbf_get_scene_layout(const pbf_solver* s, int scene, int* cell_base, int* ncells, int* pbase, int* pcount) {
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (scene < 0 || scene >= (int)s->scenes_h.size()) return fail(PBF_ERR_INVALID, "scene %d out of range", scene);
    const SceneView& v = s->scenes_h[scene];
    if (cell_base) *cell_base = v.cell_base;
    if (ncells) *ncells = v.ncells;
    if (pbase) *pbase = v.pbase;
    if (pcount) *pcount = v.pcount;
    return PBF_OK;
}

}  // extern "C"

namespace {

int create_common(const pbf_solver_parameter* para, int nscenes, const pbf_scene_desc* descs,
                  const pbf_ext_params* ext, pbf_solver** out) {
    int rc = PBF_OK;
    pbf_solver* s = new (std::nothrow) pbf_solver();
    if (!s) return fail(PBF_ERR_ALLOC, "host allocation failed");
    s->para = *para;
    s->ext = *ext;
    std::memcpy(s->grid_space, descs[0].grid_space, sizeof s->grid_space);
    std::memcpy(s->boundary, descs[0].boundary, sizeof s->boundary);
    s->n = para->nParticles;
    // scene table: keys of scene i are [cell_base, cell_base + ncells], the last
    // being its out-of-grid bin; its particles occupy slots [pbase, pbase + pcount)
    long long keys = 0, slots = 0;
    for (int i = 0; i < nscenes; ++i) {
        const pbf_scene_desc& d = descs[i];
        SceneView v{};
        for (int a = 0; a < 3; ++a) {
            v.gmin[a] = d.grid_space[a];
            v.bmin[a] = d.boundary[a];
            v.bmax[a] = d.boundary[3 + a];
            v.dims[a] = d.grid_dims[a];
        }
        for (int a = 0; a < 4; ++a) v.sphere[a] = d.sphere[a];
        v.ncells = d.grid_dims[0] * d.grid_dims[1] * d.grid_dims[2];
        v.cell_base = (int)keys;
        v.pbase = (int)slots;
        v.pcount = d.nparticles;
        keys += (long long)v.ncells + 1;
        slots += d.nparticles;
        s->scenes_h.push_back(v);
    }
    if (keys >= (1ll << 31) - 1) {
        delete s;
        return fail(PBF_ERR_INVALID, "too many cells over all scenes (%lld)", keys);
    }
    s->nkeys = (int)keys;
    s->ncells = s->scenes_h[0].ncells;
    s->capacity = s->n;
    s->stride = (s->n + 31) & ~31;
    const size_t n = s->n;
    const bool dbg = ext->debug != 0;
#define AL(ptr, count)                     \
    do {                                   \
        rc = dalloc(&(ptr), (count));      \
        if (rc) {                          \
            free_all(s);                   \
            delete s;                      \
            return rc;                     \
        }                                  \
    } while (0)
    AL(s->Sx, n); AL(s->Sv, n); AL(s->Px, n); AL(s->Pv, n); AL(s->Pxold, n); AL(s->Q, n); AL(s->omega, n); AL(s->vw, n);
    AL(s->Sperm, n); AL(s->Pperm, n); AL(s->cell, n); AL(s->ticket, n); AL(s->tmp, n); AL(s->cell_sorted, n);
    AL(s->ncnt, n);
    AL(s->nbr, (size_t)ext->max_neighbors * s->stride);
    AL(s->cnt, (size_t)s->nkeys);
    AL(s->cell_start, (size_t)s->nkeys + 1);
    AL(s->lam_acc, n); AL(s->lam_prev_sorted, n); AL(s->lam0, n);
    AL(s->feat, n * (size_t)MLP_IN);
    AL(s->staging, 6 * n);
    AL(s->dstats, 1);
    if (dbg) {
        AL(s->xpred_dbg, n); AL(s->dp_dbg, n); AL(s->vort_dbg, n); AL(s->visc_dbg, n); AL(s->rho_dbg, n);
        AL(s->hash_dbg, n);
    }
    if (nscenes > 1) {
        AL(s->scenes_d, (size_t)nscenes);
        AL(s->sid, n);
    }
    {
        const size_t ws = scan_status_bytes(s->nkeys);
        cudaError_t e = cudaMalloc(&s->scan_ws, ws);
        if (e != cudaSuccess) {
            free_all(s);
            delete s;
            return fail(PBF_ERR_ALLOC, "cudaMalloc(scan workspace): %s", cudaGetErrorString(e));
        }
    }
#undef AL
    cudaError_t e = cudaMemset(s->cnt, 0, sizeof(int) * (size_t)s->nkeys);
    if (e == cudaSuccess && nscenes > 1) {
        e = cudaMemcpy(s->scenes_d, s->scenes_h.data(), sizeof(SceneView) * nscenes, cudaMemcpyHostToDevice);
        std::vector<int> sid(n);
        for (int i = 0; i < nscenes; ++i)
            for (int k = 0; k < s->scenes_h[i].pcount; ++k) sid[s->scenes_h[i].pbase + k] = i;
        if (e == cudaSuccess) e = cudaMemcpy(s->sid, sid.data(), sizeof(int) * n, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemset(s->dstats, 0, sizeof(DevStats));
    if (e == cudaSuccess) e = cudaMemset(s->lam_acc, 0, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMemset(s->lam0, 0, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->body_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        free_all(s);
        delete s;
        return fail(PBF_ERR_CUDA, "setup: %s", cudaGetErrorString(e));
    }
    s->kp = make_kparams(*s);
    *out = s;
    return PBF_OK;
}

}  // namespace

namespace pbf {
// Current positions of a solver (float4, slot order) for the renderer.
int solver_positions(pbf_solver* s, const float4** x, int* n) {
    if (!s) return set_last_error(PBF_ERR_INVALID, "null handle");
    if (!s->uploaded) return set_last_error(PBF_ERR_STATE, "render before pbf_upload");
    *x = s->Sx;
    *n = s->n;
    return PBF_OK;
}
}  // namespace pbf

extern "C" {

int pbf_destroy(pbf_solver* s) {
    if (!s) return PBF_OK;
    cudaStreamSynchronize(s->last_stream);  // NULL is the legacy default stream
    cudaDeviceSynchronize();
    free_all(s);
    delete s;
    return PBF_OK;
}

int pbf_upload_device(pbf_solver* s, const float* d_pos, const float* d_vel, int n, void* stream) {
    NvtxRange range("pbf_upload_device");
    if (!s || !d_pos || !d_vel) return fail(PBF_ERR_INVALID, "null argument");
    if (n != s->n) return fail(PBF_ERR_INVALID, "n (%d) differs from nParticles (%d)", n, s->n);
    cudaStream_t st = (cudaStream_t)stream;
    CK(cudaMemsetAsync(s->dstats, 0, sizeof(DevStats), st));
    launch_from_aos(n, d_pos, d_vel, s->Sx, s->Sv, s->Sperm, &s->dstats->err, st);
    CK(cudaGetLastError());
    CK(cudaMemsetAsync(s->lam_acc, 0, sizeof(float) * n, st));
    // the first substep's grid hash (later substeps get theirs from the
    // vorticity pass before them)
    CK(cudaMemsetAsync(s->cnt, 0, sizeof(int) * (size_t)s->nkeys, st));
    launch_hash(s->kp, true, s->Sx, s->Sv, s->cell, s->ticket, s->cnt, &s->dstats->err, st);
    CK(cudaGetLastError());
    s->last_stream = st;
    s->uploaded = true;
    s->substeps = s->total_iters = s->fallbacks = 0;
    return PBF_OK;
}

int pbf_upload(pbf_solver* s, const float* pos, const float* vel, int n) {
    NvtxRange range("pbf_upload");
    if (!s || !pos || !vel) return fail(PBF_ERR_INVALID, "null argument");
    if (n != s->n) return fail(PBF_ERR_INVALID, "n (%d) differs from nParticles (%d)", n, s->n);
    for (size_t i = 0; i < (size_t)3 * n; ++i)
        if (!std::isfinite(pos[i]) || !std::isfinite(vel[i]))
            return fail(PBF_ERR_NONFINITE, "non-finite input at float %zu", i);
    CK(cudaMemcpy(s->staging, pos, sizeof(float) * 3 * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->staging + 3 * (size_t)n, vel, sizeof(float) * 3 * n, cudaMemcpyHostToDevice));
    int rc = pbf_upload_device(s, s->staging, s->staging + 3 * (size_t)n, n, nullptr);
    if (rc) return rc;
    CK(cudaStreamSynchronize(nullptr));
    return PBF_OK;
}

int pbf_bind_position(pbf_solver* s, float* d_pos) {
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    s->bound_pos = d_pos;
    return PBF_OK;
}

int pbf_step(pbf_solver* s, int substeps, void* stream) {
    NvtxRange range("pbf_step");
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (!s->uploaded) return fail(PBF_ERR_STATE, "pbf_step before pbf_upload");
    if (substeps < 0) return fail(PBF_ERR_INVALID, "negative substep count");
    if (s->ext.warm_start && !s->mlp_w) return fail(PBF_ERR_STATE, "warm_start set but no weights installed");
    if (!s->exec) {
        int rc = build_graph(s);
        if (rc) return rc;
    }
    cudaStream_t st = (cudaStream_t)stream;
    for (int i = 0; i < substeps; ++i) CK(cudaGraphLaunch(s->exec, st));
    if (s->bound_pos && substeps > 0) {
        launch_to_aos(s->n, s->Sx, s->Sperm, s->bound_pos, &s->dstats->err, st);
        CK(cudaGetLastError());
    }
    s->last_stream = st;
    s->substeps += substeps;
    return PBF_OK;
}

int pbf_step_host(pbf_solver* s, const float* pos, const float* vel, float* pos_out, int substeps, void* stream) {
    NvtxRange range("pbf_step_host");
    if (!s || !pos || !vel || !pos_out) return fail(PBF_ERR_INVALID, "null argument");
    if (substeps < 0) return fail(PBF_ERR_INVALID, "negative substep count");
    if (!s->hp) {
        // built aside and attached only once every stream, buffer and event
        // exists, so a failed set-up leaves the handle as it was and the next
        // call tries again
        HostPipe* hp = new (std::nothrow) HostPipe();
        if (!hp) return fail(PBF_ERR_ALLOC, "host allocation failed");
        const size_t n = s->capacity;
        cudaError_t e = cudaStreamCreateWithFlags(&hp->h2d, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&hp->d2h, cudaStreamNonBlocking);
        for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
            e = staging_malloc((void**)&hp->in[b], sizeof(float) * 6 * std::max<size_t>(n, 1));
            if (e == cudaSuccess) e = staging_malloc((void**)&hp->out[b], sizeof(float) * 3 * std::max<size_t>(n, 1));
            for (cudaEvent_t* ev : {&hp->in_ready[b], &hp->in_free[b], &hp->out_ready[b], &hp->out_free[b]})
                if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
        }
        if (e != cudaSuccess) {
            free_host_pipe(hp);
            return fail(PBF_ERR_ALLOC, "pbf_step_host staging: %s", cudaGetErrorString(e));
        }
        s->hp = hp;
    }
    HostPipe& hp = *s->hp;
    cudaStream_t st = (cudaStream_t)stream;
    const int b = (int)(hp.calls & 1);
    const size_t bytes = sizeof(float) * 3 * (size_t)s->n;
    // inputs: into staging b once the upload of two calls ago has read it
    CK(cudaStreamWaitEvent(hp.h2d, hp.in_free[b], 0));
    CK(cudaMemcpyAsync(hp.in[b], pos, bytes, cudaMemcpyHostToDevice, hp.h2d));
    CK(cudaMemcpyAsync(hp.in[b] + 3 * (size_t)s->n, vel, bytes, cudaMemcpyHostToDevice, hp.h2d));
    CK(cudaEventRecord(hp.in_ready[b], hp.h2d));
    CK(cudaStreamWaitEvent(st, hp.in_ready[b], 0));
    int rc = pbf_upload_device(s, hp.in[b], hp.in[b] + 3 * (size_t)s->n, s->n, stream);
    if (rc) return rc;
    CK(cudaEventRecord(hp.in_free[b], st));
    rc = pbf_step(s, substeps, stream);
    if (rc) return rc;
    // result: into staging b once the copy-out of two calls ago has read it
    CK(cudaStreamWaitEvent(st, hp.out_free[b], 0));
    rc = pbf_download_device(s, hp.out[b], nullptr, stream);
    if (rc) return rc;
    CK(cudaEventRecord(hp.out_ready[b], st));
    CK(cudaStreamWaitEvent(hp.d2h, hp.out_ready[b], 0));
    CK(cudaMemcpyAsync(pos_out, hp.out[b], bytes, cudaMemcpyDeviceToHost, hp.d2h));
    CK(cudaEventRecord(hp.out_free[b], hp.d2h));
    ++hp.calls;
    return PBF_OK;
}

int pbf_debug_expire_wait(int which, int* error_bits) {
    if (!error_bits) return fail(PBF_ERR_INVALID, "null argument");
    if (which != 0 && which != 1) return fail(PBF_ERR_INVALID, "which must be 0 (scan) or 1 (tensor-core barrier)");
    *error_bits = 0;
    const int m = 3 * 8192;  // three scan tiles; 192 feature rows for the network
    int *d_in = nullptr, *d_out = nullptr, *d_err = nullptr;
    void* ws = nullptr;
    uint16_t* w = nullptr;
    float *b = nullptr, *feat = nullptr, *out = nullptr;
    cudaError_t e = cudaMalloc(&d_err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(d_err, 0, sizeof(int));
    if (e == cudaSuccess && which == 0) {
        e = cudaMalloc(&d_in, sizeof(int) * m);
        if (e == cudaSuccess) e = cudaMemset(d_in, 0, sizeof(int) * m);
        if (e == cudaSuccess) e = cudaMalloc(&d_out, sizeof(int) * (m + 1));
        if (e == cudaSuccess) e = cudaMalloc(&ws, scan_status_bytes(m));
        // tile 0 never publishes; its successors give up after 4,096 polls
        if (e == cudaSuccess) launch_scan_silent_tile(d_in, d_out, m, ws, d_err, 0, 4096, nullptr);
    } else if (e == cudaSuccess) {
        const int rows = 192;
        e = cudaMalloc(&w, sizeof(uint16_t) * MLP_NUM_WEIGHTS);
        if (e == cudaSuccess) e = cudaMemset(w, 0, sizeof(uint16_t) * MLP_NUM_WEIGHTS);
        if (e == cudaSuccess) e = cudaMalloc(&b, sizeof(float) * MLP_NUM_BIASES);
        if (e == cudaSuccess) e = cudaMemset(b, 0, sizeof(float) * MLP_NUM_BIASES);
        if (e == cudaSuccess) e = cudaMalloc(&feat, sizeof(float) * MLP_IN * rows);
        if (e == cudaSuccess) e = cudaMemset(feat, 0, sizeof(float) * MLP_IN * rows);
        if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(float) * rows);
        if (e == cudaSuccess && mlp_infer_uncommitted(w, b, feat, rows, out, 4096, d_err, nullptr))
            e = cudaErrorLaunchFailure;
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(error_bits, d_err, sizeof(int), cudaMemcpyDeviceToHost);
    for (void* p : {(void*)d_in, (void*)d_out, (void*)d_err, ws, (void*)w, (void*)b, (void*)feat, (void*)out})
        if (p) cudaFree(p);
    if (e != cudaSuccess) return fail(PBF_ERR_CUDA, "pbf_debug_expire_wait: %s", cudaGetErrorString(e));
    if (*error_bits) return fail(PBF_ERR_DEVICE, "kernel error bits 0x%x", *error_bits);
    return PBF_OK;
}

int pbf_measure_fp32_peak(double* scalar_tflops, double* packed_tflops) {
    if (!scalar_tflops || !packed_tflops) return fail(PBF_ERR_INVALID, "null argument");
    NvtxRange range("pbf_measure_fp32_peak");
    if (measure_fp32_peak(scalar_tflops, packed_tflops)) return fail(PBF_ERR_CUDA, "FP32 throughput probe failed");
    return PBF_OK;
}

int pbf_debug_fail_staging_alloc(int k) {
    if (k < 0) return fail(PBF_ERR_INVALID, "k must be >= 0");
    g_fail_staging_alloc.store(k);
    return PBF_OK;
}

int pbf_host_fence(pbf_solver* s, void* stream) {
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (!s->hp || s->hp->calls == 0) return PBF_OK;
    // copies of one direction complete in call order; the last copy-out comes
    // after its call's copy-in
    CK(cudaStreamWaitEvent((cudaStream_t)stream, s->hp->out_free[(s->hp->calls - 1) & 1], 0));
    return PBF_OK;
}

int pbf_set_parameter(pbf_solver* s, const pbf_solver_parameter* para) {
    if (!s || !para) return fail(PBF_ERR_INVALID, "null argument");
    if (para->nParticles != s->n)
        return fail(PBF_ERR_INVALID, "nParticles (%d) differs from the solver's %d particles", para->nParticles, s->n);
    const int rc = validate(para, s->grid_space, s->boundary, &s->ext);
    if (rc) return rc;
    if (std::memcmp(para, &s->para, sizeof *para) == 0) return PBF_OK;
    s->para = *para;
    s->kp = make_kparams(*s);
    if (s->exec) {  // constants and the iteration count live in the captured graph
        cudaGraphExecDestroy(s->exec);
        s->exec = nullptr;
    }
    if (s->uploaded) {
        // The next substep's grid hash (prediction with dt and gravity, cell keys
        // with h) was made with the old values; make it again from the state.
        cudaStream_t st = s->last_stream;
        CK(cudaMemsetAsync(s->cnt, 0, sizeof(int) * (size_t)s->nkeys, st));
        launch_hash(s->kp, true, s->Sx, s->Sv, s->cell, s->ticket, s->cnt, &s->dstats->err, st);
        CK(cudaGetLastError());
    }
    return PBF_OK;
}

int pbf_resize(pbf_solver* s, int n) {
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (s->scenes_h.size() != 1) return fail(PBF_ERR_INVALID, "pbf_resize needs a single-scene solver");
    if (n < 1 || n > s->capacity) return fail(PBF_ERR_INVALID, "n (%d) outside [1, %d]", n, s->capacity);
    CK(cudaDeviceSynchronize());  // nothing of the old size may still run
    s->n = n;
    s->para.nParticles = n;
    s->scenes_h[0].pcount = n;
    s->kp = make_kparams(*s);
    if (s->exec) {  // grid sizes change: capture again at the next pbf_step
        cudaGraphExecDestroy(s->exec);
        s->exec = nullptr;
    }
    s->uploaded = false;
    return PBF_OK;
}

int pbf_download_sorted_device(pbf_solver* s, float* d_pos, float* d_vel, int* d_ids, int* d_key, int* d_rank,
                               void* stream) {
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (s->substeps == 0) return fail(PBF_ERR_STATE, "no substep has run since the upload");
    cudaStream_t st = (cudaStream_t)stream;
    launch_sorted_state(s->n, s->Sx, s->Sv, s->Sperm, s->cell_sorted, s->cell_start, d_pos, d_vel, d_ids, d_key,
                        d_rank, st);
    CK(cudaGetLastError());
    s->last_stream = st;
    return PBF_OK;
}

int pbf_build_grid(pbf_solver* s, void* stream) {
    NvtxRange range("pbf_build_grid");
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (!s->uploaded) return fail(PBF_ERR_STATE, "pbf_build_grid before pbf_upload");
    cudaStream_t st = (cudaStream_t)stream;
    const KParams& kp = s->kp;
    int* err = &s->dstats->err;
    CK(cudaMemsetAsync(s->cnt, 0, sizeof(int) * (size_t)s->nkeys, st));  // drop the next substep's counts
    launch_hash(kp, false, s->Sx, s->Sv, s->cell, s->ticket, s->cnt, err, st);
    if (s->hash_dbg) CK(cudaMemcpyAsync(s->hash_dbg, s->cell, sizeof(int) * s->n, cudaMemcpyDeviceToDevice, st));
    launch_scan(s->cnt, s->cell_start, s->nkeys, s->scan_ws, err, st);
    launch_scatter(s->n, s->cell, s->ticket, s->cell_start, s->tmp, err, st);
    launch_reorder(kp, false, s->Sx, s->Sv, s->Sperm, s->cell, s->cell_start, s->tmp, s->Px, s->Pv, s->Pxold, s->Pperm,
                   s->cell_sorted, nullptr, nullptr, err, st);
    launch_neighbors(kp, s->Px, s->cell_start, s->nbr, s->ncnt, st);
    CK(cudaGetLastError());
    // the sorted state becomes the current state
    CK(cudaMemcpyAsync(s->Sx, s->Px, sizeof(float4) * s->n, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->Sv, s->Pv, sizeof(float4) * s->n, cudaMemcpyDeviceToDevice, st));
    CK(cudaMemcpyAsync(s->Sperm, s->Pperm, sizeof(int) * s->n, cudaMemcpyDeviceToDevice, st));
    // the next substep's grid hash of that state (the scan left the counts zero)
    launch_hash(kp, true, s->Sx, s->Sv, s->cell, s->ticket, s->cnt, err, st);
    CK(cudaGetLastError());
    s->last_stream = st;
    return PBF_OK;
}

int pbf_download_device(pbf_solver* s, float* d_pos, float* d_vel, void* stream) {
    NvtxRange range("pbf_download_device");
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (!s->uploaded) return fail(PBF_ERR_STATE, "pbf_download before pbf_upload");
    cudaStream_t st = (cudaStream_t)stream;
    if (d_pos) launch_to_aos(s->n, s->Sx, s->Sperm, d_pos, &s->dstats->err, st);
    if (d_vel) launch_to_aos(s->n, s->Sv, s->Sperm, d_vel, &s->dstats->err, st);
    CK(cudaGetLastError());
    s->last_stream = st;
    return PBF_OK;
}

int pbf_download(pbf_solver* s, float* pos, float* vel) {
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (!s->uploaded) return fail(PBF_ERR_STATE, "pbf_download before pbf_upload");
    const size_t n = s->n;
    CK(cudaStreamSynchronize(s->last_stream));  // NULL is the legacy default stream
    int rc = pbf_download_device(s, s->staging, s->staging + 3 * n, nullptr);
    if (rc) return rc;
    CK(cudaStreamSynchronize(nullptr));
    if (pos) CK(cudaMemcpy(pos, s->staging, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost));
    if (vel) CK(cudaMemcpy(vel, s->staging + 3 * n, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost));
    return PBF_OK;
}

int pbf_get_stats(pbf_solver* s, pbf_stats* out) {
    if (!s || !out) return fail(PBF_ERR_INVALID, "null argument");
    CK(cudaStreamSynchronize(s->last_stream));  // NULL is the legacy default stream
    CK(cudaDeviceSynchronize());
    DevStats h;
    CK(cudaMemcpy(&h, s->dstats, sizeof h, cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof *out);
    out->substeps = s->substeps;
    out->error_bits = h.err;
    int slot = kSlots - 1;
    if (s->ext.adaptive) {
        out->last_iterations = s->first_corrections + h.iters;
        slot = h.done ? h.conv_slot : s->ext.max_iterations;
    } else {
        out->last_iterations = s->para.iterations;
    }
    slot = std::min(std::max(slot, 0), kSlots - 1);
    out->fallbacks = h.fallback;
    double m;
    std::memcpy(&m, &h.max_bits[slot], sizeof m);
    out->max_density_error = m;
    out->mean_density_error = h.sum[slot] / (double)s->n;
    out->total_iterations = s->ext.adaptive ? h.total_iters : s->substeps * (long long)s->para.iterations;
    if (h.err) return fail(PBF_ERR_DEVICE, "kernel error bits 0x%x", h.err);
    return PBF_OK;
}

int pbf_stage_times(pbf_solver* s, float* ms, int nstages) {
    if (!s || !ms || nstages <= 0) return fail(PBF_ERR_INVALID, "null argument");
    if (s->prof.empty()) return fail(PBF_ERR_STATE, "stage times need ext.profile and a pbf_step");
    CK(cudaStreamSynchronize(s->last_stream));  // NULL is the legacy default stream
    for (int i = 0; i < nstages; ++i) ms[i] = 0.0f;
    for (const auto& e : s->prof) {
        float t = 0.0f;
        CK(cudaEventElapsedTime(&t, e.a, e.b));
        if (e.stage < nstages) ms[e.stage] += t;
    }
    return PBF_OK;
}

int pbf_graph_kernel_count(pbf_solver* s) {
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (!s->exec) {
        int rc = build_graph(s);
        if (rc) return rc;
    }
    return s->kernel_nodes;
}

int pbf_measure_density_error(pbf_solver* s, double* max_err, double* mean_err, void* stream) {
    if (!s || !max_err || !mean_err) return fail(PBF_ERR_INVALID, "null argument");
    if (!s->uploaded || s->substeps == 0) return fail(PBF_ERR_STATE, "no substep has run");
    cudaStream_t st = (cudaStream_t)stream;
    DevStats* ds = s->dstats;
    CK(cudaMemsetAsync(&ds->max_bits[kSlots - 1], 0, sizeof(unsigned long long), st));
    CK(cudaMemsetAsync(&ds->sum[kSlots - 1], 0, sizeof(double), st));
    launch_density_error(s->kp, s->Sx, s->nbr, s->ncnt, &ds->max_bits[kSlots - 1], &ds->sum[kSlots - 1], nullptr, st);
    CK(cudaGetLastError());
    unsigned long long mb = 0;
    double sum = 0.0;
    CK(cudaMemcpyAsync(&mb, &ds->max_bits[kSlots - 1], sizeof mb, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&sum, &ds->sum[kSlots - 1], sizeof sum, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::memcpy(max_err, &mb, sizeof mb);
    *mean_err = sum / (double)s->n;
    return PBF_OK;
}

size_t pbf_field_bytes(const pbf_solver* s, int field) {
    if (!s) return 0;
    const size_t n = s->n;
    switch (field) {
        case PBF_FIELD_X: case PBF_FIELD_V: case PBF_FIELD_XOLD: case PBF_FIELD_XPRED: case PBF_FIELD_XL:
        case PBF_FIELD_DP: case PBF_FIELD_CURL: case PBF_FIELD_VORT: case PBF_FIELD_VISC:
            return n * sizeof(float4);
        case PBF_FIELD_RHO: case PBF_FIELD_LAMBDA0: case PBF_FIELD_LAMBDA_TOTAL: return n * sizeof(float);
        case PBF_FIELD_FEATURES: return n * MLP_IN * sizeof(float);
        case PBF_FIELD_CELL: case PBF_FIELD_PERM: case PBF_FIELD_NCNT: case PBF_FIELD_HASH: return n * sizeof(int);
        case PBF_FIELD_CELL_START: return ((size_t)s->nkeys + 1) * sizeof(int);
        case PBF_FIELD_NBR: return (size_t)s->ext.max_neighbors * s->stride * sizeof(int);
        default: return 0;
    }
}

int pbf_fetch(pbf_solver* s, int field, void* dst, size_t bytes) {
    if (!s || !dst) return fail(PBF_ERR_INVALID, "null argument");
    const size_t want = pbf_field_bytes(s, field);
    if (want == 0) return fail(PBF_ERR_INVALID, "unknown field %d", field);
    if (bytes != want) return fail(PBF_ERR_INVALID, "field %d needs %zu bytes, got %zu", field, want, bytes);
    const void* src = nullptr;
    switch (field) {
        case PBF_FIELD_X: src = s->Sx; break;
        case PBF_FIELD_V: src = s->Sv; break;
        case PBF_FIELD_XOLD: src = s->Pxold; break;
        case PBF_FIELD_XPRED: src = s->xpred_dbg; break;
        case PBF_FIELD_XL: src = s->Q; break;
        case PBF_FIELD_RHO: src = s->rho_dbg; break;
        case PBF_FIELD_DP: src = s->dp_dbg; break;
        case PBF_FIELD_CURL: src = s->omega; break;
        case PBF_FIELD_VORT: src = s->vort_dbg; break;
        case PBF_FIELD_VISC: src = s->visc_dbg; break;
        case PBF_FIELD_CELL: src = s->cell_sorted; break;
        case PBF_FIELD_CELL_START: src = s->cell_start; break;
        case PBF_FIELD_PERM: src = s->Sperm; break;
        case PBF_FIELD_NCNT: src = s->ncnt; break;
        case PBF_FIELD_NBR: src = s->nbr; break;
        case PBF_FIELD_HASH: src = s->hash_dbg; break;
        case PBF_FIELD_LAMBDA0: src = s->lam0; break;
        case PBF_FIELD_FEATURES: src = s->feat; break;
        case PBF_FIELD_LAMBDA_TOTAL: src = s->lam_acc; break;
        default: break;
    }
    if (!src) return fail(PBF_ERR_STATE, "field %d is kept only when ext.debug is set", field);
    CK(cudaStreamSynchronize(s->last_stream));  // NULL is the legacy default stream
    CK(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
    return PBF_OK;
}

int pbf_get_layout(const pbf_solver* s, int* ncells, int* stride, int* max_neighbors) {
    if (!s) return fail(PBF_ERR_INVALID, "null handle");
    if (ncells) *ncells = s->ncells;
    if (stride) *stride = s->stride;
    if (max_neighbors) *max_neighbors = s->ext.max_neighbors;
    return PBF_OK;
}

int pbf_set_warm_start(pbf_solver* s, const unsigned short* w_bf16, size_t n_w, const float* b_f32, size_t n_b) {
    if (!s || !w_bf16 || !b_f32) return fail(PBF_ERR_INVALID, "null argument");
    if (n_w != (size_t)MLP_NUM_WEIGHTS || n_b != (size_t)MLP_NUM_BIASES)
        return fail(PBF_ERR_INVALID, "warm start needs %d bf16 weights and %d floats", MLP_NUM_WEIGHTS,
                    MLP_NUM_BIASES);
    for (size_t i = 0; i < n_b; ++i)
        if (!std::isfinite(b_f32[i])) return fail(PBF_ERR_NONFINITE, "non-finite warm-start constant %zu", i);
    if (!s->mlp_w) {
        int rc = dalloc(&s->mlp_w, (size_t)MLP_NUM_WEIGHTS);
        if (!rc) rc = dalloc(&s->mlp_b, (size_t)MLP_NUM_BIASES);
        if (rc) return rc;
    }
    CK(cudaMemcpy(s->mlp_w, w_bf16, sizeof(uint16_t) * MLP_NUM_WEIGHTS, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(s->mlp_b, b_f32, sizeof(float) * MLP_NUM_BIASES, cudaMemcpyHostToDevice));
    if (s->exec) {  // the substep graph depends on whether a warm start is installed
        cudaGraphExecDestroy(s->exec);
        s->exec = nullptr;
    }
    return PBF_OK;
}

int pbf_gather_training_rows(pbf_solver* s, const int* d_slots, int count, float* d_feat, float* d_target,
                             void* stream) {
    if (!s || !d_slots || !d_feat || !d_target) return fail(PBF_ERR_INVALID, "null argument");
    if (!s->ext.record_features && !s->ext.warm_start)
        return fail(PBF_ERR_STATE, "features are kept only with ext.record_features or ext.warm_start");
    if (count < 0) return fail(PBF_ERR_INVALID, "negative count");
    cudaStream_t st = (cudaStream_t)stream;
    launch_gather_rows(d_slots, count, s->n, s->feat, s->lam_acc, d_feat, d_target, &s->dstats->err, st);
    CK(cudaGetLastError());
    s->last_stream = st;
    return PBF_OK;
}

struct pbf_mlp_trainer {
    MlpTrainer* t;
    int max_batch;
};

int pbf_mlp_trainer_create(int max_batch, const float* w32, const float* b32, pbf_mlp_trainer** out) {
    if (!out || !w32 || !b32) return fail(PBF_ERR_INVALID, "null argument");
    *out = nullptr;
    if (max_batch < 1 || max_batch > (1 << 24)) return fail(PBF_ERR_INVALID, "max_batch out of range");
    for (int i = 0; i < MLP_NUM_WEIGHTS; ++i)
        if (!std::isfinite(w32[i])) return fail(PBF_ERR_NONFINITE, "non-finite weight %d", i);
    for (int i = 0; i < MLP_NUM_BIASES; ++i)
        if (!std::isfinite(b32[i])) return fail(PBF_ERR_NONFINITE, "non-finite bias %d", i);
    MlpTrainer* t = mlp_trainer_create(max_batch, w32, b32);
    if (!t) return fail(PBF_ERR_ALLOC, "trainer buffers");
    *out = new pbf_mlp_trainer{t, max_batch};
    return PBF_OK;
}

int pbf_mlp_trainer_destroy(pbf_mlp_trainer* tr) {
    if (!tr) return PBF_OK;
    cudaDeviceSynchronize();
    mlp_trainer_destroy(tr->t);
    delete tr;
    return PBF_OK;
}

int pbf_mlp_gradients(pbf_mlp_trainer* tr, const float* d_feat, const float* d_target, int batch, float* h_gw,
                      float* h_gb, float* h_loss, void* stream) {
    if (!tr || !d_feat || !d_target) return fail(PBF_ERR_INVALID, "null argument");
    if (batch < 1 || batch > tr->max_batch) return fail(PBF_ERR_INVALID, "batch must lie in [1, max_batch]");
    cudaStream_t st = (cudaStream_t)stream;
    if (mlp_gradients(tr->t, d_feat, d_target, batch, st)) return fail(PBF_ERR_CUDA, "gradient kernels failed");
    if (h_gw || h_gb || h_loss) {
        CK(cudaStreamSynchronize(st));
        int err = 0;
        mlp_read(tr->t, nullptr, nullptr, h_gw, h_gb, h_loss, &err);
        if (err) return fail(PBF_ERR_DEVICE, "tensor-core pipeline error bits 0x%x", err);
    }
    return PBF_OK;
}

int pbf_mlp_train_step(pbf_mlp_trainer* tr, const float* d_feat, const float* d_target, int batch, float lr,
                       float* h_loss, void* stream) {
    int rc = pbf_mlp_gradients(tr, d_feat, d_target, batch, nullptr, nullptr, nullptr, stream);
    if (rc) return rc;
    if (!(lr > 0.0f) || !std::isfinite(lr)) return fail(PBF_ERR_INVALID, "learning rate must be positive");
    cudaStream_t st = (cudaStream_t)stream;
    if (mlp_adam(tr->t, lr, 0.9f, 0.999f, 1e-8f, st)) return fail(PBF_ERR_CUDA, "Adam kernels failed");
    if (h_loss) {
        CK(cudaStreamSynchronize(st));
        int err = 0;
        mlp_read(tr->t, nullptr, nullptr, nullptr, nullptr, h_loss, &err);
        if (err) return fail(PBF_ERR_DEVICE, "tensor-core pipeline error bits 0x%x", err);
    }
    return PBF_OK;
}

int pbf_mlp_get_params(pbf_mlp_trainer* tr, float* w32, float* b32, unsigned short* w_bf16) {
    if (!tr) return fail(PBF_ERR_INVALID, "null handle");
    CK(cudaDeviceSynchronize());
    mlp_read(tr->t, w32, b32, nullptr, nullptr, nullptr, nullptr);
    if (w_bf16)
        CK(cudaMemcpy(w_bf16, mlp_weights_bf16(tr->t), sizeof(uint16_t) * MLP_NUM_WEIGHTS, cudaMemcpyDeviceToHost));
    return PBF_OK;
}

int pbf_mlp_forward(pbf_mlp_trainer* tr, const float* d_feat, int batch, float* d_out, void* stream) {
    if (!tr || !d_feat || !d_out) return fail(PBF_ERR_INVALID, "null argument");
    if (batch < 1) return fail(PBF_ERR_INVALID, "batch must be positive");
    static int* d_err = nullptr;
    if (!d_err) CK(cudaMalloc(&d_err, sizeof(int)));
    cudaStream_t st = (cudaStream_t)stream;
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    if (mlp_infer(mlp_weights_bf16(tr->t), mlp_biases(tr->t), d_feat, batch, d_out, nullptr, nullptr, 0.0f, 0, d_err,
                  st))
        return fail(PBF_ERR_CUDA, "inference kernel failed");
    int h = 0;
    CK(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h) return fail(PBF_ERR_DEVICE, "tensor-core pipeline error bits 0x%x", h);
    return PBF_OK;
}

int pbf_tc_gemm_bf16(const void* d_a, const void* d_b, float* d_d, int n, int k, void* stream) {
    if (!d_a || !d_b || !d_d) return fail(PBF_ERR_INVALID, "null argument");
    if (n < 16 || n > 256 || n % 16 || k < 16 || k > 256 || k % 16)
        return fail(PBF_ERR_INVALID, "n and k must be multiples of 16 in [16, 256]");
    static int* d_err = nullptr;
    if (!d_err) CK(cudaMalloc(&d_err, sizeof(int)));
    cudaStream_t st = (cudaStream_t)stream;
    CK(cudaMemsetAsync(d_err, 0, sizeof(int), st));
    if (tc_gemm_bf16(d_a, d_b, d_d, n, k, d_err, st)) return fail(PBF_ERR_CUDA, "tensor-core GEMM launch failed");
    int h = 0;
    CK(cudaMemcpyAsync(&h, d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (h) return fail(PBF_ERR_DEVICE, "tensor-core pipeline wait expired (error bits 0x%x)", h);
    return PBF_OK;
}

size_t pbf_scan_workspace_bytes(int n) {
    if (n <= 0 || n > PBF_SCAN_MAX_COUNT) return 0;
    return scan_status_bytes(n) + 16;
}

int pbf_scan_exclusive_i32(const int* d_in, int* d_out, int n, void* d_ws, size_t ws_bytes, void* stream) {
    if (!d_in || !d_out || !d_ws) return fail(PBF_ERR_INVALID, "null argument");
    if (n <= 0) return fail(PBF_ERR_INVALID, "n must be positive");
    if (n > PBF_SCAN_MAX_COUNT) return fail(PBF_ERR_INVALID, "n exceeds the scan's maximum of 2^30 counts");
    if (ws_bytes < pbf_scan_workspace_bytes(n)) return fail(PBF_ERR_INVALID, "workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    int* err = (int*)((char*)d_ws + scan_status_bytes(n));
    CK(cudaMemsetAsync(err, 0, sizeof(int), st));
    launch_scan_const(d_in, d_out, n, d_ws, err, st);
    CK(cudaGetLastError());
    int herr = 0;
    CK(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (herr) return fail(PBF_ERR_DEVICE, "scan error bits 0x%x", herr);
    return PBF_OK;
}

}  // extern "C"
