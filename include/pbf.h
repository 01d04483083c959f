/*
 * pbf.h -- C ABI of the B200-native Position Based Fluids solver step.
 *
 * Drop-in boundary for the reference's solver interface:
 *   kernels/cudaPBF.h:8-12      initCUDASolverDataBuffer / cudaPBFSolve / freeCUDASolverDataBuffer
 *   include/solverBase.h:16-64  SolverParameter, SolverData
 *   include/solver.h:86-111     PBFSolver(para, box, fext) / solve(Particle*)
 * Plain C types only; no CUDA or torch types in any signature (a stream is a
 * void* holding a cudaStream_t, NULL = the legacy default stream).
 *
 * Every function returns PBF_OK (0) or a negative status and never exits the
 * process; pbf_last_error() gives a message for the calling thread. Calls on one
 * handle are stream-ordered and not thread-safe without external locking.
 */
#ifndef PBF_B200_PBF_H
#define PBF_B200_PBF_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PBF_ABI_VERSION 1

/* status codes */
#define PBF_OK 0
#define PBF_ERR_INVALID (-1)   /* bad argument or parameter */
#define PBF_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define PBF_ERR_ALLOC (-3)     /* device or host allocation failed */
#define PBF_ERR_DEVICE (-4)    /* a kernel reported an error bit (see pbf_stats.error_bits) */
#define PBF_ERR_STATE (-5)     /* call out of order, e.g. pbf_step before pbf_upload */
#define PBF_ERR_NONFINITE (-6) /* NaN or Inf in positions or velocities */

/* error_bits reported by kernels */
#define PBF_DEVERR_SCAN_TIMEOUT 1 /* scan look-back wait expired */
#define PBF_DEVERR_BAD_INDEX 2    /* an index fell outside its array */
#define PBF_DEVERR_NONFINITE 4    /* a non-finite position appeared */
#define PBF_DEVERR_MLP_TIMEOUT 8  /* tensor-core pipeline wait expired */

/* Same layout and meaning as the reference SolverParameter
 * (include/solverBase.h:16-40); 13 x 4 bytes. */
typedef struct pbf_solver_parameter {
    float h;          /* kernel radius */
    int nParticles;
    float restRho;    /* rest density rho0 */
    float epsilon;    /* constraint relaxation */
    float k;          /* s_corr strength */
    float n;          /* s_corr exponent */
    float deltaq;     /* s_corr reference distance */
    float c;          /* XSPH viscosity */
    float dt;         /* substep */
    float invDt;      /* accepted for layout compatibility; the step divides by dt */
    int iterations;   /* Jacobi iterations (minimum count when adaptive) */
    float vorticityConfinementEpilon;
    float radius;     /* particle radius (the reference app shrinks the box by it) */
} pbf_solver_parameter;

/* stable-mode flags (each is a named departure from the reference formulas) */
#define PBF_FLAG_CLAMP_C 1u   /* unilateral density constraint C = max(C, 0) */
#define PBF_FLAG_XSPH_RHO 2u  /* XSPH weight c / rho0 instead of c */
#define PBF_FLAG_WALL_DENSITY 4u /* boundary faces add the density of a fluid half-space */

/* Everything the reference fixes at compile time or does not have. Fill with
 * pbf_ext_params_default() and change what you need. */
typedef struct pbf_ext_params {
    float gravity[3];    /* default (0,-49,0): kernels/cudaPBFSolver.cu:9 */
    int grid_dims[3];    /* default 64^3: include/solverBase.h:10-12 */
    float cell_scale;    /* cell edge = h * cell_scale, >= 0.25 (default 1); below 1 the
                            stencil reaches ceil(1 / cell_scale) cells each way */
    float wall_jitter;   /* wall offset coefficient (default 0.01, RANDOM_OFFSET_COEFF) */
    float grad_rmin;     /* spiky gradient lower cutoff (default 0.01, cuh:107) */
    int max_neighbors;   /* neighbour cap, 1..127 (default 63, MAX_NEIGHBOR) */
    int cell_order;      /* 0 ascending (stable) or 1 descending slot order within a cell */
    unsigned flags;      /* PBF_FLAG_* */
    float scorr_scale;   /* multiplies s_corr (default 1) */
    float sphere[4];     /* static sphere obstacle: centre xyz, radius (<= 0: none) */
    int adaptive;        /* 1: iterate until max density error <= density_tol */
    float density_tol;   /* one-sided max density error tolerance (default 0.01) */
    int max_iterations;  /* cap for adaptive iterations and warm-start fallback (default 16) */
    int measure_error;   /* 1: record max/mean density error of every substep */
    int debug;           /* 1: keep per-stage intermediates for pbf_fetch */
    int warm_start;      /* 1: learned lambda warm start (needs installed weights) */
    int profile;         /* 1: time every launch with CUDA events (pbf_stage_times) */
    int block_size;      /* threads per block of the neighbour passes: 0 (= 256), 64, 128 or 256 */
    int record_features; /* 1: keep warm-start features and total lambda (training data) */
    float warm_clamp;    /* warm start: lambda0 keeps the sign of the plain lambda of its
                            pass and at most warm_clamp times its magnitude (default 4; 0: off) */
    int pair_lanes;      /* threads sharing one particle's neighbour sums: 1, 2, 4 or 8 (default 2;
                            0 = 2). Lane t takes list entries t, t+L, ...; lane sums are combined
                            pairwise, so the value changes the FP32 summation order */
    int persistent;      /* 1: each neighbour pass (search, lambda, dp, curl, vorticity) is one
                            persistent launch: the blocks resident at once stride over all
                            scenes' tiles of slots (default 0: one block per tile). Same results */
    int warm_unfused;    /* 1: the warm start's feature pass and network as two launches with the
                            features through HBM (default 0: one fused launch, the features go
                            from the feature pass to the tensor cores through shared memory).
                            Same results; kept for measurement */
    int warm_floor;      /* 1: with warm_clamp > 0, lambda0 is also at least as strong as the plain
                            lambda of its pass (between it and warm_clamp times it), so the first
                            correction never pushes less than a plain iteration would (default 0) */
} pbf_ext_params;

typedef struct pbf_stats {
    long long substeps;         /* substeps run since upload */
    long long total_iterations; /* Jacobi iterations run since upload */
    long long fallbacks;        /* warm-start substeps that needed plain iterations */
    int last_iterations;        /* iterations used by the last substep */
    int error_bits;             /* PBF_DEVERR_* accumulated since upload */
    double max_density_error;   /* last substep: max_i max(rho_i/rho0 - 1, 0), FP64 */
    double mean_density_error;  /* last substep: mean of the same */
} pbf_stats;

typedef struct pbf_solver pbf_solver;

/* pbf_fetch field ids: internal arrays in cell-sorted slot order */
#define PBF_FIELD_X 0          /* float4[n] positions after the substep */
#define PBF_FIELD_V 1          /* float4[n] velocities after the substep */
#define PBF_FIELD_XOLD 2       /* float4[n] positions before prediction */
#define PBF_FIELD_XPRED 3      /* float4[n] predicted positions (debug) */
#define PBF_FIELD_XL 4         /* float4[n] last lambda pass: xyz, lambda in w */
#define PBF_FIELD_RHO 5        /* float[n] last density (debug) */
#define PBF_FIELD_DP 6         /* float4[n] last position correction (debug) */
#define PBF_FIELD_CURL 7       /* float4[n] vorticity omega */
#define PBF_FIELD_VORT 8       /* float4[n] confinement force (debug) */
#define PBF_FIELD_VISC 9       /* float4[n] XSPH term (debug) */
#define PBF_FIELD_CELL 10      /* int[n] cell key per slot (ncells = outside the grid) */
#define PBF_FIELD_CELL_START 11 /* int[ncells + 2] cell starts, out-of-grid bin, n */
#define PBF_FIELD_PERM 12      /* int[n] slot -> original particle id */
#define PBF_FIELD_NCNT 13      /* int[n] neighbour counts */
#define PBF_FIELD_NBR 14       /* int[max_neighbors * stride] slot-major neighbour slots */
#define PBF_FIELD_HASH 15      /* int[n] cell key per particle before sorting (debug) */
#define PBF_FIELD_LAMBDA0 16   /* float[n] warm-start lambda of the last substep */
#define PBF_FIELD_FEATURES 17  /* float[n * 12] warm-start features of the last substep */
#define PBF_FIELD_LAMBDA_TOTAL 18 /* float[n] total lambda applied in the last substep */

void pbf_ext_params_default(pbf_ext_params* ext);

/* Replaces initCUDASolverDataBuffer (kernels/cudaPBF.cu:4-30) and the
 * PBFSolver constructor (include/solver.h:86-110): allocates every device
 * buffer for para->nParticles particles. grid_space and boundary are AABBs
 * (pMin xyz, pMax xyz): grid_space anchors the uniform grid, boundary is the
 * wall the particles are clamped to. */
int pbf_create(const pbf_solver_parameter* para, const float grid_space[6], const float boundary[6],
               const pbf_ext_params* ext, pbf_solver** out);

/* One scene of a batch (no reference counterpart): its grid anchor and wall
 * box, grid cells per axis, particle count and sphere obstacle. */
typedef struct pbf_scene_desc {
    float grid_space[6];
    float boundary[6];
    int grid_dims[3];
    int nparticles;
    float sphere[4];  /* centre xyz, radius (<= 0: none) */
} pbf_scene_desc;

/* Many independent scenes advanced together: every phase of a substep is one
 * launch over all scenes' particles, and one scan over the concatenated cell
 * keys of all scenes sorts every scene at once. para->nParticles must be the
 * sum of the scenes' counts; positions and velocities are uploaded and
 * downloaded concatenated in scene order. ext->grid_dims and ext->sphere are
 * taken from the scene descriptions instead. */
int pbf_create_batch(const pbf_solver_parameter* para, int nscenes, const pbf_scene_desc* scenes,
                     const pbf_ext_params* ext, pbf_solver** out);

/* Layout of scene `scene`: first cell key, real cells, first particle slot,
 * particle count. */
int pbf_get_scene_layout(const pbf_solver* s, int scene, int* cell_base, int* ncells, int* pbase, int* pcount);

/* Replaces freeCUDASolverDataBuffer (kernels/cudaPBF.cu:32-48). */
int pbf_destroy(pbf_solver* s);

/* Host positions and velocities, AoS xyz, n == nParticles; the cudaMemcpy of
 * kernels/cudaPBF.cu:26-27. Resets the stats. */
int pbf_upload(pbf_solver* s, const float* pos, const float* vel, int n);

/* Same from device memory (AoS xyz float[3n]), stream-ordered. */
int pbf_upload_device(pbf_solver* s, const float* d_pos, const float* d_vel, int n, void* stream);

/* Caller-owned device buffer float[3n] that receives positions in original
 * order after every pbf_step, as data.position did (src/renderapp.cpp:246-249,
 * kernels/cudaPBF.cu:7). NULL unbinds. */
int pbf_bind_position(pbf_solver* s, float* d_pos);

/* Replaces cudaPBFSolve (kernels/cudaPBF.cu:50-115), once per substep: replays
 * the captured substep graph `substeps` times on `stream`. */
int pbf_step(pbf_solver* s, int substeps, void* stream);

/* New SolverParameter values for the following substeps, as the reference's
 * cudaPBFSolve(data, para) takes them on every call (kernels/cudaPBF.cu:50-115
 * reads h, dt, iterations, restRho, epsilon, k, n, deltaq, c and the vorticity
 * epsilon from para each time). para->nParticles must equal the solver's
 * particle count. Unchanged values cost nothing; changed ones take effect from
 * the next pbf_step, which captures its graph again, and the grid hash the next
 * substep starts from is made again with them (stream-ordered on the stream of
 * the last call). */
int pbf_set_parameter(pbf_solver* s, const pbf_solver_parameter* para);

/* One frame from and to host memory, asynchronous and pipelined across calls
 * (no reference counterpart; the host side of initCUDASolverDataBuffer's
 * copies and cudaPBFSolve in one call): copies pos and vel (AoS xyz float[3n];
 * page-locked memory lets the copies overlap) to the device on an internal
 * stream, uploads them as pbf_upload_device does and runs `substeps` substeps
 * on `stream`, then copies the positions (original order) to pos_out on a
 * second internal stream. Device staging is double-buffered, so the copies of
 * neighbouring calls overlap the substeps. The three host buffers must stay
 * untouched until the call's copies are done: pbf_host_fence(s, stream) makes
 * `stream` wait for every copy issued so far; synchronise that stream before
 * reading pos_out. */
int pbf_step_host(pbf_solver* s, const float* pos, const float* vel, float* pos_out, int substeps, void* stream);
int pbf_host_fence(pbf_solver* s, void* stream);

/* Testing hook (host-side fault injection, no reference counterpart): the k-th
 * device allocation of the next pbf_step_host staging set-up (1-based; four per
 * set-up) fails as if the device were out of memory; 0 turns it off. A failed
 * set-up returns PBF_ERR_ALLOC and leaves the handle as it was, so the next call
 * sets the staging up again. */
int pbf_debug_fail_staging_alloc(int k);

/* Testing hook (failure injection on the device without a fault, no reference
 * counterpart; the reference's CHECK_CUDA exits the process instead,
 * kernels/cudaPBFSolver.cuh:5-10). Runs one production kernel with a wait that
 * nothing will satisfy and a short limit: which = 0, the exclusive scan with a
 * tile that never publishes its status (the look-back waits of its successors
 * run out); which = 1, the warm-start network's forward kernel with nothing
 * committed to its tensor-core barrier. The kernel records the expired wait in
 * its error word, frees what it holds and returns; *error_bits receives the
 * word (PBF_DEVERR_SCAN_TIMEOUT or PBF_DEVERR_MLP_TIMEOUT) and the call returns
 * PBF_ERR_DEVICE, with the CUDA context still usable. Synchronises the device. */
int pbf_debug_expire_wait(int which, int* error_bits);

/* Measured FP32 fused multiply-add throughput of the current device in TFLOP/s
 * (no reference counterpart): scalar FFMA and packed two-lane f32x2 FMA chains,
 * 8 per thread on 8 blocks of 256 per SM, best of three CUDA-event-timed
 * launches. The denominator the neighbour passes' FP32 rate is reported
 * against. Synchronises the device. */
int pbf_measure_fp32_peak(double* scalar_tflops, double* packed_tflops);

/* Changes the particle count of a single-scene solver to n (1 <= n <= the
 * nParticles it was created with); the next pbf_step captures its graph again
 * and needs a new upload first. Synchronises the device. */
int pbf_resize(pbf_solver* s, int n);

/* The state after the last pbf_step in slot order (cell order): AoS positions
 * and velocities, each slot's index in the uploaded order, the key of the cell
 * the slot was sorted into and the slot's rank within that cell. The next
 * substep sorts stably by (key, rank), which is what a caller that splits and
 * merges states (slab decomposition) needs to keep the order. Any pointer may
 * be NULL; stream-ordered. */
int pbf_download_sorted_device(pbf_solver* s, float* d_pos, float* d_vel, int* d_ids, int* d_key, int* d_rank,
                               void* stream);

/* Host copies of positions / velocities in original order (either may be NULL). */
int pbf_download(pbf_solver* s, float* pos, float* vel);

/* Same into device buffers, stream-ordered (either may be NULL). */
int pbf_download_device(pbf_solver* s, float* d_pos, float* d_vel, void* stream);

/* Synchronises the handle's last stream and reports stats; returns
 * PBF_ERR_DEVICE when a kernel has set an error bit. */
int pbf_get_stats(pbf_solver* s, pbf_stats* st);

/* Copies an internal array (PBF_FIELD_*) to host memory; bytes must equal the
 * field size given by pbf_field_bytes. Synchronises. */
int pbf_fetch(pbf_solver* s, int field, void* dst, size_t bytes);
size_t pbf_field_bytes(const pbf_solver* s, int field);

/* Grid build only, on the current positions and without prediction: hash,
 * histogram, scan, sort and neighbour search (buildNeighborhood's job,
 * kernels/cudaPBFSolver.cu:31-154; src/solver.cpp:3-58). */
int pbf_build_grid(pbf_solver* s, void* stream);

/* Sizes: number of cells, neighbour-list stride. */
int pbf_get_layout(const pbf_solver* s, int* ncells, int* stride, int* max_neighbors);

/* Profiling (ext.profile = 1): milliseconds per stage in the last substep, summed
 * over the launches of each stage. Stages: 0 hash (0 within a substep: the
 * previous substep's vorticity pass hashes the state it writes), 1 scan, 2 scatter,
 * 3 reorder, 4 neighbours, 5 lambda, 6 dp, 7 velocity, 8 curl, 9 vorticity,
 * 10 copy, 11 density measurement, 12 warm-start MLP. */
#define PBF_NUM_STAGES 13
int pbf_stage_times(pbf_solver* s, float* ms, int nstages);

/* Number of kernel launches in one substep (kernel nodes of the substep graph);
 * negative status on error. With ext.adaptive (and ext.profile off) the
 * corrections run in a device-side loop (a graph while node): its body's
 * kernels count once here and launch once per pass. */
int pbf_graph_kernel_count(pbf_solver* s);

/* One-sided density error max_i max(rho_i/rho0 - 1, 0) and its mean over the
 * current positions (FP64 accumulation over each neighbour list); synchronises
 * `stream`. */
int pbf_measure_density_error(pbf_solver* s, double* max_err, double* mean_err, void* stream);

/* Exclusive scan of int32 with decoupled look-back (calculatePrefixSum +
 * addBlockSum, kernels/cudaPBFSolver.cu:42-96, for 1 <= n <= PBF_SCAN_MAX_COUNT;
 * larger n is rejected with PBF_ERR_INVALID and pbf_scan_workspace_bytes returns
 * 0 for it). d_out receives n + 1 ints (the total last). d_ws must hold
 * pbf_scan_workspace_bytes(n) bytes. The input is left unchanged. */
#define PBF_SCAN_MAX_COUNT (1 << 30)
size_t pbf_scan_workspace_bytes(int n);
int pbf_scan_exclusive_i32(const int* d_in, int* d_out, int n, void* d_ws, size_t ws_bytes, void* stream);

/* ---- Learned lambda warm start (no reference counterpart) --------------------
 * A per-particle MLP, 12 features -> 64 -> 64 -> 64 -> 1 with GELU, BF16
 * weights and FP32 accumulation on the tensor cores, predicts the substep's
 * total lambda from the features of the first lambda pass; that prediction is
 * applied as the first correction, then the plain Jacobi iterations follow (and,
 * with ext.adaptive, continue while the density error exceeds ext.density_tol).
 * Weights: W1[64][16], W2[64][64], W3[64][64], w4[64] row-major [out][in]
 * (9,280 values); constants: b1[64], b2[64], b3[64], b4, feature mean[16],
 * feature 1/std[16], output scale (226 floats). */
#define PBF_MLP_NUM_WEIGHTS 9280
#define PBF_MLP_NUM_BIASES 226

/* Installs warm-start weights (BF16 bit patterns) and constants in a solver. */
int pbf_set_warm_start(pbf_solver* s, const unsigned short* w_bf16, size_t n_w, const float* b_f32, size_t n_b);

/* Training rows from the last substep (ext.record_features): for each slot in
 * d_slots, its 12 features to d_feat[i * 12] and its total lambda to d_target[i]. */
int pbf_gather_training_rows(pbf_solver* s, const int* d_slots, int count, float* d_feat, float* d_target,
                             void* stream);

/* Trainer: FP32 master weights, Adam state, and tensor-core forward/backward
 * kernels; loss = mean (output - target / output scale)^2. */
typedef struct pbf_mlp_trainer pbf_mlp_trainer;
int pbf_mlp_trainer_create(int max_batch, const float* w32, const float* b32, pbf_mlp_trainer** out);
int pbf_mlp_trainer_destroy(pbf_mlp_trainer* t);
/* Gradients of the loss over a batch (device features [batch][12], targets
 * [batch]); copies them (9,280 + 226 floats, zeros for the constants) and the
 * loss to host memory when the pointers are not null. */
int pbf_mlp_gradients(pbf_mlp_trainer* t, const float* d_feat, const float* d_target, int batch, float* h_gw,
                      float* h_gb, float* h_loss, void* stream);
/* Gradients plus one Adam step (beta 0.9 / 0.999, eps 1e-8). */
int pbf_mlp_train_step(pbf_mlp_trainer* t, const float* d_feat, const float* d_target, int batch, float lr,
                       float* h_loss, void* stream);
int pbf_mlp_get_params(pbf_mlp_trainer* t, float* w32, float* b32, unsigned short* w_bf16);
/* lambda0 for a batch of feature rows with the trainer's current weights. */
int pbf_mlp_forward(pbf_mlp_trainer* t, const float* d_feat, int batch, float* d_out, void* stream);

/* Tile GEMM on the 5th-generation tensor cores (tcgen05, TMEM accumulator):
 * d_d[128 x n] = d_a[128 x k] * d_b[n x k]^T with BF16 row-major inputs and an
 * FP32 row-major output; n and k multiples of 16 in [16, 256]. The building
 * block of the warm-start MLP, exported for testing. Synchronises `stream`. */
int pbf_tc_gemm_bf16(const void* d_a, const void* d_b, float* d_d, int n, int k, void* stream);

/* The same exclusive scan for callers that cannot allocate device memory (no
 * counterpart in the reference). A render or simulation loop that must not
 * stall on cudaMalloc, or a plug-in whose host application owns every device
 * allocation, has no workspace to pass; this variant keeps its scratch (about
 * 33 KB) in a device array inside the library, so it calls no cudaMalloc,
 * cudaFree or allocating library routine. Limit: n <= 16,777,216 (larger n is
 * rejected with PBF_ERR_INVALID). The first call on each device looks up the
 * array's device address, so make that first call before any stream capture.
 * All calls share the array: calls that overlap on the GPU race, so issue them
 * on one stream or serialise them. d_out receives n + 1 ints (total last);
 * the input is left unchanged. Synchronises `stream`. */
int pbf_scan_exclusive_i32_noalloc(const int* d_in, int* d_out, int n, void* stream);

/* ---- headless screen-space fluid rendering ----------------------------------
 * The reference draws the fluid with OpenGL shader passes (src/renderapp.cpp:
 * 400-466): point-sprite depth (shaders/depth.vert, depth.frag), 60 curvature-
 * flow smoothing passes (smooth.frag), additive thickness (thickness.frag),
 * normals from depth (normal.frag), the room (background.frag) and the fluid
 * shading (shadingParticle.frag). Here each pass is a CUDA kernel writing device
 * images of width x height pixels (row 0 at the bottom, as in the GL window). */
typedef struct pbf_render pbf_render;

typedef struct pbf_camera {
    float view[16];            /* world -> view, column-major (glm::lookAt) */
    float proj[16];            /* view -> clip, column-major (glm::perspective) */
    float cam_pos[3];          /* eye position, world */
    float radius;              /* sprite radius, world units (SolverParameter.radius) */
    float point_coeff;         /* sprite size in pixels = -point_coeff * radius / z_view */
    float tan_half_fov;        /* surface reconstruction of the shading pass */
    float light_pos[3];        /* fluid light, world (reference (0, 50, -20)) */
    float light_diffuse[3];    /* (0.8, 0.8, 0.8) */
    float roi;                 /* Fresnel ratio (1.3) */
    float room_light_pos[3];   /* room light, world (reference (0, 50, 0)) */
    float room_light_diffuse[3];
    float room[6];             /* room walls: xmin, ymin (floor), zmin (back), xmax, ymax, zmax */
    int smooth_iterations;     /* curvature-flow passes (60) */
    int reserved[5];
} pbf_camera;

/* images readable with pbf_render_read (floats per pixel in brackets) */
#define PBF_IMAGE_DEPTH_RAW 0  /* [1] -z of the nearest sprite surface, 0 where empty */
#define PBF_IMAGE_DEPTH 1      /* [1] after the smoothing passes */
#define PBF_IMAGE_THICKNESS 2  /* [1] summed sprite thickness */
#define PBF_IMAGE_NORMAL 3     /* [4] view-space normal xyz, 0 */
#define PBF_IMAGE_ROOM 4       /* [4] room colour rgba (8-bit quantised, as the GL texture) */
#define PBF_IMAGE_COLOR 5      /* [4] final colour rgba */

int pbf_render_create(int width, int height, pbf_render** out);
int pbf_render_destroy(pbf_render* r);
/* Renders n particles whose xyz lie at d_pos + i * stride floats (stride 3 for
 * AoS positions, 4 for float4) on `stream`. */
int pbf_render_frame(pbf_render* r, const float* d_pos, int n, int stride, const pbf_camera* cam, void* stream);
/* Renders a solver's current state. */
int pbf_render_frame_solver(pbf_render* r, pbf_solver* s, const pbf_camera* cam, void* stream);
/* Copies one image to host memory (count = floats available at host); synchronises. */
int pbf_render_read(pbf_render* r, int image, float* host, size_t count);

const char* pbf_last_error(void);
int pbf_abi_version(void);

/* sizeof of the ABI structs, for FFI bindings to check their layouts:
 * 0 pbf_solver_parameter, 1 pbf_ext_params, 2 pbf_stats, 3 pbf_camera. */
size_t pbf_struct_size(int which);

#ifdef __cplusplus
}
#endif

#endif /* PBF_B200_PBF_H */
