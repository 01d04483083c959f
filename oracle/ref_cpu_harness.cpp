// TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline, never the product).
//
// C entry points around the reference's own CPU solver, PBFSolver
// (include/solver.h:83-222, src/solver.cpp:3-156), compiled from the reference
// sources where they lie by oracle/Makefile into oracle/_ref/libpbfref_cpu.so.
// Nothing here changes the reference algorithm: the harness constructs the
// solver, optionally resizes its uniform grid (the reference sizes it from the
// 64^3 macros of include/solverBase.h:10-12), calls solve() or
// buildNeiborhood() and copies the solver's internal arrays out.
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include <omp.h>

#include "config.h"
#include "AABB.h"
#include "particle.h"
#include "solverBase.h"

// The harness reads the solver's private arrays (grids, neighbour lists, lambda).
#define private public
#include "solver.h"
#undef private

namespace {

struct RefCpu {
    PBFSolver* solver = nullptr;
    std::vector<Particle> particles;
    int n = 0;
};

}  // namespace

extern "C" {

// para13: the 13 fields of SolverParameter in declaration order
// (include/solverBase.h:16-40); box: pMin xyz, pMax xyz (the solver shrinks it by
// para.radius for the wall, include/solver.h:97); dims: grid cells per axis.
void* refcpu_create(const void* para13, const float* box, const int* dims) {
    SolverParameter para;
    std::memcpy(&para, para13, sizeof(SolverParameter));
    AABB b(glm::vec3(box[0], box[1], box[2]), glm::vec3(box[3], box[4], box[5]));
    RefCpu* r = new RefCpu();
    r->n = para.nParticles;
    r->solver = new PBFSolver(para, b);
    PBFSolver& s = *r->solver;
    if (dims && (dims[0] != s.gridDimSize[0] || dims[1] != s.gridDimSize[1] || dims[2] != s.gridDimSize[2])) {
        delete[] s.grids;
        delete[] s.gridParticlesCnt;
        for (int a = 0; a < 3; ++a) s.gridDimSize[a] = dims[a];
        s.gridsCnt = dims[0] * dims[1] * dims[2];
        s.grids = new Grid[s.gridsCnt];
    } else {
        delete[] s.gridParticlesCnt;
    }
    // The constructor's memset covers sizeof(pointer) bytes only (include/solver.h:102);
    // start from an all-zero count array as a fresh mmap'd allocation would.
    s.gridParticlesCnt = new int[s.gridsCnt]();
    r->particles.resize(r->n);
    return r;
}

void refcpu_set_threads(int t) {
    if (t > 0) omp_set_num_threads(t);
}

int refcpu_max_threads() { return omp_get_max_threads(); }

static void load(RefCpu* r, const float* pos, const float* vel) {
    for (int i = 0; i < r->n; ++i) {
        r->particles[i].position = glm::vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        if (vel) r->particles[i].velocity = glm::vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
}

// One PBFSolver::solve on the given particles (in/out). quiet != 0 sends the
// solver's per-particle printf (src/solver.cpp:94) to /dev/null.
int refcpu_solve(void* hv, float* pos, float* vel, int substeps, int quiet) {
    RefCpu* r = (RefCpu*)hv;
    if (!r) return -1;
    load(r, pos, vel);
    int saved = -1, devnull = -1;
    if (quiet) {
        fflush(stdout);
        saved = dup(1);
        devnull = open("/dev/null", O_WRONLY);
        if (saved >= 0 && devnull >= 0) dup2(devnull, 1);
    }
    for (int s = 0; s < substeps; ++s) r->solver->solve(r->particles.data());
    if (quiet) {
        fflush(stdout);
        if (saved >= 0) { dup2(saved, 1); close(saved); }
        if (devnull >= 0) close(devnull);
    }
    for (int i = 0; i < r->n; ++i) {
        const glm::vec3& p = r->particles[i].position;
        const glm::vec3& v = r->particles[i].velocity;
        pos[3 * i] = p.x; pos[3 * i + 1] = p.y; pos[3 * i + 2] = p.z;
        vel[3 * i] = v.x; vel[3 * i + 1] = v.y; vel[3 * i + 2] = v.z;
    }
    return 0;
}

// buildNeiborhood (src/solver.cpp:3-58) on the given positions only.
int refcpu_build(void* hv, const float* pos) {
    RefCpu* r = (RefCpu*)hv;
    if (!r) return -1;
    load(r, pos, nullptr);
    r->solver->buildNeiborhood(r->particles.data(), r->n, r->solver->para.h);
    return 0;
}

// field ids: 0 lambda, 1 offset(3), 2 curl(3), 3 vorticity(3), 4 viscosity(3),
// 5 oldPosition(3), 6 particlesGid, 7 grid start, 8 grid end, 9 gridParticlesID,
// 10 neighbour counts, 11 neighbour ids (n x 63, unused slots -1)
int refcpu_get(void* hv, int field, double* outd, int* outi) {
    RefCpu* r = (RefCpu*)hv;
    if (!r) return -1;
    PBFSolver& s = *r->solver;
    const int n = r->n;
    auto put3 = [&](const std::vector<glm::vec3>& a) {
        for (int i = 0; i < n; ++i) { outd[3 * i] = a[i].x; outd[3 * i + 1] = a[i].y; outd[3 * i + 2] = a[i].z; }
    };
    switch (field) {
        case 0: for (int i = 0; i < n; ++i) outd[i] = s.lambda[i]; return 0;
        case 1: put3(s.particlesOffset); return 0;
        case 2: put3(s.particlesCurl); return 0;
        case 3: put3(s.particlesVorticity); return 0;
        case 4: put3(s.particlesViscosity); return 0;
        case 5: put3(s.oldPosition); return 0;
        case 6: std::memcpy(outi, s.particlesGid, sizeof(int) * n); return 0;
        case 7: for (int c = 0; c < s.gridsCnt; ++c) outi[c] = (int)s.grids[c].startIdx; return 0;
        case 8: for (int c = 0; c < s.gridsCnt; ++c) outi[c] = (int)s.grids[c].endIdx; return 0;
        case 9: std::memcpy(outi, s.gridParticlesID, sizeof(int) * n); return 0;
        case 10: for (int i = 0; i < n; ++i) outi[i] = s.neighbors[i][maxNeighborCnt]; return 0;
        case 11:
            for (int i = 0; i < n; ++i)
                for (int q = 0; q < (int)maxNeighborCnt; ++q)
                    outi[i * maxNeighborCnt + q] = q < s.neighbors[i][maxNeighborCnt] ? s.neighbors[i][q] : -1;
            return 0;
        default: return -1;
    }
}

int refcpu_ncells(void* hv) { return ((RefCpu*)hv)->solver->gridsCnt; }

void refcpu_destroy(void* hv) {
    RefCpu* r = (RefCpu*)hv;
    if (!r) return;
    PBFSolver& s = *r->solver;
    delete[] s.grids;
    delete[] s.gridParticlesCnt;
    delete[] s.particlesGid;
    delete[] s.gridParticlesID;
    for (int i = 0; i < r->n; ++i) delete[] s.neighbors[i];
    delete[] s.neighbors;
    delete r->solver;
    delete r;
}

}  // extern "C"
