// The reference's three solver entry points (kernels/cudaPBF.h:8-12) on top of
// the C ABI in include/pbf.h, so the reference app's call sites
// (src/renderapp.cpp:251, :499, :508) link unchanged against libpbf_b200.so.
//
// Compiled against the reference's headers (solverBase.h, AABB.h and glm), as
// part of the app that calls these functions. The handle owns its buffers and
// is looked up by the address of the caller's SolverData; of that struct only
// position is used, the caller-owned device buffer (the GL-mapped VBO in the
// reference app) that receives positions after every substep.
//
// The reference has no error path (CHECK_CUDA prints and exits,
// kernels/cudaPBFSolver.cuh:5-10) and these signatures return nothing, so a
// failure is printed to stderr with the library's message and the call returns;
// a later call on a SolverData whose set-up failed prints that too instead of
// doing nothing silently.
#include <cstdio>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "AABB.h"
#include "solverBase.h"
#include "pbf.h"

namespace {

struct Entry {
    pbf_solver* h = nullptr;
    pbf_solver_parameter para{};  // the values of the last call
};

std::mutex g_mu;
std::unordered_map<const SolverData*, Entry> g_handles;

void report(const char* call, int rc) {
    std::fprintf(stderr, "pbf_b200: %s failed (status %d): %s\n", call, rc, pbf_last_error());
}

}  // namespace

void initCUDASolverDataBuffer(const std::vector<glm::vec3>& position, const std::vector<glm::vec3>& velocity,
                              SolverData& data, const SolverParameter& para, const AABB& gridSpace,
                              const AABB& boundary) {
    static_assert(sizeof(SolverParameter) == sizeof(pbf_solver_parameter), "SolverParameter layout");
    pbf_ext_params ext;
    pbf_ext_params_default(&ext);  // gravity (0,-49,0), 64^3 grid, 63 neighbours: the reference's constants
    const float gs[6] = {gridSpace.pMin.x, gridSpace.pMin.y, gridSpace.pMin.z,
                         gridSpace.pMax.x, gridSpace.pMax.y, gridSpace.pMax.z};
    const float bd[6] = {boundary.pMin.x, boundary.pMin.y, boundary.pMin.z,
                         boundary.pMax.x, boundary.pMax.y, boundary.pMax.z};
    Entry e;
    std::memcpy(&e.para, &para, sizeof e.para);
    int rc = pbf_create(&e.para, gs, bd, &ext, &e.h);
    if (rc != PBF_OK) {
        report("initCUDASolverDataBuffer: pbf_create", rc);
    } else if ((rc = pbf_upload(e.h, reinterpret_cast<const float*>(position.data()),
                                reinterpret_cast<const float*>(velocity.data()), para.nParticles)) != PBF_OK) {
        report("initCUDASolverDataBuffer: pbf_upload", rc);
        pbf_destroy(e.h);
        e.h = nullptr;
    } else {
        // as the reference's init does (kernels/cudaPBF.cu:26), data.position
        // holds the uploaded positions; every substep refreshes it
        float* dpos = reinterpret_cast<float*>(data.position);
        pbf_bind_position(e.h, dpos);
        if (dpos && (rc = pbf_download_device(e.h, dpos, nullptr, nullptr)) != PBF_OK)
            report("initCUDASolverDataBuffer: copy to data.position", rc);
    }
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_handles.find(&data);
    if (it != g_handles.end() && it->second.h) pbf_destroy(it->second.h);  // a second init replaces the first
    g_handles[&data] = e;  // kept even when set-up failed, so later calls can say so
}

void cudaPBFSolve(SolverData& data, const SolverParameter& para) {
    pbf_solver* h = nullptr;
    bool changed = false;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_handles.find(&data);
        if (it == g_handles.end()) {
            std::fprintf(stderr, "pbf_b200: cudaPBFSolve on a SolverData that initCUDASolverDataBuffer did not set up\n");
            return;
        }
        h = it->second.h;
        changed = std::memcmp(&it->second.para, &para, sizeof para) != 0;
    }
    if (!h) {
        std::fprintf(stderr, "pbf_b200: cudaPBFSolve skipped: initCUDASolverDataBuffer failed for this SolverData\n");
        return;
    }
    int rc;
    // the reference reads every SolverParameter value on every call
    if (changed) {
        if ((rc = pbf_set_parameter(h, reinterpret_cast<const pbf_solver_parameter*>(&para))) != PBF_OK) {
            report("cudaPBFSolve: pbf_set_parameter", rc);
            return;
        }
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_handles.find(&data);
        if (it != g_handles.end()) std::memcpy(&it->second.para, &para, sizeof para);
    }
    if ((rc = pbf_step(h, 1, nullptr)) != PBF_OK) report("cudaPBFSolve: pbf_step", rc);
}

void freeCUDASolverDataBuffer(SolverData& data) {
    pbf_solver* h = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_handles.find(&data);
        if (it == g_handles.end()) return;
        h = it->second.h;
        g_handles.erase(it);
    }
    if (h) pbf_destroy(h);
}
