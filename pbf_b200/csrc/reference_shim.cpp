// The reference's three solver entry points (kernels/cudaPBF.h:8-12) on top of
// the C ABI in include/pbf.h, so the reference app's call sites
// (src/renderapp.cpp:251, :499, :508) link unchanged against libpbf_b200.so.
//
// Compiled inside the reference's tree (it needs the reference's solverBase.h,
// AABB.h and glm); see INTEGRATION.md. The SolverData fields other than
// position are not used: the handle owns its buffers and is looked up by the
// address of the caller's SolverData.
#include <mutex>
#include <unordered_map>
#include <vector>

#include "AABB.h"
#include "solverBase.h"
#include "pbf.h"

namespace {

std::mutex g_mu;
std::unordered_map<const SolverData*, pbf_solver*> g_handles;

pbf_solver* handle_of(const SolverData& d) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_handles.find(&d);
    return it == g_handles.end() ? nullptr : it->second;
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
    pbf_solver* h = nullptr;
    if (pbf_create(reinterpret_cast<const pbf_solver_parameter*>(&para), gs, bd, &ext, &h) != PBF_OK) return;
    pbf_upload(h, reinterpret_cast<const float*>(position.data()), reinterpret_cast<const float*>(velocity.data()),
               para.nParticles);
    pbf_bind_position(h, reinterpret_cast<float*>(data.position));  // the GL-mapped buffer
    // the first substep writes data.position; until then it holds the caller's upload
    std::lock_guard<std::mutex> lk(g_mu);
    g_handles[&data] = h;
}

void cudaPBFSolve(SolverData& data, const SolverParameter& para) {
    (void)para;
    if (pbf_solver* h = handle_of(data)) pbf_step(h, 1, nullptr);
}

void freeCUDASolverDataBuffer(SolverData& data) {
    pbf_solver* h = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_handles.find(&data);
        if (it == g_handles.end()) return;
        h = it->second;
        g_handles.erase(it);
    }
    pbf_destroy(h);
}
