// TEST INFRASTRUCTURE ONLY (fixture generator, never the product).
//
// C entry point around the reference's own CUDA solver, built by oracle/Makefile
// from kernels/cudaPBF.cu and kernels/cudaPBFSolver.cu where they lie, into
// oracle/_ref/libpbfref_gpu.so. It allocates the position buffer that the
// reference app would map from an OpenGL VBO (src/renderapp.cpp:246-249), calls
// initCUDASolverDataBuffer / cudaPBFSolve (kernels/cudaPBF.cu:4-115) unchanged,
// and copies every SolverData array back to the host.
#include <cstdio>
#include <cstring>
#include <vector>

#include "cudaPBF.h"
#include "cudaPBFSolver.cuh"

extern "C" {

// para13: SolverParameter (include/solverBase.h:16-40) as raw bytes;
// grid_space / boundary: pMin xyz, pMax xyz. Outputs may be null.
// nbr receives n x 64 ints (63 ids + count, the reference layout).
// grid receives 2 x 64^3 uints (startIdx, endIdx pairs).
int refgpu_run(const void* para13, const float* grid_space, const float* boundary, const float* pos,
               const float* vel, int substeps, float* out_pos, float* out_vel, float* out_oldpos,
               float* out_lambda, float* out_offset, float* out_curl, float* out_vort, float* out_visc,
               int* out_nbr, unsigned* out_grid, int* out_ids, int* out_prefix) {
    SolverParameter para;
    std::memcpy(&para, para13, sizeof(SolverParameter));
    const int n = para.nParticles;
    std::vector<glm::vec3> p(n), v(n);
    for (int i = 0; i < n; ++i) {
        p[i] = glm::vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        v[i] = glm::vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
    AABB gs(glm::vec3(grid_space[0], grid_space[1], grid_space[2]), glm::vec3(grid_space[3], grid_space[4], grid_space[5]));
    AABB bd(glm::vec3(boundary[0], boundary[1], boundary[2]), glm::vec3(boundary[3], boundary[4], boundary[5]));
    SolverData d;
    if (cudaMalloc((void**)&d.position, (size_t)n * 3 * sizeof(float)) != cudaSuccess) return -1;
    initCUDASolverDataBuffer(p, v, d, para, gs, bd);
    for (int s = 0; s < substeps; ++s) cudaPBFSolve(d, para);
    if (cudaDeviceSynchronize() != cudaSuccess) return -2;
    const size_t v3 = (size_t)n * 3 * sizeof(float);
    const unsigned cells = UNIFORM_GRID_DIM_SIZE_X * UNIFORM_GRID_DIM_SIZE_Y * UNIFORM_GRID_DIM_SIZE_Z;
    if (out_pos) cudaMemcpy(out_pos, d.position, v3, cudaMemcpyDeviceToHost);
    if (out_vel) cudaMemcpy(out_vel, d.velocity, v3, cudaMemcpyDeviceToHost);
    if (out_oldpos) cudaMemcpy(out_oldpos, d.oldPosition, v3, cudaMemcpyDeviceToHost);
    if (out_lambda) cudaMemcpy(out_lambda, d.lambda, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost);
    if (out_offset) cudaMemcpy(out_offset, d.particlesOffset, v3, cudaMemcpyDeviceToHost);
    if (out_curl) cudaMemcpy(out_curl, d.particlesCurl, v3, cudaMemcpyDeviceToHost);
    if (out_vort) cudaMemcpy(out_vort, d.particlesVorticity, v3, cudaMemcpyDeviceToHost);
    if (out_visc) cudaMemcpy(out_visc, d.particlesViscosity, v3, cudaMemcpyDeviceToHost);
    if (out_nbr) cudaMemcpy(out_nbr, d.neighbors, (size_t)n * (MAX_NEIGHBOR + 1) * sizeof(int), cudaMemcpyDeviceToHost);
    if (out_grid) cudaMemcpy(out_grid, d.grid, (size_t)cells * 2 * sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (out_ids) cudaMemcpy(out_ids, d.gridParticlesID, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost);
    if (out_prefix) cudaMemcpy(out_prefix, d.prefixSum, (size_t)cells * sizeof(int), cudaMemcpyDeviceToHost);
    const cudaError_t e = cudaDeviceSynchronize();
    freeCUDASolverDataBuffer(d);
    cudaFree(d.position);
    return e == cudaSuccess ? 0 : -3;
}

}  // extern "C"
