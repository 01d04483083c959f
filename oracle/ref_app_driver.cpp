// TEST INFRASTRUCTURE ONLY (a test program, never the product).
//
// Drives the library through the reference's own three entry points the way the
// reference app does (src/renderapp.cpp:246-251 and :499): the caller owns the
// device buffer data.position (cudaMalloc here, a mapped GL buffer there),
// calls initCUDASolverDataBuffer once, then cudaPBFSolve(data, para) once per
// frame, reading data.position after each call, and frees with
// freeCUDASolverDataBuffer. It is compiled against the reference's headers
// (kernels/cudaPBF.h, include/solverBase.h, include/AABB.h) and linked with
// pbf_b200/csrc/reference_shim.cpp and libpbf_b200.so by oracle/Makefile.
//
//   ref_app_driver <input> <output>
// input (raw little-endian): int n, int calls, int change_at, SolverParameter
// para (52 bytes), SolverParameter para2 (used from call change_at on), float
// gridSpace[6], float boundary[6], float pos[3n], float vel[3n].
// output: float positions[calls + 1][3n] read from data.position after the init
// and after every cudaPBFSolve.
#include <cstdio>
#include <cstring>
#include <vector>

#include "cudaPBF.h"

static bool rd(FILE* f, void* p, size_t bytes) { return std::fread(p, 1, bytes, f) == bytes; }

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <input> <output>\n", argv[0]);
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int n = 0, calls = 0, change_at = 0;
    SolverParameter para, para2;
    float gs[6], bd[6];
    bool ok = rd(f, &n, 4) && rd(f, &calls, 4) && rd(f, &change_at, 4) && rd(f, &para, sizeof para) &&
              rd(f, &para2, sizeof para2) && rd(f, gs, sizeof gs) && rd(f, bd, sizeof bd);
    if (!ok || n <= 0 || calls < 0) return 2;
    std::vector<glm::vec3> position(n), velocity(n);
    ok = rd(f, position.data(), sizeof(glm::vec3) * n) && rd(f, velocity.data(), sizeof(glm::vec3) * n);
    std::fclose(f);
    if (!ok) return 2;

    SolverData data;
    std::memset(&data, 0, sizeof data);
    if (cudaMalloc((void**)&data.position, sizeof(float) * 3 * n) != cudaSuccess) return 3;
    const AABB box(glm::vec3(gs[0], gs[1], gs[2]), glm::vec3(gs[3], gs[4], gs[5]));
    const AABB boundary(glm::vec3(bd[0], bd[1], bd[2]), glm::vec3(bd[3], bd[4], bd[5]));
    initCUDASolverDataBuffer(position, velocity, data, para, box, boundary);

    FILE* o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    std::vector<float> host(3 * (size_t)n);
    int rc = 0;
    for (int k = 0; k <= calls && rc == 0; ++k) {
        if (k > 0) cudaPBFSolve(data, k >= change_at ? para2 : para);
        if (cudaMemcpy(host.data(), data.position, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = 3;
        else if (std::fwrite(host.data(), sizeof(float), host.size(), o) != host.size())
            rc = 2;
    }
    std::fclose(o);
    freeCUDASolverDataBuffer(data);
    cudaFree(data.position);
    return rc;
}
