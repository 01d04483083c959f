// Exclusive scan that allocates nothing (no counterpart in the reference).
//
// Some callers cannot call cudaMalloc: a render or simulation loop that must
// not stall (cudaMalloc can synchronise the device), a plug-in inside a host
// application that owns every device allocation through its own pool, or code
// running with a device-memory budget fixed at start-up. For them this entry
// point runs the same decoupled look-back scan as pbf_scan_exclusive_i32 with
// its scratch (one status word per tile of the scan, a tile counter and an
// error word) in a file-scope device array instead of a caller workspace.
//
// The array is a static __device__ object: every GPU that loads this library
// holds it (about 33 KB) until the process exits. Host code cannot use the
// array's name as a device address, so the first call on each device looks the
// address up with cudaGetSymbolAddress while that device is current, and later
// calls reuse it. Every call shares the one array; its status words and counter
// are cleared at the start of each call, and calls that overlap on the GPU (on
// different streams) race on it.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/pbf.h"
#include "pbf_kernels.h"

namespace {

constexpr int kMaxTiles = 4096;                         // room for 4,096 status words
constexpr long long kMaxElements = 16777216ll;          // largest n accepted
constexpr int kScratchBytes = kMaxTiles * 8 + 16 + 64;  // status words, counter, error word

static __device__ __align__(256) unsigned char g_scan_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {nullptr};

// errors are reported through pbf_last_error()
int fail(int code, const char* msg) { return pbf::set_last_error(code, msg); }

// Device address of the scratch array on the current device (looked up once).
int scratch_ptr(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(PBF_ERR_CUDA, "no current CUDA device");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scan_scratch);
        if (e != cudaSuccess || !p) return fail(PBF_ERR_CUDA, "cudaGetSymbolAddress of the scan scratch failed");
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return PBF_OK;
}

}  // namespace

extern "C" {

int pbf_scan_exclusive_i32_noalloc(const int* d_in, int* d_out, int n, void* stream) {
    if (!d_in || !d_out) return fail(PBF_ERR_INVALID, "null argument");
    if (n <= 0) return fail(PBF_ERR_INVALID, "n must be positive");
    if ((long long)n > kMaxElements)
        return fail(PBF_ERR_INVALID, "n exceeds the allocation-free scan's maximum of 16,777,216 elements");
    void* scratch = nullptr;
    int rc = scratch_ptr(&scratch);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t status = pbf::scan_status_bytes(n);  // status words and tile counter
    if (((status + 15) & ~(size_t)15) + sizeof(int) > (size_t)kScratchBytes)
        return fail(PBF_ERR_INVALID, "n needs more scan tiles than the allocation-free scratch holds");
    int* err = (int*)((char*)scratch + ((status + 15) & ~(size_t)15));
    if (cudaMemsetAsync(err, 0, sizeof(int), st) != cudaSuccess) return fail(PBF_ERR_CUDA, "clearing the error word");
    pbf::launch_scan_const(d_in, d_out, n, scratch, err, st);  // clears the status words, then scans
    if (cudaGetLastError() != cudaSuccess) return fail(PBF_ERR_CUDA, "scan launch failed");
    int h = 0;
    if (cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(PBF_ERR_CUDA, "reading the scan status");
    if (h) return fail(PBF_ERR_DEVICE, "scan look-back wait expired");
    return PBF_OK;
}

}  // extern "C"
