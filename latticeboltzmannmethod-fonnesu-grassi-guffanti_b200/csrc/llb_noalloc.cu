// llb_flow_forces_noalloc: the lift/drag reduction without any device allocation.
//
// Who needs it: a caller whose device memory is committed up front -- a solve
// server that admits lattices under a fixed HBM budget, or a host that hands
// the whole GPU to one caching allocator -- cannot let a library call
// cudaMalloc in the middle of its loop: the allocation may fail once the
// budget is spent, and cudaMalloc/cudaFree can synchronise the whole device,
// stalling every other lattice in flight.  llb_set_force_points and
// llb_flow_forces allocate device buffers for the considered points and the
// per-block partial sums; this entry point instead keeps both in one
// file-scope device array.  CUDA loads the library's device code on a device
// lazily, so the array is reserved there at the latest by the first call's
// set-up below, not by any later call.
//
// The array is shared by every call in the process (per device) and holds
// whatever the last call left there.  Nothing in it has to start at zero:
// each call overwrites the point list it uses and every partial sum it folds.
// Two calls whose work overlaps on the GPU (different streams or handles at
// the same time) race on the array; callers must serialise them.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress (with that device current) and caches it; that lookup
// is where the device memory is taken.  Make that first call before the loop
// that must not allocate and before any stream capture begins on the device.
// A cudaDeviceReset frees the array with every other allocation of the
// context (the library's lattices included), so the cached address is only
// valid while the context that looked it up lives.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/llalbm_cuda.h"
#include "llb_internal.cuh"
#include "llb_launch.h"

namespace {

constexpr long long MAX_POINTS = LLB_NOALLOC_MAX_FORCE_POINTS;
constexpr int MAX_BLOCKS = llb::FORCE_MAX_BLOCKS;  // partial-sum slots (grid of the force kernel)
constexpr size_t PTS_BYTES = sizeof(int64_t) * 2 * MAX_POINTS;
constexpr size_t DIRS_BYTES = (sizeof(uint16_t) * MAX_POINTS + 255) / 256 * 256;
constexpr size_t PARTIAL_BYTES = sizeof(double2) * 3 * MAX_BLOCKS;
constexpr size_t SCRATCH_BYTES = PTS_BYTES + DIRS_BYTES + PARTIAL_BYTES;

// points (i, j) | direction bits | per-block partial sums
static __device__ __align__(256) unsigned char g_force_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
void* g_scratch[MAX_DEVICES] = {};

// Device address of the scratch array on the current device (looked up once).
cudaError_t scratch_address(int device, void** out) {
    if (device < 0 || device >= MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_force_scratch);
        if (e != cudaSuccess) return e;
        g_scratch[device] = p;
    }
    *out = g_scratch[device];
    return cudaSuccess;
}

}  // namespace

namespace llb {
// Hooks into the handle, defined in llb_capi.cu.
int handle_force_context(llb_handle h, LaunchCtx* ctx, const void** fin, double** d_out, int* storage,
                         int* device, int64_t* rows, int64_t* cols);
int handle_fail(llb_handle h, int code, const char* msg);
}  // namespace llb

extern "C" int llb_flow_forces_noalloc(llb_handle h, const int64_t* ij, const uint16_t* dirs, int64_t n,
                                       double lift_drag[2]) {
    using namespace llb;
    if (!h || !lift_drag || n < 0 || (n > 0 && (!ij || !dirs)))
        return handle_fail(h, LLB_E_INVALID, "bad arguments");
    if (n > MAX_POINTS)
        return handle_fail(h, LLB_E_INVALID,
                           "llb_flow_forces_noalloc: more points than LLB_NOALLOC_MAX_FORCE_POINTS (65536)");
    LaunchCtx x;
    const void* fin = nullptr;
    double* d_out = nullptr;
    int storage = 0, device = 0;
    int64_t R = 0, C = 0;
    int rc = handle_force_context(h, &x, &fin, &d_out, &storage, &device, &R, &C);
    if (rc != LLB_OK) return rc;
    for (int64_t q = 0; q < n; ++q)
        if (ij[2 * q] < 0 || ij[2 * q + 1] < 0 || ij[2 * q] >= R || ij[2 * q + 1] >= C)
            return handle_fail(h, LLB_E_INVALID, "force point out of range");
    void* base = nullptr;
    cudaError_t e = scratch_address(device, &base);
    if (e != cudaSuccess) return handle_fail(h, LLB_E_CUDA, "cudaGetSymbolAddress of the force scratch failed");
    auto* d_pts = static_cast<int64_t*>(base);
    auto* d_dirs = reinterpret_cast<uint16_t*>(static_cast<unsigned char*>(base) + PTS_BYTES);
    auto* d_partials = reinterpret_cast<double2*>(static_cast<unsigned char*>(base) + PTS_BYTES + DIRS_BYTES);
    if (n > 0) {
        e = cudaMemcpyAsync(d_pts, ij, sizeof(int64_t) * 2 * n, cudaMemcpyHostToDevice, x.stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(d_dirs, dirs, sizeof(uint16_t) * n, cudaMemcpyHostToDevice, x.stream);
        if (e != cudaSuccess) return handle_fail(h, LLB_E_CUDA, "copy of the force points failed");
    }
    // same grid rule as llb_flow_forces, so both sum in the same order
    const int nb = force_blocks(n);
    e = launch_flow_forces(storage, x, fin, d_pts, d_dirs, n, d_partials, nb, d_out);
    if (e == cudaSuccess) e = cudaMemcpyAsync(lift_drag, d_out, sizeof(double) * 2, cudaMemcpyDeviceToHost, x.stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(x.stream);
    if (e != cudaSuccess) return handle_fail(h, LLB_E_CUDA, cudaGetErrorString(e));
    return LLB_OK;
}
