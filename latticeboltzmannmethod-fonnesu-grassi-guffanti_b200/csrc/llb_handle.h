// The lattice handle (struct llb_lattice) shared by the C-ABI translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/llalbm_cuda.h"
#include "llb_launch.h"

using llb::Collision;
using llb::TmaPlan;

struct llb_lattice {
    // one lattice on one device: stream, node mask, resident populations
    // (ping-pong), boundary-value ring, outputs, graphs and pipeline state
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = true;  // false when the stream belongs to a batch
    int storage = LLB_STORE_F64, pattern = LLB_PATTERN_AB;
    int64_t R = 0, C = 0;
    int ld = 0;
    long long plane = 0;
    size_t elem = 8;
    void* f[2] = {nullptr, nullptr};
    int cur = 0;
    uint8_t* d_mask = nullptr;
    int32_t* d_open_idx = nullptr;
    double2* d_open = nullptr;
    int n_open = 0, cap = 1;
    double* d_rho = nullptr;
    double* d_u = nullptr;
    double* d_dense = nullptr;
    long long* d_step = nullptr;  // step index at the start of a graph replay
    unsigned* d_flags = nullptr;
    int block_y = 4;
    double2* d_partials = nullptr;
    int partial_blocks = 0;
    double* d_red = nullptr;
    int64_t* d_fpts = nullptr;
    uint16_t* d_fdirs = nullptr;
    int64_t n_fpts = 0;
    double* d_gather = nullptr;
    Collision coll{};
    int64_t step = 0;
    bool initialized = false;
    bool macro_valid = false;
    cudaEvent_t ev[8] = {};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int64_t bytes = 0;
    std::string err;
    // TMA-pipelined step kernel (plain steps); tma_cfg < 0 selects the
    // one-thread-per-node kernel.
    int tma_cfg = 0;
    TmaPlan plan;
    bool maps_ready = false;
    CUtensorMap pmap[2];  // populations f[0], f[1]
    CUtensorMap mmap;     // node mask
    int sm_count = 148;
};

namespace llb {
// Launch context of a handle's current state (defined in llb_capi.cu).
LaunchCtx handle_ctx(llb_handle h);
// Error reporting on a handle.
int handle_fail(llb_handle h, int code, const char* msg);
}  // namespace llb
