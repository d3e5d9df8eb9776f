// The lattice handle (struct llb_lattice) shared by the C-ABI translation units.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

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
    uint8_t* d_bb = nullptr;
    uint8_t* d_ps = nullptr;   // partially saturated obstacles only
    double* d_psb = nullptr;
    int32_t* d_sectors = nullptr;  // active-sector list (lattices of fewer than 2^31 slots per plane)
    uint8_t* d_smask = nullptr;    // mask and bounce bytes of the listed nodes
    uint8_t* d_sbb = nullptr;
    int n_sectors = 0;
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
    // split numerics checks: pinned host copies of the flag word and the
    // events that mark their arrival, one per slot (allocated on first use)
    unsigned* h_flags = nullptr;
    cudaEvent_t flag_ev[8] = {};
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int64_t bytes = 0;
    std::string err;
    // plain-step kernel: tma_cfg >= 0 the TMA pipeline configuration,
    // PIPE_GRID the one-thread-per-node grid, PIPE_LIST the active-sector list,
    // PIPE_COMPACT the compacted planes, PIPE_CLUSTER one cluster
    int tma_cfg = 0;
    TmaPlan plan;
    bool maps_ready = false;
    CUtensorMap pmap[2];  // populations f[0], f[1]
    CUtensorMap mmap;     // node mask
    CUtensorMap bmap;     // bounce bytes (configurations that load them)
    int sm_count = 148;
    // active nodes with a wall, obstacle, dead or outside source (not PLAIN)
    int64_t n_active = 0, n_nonplain = 0;
    // column-compacted planes of the active nodes (pipeline PIPE_COMPACT,
    // built on first use) and their addressing tables
    void* cf[2] = {nullptr, nullptr};
    uint32_t* d_cnb = nullptr;
    int2* d_cseg = nullptr;
    int2* d_cchunk = nullptr;
    int32_t* d_ccol = nullptr;
    uint16_t* d_cinfo = nullptr;
    int cnseg = 0, c_chunks = 0;
    long long cplane = 0, c_slots = 0;
    int64_t compact_bytes = 0;
    // where the resident state f*[cur] lives: RES_DENSE, RES_COMPACT or both
    int where = 0;
    // polls of the pipelined kernels' stage waits before they give up
    long long wait_limit = llb::DEFAULT_WAIT_LIMIT;
    // per (32-row segment ti, column j), plain_seg[j * ceil(R / 32) + ti]: 1
    // when all 32 rows of the segment exist and are PLAIN fluid nodes (built
    // with the mask; a batch flags its all-PLAIN dense tiles from it)
    std::vector<uint8_t> plain_seg;
    // the lattice resident in one thread-block cluster (pipeline
    // PIPE_CLUSTER): its plan, looked up once (cl_state 0 not yet, 1 it
    // fits, -1 it does not)
    llb::ClusterPlan cl_plan;
    int cl_state = 0;
};

// Residence of the state (llb_lattice::where).  Steps of the compacted
// pipeline leave it in the compacted planes; every other kernel reads and
// writes the dense planes, and a copy brings the state across when needed.
constexpr int RES_DENSE = 0, RES_COMPACT = 1, RES_BOTH = 2;

// Default plain-step kernel of a lattice, from measurements on B200 (cavities,
// channels, cylinders and porous media from 256^2 to 4096^2, every storage
// form):
//  * at least 5 % of the active nodes not PLAIN (porous media) and at least
//    2^18 nodes: the compacted planes (only active nodes stored and read; on
//    porous 4096^2 FP64 63.1k MLUPS against 46.8k for the best dense kernel,
//    which also pulls the obstacle interiors through DRAM);
//  * otherwise the dense kernels: below 2^19 nodes one thread per node; open
//    flow whose resident state (two buffers of 9 planes) exceeds the L2 cache
//    several times over: two steps per pass for FP64 and FP32 (configuration
//    3, from 2^28 bytes), the TMA pipeline for FP16 (from 2^27 bytes); else
//    one thread per node, which runs close to the copy bandwidth on open flow
//    (there every node is active and the compacted planes only add their
//    6 bytes of addressing per node);
//  * lattices resident in one 16-block cluster (their slabs fit its shared
//    memory) up to 12 000 nodes (FP64, FP32) or 26 000 (FP16): the cluster
//    runs a chunk of steps per launch (chosen at creation, where the device
//    is known).  96^2 steps in 2.2 us against 3.0 us on the one-thread grid;
//    at config 1 (129^2) the 16 SMs of one cluster are bound by the FP64
//    arithmetic of 16 641 nodes (3.6 us against 3.1 us), so the grid keeps it.
constexpr int PIPE_GRID = -1, PIPE_LIST = -2, PIPE_COMPACT = -3, PIPE_CLUSTER = -4;
inline bool cluster_default_size(const llb_lattice& h) {
    return h.R * h.C <= (h.storage == LLB_STORE_F16S ? 26000 : 12000);
}
constexpr int64_t TMA_MIN_NODES = 1 << 19;
constexpr double TMA_MIN_NONPLAIN = 0.05;
constexpr int64_t COMPACT_MIN_NODES = 1 << 18;
inline bool obstacle_rich(const llb_lattice& h) {
    return h.n_active > 0 &&
           static_cast<double>(h.n_nonplain) >= TMA_MIN_NONPLAIN * static_cast<double>(h.n_active);
}
// The best dense kernel (also the choice for lattices without compacted planes).
inline int default_dense_pipeline(const llb_lattice& h) {
    const int64_t n = h.R * h.C;
    if (n < TMA_MIN_NODES || h.n_active == 0) return PIPE_GRID;
    if (static_cast<double>(h.n_nonplain) >= TMA_MIN_NONPLAIN * static_cast<double>(h.n_active))
        return h.storage == LLB_STORE_F64 ? (n >= (int64_t{1} << 21) ? 1 : 0) : 6;
    const double state = 2.0 * 9.0 * static_cast<double>(h.elem) * static_cast<double>(n);
    if (h.storage == LLB_STORE_F16S) return state >= static_cast<double>(int64_t{1} << 27) ? 0 : PIPE_GRID;
    return state >= static_cast<double>(int64_t{1} << 28) ? llb::FIRST_PAIR_CONFIG : PIPE_GRID;
}
inline int default_pipeline(const llb_lattice& h) {
    if (obstacle_rich(h) && h.R * h.C >= COMPACT_MIN_NODES) return PIPE_COMPACT;
    return default_dense_pipeline(h);
}

namespace llb {
// Launch context of a handle's current state (defined in llb_capi.cu).
LaunchCtx handle_ctx(llb_handle h);
// Error reporting on a handle.
int handle_fail(llb_handle h, int code, const char* msg);
// Brings the state of a handle into its dense planes (a copy when the last
// steps ran on the compacted ones); LLB_OK or an error code.
int handle_dense_state(llb_handle h);
// Before a batch takes a handle: its state in the dense planes, and a handle
// on the compacted pipeline moves to the one-thread-per-node kernel.
int handle_leave_compact(llb_handle h);
// The compacted planes and tables of a handle (built once; host work and a
// synchronisation of the handle's stream).  LLB_OK, or an error when the
// lattice has none (partially saturated obstacles, too large).
int handle_prepare_compact(llb_handle h);
// The state of a handle moved into the layout a batch steps (a copy kernel on
// the handle's stream when needed).
int handle_batch_layout(llb_handle h, bool compact);
// A batch has stepped the handle's lattice in that layout.
void handle_batch_stepped(llb_handle h, bool compact);
// Addressing tables of the handle's compacted planes (after handle_prepare_compact).
CompactGeo handle_compact_geo(llb_handle h);
}  // namespace llb
