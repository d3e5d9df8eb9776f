// Host-side launch interface between the C ABI (llb_capi.cu) and the
// per-storage kernel translation units (llb_f64.cu, llb_lowp.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "llb_internal.cuh"

namespace llb {

struct LaunchCtx {
    Geometry g;
    OpenTable ot;
    Collision c;
    MacroOut mo;
    StepSync ss;
    cudaStream_t stream;
    int block_y;        // columns per block of the step kernel (1..8)
};

// Storage-specific entry points; `storage` is LLB_STORE_* and selects the
// translation unit.  All launches go to ctx.stream and return the launch error.
cudaError_t launch_step(int storage, const LaunchCtx& ctx, const void* fin, void* fout, bool init, bool macro);
cudaError_t launch_finalize(int storage, const LaunchCtx& ctx, const void* fin, double* out, long long t);
cudaError_t launch_export(int storage, const LaunchCtx& ctx, const void* fin, double* out);
cudaError_t launch_mass_momentum(int storage, const LaunchCtx& ctx, const void* fin, double2* partials,
                                 int nblocks, double* out3);
cudaError_t launch_flow_forces(int storage, const LaunchCtx& ctx, const void* fin, const int64_t* pts,
                               const uint16_t* dirs, long long n, double2* partials, int nblocks, double* out2);
cudaError_t launch_gather_forces(int storage, const LaunchCtx& ctx, const void* fin, const int64_t* pts,
                                 const uint16_t* dirs, long long n, double* out);

cudaError_t launch_fill_keep(int storage, const LaunchCtx& ctx, void* buf);

// Column-compacted storage (llb_compact.cuh): one plain step between compacted
// planes, and copies between the dense and the compacted planes.
cudaError_t launch_step_compact(int storage, const LaunchCtx& ctx, const CompactGeo& cg, const void* fin, void* fout);
cudaError_t launch_compact_copy(int storage, const LaunchCtx& ctx, const CompactGeo& cg, void* dense, void* comp,
                                bool to_compact);
cudaError_t launch_step_compact_f64(const LaunchCtx&, const CompactGeo&, const void*, void*);
cudaError_t launch_compact_copy_f64(const LaunchCtx&, const CompactGeo&, void*, void*, bool);
cudaError_t launch_step_compact_lowp(int storage, const LaunchCtx&, const CompactGeo&, const void*, void*);
cudaError_t launch_compact_copy_lowp(int storage, const LaunchCtx&, const CompactGeo&, void*, void*, bool);

// Small lattices resident in one thread-block cluster (llb_cluster.cuh):
// `steps` plain steps from step index t0 in one launch, state f[cur]
// ping-ponging between f0 and f1.  The host splits longer runs into chunks of
// CLUSTER_CHUNK steps.
struct ClusterPlan {
    int nc = 0;          // blocks of the cluster
    int wmax = 0;        // columns of the widest slab
    long long smem = 0;  // dynamic shared memory per block
};
constexpr int CLUSTER_CHUNK = 4096;
bool cluster_plan(int storage, int R, int C, int device, ClusterPlan* plan);
cudaError_t launch_step_cluster(int storage, const LaunchCtx& ctx, const ClusterPlan& plan, void* f0, void* f1,
                                int cur, long long t0, int steps);
bool cluster_plan_f64(int R, int C, int device, ClusterPlan* plan);
bool cluster_plan_lowp(int storage, int R, int C, int device, ClusterPlan* plan);
cudaError_t launch_step_cluster_f64(const LaunchCtx&, const ClusterPlan&, void*, void*, int, long long, int);
cudaError_t launch_step_cluster_lowp(int storage, const LaunchCtx&, const ClusterPlan&, void*, void*, int, long long,
                                     int);

struct BatchLattice;
// Batched step over a work list (llb_batch.cuh).  `cooperative` launches the
// grid cooperatively (required when steps > 1).
struct BatchLaunch {
    const BatchLattice* lats;
    const int2* items;     // dense tiles first, then compacted slot blocks
    int n_items;
    int n_dense;          // items[0, n_dense) are dense tiles
    const long long* sbase;
    long long soff;
    int steps;
    unsigned* bar;
    unsigned* err;
    long long bar_limit;   // polls of the grid barrier before a block gives up
    int grid;
    int block_y;
    bool cooperative;
    cudaStream_t stream;
};
cudaError_t launch_batch_step(int storage, const BatchLaunch& b);
// Largest co-resident grid of the batched kernel for a block of 32 x block_y.
int batch_max_grid(int storage, int block_y, int sm_count);
cudaError_t launch_macro_now(int storage, const LaunchCtx& ctx, const void* fin, long long t, double* rho, double* u);

// per translation unit
cudaError_t launch_batch_step_f64(const BatchLaunch&);
cudaError_t launch_batch_step_lowp(int storage, const BatchLaunch&);
int batch_max_grid_f64(int block_y, int sm_count);
int batch_max_grid_lowp(int storage, int block_y, int sm_count);
cudaError_t launch_macro_now_f64(const LaunchCtx&, const void*, long long, double*, double*);
cudaError_t launch_macro_now_lowp(int storage, const LaunchCtx&, const void*, long long, double*, double*);
cudaError_t launch_fill_keep_f64(const LaunchCtx&, void*);
cudaError_t launch_fill_keep_lowp(int storage, const LaunchCtx&, void*);
cudaError_t launch_step_f64(const LaunchCtx&, const void*, void*, bool, bool);
cudaError_t launch_finalize_f64(const LaunchCtx&, const void*, double*, long long);
cudaError_t launch_export_f64(const LaunchCtx&, const void*, double*);
cudaError_t launch_mass_momentum_f64(const LaunchCtx&, const void*, double2*, int, double*);
cudaError_t launch_flow_forces_f64(const LaunchCtx&, const void*, const int64_t*, const uint16_t*, long long,
                                   double2*, int, double*);
cudaError_t launch_gather_forces_f64(const LaunchCtx&, const void*, const int64_t*, const uint16_t*, long long,
                                     double*);
cudaError_t launch_step_lowp(int storage, const LaunchCtx&, const void*, void*, bool, bool);
cudaError_t launch_finalize_lowp(int storage, const LaunchCtx&, const void*, double*, long long);
cudaError_t launch_export_lowp(int storage, const LaunchCtx&, const void*, double*);
cudaError_t launch_mass_momentum_lowp(int storage, const LaunchCtx&, const void*, double2*, int, double*);
cudaError_t launch_flow_forces_lowp(int storage, const LaunchCtx&, const void*, const int64_t*, const uint16_t*,
                                    long long, double2*, int, double*);
cudaError_t launch_gather_forces_lowp(int storage, const LaunchCtx&, const void*, const int64_t*,
                                      const uint16_t*, long long, double*);

// One configuration of the TMA-pipelined step kernel (tile TI x TJ nodes,
// S shared-memory stages, W consumer warps + 1 producer warp).
struct TmaPlan {
    int cfg = -1;
    bool pair = false;     // two steps per launch (k_step_pair)
    int ctas_per_sm = 1;   // persistent grid = ctas_per_sm x SM count
    bool bbx = false;      // the producer also loads a TI x TJ box of bounce bytes
    int TI = 0, TJ = 0, S = 0, W = 0;
    int BI = 0;            // rows of a population box
    int BJ = 0;            // columns of a population box
    int BIM = 0, BJM = 0;  // rows / columns of the mask box
    int smem = 0;          // dynamic shared memory bytes
    int threads = 0;
};
// Configurations 0..2 and 6: one step per launch (k_step_tma; 6 also loads the
// tile's bounce bytes); 3..5: two steps per launch (k_step_pair).
constexpr int TMA_CONFIGS = 7;
constexpr int FIRST_PAIR_CONFIG = 3;
// Fills `out` for configuration `cfg` (0..TMA_CONFIGS-1) of a storage form.
bool tma_plan(int storage, int cfg, TmaPlan* out);
cudaError_t launch_step_tma(int storage, const TmaPlan& p, const LaunchCtx& ctx, const CUtensorMap* pmap,
                            const CUtensorMap* mmap, const CUtensorMap* bmap, const void* fin, void* fout, int grid);
bool tma_plan_f64(int cfg, TmaPlan* out);
cudaError_t launch_step_tma_f64(const TmaPlan&, const LaunchCtx&, const CUtensorMap*, const CUtensorMap*,
                                const CUtensorMap*, const void*, void*, int);
bool tma_plan_lowp(int storage, int cfg, TmaPlan* out);
cudaError_t launch_step_tma_lowp(int storage, const TmaPlan&, const LaunchCtx&, const CUtensorMap*,
                                 const CUtensorMap*, const CUtensorMap*, const void*, void*, int);

// Blocks of the lift/drag reduction, at most: llb_flow_forces and
// llb_flow_forces_noalloc size their grids by the same rule, so both fold the
// per-block partial sums in the same order.
constexpr int FORCE_MAX_BLOCKS = 148 * 4;
inline int force_blocks(long long n) {
    return static_cast<int>(n > 0 ? ((n + 255) / 256 < FORCE_MAX_BLOCKS ? (n + 255) / 256 : FORCE_MAX_BLOCKS) : 1);
}

inline dim3 node_grid(const Geometry& g, int bx, int by) {
    return dim3(static_cast<unsigned>((g.rows + bx - 1) / bx), static_cast<unsigned>((g.cols + by - 1) / by));
}

}  // namespace llb
