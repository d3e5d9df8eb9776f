// Shifted low-precision kernels (populations stored as f - w in FP32 or FP16,
// arithmetic in FP32).  Compiled with --fmad=false: the model writes its
// multiply-adds out, so every kernel of a form gives the same bits.
#include "llb_kernel_inst.cuh"

#include "../../include/llalbm_cuda.h"

namespace llb {

using ModelF32S = ModelShift<float>;
using ModelF16S = ModelShift<__half>;

#define LLB_DISPATCH(call_f32, call_f16) \
    return storage == LLB_STORE_F32S ? (call_f32) : (call_f16)

cudaError_t launch_step_lowp(int storage, const LaunchCtx& x, const void* fin, void* fout, bool init, bool macro) {
    LLB_DISPATCH((do_step<ModelF32S>(x, fin, fout, init, macro)), (do_step<ModelF16S>(x, fin, fout, init, macro)));
}
cudaError_t launch_fill_keep_lowp(int storage, const LaunchCtx& x, void* buf) {
    LLB_DISPATCH((do_fill_keep<ModelF32S>(x, buf)), (do_fill_keep<ModelF16S>(x, buf)));
}
cudaError_t launch_step_compact_lowp(int storage, const LaunchCtx& x, const CompactGeo& cg, const void* fin, void* fout) {
    LLB_DISPATCH((do_step_compact<ModelF32S>(x, cg, fin, fout)), (do_step_compact<ModelF16S>(x, cg, fin, fout)));
}
bool cluster_plan_lowp(int storage, int R, int C, int device, ClusterPlan* plan) {
    LLB_DISPATCH((do_cluster_plan<ModelF32S>(R, C, device, plan)), (do_cluster_plan<ModelF16S>(R, C, device, plan)));
}
cudaError_t launch_step_cluster_lowp(int storage, const LaunchCtx& x, const ClusterPlan& p, void* f0, void* f1, int cur,
                                     long long t0, int steps) {
    LLB_DISPATCH((do_step_cluster<ModelF32S>(x, p, f0, f1, cur, t0, steps)),
                 (do_step_cluster<ModelF16S>(x, p, f0, f1, cur, t0, steps)));
}
cudaError_t launch_compact_copy_lowp(int storage, const LaunchCtx& x, const CompactGeo& cg, void* dense, void* comp,
                                     bool to_compact) {
    LLB_DISPATCH((do_compact_copy<ModelF32S>(x, cg, dense, comp, to_compact)),
                 (do_compact_copy<ModelF16S>(x, cg, dense, comp, to_compact)));
}
cudaError_t launch_finalize_lowp(int storage, const LaunchCtx& x, const void* fin, double* out, long long t) {
    LLB_DISPATCH((do_finalize<ModelF32S>(x, fin, out, t)), (do_finalize<ModelF16S>(x, fin, out, t)));
}
cudaError_t launch_export_lowp(int storage, const LaunchCtx& x, const void* fin, double* out) {
    LLB_DISPATCH((do_export<ModelF32S>(x, fin, out)), (do_export<ModelF16S>(x, fin, out)));
}
cudaError_t launch_mass_momentum_lowp(int storage, const LaunchCtx& x, const void* fin, double2* p, int nb,
                                      double* out3) {
    LLB_DISPATCH((do_mass<ModelF32S>(x, fin, p, nb, out3)), (do_mass<ModelF16S>(x, fin, p, nb, out3)));
}
cudaError_t launch_flow_forces_lowp(int storage, const LaunchCtx& x, const void* fin, const int64_t* pts,
                                    const uint16_t* dirs, long long n, double2* p, int nb, double* out2) {
    LLB_DISPATCH((do_forces<ModelF32S>(x, fin, pts, dirs, n, p, nb, out2)),
                 (do_forces<ModelF16S>(x, fin, pts, dirs, n, p, nb, out2)));
}
cudaError_t launch_gather_forces_lowp(int storage, const LaunchCtx& x, const void* fin, const int64_t* pts,
                                      const uint16_t* dirs, long long n, double* out) {
    LLB_DISPATCH((do_gather<ModelF32S>(x, fin, pts, dirs, n, out)), (do_gather<ModelF16S>(x, fin, pts, dirs, n, out)));
}

// TMA pipeline configurations (tile rows, tile columns, stages, consumer warps)
using F32Cfg0 = TmaCfg<float, 128, 8, 3, 16>;
using F32Cfg1 = TmaCfg<float, 128, 16, 2, 16>;
using F32Cfg2 = TmaCfg<float, 128, 8, 4, 24>;
using F16Cfg0 = TmaCfg<__half, 128, 24, 3, 24>;
using F16Cfg1 = TmaCfg<__half, 128, 16, 3, 16>;
using F16Cfg2 = TmaCfg<__half, 128, 32, 2, 16>;
// two steps per launch
using F32Pair3 = PairCfg<float, 32, 32, 2, 16>;
using F32Pair4 = PairCfg<float, 32, 32, 3, 16>;
using F32Pair5 = PairCfg<float, 32, 32, 1, 8, 2>;
using F16Pair3 = PairCfg<__half, 32, 64, 2, 16>;
using F16Pair4 = PairCfg<__half, 64, 32, 2, 16>;
using F16Pair5 = PairCfg<__half, 32, 64, 1, 8, 2>;
// configuration 0 with the tile's bounce bytes
using F32Cfg6 = TmaCfg<float, 128, 8, 3, 16, true>;
using F16Cfg6 = TmaCfg<__half, 128, 24, 3, 24, true>;

bool tma_plan_lowp(int storage, int cfg, TmaPlan* p) {
    if (storage == LLB_STORE_F32S) {
        switch (cfg) {
        case 0: fill_plan<ModelF32S, F32Cfg0>(0, p); return true;
        case 1: fill_plan<ModelF32S, F32Cfg1>(1, p); return true;
        case 2: fill_plan<ModelF32S, F32Cfg2>(2, p); return true;
        case 3: fill_plan<ModelF32S, F32Pair3>(3, p); return true;
        case 4: fill_plan<ModelF32S, F32Pair4>(4, p); return true;
        case 5: fill_plan<ModelF32S, F32Pair5>(5, p); return true;
        case 6: fill_plan<ModelF32S, F32Cfg6>(6, p); return true;
        default: return false;
        }
    }
    switch (cfg) {
    case 0: fill_plan<ModelF16S, F16Cfg0>(0, p); return true;
    case 1: fill_plan<ModelF16S, F16Cfg1>(1, p); return true;
    case 2: fill_plan<ModelF16S, F16Cfg2>(2, p); return true;
    case 3: fill_plan<ModelF16S, F16Pair3>(3, p); return true;
    case 4: fill_plan<ModelF16S, F16Pair4>(4, p); return true;
    case 5: fill_plan<ModelF16S, F16Pair5>(5, p); return true;
    case 6: fill_plan<ModelF16S, F16Cfg6>(6, p); return true;
    default: return false;
    }
}

cudaError_t launch_step_tma_lowp(int storage, const TmaPlan& p, const LaunchCtx& x, const CUtensorMap* pm,
                                 const CUtensorMap* mm, const CUtensorMap* bm, const void* fin, void* fout,
                                 int grid) {
    if (storage == LLB_STORE_F32S) {
        switch (p.cfg) {
        case 0: return do_step_tma<ModelF32S, F32Cfg0>(x, pm, mm, bm, fin, fout, grid);
        case 1: return do_step_tma<ModelF32S, F32Cfg1>(x, pm, mm, bm, fin, fout, grid);
        case 2: return do_step_tma<ModelF32S, F32Cfg2>(x, pm, mm, bm, fin, fout, grid);
        case 3: return do_step_pair<ModelF32S, F32Pair3>(x, pm, mm, bm, fin, fout, grid);
        case 4: return do_step_pair<ModelF32S, F32Pair4>(x, pm, mm, bm, fin, fout, grid);
        case 5: return do_step_pair<ModelF32S, F32Pair5>(x, pm, mm, bm, fin, fout, grid);
        case 6: return do_step_tma<ModelF32S, F32Cfg6>(x, pm, mm, bm, fin, fout, grid);
        default: return cudaErrorInvalidValue;
        }
    }
    switch (p.cfg) {
    case 0: return do_step_tma<ModelF16S, F16Cfg0>(x, pm, mm, bm, fin, fout, grid);
    case 1: return do_step_tma<ModelF16S, F16Cfg1>(x, pm, mm, bm, fin, fout, grid);
    case 2: return do_step_tma<ModelF16S, F16Cfg2>(x, pm, mm, bm, fin, fout, grid);
    case 3: return do_step_pair<ModelF16S, F16Pair3>(x, pm, mm, bm, fin, fout, grid);
    case 4: return do_step_pair<ModelF16S, F16Pair4>(x, pm, mm, bm, fin, fout, grid);
    case 5: return do_step_pair<ModelF16S, F16Pair5>(x, pm, mm, bm, fin, fout, grid);
    case 6: return do_step_tma<ModelF16S, F16Cfg6>(x, pm, mm, bm, fin, fout, grid);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batch_step_lowp(int storage, const BatchLaunch& b) {
    LLB_DISPATCH((do_batch_step<ModelF32S>(b)), (do_batch_step<ModelF16S>(b)));
}
int batch_max_grid_lowp(int storage, int block_y, int sm_count) {
    LLB_DISPATCH((do_batch_max_grid<ModelF32S>(block_y, sm_count)), (do_batch_max_grid<ModelF16S>(block_y, sm_count)));
}
cudaError_t launch_macro_now_lowp(int storage, const LaunchCtx& x, const void* fin, long long t, double* rho,
                                  double* u) {
    LLB_DISPATCH((do_macro_now<ModelF32S>(x, fin, t, rho, u)), (do_macro_now<ModelF16S>(x, fin, t, rho, u)));
}

}  // namespace llb
