// FP64 kernels.  This translation unit is compiled with --fmad=false so that no
// multiply and add are fused: the arithmetic then rounds exactly like the
// reference's default x86-64 build, and results match it bit for bit.
#include "llb_kernel_inst.cuh"

namespace llb {

cudaError_t launch_step_f64(const LaunchCtx& x, const void* fin, void* fout, bool init, bool macro) {
    return do_step<ModelF64>(x, fin, fout, init, macro);
}
cudaError_t launch_fill_keep_f64(const LaunchCtx& x, void* buf) { return do_fill_keep<ModelF64>(x, buf); }
cudaError_t launch_step_compact_f64(const LaunchCtx& x, const CompactGeo& cg, const void* fin, void* fout) {
    return do_step_compact<ModelF64>(x, cg, fin, fout);
}
bool cluster_plan_f64(int R, int C, int device, ClusterPlan* plan) { return do_cluster_plan<ModelF64>(R, C, device, plan); }
cudaError_t launch_step_cluster_f64(const LaunchCtx& x, const ClusterPlan& p, void* f0, void* f1, int cur, long long t0,
                                    int steps) {
    return do_step_cluster<ModelF64>(x, p, f0, f1, cur, t0, steps);
}
cudaError_t launch_compact_copy_f64(const LaunchCtx& x, const CompactGeo& cg, void* dense, void* comp, bool to_compact) {
    return do_compact_copy<ModelF64>(x, cg, dense, comp, to_compact);
}
cudaError_t launch_finalize_f64(const LaunchCtx& x, const void* fin, double* out, long long t) {
    return do_finalize<ModelF64>(x, fin, out, t);
}
cudaError_t launch_export_f64(const LaunchCtx& x, const void* fin, double* out) { return do_export<ModelF64>(x, fin, out); }
cudaError_t launch_mass_momentum_f64(const LaunchCtx& x, const void* fin, double2* p, int nb, double* out3) {
    return do_mass<ModelF64>(x, fin, p, nb, out3);
}
cudaError_t launch_flow_forces_f64(const LaunchCtx& x, const void* fin, const int64_t* pts, const uint16_t* dirs,
                                   long long n, double2* p, int nb, double* out2) {
    return do_forces<ModelF64>(x, fin, pts, dirs, n, p, nb, out2);
}
cudaError_t launch_gather_forces_f64(const LaunchCtx& x, const void* fin, const int64_t* pts, const uint16_t* dirs,
                                     long long n, double* out) {
    return do_gather<ModelF64>(x, fin, pts, dirs, n, out);
}

// TMA pipeline configurations of the FP64 step (tile rows, tile columns, stages, consumer warps)
using F64Cfg0 = TmaCfg<double, 128, 4, 4, 16>;
using F64Cfg1 = TmaCfg<double, 128, 8, 2, 16>;
using F64Cfg2 = TmaCfg<double, 128, 4, 4, 20>;
// two steps per launch (tile rows, tile columns, stages, consumer warps)
using F64Pair3 = PairCfg<double, 32, 16, 2, 16>;
using F64Pair4 = PairCfg<double, 32, 16, 3, 16>;
using F64Pair5 = PairCfg<double, 32, 16, 1, 8, 2>;
// configuration 1 with the tile's bounce bytes
using F64Cfg6 = TmaCfg<double, 128, 8, 2, 16, true>;

bool tma_plan_f64(int cfg, TmaPlan* p) {
    switch (cfg) {
    case 0: fill_plan<ModelF64, F64Cfg0>(0, p); return true;
    case 1: fill_plan<ModelF64, F64Cfg1>(1, p); return true;
    case 2: fill_plan<ModelF64, F64Cfg2>(2, p); return true;
    case 3: fill_plan<ModelF64, F64Pair3>(3, p); return true;
    case 4: fill_plan<ModelF64, F64Pair4>(4, p); return true;
    case 5: fill_plan<ModelF64, F64Pair5>(5, p); return true;
    case 6: fill_plan<ModelF64, F64Cfg6>(6, p); return true;
    default: return false;
    }
}

cudaError_t launch_step_tma_f64(const TmaPlan& p, const LaunchCtx& x, const CUtensorMap* pm, const CUtensorMap* mm,
                                const CUtensorMap* bm, const void* fin, void* fout, int grid) {
    switch (p.cfg) {
    case 0: return do_step_tma<ModelF64, F64Cfg0>(x, pm, mm, bm, fin, fout, grid);
    case 1: return do_step_tma<ModelF64, F64Cfg1>(x, pm, mm, bm, fin, fout, grid);
    case 2: return do_step_tma<ModelF64, F64Cfg2>(x, pm, mm, bm, fin, fout, grid);
    case 3: return do_step_pair<ModelF64, F64Pair3>(x, pm, mm, bm, fin, fout, grid);
    case 4: return do_step_pair<ModelF64, F64Pair4>(x, pm, mm, bm, fin, fout, grid);
    case 5: return do_step_pair<ModelF64, F64Pair5>(x, pm, mm, bm, fin, fout, grid);
    case 6: return do_step_tma<ModelF64, F64Cfg6>(x, pm, mm, bm, fin, fout, grid);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_batch_step_f64(const BatchLaunch& b) { return do_batch_step<ModelF64>(b); }
int batch_max_grid_f64(int block_y, int sm_count) { return do_batch_max_grid<ModelF64>(block_y, sm_count); }
cudaError_t launch_macro_now_f64(const LaunchCtx& x, const void* fin, long long t, double* rho, double* u) {
    return do_macro_now<ModelF64>(x, fin, t, rho, u);
}

}  // namespace llb
