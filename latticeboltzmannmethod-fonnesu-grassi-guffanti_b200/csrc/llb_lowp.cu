// Shifted low-precision kernels (populations stored as f - w in FP32 or FP16,
// arithmetic in FP32).  Multiply-add contraction is allowed here.
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

}  // namespace llb
