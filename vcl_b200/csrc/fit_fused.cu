// Fused fit iteration (placeholder until the fused kernels land).
#include "fit.cuh"

vcl_status fit_step_fused(vcl_fit* f, cudaStream_t) {
    return vcl_fail(f->ctx, VCL_ERR_STATE, "fused strategy not built");
}
int fit_fused_launches(const vcl_fit*) { return 0; }
void fit_fused_release(vcl_fit*) {}
