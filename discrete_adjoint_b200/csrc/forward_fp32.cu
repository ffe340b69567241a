// FP32-split path of the forward step: state, fluxes and sources in FP32 (FMA allowed);
// the dt min-reduction, dt arithmetic and the volume sum stay in FP64.
#include "forward_impl.cuh"

namespace da {

int launch_forward_step_fp32(da_ctx *ctx, uint8_t *record_mask) {
    return fwd::launch_step_t<float>(ctx, record_mask);
}
int launch_forward_steps_fp32(da_ctx *ctx, int nsteps, void *pre, void *post, const MidStoreList *mid) {
    return fwd::launch_steps_t<float>(ctx, nsteps, pre, post, mid);
}
int launch_step_half_fp32(da_ctx *ctx, int half, double *bounds) {
    return fwd::launch_step_half_t<float>(ctx, half, bounds);
}
int launch_refine_info_fp32(da_ctx *ctx, double *e, uint8_t *f, double *parts, double *t) {
    return fwd::refine_info_t<float>(ctx, e, f, parts, t);
}

}  // namespace da
