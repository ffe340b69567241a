// FP64 adjoint kernels, built without FMA contraction like the forward step: the fused reverse
// step replays the forward step and must reproduce it bit for bit.
#include "adjoint_kernels.cuh"

namespace da {
int launch_adjoint_step_fp64(da_ctx *ctx, int a, int b, const double *sec2, double c) {
    return adj::step_t<double>(ctx, a, b, sec2, c);
}
int launch_adjoint_reduce_fp64(da_ctx *ctx, int a, int np) { return adj::reduce_t<double>(ctx, a, np); }
int launch_youturn_fp64(da_ctx *ctx, int a, int b, const double *sec2, double c, bool seed, const double *box,
                        void *pre) {
    return adj::youturn_t<double>(ctx, a, b, sec2, c, seed, box, pre);
}
int launch_functional_fp64(da_ctx *ctx, double *out) { return adj::functional_t<double>(ctx, out); }
// the volume of every ensemble member from the segments' volume parts (fixed order)
int launch_member_volume(da_ctx *ctx, double *out) {
    adj::k_inst_sum<<<ctx->ninst, adj::kBlock, 0, ctx->stream>>>(ctx->seg_vol, ctx->ia.seg0, ctx->nseg, out);
    return cuda_check(ctx, cudaGetLastError(), "member volume launch");
}
int launch_adjoint_reduce_inst_fp64(da_ctx *ctx, int a) { return adj::reduce_inst_t<double>(ctx, a); }
}  // namespace da
