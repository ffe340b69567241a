// FP64 adjoint kernels, built without FMA contraction like the forward step: the fused reverse
// step replays the forward step and must reproduce it bit for bit.
#include "adjoint_kernels.cuh"

namespace da {
int launch_adjoint_step_fp64(da_ctx *ctx, int a, int b, const double *sec2, double c) {
    return adj::step_t<double>(ctx, a, b, sec2, c);
}
int launch_adjoint_seed_fp64(da_ctx *ctx, int b, const double box[4]) { return adj::seed_t<double>(ctx, b, box); }
int launch_adjoint_reduce_fp64(da_ctx *ctx, int a, int np) { return adj::reduce_t<double>(ctx, a, np); }
int launch_youturn_fp64(da_ctx *ctx, int a, int b, const double *sec2, double c) {
    return adj::youturn_t<double>(ctx, a, b, sec2, c);
}
}  // namespace da
