// FP32-split adjoint kernels: FP32 state and adjoint fields, FP64 sums and parameter sensitivities.
#include "adjoint_kernels.cuh"

namespace da {
int launch_adjoint_step_fp32(da_ctx *ctx, int a, int b, const double *sec2, double c) {
    return adj::step_t<float>(ctx, a, b, sec2, c);
}
int launch_adjoint_seed_fp32(da_ctx *ctx, int b, const double box[4]) { return adj::seed_t<float>(ctx, b, box); }
int launch_adjoint_reduce_fp32(da_ctx *ctx, int a, int np) { return adj::reduce_t<float>(ctx, a, np); }
int launch_youturn_fp32(da_ctx *ctx, int a, int b, const double *sec2, double c) {
    return adj::youturn_t<float>(ctx, a, b, sec2, c);
}
}  // namespace da
