// FP64 adjoint kernels.
#include "adjoint_kernels.cuh"

namespace da {
int launch_adjoint_step_fp64(da_ctx *ctx, int a, int b, const double *sec2, double c) {
    return adj::step_t<double>(ctx, a, b, sec2, c);
}
int launch_adjoint_seed_fp64(da_ctx *ctx, int b, const double box[4]) { return adj::seed_t<double>(ctx, b, box); }
int launch_adjoint_reduce_fp64(da_ctx *ctx, int a, int np) { return adj::reduce_t<double>(ctx, a, np); }
}  // namespace da
