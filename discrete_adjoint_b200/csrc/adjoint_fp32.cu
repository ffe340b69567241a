// FP32-split adjoint kernels: FP32 state and adjoint fields, FP64 sums and parameter sensitivities.
#include "adjoint_kernels.cuh"

namespace da {
int launch_adjoint_step_fp32(da_ctx *ctx, int a, int b, const double *sec2, double c) {
    return adj::step_t<float>(ctx, a, b, sec2, c);
}
int launch_adjoint_reduce_fp32(da_ctx *ctx, int a, int np) { return adj::reduce_t<float>(ctx, a, np); }
int launch_youturn_fp32(da_ctx *ctx, int a, int b, const double *sec2, double c, bool seed, const double *box,
                        void *pre) {
    return adj::youturn_t<float>(ctx, a, b, sec2, c, seed, box, pre);
}
int launch_functional_fp32(da_ctx *ctx, double *out) { return adj::functional_t<float>(ctx, out); }
int launch_adjoint_reduce_inst_fp32(da_ctx *ctx, int a) { return adj::reduce_inst_t<float>(ctx, a); }
}  // namespace da
