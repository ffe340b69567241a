// FP64 plain path of the forward step.  Built with --fmad=false: every multiply and add
// rounds on its own, in the reference's expression order, so results match the CPU
// reference (compiled without FMA) bit for bit.
#include "forward_impl.cuh"

namespace da {

int launch_forward_step_fp64(da_ctx *ctx, cudaEvent_t *ev) { return fwd::launch_step_t<double>(ctx, ev); }

int forward_alloc(da_ctx *ctx) {
    const size_t n = (size_t)ctx->mesh.n;
    const size_t rs = ctx->p.precision == DA_PREC_FP64 ? sizeof(double) : sizeof(float);
    // grid-stride kernels: at most 8 blocks of 256 threads per SM (2048 resident threads)
    const size_t want = (n + fwd::kBlock - 1) / fwd::kBlock;
    const size_t cap = (size_t)(ctx->sm_count > 0 ? ctx->sm_count : 148) * 8;
    ctx->nblocks = int(want < cap ? want : cap);
    if (ctx->nblocks < 1) ctx->nblocks = 1;
    int st = DA_OK;
    for (int b = 0; b < 2 && !st; ++b)
        for (int v = 0; v < 3 && !st; ++v) {
            st = cuda_check(ctx, cudaMalloc(&ctx->U[b][v], rs * n), "cudaMalloc(state)");
            if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->U[b][v], 0, rs * n, ctx->stream), "memset");
        }
    if (!st) st = cuda_check(ctx, cudaMalloc(&ctx->kact, rs * n), "cudaMalloc(kact)");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->vol_part, sizeof(double) * ctx->nblocks), "cudaMalloc(vol)");
    return st;
}

int launch_forward_step(da_ctx *ctx, cudaEvent_t *ev) {
    if (ctx->p.precision == DA_PREC_FP64) return launch_forward_step_fp64(ctx, ev);
    return launch_forward_step_fp32(ctx, ev);
}

}  // namespace da
