// FP64 plain path of the forward step.  Built with --fmad=false: every multiply and add
// rounds on its own, in the reference's expression order, so results match the CPU
// reference (compiled without FMA) bit for bit.
#include "forward_impl.cuh"

namespace da {

int launch_forward_step_fp64(da_ctx *ctx, uint8_t *record_mask) {
    return fwd::launch_step_t<double>(ctx, record_mask);
}
int launch_forward_steps_fp64(da_ctx *ctx, int nsteps, void *pre, void *post, const MidStoreList *mid) {
    return fwd::launch_steps_t<double>(ctx, nsteps, pre, post, mid);
}
int launch_refine_info_fp64(da_ctx *ctx, double *e, uint8_t *f, double *parts, double *t) {
    return fwd::refine_info_t<double>(ctx, e, f, parts, t);
}

int launch_step_half_fp64(da_ctx *ctx, int half, double *bounds) {
    return fwd::launch_step_half_t<double>(ctx, half, bounds);
}

int launch_volume(da_ctx *ctx) { return fwd::launch_volume_t(ctx); }

namespace {
// Every block but block 0 waits at the grid barrier; block 0 returns without arriving, so the wait
// runs out after limit_ns and raises DA_ERR_TIMEOUT.
__global__ void k_barrier_selftest(DevScalars *sc, unsigned long long limit_ns) {
    if (blockIdx.x == 0) return;
    fwd::grid_sync(sc, limit_ns);
}
}  // namespace

int launch_barrier_selftest(da_ctx *ctx, unsigned long long limit_ns) {
    // one block per SM: co-resident, as the cooperative launch checks
    const int grid = ctx->sm_count > 1 ? ctx->sm_count : 2;
    DevScalars *sc = ctx->dsc;
    void *args[] = {&sc, &limit_ns};
    return cuda_check(ctx, cudaLaunchCooperativeKernel((const void *)k_barrier_selftest, grid, 32, args, 0, ctx->stream),
                      "barrier self-test launch");
}

int forward_alloc(da_ctx *ctx) {
    const size_t n = (size_t)ctx->mesh.n;
    const size_t rs = ctx->p.precision == DA_PREC_FP64 ? sizeof(double) : sizeof(float);
    ctx->ntiles = int((n + fwd::kBlock - 1) / fwd::kBlock);
    ctx->nseg = ctx->ntiles * (fwd::kBlock / 32);
    // seed kernel grid: 4 blocks of 256 threads per SM, never more blocks than tiles
    const int cap = (ctx->sm_count > 0 ? ctx->sm_count : 148) * 4;
    ctx->nblocks = ctx->ntiles < cap ? ctx->ntiles : cap;
    update_grid(ctx);
    const size_t nseg = (size_t)ctx->nseg;
    int st = DA_OK;
    for (int b = 0; b < 2 && !st; ++b)
        for (int v = 0; v < 3 && !st; ++v) {
            st = cuda_check(ctx, cudaMalloc(&ctx->U[b][v], rs * n), "cudaMalloc(state)");
            if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->U[b][v], 0, rs * n, ctx->stream), "memset");
        }
    if (!st) st = cuda_check(ctx, cudaMalloc(&ctx->kact, rs * n), "cudaMalloc(kact)");
    if (!st) st = cuda_check(ctx, cudaMalloc(&ctx->slopes, 6 * rs * n), "cudaMalloc(slopes)");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->seg_wet, nseg), "cudaMalloc(seg_wet)");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->tile_epoch, sizeof(int) * ctx->ntiles), "cudaMalloc(epoch)");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->tile_epoch, 0xff, sizeof(int) * ctx->ntiles, ctx->stream), "memset");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->seg_act, nseg), "cudaMalloc(seg_act)");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->lam_clean, nseg), "cudaMalloc(lam_clean)");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->lam_clean, 0, nseg, ctx->stream), "memset");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->seg_vol, sizeof(double) * nseg), "cudaMalloc(vol)");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->seg_vol, 0, sizeof(double) * nseg, ctx->stream), "memset");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->vol_parts, sizeof(double) * fwd::kVolParts), "cudaMalloc(vol)");
    // the active bitmask is padded to whole tiles (8 words each) for the 16-byte tile tests
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->active, sizeof(unsigned) * nseg), "cudaMalloc(active)");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->active, 0, sizeof(unsigned) * nseg, ctx->stream), "memset");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->seg_clean, nseg), "cudaMalloc(clean)");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->seg_clean, 0, nseg, ctx->stream), "memset");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->seg_dirty, nseg), "cudaMalloc(dirty)");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->seg_dirty, 1, nseg, ctx->stream), "memset");
    return st;
}

int forward_state_changed(da_ctx *ctx) {
    // the buffers no longer hold the same segments, any segment may be wet, no cell is marked active
    const size_t nseg = (size_t)ctx->nseg;
    int st = cuda_check(ctx, cudaMemsetAsync(ctx->seg_clean, 0, nseg, ctx->stream), "memset");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->seg_wet, 1, nseg, ctx->stream), "memset");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->active, 0, sizeof(unsigned) * nseg, ctx->stream), "memset");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->seg_dirty, 1, nseg, ctx->stream), "memset");
    return st;
}

// A context with ghost cells (da_set_owned) must not form dt from its own cells alone: it steps
// through da_step_bounds / da_step_apply, with the bounds combined over the subdomains, or with a
// replayed dt sequence (da_set_dt_replay: the subdomains' reverse steps).
static bool ghosts_refused(da_ctx *ctx) {
    if (ctx->mesh.n_owned == ctx->mesh.n || ctx->tc.dt_replay) return false;
    set_error(ctx, DA_ERR_UNSUPPORTED,
              "context with ghost cells: step it with da_step_bounds / da_step_apply or a replayed dt");
    return true;
}

int launch_forward_steps(da_ctx *ctx, int nsteps, void *pre_slot, void *post_slot, const MidStoreList *mid) {
    if (ghosts_refused(ctx)) return DA_ERR_UNSUPPORTED;
    if (ctx->p.precision == DA_PREC_FP64) return launch_forward_steps_fp64(ctx, nsteps, pre_slot, post_slot, mid);
    return launch_forward_steps_fp32(ctx, nsteps, pre_slot, post_slot, mid);
}

int launch_forward_step(da_ctx *ctx, uint8_t *record_mask) {
    if (ghosts_refused(ctx)) return DA_ERR_UNSUPPORTED;
    if (ctx->p.precision == DA_PREC_FP64) return launch_forward_step_fp64(ctx, record_mask);
    return launch_forward_step_fp32(ctx, record_mask);
}

}  // namespace da
