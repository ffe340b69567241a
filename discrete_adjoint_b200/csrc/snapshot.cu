// Checkpoint copies as a launch of their own (the base store before the reverse sweep, the base
// restore after it, and the ensemble and single-step paths); the copy phases themselves, and the
// slot layout, are in snapshot_impl.cuh, shared with the cooperative step kernels.
#include <cuda_runtime.h>

#include "snapshot_impl.cuh"

namespace da {
namespace {

constexpr int kBlock = 256;

template <class R>
__global__ void __launch_bounds__(kBlock) k_snapshot(snap::SnapArgs<R> a) {
    snap::snap_segments<R>(a);
    snap::snap_scalars<R>(a);
}

template <class R>
int launch_t(da_ctx *ctx, void *slot, bool store) {
    const snap::SnapArgs<R> a = snap::snap_args<R>(ctx, slot, store, ctx->cur);
    const int grid = (ctx->sm_count > 0 ? ctx->sm_count : 148) * 4;
    trace_begin(ctx, TR_SNAPSHOT);
    k_snapshot<R><<<grid, kBlock, 0, ctx->stream>>>(a);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "snapshot copy");
}

}  // namespace

size_t snapshot_bytes(const da_ctx *ctx) {
    const size_t rs = ctx->p.precision == DA_PREC_FP64 ? sizeof(double) : sizeof(float);
    return 3 * snap::align256(rs * (size_t)ctx->mesh.n) + snap::align256((size_t)ctx->nseg) +
           snap::align256(sizeof(DevScalars)) + sizeof(double) * (size_t)ctx->ninst;
}

int launch_snapshot(da_ctx *ctx, void *slot, bool store) {
    return ctx->p.precision == DA_PREC_FP64 ? launch_t<double>(ctx, slot, store) : launch_t<float>(ctx, slot, store);
}

}  // namespace da
