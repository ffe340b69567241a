// Checkpoint copies of the adjoint's reverse sweep: one launch per store or restore.
// A snapshot holds the state (3 arrays), the per-segment wet flags and the step scalars.  A
// restore writes the state into both ping-pong buffers, so every segment is clean afterwards and
// the next steps keep their tile culling.
#include <cuda_runtime.h>

#include "da_internal.h"

namespace da {
namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ void copy_bytes(const unsigned char *__restrict__ src, unsigned char *__restrict__ dst,
                                           unsigned char *__restrict__ dst2, size_t bytes) {
    const size_t nv = bytes / 16;
    const uint4 *s4 = (const uint4 *)src;
    uint4 *d4 = (uint4 *)dst;
    uint4 *e4 = (uint4 *)dst2;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < nv; k += stride) {
        const uint4 v = s4[k];
        d4[k] = v;
        if (dst2) e4[k] = v;
    }
    for (size_t k = nv * 16 + (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < bytes; k += stride) {
        dst[k] = src[k];
        if (dst2) dst2[k] = src[k];
    }
}

struct SnapArgs {
    const unsigned char *src[3];
    unsigned char *dst[3];
    unsigned char *dst2[3];  // second destination (the other ping-pong buffer) or null
    size_t bytes;            // per state array
    const unsigned char *flags_src;
    unsigned char *flags_dst;
    size_t flag_bytes;
    const DevScalars *sc_src;
    DevScalars *sc_dst;
    uint8_t *clean;          // set to 1 for every segment when not null
    int nseg;
};

__global__ void __launch_bounds__(kBlock) k_snapshot(SnapArgs a) {
    for (int v = 0; v < 3; ++v) copy_bytes(a.src[v], a.dst[v], a.dst2[v], a.bytes);
    copy_bytes(a.flags_src, a.flags_dst, nullptr, a.flag_bytes);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (a.clean)
        for (size_t t = tid; t < (size_t)a.nseg; t += stride) a.clean[t] = 1;
    if (tid == 0) *a.sc_dst = *a.sc_src;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace

size_t snapshot_bytes(const da_ctx *ctx) {
    const size_t rs = ctx->p.precision == DA_PREC_FP64 ? sizeof(double) : sizeof(float);
    return 3 * align256(rs * (size_t)ctx->mesh.n) + align256((size_t)ctx->nseg) + sizeof(DevScalars);
}

int launch_snapshot(da_ctx *ctx, void *slot, bool store) {
    const size_t rs = ctx->p.precision == DA_PREC_FP64 ? sizeof(double) : sizeof(float);
    const size_t bytes = rs * (size_t)ctx->mesh.n, ab = align256(bytes);
    unsigned char *base = (unsigned char *)slot;
    unsigned char *flags = base + 3 * ab;
    DevScalars *ssc = (DevScalars *)(flags + align256((size_t)ctx->nseg));
    SnapArgs a{};
    a.bytes = bytes;
    a.flag_bytes = (size_t)ctx->nseg;
    a.nseg = ctx->nseg;
    for (int v = 0; v < 3; ++v) {
        if (store) {
            a.src[v] = (const unsigned char *)ctx->U[ctx->cur][v];
            a.dst[v] = base + v * ab;
            a.dst2[v] = nullptr;
        } else {
            a.src[v] = base + v * ab;
            a.dst[v] = (unsigned char *)ctx->U[ctx->cur][v];
            a.dst2[v] = (unsigned char *)ctx->U[1 - ctx->cur][v];
        }
    }
    if (store) {
        a.flags_src = ctx->seg_wet;
        a.flags_dst = flags;
        a.sc_src = ctx->dsc;
        a.sc_dst = ssc;
        a.clean = nullptr;
    } else {
        a.flags_src = flags;
        a.flags_dst = ctx->seg_wet;
        a.sc_src = ssc;
        a.sc_dst = ctx->dsc;
        a.clean = ctx->seg_clean;
    }
    int grid = (ctx->sm_count > 0 ? ctx->sm_count : 148) * 4;
    trace_begin(ctx, TR_SNAPSHOT);
    k_snapshot<<<grid, kBlock, 0, ctx->stream>>>(a);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "snapshot copy");
}

}  // namespace da
