// Checkpoint copies of the adjoint's reverse sweep: one launch per store or restore, one warp
// per 32-cell segment.
//
// Slot 0 is the base checkpoint: a full copy of the state; storing it also copies the live state
// into the other ping-pong buffer wherever the two differ, so that afterwards every segment holds
// the base in both buffers and none is dirty.  Every later store copies only the
// segments that an update has changed since the base ("dirty" segments, seg_dirty), so a flow that
// covers a small part of the mesh is checkpointed at the cost of its footprint.  A restore writes
// into both ping-pong buffers the snapshot's dirty segments, and the base copy of the segments
// that are dirty now but were not at the snapshot; every other segment already holds the base
// state in both buffers.  Each restored segment gets its wet flag and volume partial recomputed
// from the restored depths (the same sums as the update), so culling and the volume stay exact.
// Afterwards every segment is clean and the live dirty flags are the snapshot's.
#include <cuda_runtime.h>

#include "fv_device.cuh"

namespace da {
namespace {

using namespace fv;

constexpr int kBlock = 256;

enum SnapMode { STORE_BASE = 0, STORE = 1, RESTORE_BASE = 2, RESTORE = 3 };

template <class R>
struct SnapArgs {
    MeshArgs m;
    R *buf[2][3];          // the two ping-pong buffers (h, hu, hv)
    int cur;               // live buffer
    R *snap[3];            // this slot's state arrays (only dirty segments are valid after STORE)
    const R *base[3];      // slot 0's state arrays
    uint8_t *snap_dirty;   // [nseg] the slot's dirty flags
    DevScalars *snap_sc;   // the slot's step scalars
    uint8_t *seg_dirty;    // live flags
    uint8_t *seg_clean;
    uint8_t *seg_wet;
    double *seg_vol;
    DevScalars *sc;
    double *times;         // ensemble: the members' times (null in a single context)
    double *snap_times;
    int ninst;
    int nseg;
    int mode;
};

template <class R>
__global__ void __launch_bounds__(kBlock) k_snapshot(SnapArgs<R> a) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < a.nseg; s += warps) {
        const int i = s * 32 + lane;
        const bool in = i < a.m.n;
        if (a.mode == STORE) {
            if (a.seg_dirty[s] && in)
                for (int v = 0; v < 3; ++v) a.snap[v][i] = a.buf[a.cur][v][i];
            if (lane == 0) a.snap_dirty[s] = a.seg_dirty[s];
            continue;
        }
        if (a.mode == STORE_BASE) {
            const bool differ = !a.seg_clean[s];
            double vol = 0.0;
            bool wet = false;
            if (in) {
                R val[3];
                for (int v = 0; v < 3; ++v) {
                    val[v] = a.buf[a.cur][v][i];
                    a.snap[v][i] = val[v];
                    if (differ) a.buf[a.cur ^ 1][v][i] = val[v];
                }
                vol = double(cell_dx<R>(a.m, i)) * double(cell_dy<R>(a.m, i)) * double(val[0]);
                wet = val[0] >= R(DA_TINY);
            }
            if (differ) {
                // flags of a segment set wholesale by a state change: recompute them
                const unsigned wet_bits = __ballot_sync(0xffffffffu, wet);
                vol = warp_sum(vol);
                if (lane == 0) {
                    a.seg_vol[s] = vol;
                    a.seg_wet[s] = wet_bits ? 1 : 0;
                }
            }
            if (lane == 0) {
                a.seg_dirty[s] = 0;
                a.seg_clean[s] = 1;
            }
            continue;
        }
        // restores
        const uint8_t sd = a.mode == RESTORE_BASE ? 0 : a.snap_dirty[s];
        const uint8_t ld = a.seg_dirty[s];
        if (sd || ld) {
            double vol = 0.0;
            bool wet = false;
            if (in) {
                R val[3];
                for (int v = 0; v < 3; ++v) {
                    val[v] = sd ? a.snap[v][i] : a.base[v][i];
                    a.buf[0][v][i] = val[v];
                    a.buf[1][v][i] = val[v];
                }
                vol = double(cell_dx<R>(a.m, i)) * double(cell_dy<R>(a.m, i)) * double(val[0]);
                wet = val[0] >= R(DA_TINY);
            }
            const unsigned wet_bits = __ballot_sync(0xffffffffu, wet);
            vol = warp_sum(vol);
            if (lane == 0) {
                a.seg_vol[s] = vol;
                a.seg_wet[s] = wet_bits ? 1 : 0;
            }
        }
        if (lane == 0) {
            a.seg_dirty[s] = sd;
            a.seg_clean[s] = 1;
        }
    }
    if (blockIdx.x == 0) {
        const bool st = a.mode == STORE_BASE || a.mode == STORE;
        if (threadIdx.x == 0) {
            if (st)
                *a.snap_sc = *a.sc;
            else
                *a.sc = *a.snap_sc;
        }
        for (int k = threadIdx.x; k < a.ninst; k += blockDim.x) {
            if (st)
                a.snap_times[k] = a.times[k];
            else
                a.times[k] = a.snap_times[k];
        }
    }
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

template <class R>
int launch_t(da_ctx *ctx, void *slot, bool store) {
    const size_t n = (size_t)ctx->mesh.n, ab = align256(sizeof(R) * n);
    const bool is_base = slot == ctx->snaps[0];
    unsigned char *b = (unsigned char *)slot, *b0 = (unsigned char *)ctx->snaps[0];
    SnapArgs<R> a{};
    a.m = mesh_args(ctx);
    for (int q = 0; q < 2; ++q)
        for (int v = 0; v < 3; ++v) a.buf[q][v] = (R *)ctx->U[q][v];
    a.cur = ctx->cur;
    for (int v = 0; v < 3; ++v) {
        a.snap[v] = (R *)(b + v * ab);
        a.base[v] = (const R *)(b0 + v * ab);
    }
    a.snap_dirty = b + 3 * ab;
    a.snap_sc = (DevScalars *)(b + 3 * ab + align256((size_t)ctx->nseg));
    a.snap_times = (double *)(b + 3 * ab + align256((size_t)ctx->nseg) + align256(sizeof(DevScalars)));
    a.times = ctx->ia.time;
    a.ninst = ctx->ninst;
    a.seg_dirty = ctx->seg_dirty;
    a.seg_clean = ctx->seg_clean;
    a.seg_wet = ctx->seg_wet;
    a.seg_vol = ctx->seg_vol;
    a.sc = ctx->dsc;
    a.nseg = ctx->nseg;
    a.mode = store ? (is_base ? STORE_BASE : STORE) : (is_base ? RESTORE_BASE : RESTORE);
    const int grid = (ctx->sm_count > 0 ? ctx->sm_count : 148) * 4;
    trace_begin(ctx, TR_SNAPSHOT);
    k_snapshot<R><<<grid, kBlock, 0, ctx->stream>>>(a);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "snapshot copy");
}

}  // namespace

size_t snapshot_bytes(const da_ctx *ctx) {
    const size_t rs = ctx->p.precision == DA_PREC_FP64 ? sizeof(double) : sizeof(float);
    return 3 * align256(rs * (size_t)ctx->mesh.n) + align256((size_t)ctx->nseg) + align256(sizeof(DevScalars)) +
           sizeof(double) * (size_t)ctx->ninst;
}

int launch_snapshot(da_ctx *ctx, void *slot, bool store) {
    return ctx->p.precision == DA_PREC_FP64 ? launch_t<double>(ctx, slot, store) : launch_t<float>(ctx, slot, store);
}

}  // namespace da
