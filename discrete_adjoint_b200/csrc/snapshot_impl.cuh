// Checkpoint copies of the adjoint's reverse sweep, as device phases run either by the
// stand-alone snapshot kernel or as the first (restore) or last (store) phase of the cooperative
// step kernels, which saves a launch per checkpoint.  Each thread checks one 32-cell segment's
// flags, and a warp copies the segments that need it (lane = cell).
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
#pragma once
#include <cuda_runtime.h>

#include "fv_device.cuh"

namespace da {
namespace snap {
namespace {  // internal linkage: each translation unit keeps its own copy

using namespace fv;

enum SnapMode { NONE = -1, STORE_BASE = 0, STORE = 1, RESTORE_BASE = 2, RESTORE = 3 };

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

// One segment's cells (lane = cell): the copy of the mode; flag is the snapshot's dirty flag for
// a restore, whether the two buffers differ for the base store.  Restores and the base store
// recompute the segment's wet flag and volume partial.  Called by all 32 lanes of a warp.
template <class R>
__device__ __forceinline__ void copy_segment(const SnapArgs<R> &a, int s, uint8_t flag, int lane) {
    const int i = s * 32 + lane;
    const bool in = i < a.m.n;
    if (a.mode == STORE) {
        if (in)
            for (int v = 0; v < 3; ++v) a.snap[v][i] = a.buf[a.cur][v][i];
        return;
    }
    const bool base_store = a.mode == STORE_BASE;
    double vol = 0.0;
    bool wet = false;
    if (in) {
        R val[3];
        for (int v = 0; v < 3; ++v) {
            if (base_store) {
                val[v] = a.buf[a.cur][v][i];
                a.snap[v][i] = val[v];
                if (flag) a.buf[a.cur ^ 1][v][i] = val[v];
            } else {
                val[v] = flag ? a.snap[v][i] : a.base[v][i];
                a.buf[0][v][i] = val[v];
                a.buf[1][v][i] = val[v];
            }
        }
        vol = double(cell_dx<R>(a.m, i)) * double(cell_dy<R>(a.m, i)) * double(val[0]);
        wet = val[0] >= R(DA_TINY);
    }
    if (base_store && !flag) return;  // both buffers already agree: the flags stand
    // flags of a segment restored, or set wholesale by a state change: recompute them
    const unsigned wet_bits = __ballot_sync(0xffffffffu, wet);
    vol = warp_sum(vol);
    if (lane == 0) {
        a.seg_vol[s] = vol;
        a.seg_wet[s] = wet_bits ? 1 : 0;
    }
}

// The state and segment-flag part.  Thread (warp w of W, lane l) looks after the flags of segments
// l * W + w (+ 32 W k): consecutive segments belong to consecutive warps, so the dirty segments
// of a compact flow spread over the grid and one round of flag loads covers the mesh.  Each warp
// then copies its segments that need work, one after another, all lanes on one segment.
template <class R>
__device__ __forceinline__ void snap_segments(const SnapArgs<R> &a) {
    const int lane = threadIdx.x & 31;
    const int W = (gridDim.x * blockDim.x) >> 5;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (int s0 = 0; s0 < a.nseg; s0 += 32 * W) {
        const int s = s0 + lane * W + w;
        bool work = false;
        uint8_t flag = 0;
        if (s < a.nseg) {
            if (a.mode == STORE) {
                const uint8_t d = a.seg_dirty[s];
                a.snap_dirty[s] = d;
                work = d != 0;
            } else if (a.mode == STORE_BASE) {
                flag = a.seg_clean[s] ? 0 : 1;
                a.seg_dirty[s] = 0;
                a.seg_clean[s] = 1;
                work = true;
            } else {
                flag = a.mode == RESTORE_BASE ? 0 : a.snap_dirty[s];
                const uint8_t ld = a.seg_dirty[s];
                a.seg_dirty[s] = flag;
                a.seg_clean[s] = 1;
                work = flag || ld;
            }
        }
        unsigned bits = __ballot_sync(0xffffffffu, work);
        while (bits) {
            const int k = __ffs(bits) - 1;
            bits &= bits - 1;
            copy_segment<R>(a, s0 + k * W + w, (uint8_t)__shfl_sync(0xffffffffu, flag, k), lane);
        }
    }
}

// A STORE (not the base slot) from explicit arrays, for the checkpoints a multi-step launch takes
// on its way: the live dirty flags into the slot's, and the dirty segments of the live buffer
// (h, hu, hv) into the slot's arrays (s_h, s_hu, s_hv), with snap_segments' division of the work.
template <class R>
__device__ __forceinline__ void store_segments(const R *h, const R *hu, const R *hv, R *s_h, R *s_hu, R *s_hv,
                                               const uint8_t *seg_dirty, uint8_t *snap_dirty, int nseg, int n) {
    const int lane = threadIdx.x & 31;
    const int W = (gridDim.x * blockDim.x) >> 5;
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    for (int s0 = 0; s0 < nseg; s0 += 32 * W) {
        const int s = s0 + lane * W + w;
        bool work = false;
        if (s < nseg) {
            const uint8_t d = seg_dirty[s];
            snap_dirty[s] = d;
            work = d != 0;
        }
        unsigned bits = __ballot_sync(0xffffffffu, work);
        while (bits) {
            const int k = __ffs(bits) - 1;
            bits &= bits - 1;
            const int i = (s0 + k * W + w) * 32 + lane;
            if (i < n) {
                s_h[i] = h[i];
                s_hu[i] = hu[i];
                s_hv[i] = hv[i];
            }
        }
    }
}

// The state of the time stepping (time, dt, iteration, CFL values, volume and accumulators); the
// error flag stays sticky and the barrier counters are not touched (a restore runs while the other
// blocks of a cooperative launch may already wait at the barrier).
__device__ __forceinline__ void copy_step_scalars(DevScalars *d, const DevScalars *s) {
    d->time = s->time;
    d->dt = s->dt;
    d->hmax = s->hmax;
    d->min_dxe = s->min_dxe;
    d->volume = s->volume;
    d->frict_tiny = s->frict_tiny;
    d->iter = s->iter;
    d->acc_min_dxe = s->acc_min_dxe;
    d->acc_hmax = s->acc_hmax;
    d->acc_alt_min_dxe = s->acc_alt_min_dxe;
    d->acc_alt_hmax = s->acc_alt_hmax;
}

// The step scalars and the members' times: block 0.  A store reads the scalars the caller's
// block 0 has just written (same thread), a restore writes them before the caller's barrier.
template <class R>
__device__ __forceinline__ void snap_scalars(const SnapArgs<R> &a) {
    if (blockIdx.x != 0) return;
    const bool st = a.mode == STORE_BASE || a.mode == STORE;
    if (threadIdx.x == 0) {
        if (st)
            copy_step_scalars(a.snap_sc, a.sc);
        else
            copy_step_scalars(a.sc, a.snap_sc);
    }
    for (int k = threadIdx.x; k < a.ninst; k += blockDim.x) {
        if (st)
            a.snap_times[k] = a.times[k];
        else
            a.times[k] = a.snap_times[k];
    }
}

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// The copy between the live state (buffer cur) and checkpoint slot; a slot's layout: the three
// state arrays, the dirty flags, the scalars, the members' times (each 256-byte aligned).
template <class R>
SnapArgs<R> snap_args(da_ctx *ctx, void *slot, bool store, int cur) {
    const size_t n = (size_t)ctx->mesh.n, ab = align256(sizeof(R) * n);
    const bool is_base = slot == ctx->snaps[0];
    unsigned char *b = (unsigned char *)slot, *b0 = (unsigned char *)ctx->snaps[0];
    SnapArgs<R> a{};
    a.m = mesh_args(ctx);
    for (int q = 0; q < 2; ++q)
        for (int v = 0; v < 3; ++v) a.buf[q][v] = (R *)ctx->U[q][v];
    a.cur = cur;
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
    return a;
}

template <class R>
SnapArgs<R> no_snap() {
    SnapArgs<R> a{};
    a.mode = NONE;
    return a;
}

}  // namespace
}  // namespace snap
}  // namespace da
