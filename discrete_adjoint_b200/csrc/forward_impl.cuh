// Forward step kernels (order_flag = 1) for sm_100a -- templates shared by the FP64 and
// FP32-split translation units (forward_fp64.cu is built without FMA contraction).
//
// One step() of the reference (src/geoflow/step.C:29-275) is two launches:
//   k_coef   : per wet cell the limited slopes (Element::get_slopes, element2.C:830-939), k
//              act/pass (gmfggetcoef, getcoef.f:19-66) and wave speeds (eigen.f:19-49); the CFL
//              min and hmax reductions of get_coef_and_eigen.C:86-166; the last block to finish
//              forms dt (get_coef_and_eigen.C:168-179) and applies TimeProps::incrtime
//              (properties.h:397-410).
//   k_update : the four side fluxes of every cell (xdirflux/ydirflux/riemannflux with the
//              hanging-node averaging of Element::calc_edge_states, element2.C:2745-3072, and the
//              outflow copy of boundary_flux, element2.C:3374-3411) fused with the corrector
//              update_states (residual.C:162-275); slopes are recomputed here rather than
//              stored; the last block sums the FP64 volume partials in a fixed order.
// Each edge flux is evaluated by both cells that share it from the same operands, so both see
// the same bits and no edge array is stored.  A cell whose own and neighbours' depths are all
// below GEOFLOW_TINY has zero fluxes and no sources, so its state is copied unchanged (the
// same bits the full update produces).
#pragma once
#include <cuda_runtime.h>

#include "fv_device.cuh"

namespace da {
namespace fwd {
namespace {  // internal linkage: each precision TU keeps its own copy

using namespace fv;

constexpr int kBlock = kTileCells;  // one thread per cell of a tile

// dt from the reduced CFL bound and hmax (get_coef_and_eigen.C:168-179 with the single-rank
// MPI_Allreduce(MIN)), then TimeProps::incrtime.  frict_tiny follows hpfem.C:232-235 with the
// iteration count before the increment.
__device__ void finalize_dt(DevScalars *sc, const TimeConsts &tc) {
    const double min_dxe = __longlong_as_double(*(volatile unsigned long long *)&sc->acc_min_dxe);
    const double hmax = __longlong_as_double(*(volatile unsigned long long *)&sc->acc_hmax);
    const double g0 = 0.5 * min_dxe;
    const double g1 = -0.9 * sqrt(hmax * (tc.epsilon) * (tc.gravity_scale) / 9.8);
    double dt = 0.5 * (g0 > -g1 ? -g1 : g0);
    if (dt == 0.0) dt = 0.5 * tc.influx_dt;
    const double time = sc->time;
    if (time + dt > tc.next_output) dt = tc.next_output - time;
    if (time + dt > tc.next_save) dt = tc.next_save - time;
    if (time + dt > tc.max_time) dt = tc.max_time - time;
    if (tc.dt_replay) {
        // frozen time-step sequence (tangent/finite-difference checks of the adjoint)
        const long long k = sc->iter - tc.iter0;
        dt = (k >= 0 && k < tc.n_replay) ? tc.dt_replay[k] : 0.0;
    }
    sc->frict_tiny = sc->iter < tc.frict_tiny_iters ? tc.frict_tiny_early : tc.frict_tiny_late;
    sc->dt = dt;
    sc->time = time + dt;
    sc->min_dxe = min_dxe;
    sc->hmax = hmax;
    sc->iter += 1;
    sc->acc_min_dxe = __double_as_longlong(10000000.0);  // get_coef_and_eigen.C:36
    sc->acc_hmax = 0ull;
}

// True in every thread of the block that finished last (threadfence-reduction pattern).
__device__ __forceinline__ bool last_block(unsigned *counter) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned t = atomicAdd(counter, 1u);
        last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}


// ----------------------------------------------------------------------------- k_coef
// One thread per cell of each listed tile.  With tile culling, a tile that held no wet cell
// after the last update is not listed (its depths cannot have changed since).  Wet cells
// (h >= GEOFLOW_TINY) also mark themselves and their face neighbours in the active bitmask that
// k_update reads: a cell outside that set has zero fluxes and no sources this step.
// RECORD: also writes the branch code of every cell of a listed tile into mask (0 dry / at rest,
// 1..3 for sgn(vel) = -1, 0, +1 of gmfggetcoef) for the adjoint's replay.
template <class R, bool RECORD = false>
__global__ void __launch_bounds__(kBlock) k_coef(MeshArgs m, StateRef<R> U, R *__restrict__ kact,
                                                 unsigned *__restrict__ active, const uint8_t *__restrict__ tile_wet,
                                                 int ntiles, int cull, MatConsts mc, TimeConsts tc, DevScalars *sc,
                                                 uint8_t *__restrict__ mask = nullptr) {
    __shared__ int list[kBlock];
    unsigned long long my_min = 0x7FF0000000000000ull;  // +inf
    unsigned long long my_max = 0ull;
    for (int round = 0; sched_more(round, ntiles); ++round) {
        const int tq = sched_tile(round);
        const bool need = tq < ntiles && (!cull || tile_wet[tq]);
        const int cnt = compact_tiles(need, tq, list);
        for (int q = 0; q < cnt; ++q) {
            const int i = list[q] * kBlock + threadIdx.x;
            bool wet = false;
            if (i < m.n) {
                const R h = U.h[i];
                if (!(h == h)) raise_err(sc, DA_ERR_NAN);
                wet = h >= R(DA_TINY);
                uint8_t code = 0;
                if (wet) {
                    const uint8_t bf = m.bflag[i];
#pragma unroll
                    for (int s = 0; s < 4; ++s) {
                        if (bf & (1 << s)) continue;
                        const int e = m.nbr[(size_t)s * m.n + i];
                        atomicOr(&active[e >> 5], 1u << (e & 31));
                        if (bf & (0x10 << s)) {
                            const int e2 = m.nbr[(size_t)(s + 4) * m.n + i];
                            atomicOr(&active[e2 >> 5], 1u << (e2 & 31));
                        }
                    }
                    if (!(h > R(DA_TINY))) {  // h == GEOFLOW_TINY: dry for get_coef_and_eigen, wet for the fluxes
                        kact[i] = R(mc.kact_rest);
                    } else {
                        const R ui[3] = {h, U.hu[i], U.hv[i]};
                        R s[6];
                        cell_slopes<R>(m, U, i, bf, R(mc.gamma), ui, s);
                        const R k = cell_kact<R>(mc, m.mat[i], h, ui[1], ui[2], s, &code);
                        kact[i] = k;
                        const R gz = grav<R>(m, 2, i);
                        const R vx = ui[1] / h, vy = ui[2] / h;
                        const R c = sqrt(k * gz * h);
                        const R evx = dabs(vx) + c, evy = dabs(vy) + c;
                        const R ev = evx > evy ? evx : evy;
                        if (ev > R(1000000000.)) raise_err(sc, DA_ERR_EIGEN);
                        const R dxm = cell_dx<R>(m, i), dym = cell_dy<R>(m, i);
                        const unsigned long long rb = __double_as_longlong(double((dxm > dym ? dym : dxm) / ev));
                        const unsigned long long hb = __double_as_longlong(double(h));
                        my_min = rb < my_min ? rb : my_min;
                        my_max = hb > my_max ? hb : my_max;
                    }
                }
                if (RECORD) mask[i] = code;
            }
            const unsigned self = __ballot_sync(0xffffffffu, wet);
            if (self && (threadIdx.x & 31) == 0) atomicOr(&active[i >> 5], self);
        }
    }
    my_min = warp_min_u64(my_min);
    my_max = warp_max_u64(my_max);
    if ((threadIdx.x & 31) == 0) {
        if (my_min != 0x7FF0000000000000ull) atomicMin(&sc->acc_min_dxe, my_min);
        if (my_max) atomicMax(&sc->acc_hmax, my_max);
    }
    if (last_block(&sc->blocks_done[0])) {
        if (threadIdx.x == 0) {
            finalize_dt(sc, tc);
            sc->blocks_done[0] = 0;
        }
    }
}

// Full corrector update of one active cell (fluxes + sources), reference order.
template <class R>
__device__ __forceinline__ bool update_cell(const MeshArgs &m, const StateRef<R> &U, const R *__restrict__ kact,
                                            const MatConsts &mc, int i, R dt, R ft, const R prev[3], R dxc, R dyc,
                                            R st[3]) {
    const uint8_t bf = m.bflag[i];
    const R ki = prev[0] >= R(DA_TINY) ? kact[i] : R(0);
    const R gz = grav<R>(m, 2, i);
    R div[2][3];
#pragma unroll
    for (int d = 0; d < 2; ++d) {
        if (bf & ((1 << d) | (1 << (d + 2)))) {
            // an outflow side copies the opposite side's flux: the difference is exactly 0
            div[d][0] = div[d][1] = div[d][2] = R(0);
            continue;
        }
        Hfv<R> self;
        dirflux<R>(d, prev[0], prev[1], prev[2], ki, gz, self);
        R Fm[3], Fp[3];
        side_flux<R>(m, U, kact, i, bf, d + 2, self, Fm);
        side_flux<R>(m, U, kact, i, bf, d, self, Fp);
#pragma unroll
        for (int v = 0; v < 3; ++v) div[d][v] = Fp[v] - Fm[v];
    }
    R dtdx, dtdy;
    if constexpr (sizeof(R) == 8) {
        dtdx = dt / dxc;
        dtdy = dt / dyc;
    } else {
        dtdx = dt * (1.0f / dxc);
        dtdy = dt * (1.0f / dyc);
    }
#pragma unroll
    for (int v = 0; v < 3; ++v) st[v] = prev[v] - dtdx * div[0][v] - dtdy * div[1][v];
    const bool clamped = st[0] < R(0);
    if (clamped) st[0] = R(0);
    if (prev[0] > R(DA_TINY)) {
        R s[6];
        cell_slopes<R>(m, U, i, bf, R(mc.gamma), prev, s);
        R vel0, vel1, h_inv;
        if constexpr (sizeof(R) == 8) {
            vel0 = prev[1] / prev[0];
            vel1 = prev[2] / prev[0];
            h_inv = 1. / prev[0];
        } else {
            h_inv = 1.0f / prev[0];
            vel0 = prev[1] * h_inv;
            vel1 = prev[2] * h_inv;
        }
        R tmp = h_inv * (s[4] - vel0 * s[3]);
        const R sg0 = tiny_sgn(tmp, ft);
        const R sg2 = tiny_sgn(vel0, ft);
        tmp = h_inv * (s[2] - vel1 * s[0]);
        const R sg1 = tiny_sgn(tmp, ft);
        const R sg3 = tiny_sgn(vel1, ft);
        const R sin_int = R(mc.sin_int);
        const R tan_bed = R(mc.tan_bed[m.mat[i]]);
        R s1 = grav<R>(m, 0, i) * prev[0];
        R s2 = sg0 * prev[0] * ki * (gz * s[3] + dgrav<R>(m, 1, i) * prev[0]) * sin_int;
        R s3 = sg2 * rmax(gz * prev[0] + vel0 * prev[1] * curvat<R>(m, 0, i), R(0.0)) * tan_bed;
        st[1] += dt * (s1 - s2 - s3);
        s1 = grav<R>(m, 1, i) * prev[0];
        s2 = sg1 * prev[0] * ki * (gz * s[0] + dgrav<R>(m, 0, i) * prev[0]) * sin_int;
        s3 = sg3 * rmax(gz * prev[0] + vel1 * prev[2] * curvat<R>(m, 1, i), R(0.0)) * tan_bed;
        st[2] += dt * (s1 - s2 - s3);
    }
    return clamped;
}

// Sum of a block's values in a fixed order (warp shuffle, then warps in order); thread 0 holds it.
__device__ __forceinline__ double block_sum(double v, double *red) {
    v = warp_sum(v);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
#pragma unroll
        for (int w = 0; w < kBlock / 32; ++w) t += red[w];
    return t;
}

// ---------------------------------------------------------------------------- k_update
// Tiles of kBlock consecutive cells through the strided tile list.  A tile is listed when it has
// an active cell, or when its two ping-pong buffers differ (not clean), or when culling is off.
// In a listed tile, active cells get the full update and the others are copied (their update is
// the identity).  A tile that is not listed is already identical in both buffers.  Each listed
// tile stores its volume partial, its clean flag and whether it now holds a wet cell; the last
// block sums every tile's partial in tile order, so the volume does not depend on culling.
// RECORD: every cell of a listed tile gets its full mask byte (the k_coef code of a wet cell,
// bit 3 active, bit 2 depth clamped) and the tile records the step id (tile_epoch) and whether
// it had an active cell (tile_act); masks of tiles with another epoch count as zero.
template <class R, bool RECORD = false>
__global__ void __launch_bounds__(kBlock) k_update(MeshArgs m, StateRef<R> U, StateOut<R> O,
                                                   const R *__restrict__ kact, unsigned *__restrict__ active,
                                                   uint8_t *__restrict__ clean, uint8_t *__restrict__ tile_wet,
                                                   double *__restrict__ tile_vol, int ntiles, int cull, MatConsts mc,
                                                   DevScalars *sc, double *__restrict__ vol_part,
                                                   uint8_t *__restrict__ mask = nullptr, int *__restrict__ tile_epoch = nullptr,
                                                   uint8_t *__restrict__ tile_act = nullptr, int rec_id = 0) {
    __shared__ double red[kBlock / 32];
    __shared__ int list[kBlock];
    const int lane = threadIdx.x & 31;
    const R dt = R(sc->dt);
    const R ft = R(sc->frict_tiny) > R(mc.sign_floor) ? R(sc->frict_tiny) : R(mc.sign_floor);
    for (int round = 0; sched_more(round, ntiles); ++round) {
        const int tq = sched_tile(round);
        bool need = false;
        if (tq < ntiles) {
            need = !cull || !clean[tq];
            if (!need) {
                const int w0 = tq * (kBlock / 32);
                const int nw = (m.n + 31) / 32;
                for (int w = 0; w < kBlock / 32 && !need; ++w)
                    if (w0 + w < nw && active[w0 + w]) need = true;
            }
        }
        const int cnt = compact_tiles(need, tq, list);
        for (int q = 0; q < cnt; ++q) {
            const int t = list[q];
            const int i = t * kBlock + threadIdx.x;
            const unsigned word = (i < m.n) ? active[i >> 5] : 0u;
            const bool tile_active = __syncthreads_or(word != 0u);
            double vol = 0.0;
            bool wet_after = false;
            if (i < m.n) {
                const R prev[3] = {U.h[i], U.hu[i], U.hv[i]};
                const R dxc = cell_dx<R>(m, i), dyc = cell_dy<R>(m, i);
                R st[3] = {prev[0], prev[1], prev[2]};
                const bool act = word & (1u << lane);
                bool clamped = false;
                if (act) clamped = update_cell<R>(m, U, kact, mc, i, dt, ft, prev, dxc, dyc, st);
                if (RECORD)
                    mask[i] = uint8_t((prev[0] >= R(DA_TINY) ? (mask[i] & 3) : 0) | (act ? 8 : 0) | (clamped ? 4 : 0));
                if (!isfinite(st[0]) || !isfinite(st[1]) || !isfinite(st[2])) raise_err(sc, DA_ERR_NAN);
                O.h[i] = st[0];
                O.hu[i] = st[1];
                O.hv[i] = st[2];
                vol = double(dxc) * double(dyc) * double(st[0]);
                wet_after = st[0] >= R(DA_TINY);
            }
            __syncwarp();
            if (lane == 0 && word) active[i >> 5] = 0u;
            const bool any_wet = __syncthreads_or(wet_after);
            const double tv = block_sum(vol, red);
            if (threadIdx.x == 0) {
                tile_vol[t] = tv;
                clean[t] = tile_active ? 0 : 1;
                tile_wet[t] = any_wet ? 1 : 0;
                if (RECORD) {
                    tile_epoch[t] = rec_id;
                    tile_act[t] = tile_active ? 1 : 0;
                }
            }
        }
    }
    (void)vol_part;
    if (last_block(&sc->blocks_done[1])) {
        double t = 0.0;
        for (int b = threadIdx.x; b < ntiles; b += blockDim.x) t += ((volatile double *)tile_vol)[b];
        t = block_sum(t, red);
        if (threadIdx.x == 0) {
            sc->volume = t;
            sc->blocks_done[1] = 0;
        }
    }
}

template <class R>
int launch_step_t(da_ctx *ctx, uint8_t *record_mask = nullptr) {
    const MeshArgs m = mesh_args(ctx);
    const int c = ctx->cur, o = 1 - c;
    StateRef<R> U{(const R *)ctx->U[c][0], (const R *)ctx->U[c][1], (const R *)ctx->U[c][2]};
    StateOut<R> O{(R *)ctx->U[o][0], (R *)ctx->U[o][1], (R *)ctx->U[o][2]};
    R *kact = (R *)ctx->kact;
    const int tiles = ctx->ntiles, grid = ctx->nblocks, cull = ctx->p.tile_culling;
    if (record_mask) {
        // branch recording for the adjoint: codes and flags for every cell of the listed tiles
        ++ctx->rec_id;
        trace_begin(ctx, TR_COEF_REC);
        k_coef<R, true><<<grid, kBlock, 0, ctx->stream>>>(m, U, kact, ctx->active, ctx->tile_wet, tiles, cull,
                                                          ctx->mc, ctx->tc, ctx->dsc, record_mask);
        trace_end(ctx);
        trace_begin(ctx, TR_UPDATE_REC);
        k_update<R, true><<<grid, kBlock, 0, ctx->stream>>>(m, U, O, kact, ctx->active, ctx->clean, ctx->tile_wet,
                                                            ctx->tile_vol, tiles, cull, ctx->mc, ctx->dsc, ctx->vol_part,
                                                            record_mask, ctx->tile_epoch, ctx->tile_act, ctx->rec_id);
        trace_end(ctx);
    } else {
        trace_begin(ctx, TR_COEF);
        k_coef<R><<<grid, kBlock, 0, ctx->stream>>>(m, U, kact, ctx->active, ctx->tile_wet, tiles, cull, ctx->mc,
                                                    ctx->tc, ctx->dsc);
        trace_end(ctx);
        trace_begin(ctx, TR_UPDATE);
        k_update<R><<<grid, kBlock, 0, ctx->stream>>>(m, U, O, kact, ctx->active, ctx->clean, ctx->tile_wet,
                                                      ctx->tile_vol, tiles, cull, ctx->mc, ctx->dsc, ctx->vol_part);
        trace_end(ctx);
    }
    ctx->cur = o;
    return cuda_check(ctx, cudaGetLastError(), "forward step launch");
}

}  // namespace
}  // namespace fwd
}  // namespace da
