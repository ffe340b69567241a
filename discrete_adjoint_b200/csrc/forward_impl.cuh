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

#include <type_traits>

#include "fv_device.cuh"
#include "snapshot_impl.cuh"

namespace da {
namespace fwd {
namespace {  // internal linkage: each precision TU keeps its own copy

using namespace fv;

constexpr int kBlock = kTileCells;  // one thread per cell of a tile
constexpr unsigned long long kAllSegs = 0x0101010101010101ull;  // a flag byte set in all 8 segments
constexpr int kVolParts = 256;  // fixed partition of the volume sum

// The 8 one-byte segment flags of tile t as one 8-byte load (flag arrays are padded to tiles).
__device__ __forceinline__ unsigned long long seg_flags(const uint8_t *flags, int t) {
    return *reinterpret_cast<const unsigned long long *>(flags + (size_t)t * 8);
}

// dt from the reduced CFL bound and hmax (get_coef_and_eigen.C:168-179 with the single-rank
// MPI_Allreduce(MIN)), then TimeProps::incrtime.  frict_tiny follows hpfem.C:232-235 with the
// iteration count before the increment.  Its callers report a dt that is not finite as
// DA_ERR_NAN: with no wet cell, no flux source and no output or end time it is infinite, and the
// reference's next update is NaN in every cell, which stops its run (residual.C:272-273).
__device__ __forceinline__ void step_dt(double min_dxe, double hmax, double time, long long iter,
                                        const TimeConsts &tc, double &dt_out, double &ft_out) {
    const double g0 = 0.5 * min_dxe;
    const double g1 = -0.9 * sqrt(hmax * (tc.epsilon) * (tc.gravity_scale) / 9.8);
    double dt = 0.5 * (g0 > -g1 ? -g1 : g0);
    if (dt == 0.0) dt = 0.5 * tc.influx_dt;
    if (time + dt > tc.next_output) dt = tc.next_output - time;
    if (time + dt > tc.next_save) dt = tc.next_save - time;
    if (time + dt > tc.max_time) dt = tc.max_time - time;
    if (tc.dt_replay) {
        // frozen time-step sequence (tangent/finite-difference checks of the adjoint)
        const long long k = iter - tc.iter0;
        dt = (k >= 0 && k < tc.n_replay) ? tc.dt_replay[k] : 0.0;
    }
    dt_out = dt;
    ft_out = iter < tc.frict_tiny_iters ? tc.frict_tiny_early : tc.frict_tiny_late;
}

constexpr unsigned long long kMinDxeStart = 0x416312D000000000ull;  // bits of 1e7, get_coef_and_eigen.C:36

__device__ void finalize_dt(DevScalars *sc, const TimeConsts &tc) {
    const double min_dxe = __longlong_as_double(*(volatile unsigned long long *)&sc->acc_min_dxe);
    const double hmax = __longlong_as_double(*(volatile unsigned long long *)&sc->acc_hmax);
    const double time = sc->time;
    double dt, ft;
    step_dt(min_dxe, hmax, time, sc->iter, tc, dt, ft);
    if (!isfinite(dt)) raise_err(sc, DA_ERR_NAN);
    sc->frict_tiny = ft;
    sc->dt = dt;
    sc->time = time + dt;
    sc->min_dxe = min_dxe;
    sc->hmax = hmax;
    sc->iter += 1;
    sc->acc_min_dxe = kMinDxeStart;
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


// Warp-reduced CFL min / hmax into one accumulator pair.
__device__ __forceinline__ void push_minmax(unsigned long long my_min, unsigned long long my_max,
                                            unsigned long long *acc_min, unsigned long long *acc_max) {
    my_min = warp_min_u64(my_min);
    my_max = warp_max_u64(my_max);
    if ((threadIdx.x & 31) == 0) {
        if (my_min != 0x7FF0000000000000ull) atomicMin(acc_min, my_min);
        if (my_max) atomicMax(acc_max, my_max);
    }
}

// ----------------------------------------------------------------------------- k_coef
// One thread per cell of each listed tile.  With tile culling, a tile none of whose 32-cell
// segments held a wet cell after the last update is not listed (its depths cannot have changed
// since).  Wet cells
// (h >= GEOFLOW_TINY) also mark themselves and their face neighbours in the active bitmask that
// k_update reads: a cell outside that set has zero fluxes and no sources this step.
// RECORD: also writes the branch code of every cell of a listed tile into mask (0 dry / at rest,
// 1..3 for sgn(vel) = -1, 0, +1 of gmfggetcoef) for the adjoint's replay.
// The thread's CFL min and hmax (bit patterns of positive doubles) accumulate in my_min / my_max.
// BATCH (ensemble): the tile's member gives the material constants, and the CFL values go to the
// member's accumulators after every tile.
template <class R, bool RECORD, bool BATCH = false>
__device__ __forceinline__ void coef_phase(const MeshArgs &m, const StateRef<R> &U, R *kact, unsigned *active,
                                           const uint8_t *seg_wet, int ntiles, int cull, const MatConsts &mc0,
                                           DevScalars *sc, uint8_t *mask, int *list, unsigned long long &my_min,
                                           unsigned long long &my_max, const InstArgs &ia) {
    for (int round = 0; sched_more(round, ntiles); ++round) {
        const int tq = sched_tile(round);
        const bool need = tq < ntiles && (!cull || seg_flags(seg_wet, tq) != 0ull);
        const int cnt = compact_tiles(need, tq, list);
        for (int q = 0; q < cnt; ++q) {
            const int t = list[q];
            const int inst = BATCH ? ia.tile_inst[t] : 0;
            const MatConsts &mc = BATCH ? ia.mcs[inst] : mc0;
            const int i = t * kBlock + threadIdx.x;
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
                        cell_slopes<R>(global_view<R>(m, U, kact), i, bf, R(mc.gamma), ui, s);
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
                        if (i < m.n_owned) {  // ghost cells are another subdomain's
                            my_min = rb < my_min ? rb : my_min;
                            my_max = hb > my_max ? hb : my_max;
                        }
                    }
                }
                if (RECORD) mask[i] = code;
            }
            const unsigned self = __ballot_sync(0xffffffffu, wet);
            if (self && (threadIdx.x & 31) == 0) atomicOr(&active[i >> 5], self);
            if (BATCH) {
                push_minmax(my_min, my_max, ia.acc_min + inst, ia.acc_max + inst);
                my_min = 0x7FF0000000000000ull;
                my_max = 0ull;
            }
        }
    }
}

// bounds (or null): the step's first half alone -- the last block writes the subdomain's CFL bound
// and -hmax to bounds[0..1] instead of forming dt, so that one MIN all-reduce over the two doubles
// combines the subdomains (get_coef_and_eigen.C:173) before k_apply_bounds forms dt.
template <class R, bool RECORD = false>
__global__ void __launch_bounds__(kBlock) k_coef(MeshArgs m, StateRef<R> U, R *__restrict__ kact,
                                                 unsigned *__restrict__ active, const uint8_t *__restrict__ seg_wet,
                                                 int ntiles, int cull, MatConsts mc, TimeConsts tc, DevScalars *sc,
                                                 uint8_t *__restrict__ mask = nullptr, double *bounds = nullptr) {
    __shared__ int list[kBlock];
    unsigned long long my_min = 0x7FF0000000000000ull;  // +inf
    unsigned long long my_max = 0ull;
    coef_phase<R, RECORD>(m, U, kact, active, seg_wet, ntiles, cull, mc, sc, mask, list, my_min, my_max, InstArgs{});
    push_minmax(my_min, my_max, &sc->acc_min_dxe, &sc->acc_hmax);
    if (last_block(&sc->blocks_done[0])) {
        if (threadIdx.x == 0) {
            if (bounds) {
                volatile unsigned long long *acc = &sc->acc_min_dxe, *acx = &sc->acc_hmax;
                bounds[0] = __longlong_as_double(*acc);
                bounds[1] = -__longlong_as_double(*acx);
                sc->acc_min_dxe = kMinDxeStart;
                sc->acc_hmax = 0ull;
            } else {
                finalize_dt(sc, tc);
            }
            sc->blocks_done[0] = 0;
        }
    }
}

// dt of the combined subdomains: bounds = the MIN all-reduce of every subdomain's k_coef bounds.
__global__ void k_apply_bounds(DevScalars *sc, TimeConsts tc, const double *bounds) {
    sc->acc_min_dxe = __double_as_longlong(bounds[0]);
    sc->acc_hmax = __double_as_longlong(-bounds[1]);
    finalize_dt(sc, tc);
}

// The flux differences F(+side) - F(-side) of one cell in x (div[0]) and y (div[1]): the edge
// fluxes calc_edge_states leaves on the cell's edge nodes (element2.C:2745-3072, hanging sides
// averaged on the coarse side), an outflow direction exactly 0 (boundary_flux, :3374-3411).
template <class R, class V>
__device__ __forceinline__ void flux_div(const V &v, int i, uint8_t bf, const R prev[3], R div[2][3]) {
    const R ki = prev[0] >= R(DA_TINY) ? v.k(i) : R(0);
    const R gz = v.gz(i);
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
        side_flux<R>(v, i, bf, d + 2, self, Fm);
        side_flux<R>(v, i, bf, d, self, Fp);
#pragma unroll
        for (int v = 0; v < 3; ++v) div[d][v] = Fp[v] - Fm[v];
    }
}

// Full corrector update of one active cell (fluxes + sources), reference order.  c is the cell in
// the view; cs its source coefficients (read only for a wet cell, h > GEOFLOW_TINY); hook(f,
// clamped) runs for a wet cell with the slopes, velocities and friction signs of its sources.
// pre_s (or null): the cell's limited slopes as the coefficient phase computed them from the same
// state (the same bits cell_slopes gives here).
template <class R, class V, class Hook = NoSrcHook>
__device__ __forceinline__ bool update_cell(const V &v, int c, uint8_t bf, const CellSrc<R> &cs, const MatConsts &mc,
                                            R dt, R ft, const R prev[3], R dxc, R dyc, R st[3],
                                            const R *pre_s = nullptr, const Hook &hook = Hook{}) {
    const R ki = prev[0] >= R(DA_TINY) ? v.k(c) : R(0);
    const R gz = v.gz(c);
    const R g0 = cs.g[0], g1 = cs.g[1], dg0 = cs.dg[0], dg1 = cs.dg[1], cv0 = cs.cv[0], cv1 = cs.cv[1];
    const int mat = cs.mat;
    R div[2][3];
    flux_div<R>(v, c, bf, prev, div);
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
        if (pre_s) {
#pragma unroll
            for (int j = 0; j < 6; ++j) s[j] = pre_s[j];
        } else {
            cell_slopes<R>(v, c, bf, R(mc.gamma), prev, s);
        }
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
        // the reverse step's source adjoint of this cell, from these same values (its branches)
        hook(SrcFwd<R>{{s[0], s[1], s[2], s[3], s[4], s[5]}, vel0, vel1, h_inv, sg0, sg1, sg2, sg3}, clamped);
        const R sin_int = R(mc.sin_int);
        const R tan_bed = R(mc.tan_bed[mat]);
        R s1 = g0 * prev[0];
        R s2 = sg0 * prev[0] * ki * (gz * s[3] + dg1 * prev[0]) * sin_int;
        R s3 = sg2 * rmax(gz * prev[0] + vel0 * prev[1] * cv0, R(0.0)) * tan_bed;
        st[1] += dt * (s1 - s2 - s3);
        s1 = g1 * prev[0];
        s2 = sg1 * prev[0] * ki * (gz * s[0] + dg0 * prev[0]) * sin_int;
        s3 = sg3 * rmax(gz * prev[0] + vel1 * prev[2] * cv1, R(0.0)) * tan_bed;
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
// Tiles of kBlock consecutive cells through the strided tile list; each warp owns one 32-cell
// segment of a tile and keeps that segment's flags, so a tile needs no block-wide step.  A tile
// is listed when a cell of it is active, when a segment's two ping-pong buffers differ (not
// clean), or when culling is off.  In a listed tile, active cells get the full update and the
// others are copied (their update is the identity); a tile that is not listed is already
// identical in both buffers.  Each segment stores its volume partial (the volume is their sum in
// a fixed order, so it depends neither on culling nor on the grid), its clean flag and whether it
// now holds a wet cell.
// RECORD: every cell of a listed tile gets its full mask byte (the k_coef code of a wet cell,
// bit 3 active, bit 2 depth clamped), the tile records the step id (tile_epoch) and each segment
// whether it had an active cell (seg_act); masks of tiles with another epoch count as zero.
template <class R, bool RECORD, bool BATCH = false>
__device__ __forceinline__ void update_phase(const MeshArgs &m, const StateRef<R> &U, const StateOut<R> &O,
                                             const R *kact, unsigned *active, uint8_t *seg_clean, uint8_t *seg_wet,
                                             double *seg_vol, uint8_t *seg_dirty, int ntiles, int cull,
                                             const MatConsts &mc0,
                                             DevScalars *sc, R dt0, R ft, uint8_t *mask, int *tile_epoch,
                                             uint8_t *seg_act, int rec_id, int *list, const InstArgs &ia) {
    const int lane = threadIdx.x & 31;
    for (int round = 0; sched_more(round, ntiles); ++round) {
        const int tq = sched_tile(round);
        bool need = false;
        if (tq < ntiles) {
            need = !cull || seg_flags(seg_clean, tq) != kAllSegs;
            if (!need) {
                // the tile's 8 bitmask words in two 16-byte loads (the bitmask is padded to
                // whole tiles)
                const uint4 *w4 = reinterpret_cast<const uint4 *>(active + (size_t)tq * (kBlock / 32));
                const uint4 a = w4[0], b = w4[1];
                need = (a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w) != 0u;
            }
        }
        const int cnt = compact_tiles(need, tq, list);
        for (int q = 0; q < cnt; ++q) {
            const int t = list[q];
            const int inst = BATCH ? ia.tile_inst[t] : 0;
            const MatConsts &mc = BATCH ? ia.mcs[inst] : mc0;
            const R dt = BATCH ? R(ia.dt[inst]) : dt0;
            const int i = t * kBlock + threadIdx.x;
            const int seg = i >> 5;
            const unsigned word = active[seg];  // padded: bits of cells >= n are never set
            double vol = 0.0;
            bool wet_after = false;
            if (i < m.n) {
                const R prev[3] = {U.h[i], U.hu[i], U.hv[i]};
                const R dxc = cell_dx<R>(m, i), dyc = cell_dy<R>(m, i);
                R st[3] = {prev[0], prev[1], prev[2]};
                const bool act = word & (1u << lane);
                bool clamped = false;
                if (act) {
                    const CellSrc<R> cs = prev[0] > R(DA_TINY) ? cell_src<R>(m, i) : CellSrc<R>{};
                    clamped = update_cell<R>(global_view<R>(m, U, kact), i, m.bflag[i], cs, mc, dt, ft, prev, dxc, dyc,
                                             st);
                }
                if (RECORD)
                    mask[i] = uint8_t((prev[0] >= R(DA_TINY) ? (mask[i] & 3) : 0) | (act ? 8 : 0) | (clamped ? 4 : 0));
                if (!isfinite(st[0]) || !isfinite(st[1]) || !isfinite(st[2])) raise_err(sc, DA_ERR_NAN);
                O.h[i] = st[0];
                O.hu[i] = st[1];
                O.hv[i] = st[2];
                if (i < m.n_owned) vol = double(dxc) * double(dyc) * double(st[0]);
                wet_after = st[0] >= R(DA_TINY);
            }
            const unsigned wet_bits = __ballot_sync(0xffffffffu, wet_after);
            vol = warp_sum(vol);
            if (lane == 0) {
                if (word) {
                    active[seg] = 0u;
                    seg_dirty[seg] = 1;  // changed since the base checkpoint
                }
                seg_vol[seg] = vol;
                seg_clean[seg] = word ? 0 : 1;
                seg_wet[seg] = wet_bits ? 1 : 0;
                if (RECORD) seg_act[seg] = word ? 1 : 0;
            }
            if (RECORD && threadIdx.x == 0) tile_epoch[t] = rec_id;
        }
    }
}

template <class R, bool RECORD = false>
__global__ void __launch_bounds__(kBlock) k_update(MeshArgs m, StateRef<R> U, StateOut<R> O,
                                                   const R *__restrict__ kact, unsigned *__restrict__ active,
                                                   uint8_t *__restrict__ seg_clean, uint8_t *__restrict__ seg_wet,
                                                   double *__restrict__ seg_vol, uint8_t *__restrict__ seg_dirty,
                                                   int ntiles, int cull, MatConsts mc,
                                                   DevScalars *sc, uint8_t *__restrict__ mask = nullptr,
                                                   int *__restrict__ tile_epoch = nullptr,
                                                   uint8_t *__restrict__ seg_act = nullptr, int rec_id = 0) {
    __shared__ int list[kBlock];
    const R dt = R(sc->dt);
    const R ft = R(sc->frict_tiny) > R(mc.sign_floor) ? R(sc->frict_tiny) : R(mc.sign_floor);
    update_phase<R, RECORD>(m, U, O, kact, active, seg_clean, seg_wet, seg_vol, seg_dirty, ntiles, cull, mc, sc, dt, ft, mask,
                            tile_epoch, seg_act, rec_id, list, InstArgs{});
}

// ---------------------------------------------------------------------------- volume
// sum of dx dy h over the mesh (step.C:205) from the segments' partials, in a fixed order: block
// b of kVolParts sums a fixed contiguous range of segments, then one block adds the parts.
// Launched only when the volume is asked for.
__global__ void __launch_bounds__(kBlock) k_volume_parts(const double *__restrict__ seg_vol, int nseg,
                                                         double *__restrict__ parts) {
    __shared__ double red[kBlock / 32];
    const int per = (nseg + kVolParts - 1) / kVolParts;
    const int s0 = blockIdx.x * per, s1 = min(nseg, s0 + per);
    double acc = 0.0;
    for (int s = s0 + threadIdx.x; s < s1; s += kBlock) acc += seg_vol[s];
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) parts[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kVolParts) k_volume_final(const double *__restrict__ parts, DevScalars *sc) {
    __shared__ double red[kVolParts / 32];
    const double v = warp_sum(parts[threadIdx.x]);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kVolParts / 32; ++w) t += red[w];
        sc->volume = t;
    }
}

}  // namespace
}  // namespace fwd
}  // namespace da

#include "staged_impl.cuh"

namespace da {
namespace fwd {
namespace {

// ---------------------------------------------------------------------------- k_steps
// nsteps whole steps in one cooperative launch (all blocks resident): per step the coefficient
// phase, a grid barrier, dt (every block forms the same dt from the same reduced values), the
// update phase and a second barrier.  Odd and even steps accumulate the CFL min / hmax in two
// pairs, so block 0 can restart one pair while the other is read.  time and iteration advance
// in registers; block 0 writes them and the last step's scalars at the end.  The
// state buffers alternate as in single steps and are read with coherent loads (no read-only
// cache: other blocks wrote them earlier in the same launch).
// The barrier is one 64-bit word (arrivals in the low half, generation in the high half): a block
// arrives with one atomic add (acquire-release at GPU scope, after the block's own barrier, so that
// every write of the block before it is released); the last one to arrive moves the word to the
// next generation with zero arrivals in one more such add; the others poll the word with acquire
// loads.  The waits are bounded: after ~4 s a block raises DA_ERR_TIMEOUT and returns, and the
// others give up when they see the error (checked on arrival and every 256 polls).
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long bar_add(unsigned long long *p, unsigned long long v) {
    unsigned long long old;
    asm volatile("atom.add.acq_rel.gpu.global.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned long long bar_load(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Waits for every block of the (co-resident) grid.  One atomic per block: the barrier word counts
// the arrivals since the launch began, so barrier k of a grid of G blocks is open once it reaches
// G (k + 1) -- the last arrival has nothing more to do, the others poll the word.  The wait is
// bounded: after limit_ns (4 s by default) or 2^26 polls a block raises DA_ERR_TIMEOUT and returns
// false, and so does every block that arrives or polls after that; the host restarts the barrier
// word when it reads the error.  A launch that ends normally restarts it itself (grid_exit).
__device__ __forceinline__ bool grid_sync(DevScalars *sc, unsigned long long limit_ns = 4000000000ull) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile int *err = &sc->err;
        int good = *err != DA_ERR_TIMEOUT;
        const unsigned long long old = bar_add(&sc->bar, 1ull);
        const unsigned long long G = gridDim.x;
        const unsigned long long target = (old / G + 1) * G;
        if (old + 1 != target) {
            const unsigned long long t0 = global_ns();
            for (unsigned it = 1; bar_load(&sc->bar) < target; ++it) {
                if ((it & 255u) == 0 &&
                    (*err == DA_ERR_TIMEOUT || it > (1u << 26) || global_ns() - t0 > limit_ns)) {
                    atomicCAS(&sc->err, 0, DA_ERR_TIMEOUT);
                    good = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// The end of a cooperative launch that passed all its barriers: the last block to leave (every
// other block has finished polling by then) puts the barrier word back at 0 for the next launch.
__device__ __forceinline__ void grid_exit(DevScalars *sc) {
    if (threadIdx.x == 0) {
        const unsigned long long old = bar_add(&sc->bar_exit, 1ull);
        if (old == gridDim.x - 1) {
            sc->bar = 0ull;
            sc->bar_exit = 0ull;
        }
    }
}

template <class R>
struct StatePair {
    R *h[2];
    R *hu[2];
    R *hv[2];
};

// The checkpoint stores inside a multi-step launch (MidStoreList on the device): the arrays of
// each slot and the number of segments.
template <class R>
struct MidStores {
    int n, nseg;
    int after[kMidStores];
    R *snap[kMidStores][3];
    uint8_t *dirty[kMidStores];
    DevScalars *ssc[kMidStores];
};

// Ensemble: the dt of every member from its reduced CFL values (threads over members), its time
// advanced, its accumulators restarted.  Runs between two grid barriers.
__device__ __forceinline__ void inst_dt_pass(const InstArgs &ia, long long iter, const TimeConsts &tc, DevScalars *sc) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < ia.ninst; k += gridDim.x * blockDim.x) {
        const double mn = __longlong_as_double(__ldcg(ia.acc_min + k));
        const double hx = __longlong_as_double(__ldcg(ia.acc_max + k));
        const double time = ia.time[k];
        double dt, ft;
        step_dt(mn, hx, time, iter, tc, dt, ft);
        if (!isfinite(dt)) raise_err(sc, DA_ERR_NAN);
        ia.dt[k] = dt;
        ia.time[k] = time + dt;
        ia.min_dxe[k] = mn;
        ia.hmax[k] = hx;
        ia.acc_min[k] = kMinDxeStart;
        ia.acc_max[k] = 0ull;
    }
}

// BATCH: every member of the ensemble steps with its own dt (a third barrier per step after the
// members' dt pass); the shared iteration count lives in the scalars.  OCC: resident blocks per
// SM the register budget is set for (da_params.blocks_per_sm).  STAGED: the phases stage each
// tile and its halo in dynamic shared memory (staged_impl.cuh).
template <class R, bool BATCH = false, int OCC = 2, bool STAGED = false, bool MID = false>
__global__ void __launch_bounds__(kBlock, OCC) k_steps(MeshArgs m, StatePair<R> S, int cur, int nsteps, R *kact,
                                                  unsigned *active, uint8_t *seg_clean, uint8_t *seg_wet,
                                                  double *seg_vol, uint8_t *seg_dirty, int ntiles, int cull,
                                                  MatConsts mc, TimeConsts tc, DevScalars *sc, InstArgs ia,
                                                  snap::SnapArgs<R> pre, snap::SnapArgs<R> post, HaloArgs ha,
                                                  MidStores<R> mid) {
    __shared__ int list[kBlock];
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    StageSmem<R> &stg = *reinterpret_cast<StageSmem<R> *>(dyn_smem);
    if (pre.mode != snap::NONE) {
        // a checkpoint restore first (both buffers, flags, scalars), then a barrier
        snap::snap_segments<R>(pre);
        snap::snap_scalars<R>(pre);
        if (!grid_sync(sc)) return;
    }
    double time = __ldcg(&sc->time);
    long long iter = __ldcg(&sc->iter);
    double dt = __ldcg(&sc->dt), ft = __ldcg(&sc->frict_tiny), min_dxe = __ldcg(&sc->min_dxe),
           hmax = __ldcg(&sc->hmax);
    int ms = 0;  // the next of the launch's checkpoint stores
    for (int s = 0; s < nsteps; ++s) {
        const int c = (cur + s) & 1, p = s & 1;
        unsigned long long *acc_min = p ? &sc->acc_alt_min_dxe : &sc->acc_min_dxe;
        unsigned long long *acc_max = p ? &sc->acc_alt_hmax : &sc->acc_hmax;
        const StateRef<R> U{S.h[c], S.hu[c], S.hv[c]};
        const StateOut<R> O{S.h[c ^ 1], S.hu[c ^ 1], S.hv[c ^ 1]};
        unsigned long long my_min = 0x7FF0000000000000ull, my_max = 0ull;
        if (STAGED)
            coef_phase_staged<R, false, BATCH>(m, ha, U, kact, active, seg_wet, ntiles, cull, mc, sc, nullptr, list,
                                               my_min, my_max, ia, stg);
        else
            coef_phase<R, false, BATCH>(m, U, kact, active, seg_wet, ntiles, cull, mc, sc, nullptr, list, my_min,
                                        my_max, ia);
        if (!BATCH) push_minmax(my_min, my_max, acc_min, acc_max);
        if (!grid_sync(sc)) return;
        if (BATCH) {
            ft = iter < tc.frict_tiny_iters ? tc.frict_tiny_early : tc.frict_tiny_late;
            inst_dt_pass(ia, iter, tc, sc);
            iter += 1;
            if (!grid_sync(sc)) return;
        } else {
            min_dxe = __longlong_as_double(__ldcg(acc_min));
            hmax = __longlong_as_double(__ldcg(acc_max));
            step_dt(min_dxe, hmax, time, iter, tc, dt, ft);
            time += dt;
            iter += 1;
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                if (!isfinite(dt)) raise_err(sc, DA_ERR_NAN);
                // read by every block before this step's first barrier; used again next step
                *(p ? &sc->acc_min_dxe : &sc->acc_alt_min_dxe) = kMinDxeStart;
                *(p ? &sc->acc_hmax : &sc->acc_alt_hmax) = 0ull;
            }
        }
        const R ftr = R(ft) > R(mc.sign_floor) ? R(ft) : R(mc.sign_floor);
        if (STAGED)
            update_phase_staged<R, false, BATCH>(m, ha, U, O, kact, active, seg_clean, seg_wet, seg_vol, seg_dirty,
                                                 ntiles, cull, mc, sc, R(dt), ftr, nullptr, nullptr, nullptr, 0, list,
                                                 ia, stg);
        else
            update_phase<R, false, BATCH>(m, U, O, kact, active, seg_clean, seg_wet, seg_vol, seg_dirty, ntiles, cull,
                                          mc, sc, R(dt), ftr, nullptr, nullptr, nullptr, 0, list, ia);
        if (!grid_sync(sc)) return;
        if (MID && ms < mid.n && mid.after[ms] == s) {
            // a checkpoint of the state after this step, with no barrier of its own: the next
            // two steps do not write this buffer, and the next update changes the dirty flags
            // only after the next barrier, which every block reaches after its part of the copy
            snap::store_segments<R>(O.h, O.hu, O.hv, mid.snap[ms][0], mid.snap[ms][1], mid.snap[ms][2], seg_dirty,
                                    mid.dirty[ms], mid.nseg, m.n);
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                // the step scalars as a launch ending after this step leaves them
                DevScalars *d = mid.ssc[ms];
                snap::copy_step_scalars(d, sc);
                d->time = time;
                d->dt = dt;
                d->hmax = hmax;
                d->min_dxe = min_dxe;
                d->frict_tiny = ft;
                d->iter = iter;
                d->acc_min_dxe = d->acc_alt_min_dxe = kMinDxeStart;
                d->acc_hmax = d->acc_alt_hmax = 0ull;
            }
            ++ms;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->iter = iter;
        sc->frict_tiny = ft;
        if (!BATCH) {
            sc->time = time;
            sc->dt = dt;
            sc->min_dxe = min_dxe;
            sc->hmax = hmax;
            sc->acc_min_dxe = sc->acc_alt_min_dxe = kMinDxeStart;
            sc->acc_hmax = sc->acc_alt_hmax = 0ull;
        }
    }
    if (post.mode != snap::NONE) {
        // a checkpoint store of the state after the last step (every block has passed the last
        // barrier; block 0's thread 0 has just written the scalars it copies)
        snap::snap_segments<R>(post);
        snap::snap_scalars<R>(post);
    }
    grid_exit(sc);
}

template <class R>
int launch_step_t(da_ctx *ctx, uint8_t *record_mask = nullptr) {
    const MeshArgs m = mesh_args(ctx);
    const int c = ctx->cur, o = 1 - c;
    StateRef<R> U{(const R *)ctx->U[c][0], (const R *)ctx->U[c][1], (const R *)ctx->U[c][2]};
    StateOut<R> O{(R *)ctx->U[o][0], (R *)ctx->U[o][1], (R *)ctx->U[o][2]};
    R *kact = (R *)ctx->kact;
    const int tiles = ctx->ntiles, grid = ctx->grid, cull = ctx->p.tile_culling;
    if (record_mask) {
        // branch recording for the adjoint: codes and flags for every cell of the listed tiles
        ++ctx->rec_id;
        trace_begin(ctx, TR_COEF_REC);
        k_coef<R, true><<<grid, kBlock, 0, ctx->stream>>>(m, U, kact, ctx->active, ctx->seg_wet, tiles, cull,
                                                          ctx->mc, ctx->tc, ctx->dsc, record_mask);
        trace_end(ctx);
        trace_begin(ctx, TR_UPDATE_REC);
        k_update<R, true><<<grid, kBlock, 0, ctx->stream>>>(m, U, O, kact, ctx->active, ctx->seg_clean, ctx->seg_wet,
                                                            ctx->seg_vol, ctx->seg_dirty, tiles, cull, ctx->mc, ctx->dsc,
                                                            record_mask,
                                                            ctx->tile_epoch, ctx->seg_act, ctx->rec_id);
        trace_end(ctx);
    } else {
        trace_begin(ctx, TR_COEF);
        k_coef<R><<<grid, kBlock, 0, ctx->stream>>>(m, U, kact, ctx->active, ctx->seg_wet, tiles, cull, ctx->mc,
                                                    ctx->tc, ctx->dsc);
        trace_end(ctx);
        trace_begin(ctx, TR_UPDATE);
        k_update<R><<<grid, kBlock, 0, ctx->stream>>>(m, U, O, kact, ctx->active, ctx->seg_clean, ctx->seg_wet,
                                                      ctx->seg_vol, ctx->seg_dirty, tiles, cull, ctx->mc, ctx->dsc);
        trace_end(ctx);
    }
    ctx->cur = o;
    return cuda_check(ctx, cudaGetLastError(), "forward step launch");
}

// One step in two halves for a subdomain: half 0 is the coefficient phase writing bounds (device
// memory), half 1 forms dt from the all-reduced bounds and runs the update phase.
template <class R>
int launch_step_half_t(da_ctx *ctx, int half, double *bounds) {
    const MeshArgs m = mesh_args(ctx);
    const int c = ctx->cur, o = 1 - c;
    StateRef<R> U{(const R *)ctx->U[c][0], (const R *)ctx->U[c][1], (const R *)ctx->U[c][2]};
    R *kact = (R *)ctx->kact;
    const int tiles = ctx->ntiles, grid = ctx->grid, cull = ctx->p.tile_culling;
    if (half == 0) {
        trace_begin(ctx, TR_COEF);
        k_coef<R><<<grid, kBlock, 0, ctx->stream>>>(m, U, kact, ctx->active, ctx->seg_wet, tiles, cull, ctx->mc,
                                                    ctx->tc, ctx->dsc, nullptr, bounds);
        trace_end(ctx);
    } else {
        StateOut<R> O{(R *)ctx->U[o][0], (R *)ctx->U[o][1], (R *)ctx->U[o][2]};
        k_apply_bounds<<<1, 1, 0, ctx->stream>>>(ctx->dsc, ctx->tc, bounds);
        trace_begin(ctx, TR_UPDATE);
        k_update<R><<<grid, kBlock, 0, ctx->stream>>>(m, U, O, kact, ctx->active, ctx->seg_clean, ctx->seg_wet,
                                                      ctx->seg_vol, ctx->seg_dirty, tiles, cull, ctx->mc, ctx->dsc);
        trace_end(ctx);
        ctx->cur = o;
    }
    return cuda_check(ctx, cudaGetLastError(), "forward half-step launch");
}

// nsteps steps in one cooperative launch of k_steps; the grid is capped at the number of blocks
// that can be resident at once (the launch fails otherwise, it never deadlocks).
// pre_slot / post_slot (or null): a checkpoint slot restored before the first step / stored after
// the last one, in the same launch.
template <class R>
int launch_steps_t(da_ctx *ctx, int nsteps, void *pre_slot, void *post_slot, const MidStoreList *ml = nullptr) {
    if (nsteps <= 0) return DA_OK;
    const bool batch = ctx->ninst > 0;
    const int occ3 = ctx->p.blocks_per_sm == 3;
    const bool staged = staged_ok(ctx);
    // the checkpoint stores inside a launch are compiled only into their own single-instance
    // kernels: the plain ones keep their register allocation
    const bool mids = ml && ml->n > 0 && !batch;
    const void *kern;
    if (mids)
        kern = staged ? (occ3 ? (const void *)k_steps<R, false, 3, true, true>
                              : (const void *)k_steps<R, false, 2, true, true>)
                      : (occ3 ? (const void *)k_steps<R, false, 3, false, true>
                              : (const void *)k_steps<R, false, 2, false, true>);
    else if (staged)
        kern = batch ? (occ3 ? (const void *)k_steps<R, true, 3, true> : (const void *)k_steps<R, true, 2, true>)
                     : (occ3 ? (const void *)k_steps<R, false, 3, true> : (const void *)k_steps<R, false, 2, true>);
    else
        kern = batch ? (occ3 ? (const void *)k_steps<R, true, 3> : (const void *)k_steps<R, true, 2>)
                     : (occ3 ? (const void *)k_steps<R, false, 3> : (const void *)k_steps<R, false, 2>);
    const size_t smem = staged ? stage_smem_bytes<R>() : 0;
    int &cap_ref = ctx->coop_cap[(sizeof(R) == 8) + 2 * batch + 4 * occ3 + 8 * staged + 16 * mids];
    if (cap_ref <= 0) {
        int st = DA_OK;
        if (staged)
            st = cuda_check(ctx, cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                            "shared memory attribute");
        int per_sm = 0;
        if (!st)
            st = cuda_check(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kBlock, smem),
                            "occupancy");
        if (st) return st;
        cap_ref = per_sm * (ctx->sm_count > 0 ? ctx->sm_count : 1);
    }
    const int cap = cap_ref;
    if (cap <= 0) return set_error(ctx, DA_ERR_UNSUPPORTED, "multi-step kernel cannot be resident");
    const int grid = ctx->grid < cap ? ctx->grid : cap;
    MeshArgs m = mesh_args(ctx);
    StatePair<R> S;
    for (int b = 0; b < 2; ++b) {
        S.h[b] = (R *)ctx->U[b][0];
        S.hu[b] = (R *)ctx->U[b][1];
        S.hv[b] = (R *)ctx->U[b][2];
    }
    int cur = ctx->cur, n = nsteps, ntiles = ctx->ntiles, cull = ctx->p.tile_culling;
    R *kact = (R *)ctx->kact;
    unsigned *active = ctx->active;
    uint8_t *seg_clean = ctx->seg_clean, *seg_wet = ctx->seg_wet;
    double *seg_vol = ctx->seg_vol;
    uint8_t *seg_dirty = ctx->seg_dirty;
    MatConsts mc = ctx->mc;
    TimeConsts tc = ctx->tc;
    DevScalars *sc = ctx->dsc;
    InstArgs ia = ctx->ia;
    snap::SnapArgs<R> pre = pre_slot ? snap::snap_args<R>(ctx, pre_slot, false, cur) : snap::no_snap<R>();
    snap::SnapArgs<R> post =
        post_slot ? snap::snap_args<R>(ctx, post_slot, true, (cur + nsteps) & 1) : snap::no_snap<R>();
    HaloArgs ha = halo_args(ctx);
    MidStores<R> mid{};
    if (ml && ml->n > 0) {
        if (batch || ml->n > kMidStores || post_slot)
            return set_error(ctx, DA_ERR_INVALID, "multi-step launch: checkpoint stores inside an ensemble launch");
        for (int k = 0; k < ml->n; ++k) {
            if (ml->after[k] < 0 || ml->after[k] >= nsteps || (k > 0 && ml->after[k] <= ml->after[k - 1]) ||
                ml->slot[k] == ctx->snaps[0])
                return set_error(ctx, DA_ERR_INVALID, "multi-step launch: bad checkpoint store list");
            const snap::SnapArgs<R> a = snap::snap_args<R>(ctx, ml->slot[k], true, 0);
            mid.after[k] = ml->after[k];
            for (int v = 0; v < 3; ++v) mid.snap[k][v] = a.snap[v];
            mid.dirty[k] = a.snap_dirty;
            mid.ssc[k] = a.snap_sc;
        }
        mid.n = ml->n;
        mid.nseg = ctx->nseg;
    }
    void *args[] = {&m,         &S,      &cur,  &n,  &kact, &active, &seg_clean, &seg_wet, &seg_vol,
                    &seg_dirty, &ntiles, &cull, &mc, &tc,   &sc,     &ia,        &pre,     &post, &ha, &mid};
    trace_begin(ctx, TR_STEPS);
    const cudaError_t e = cudaLaunchCooperativeKernel(kern, grid, kBlock, args, smem, ctx->stream);
    trace_end(ctx, nsteps);
    if (e != cudaSuccess) return cuda_check(ctx, e, "multi-step launch");
    ctx->cur = (cur + nsteps) & 1;
    return DA_OK;
}

// The volume of the current state into the scalars (two launches, fixed order).
inline int launch_volume_t(da_ctx *ctx) {
    k_volume_parts<<<kVolParts, kBlock, 0, ctx->stream>>>(ctx->seg_vol, ctx->nseg, ctx->vol_parts);
    k_volume_final<<<1, kVolParts, 0, ctx->stream>>>(ctx->vol_parts, ctx->dsc);
    return cuda_check(ctx, cudaGetLastError(), "volume launch");
}

// ------------------------------------------------------------------------- refinement hand-back
// After a step: per cell the flux-balance weight el_error[0] = 2 (sum_j |dF_x,j| + |dF_y,j|)^2 /
// (dx + dy) + WEIGHT_ADJUSTER (Element::calc_flux_balance, element2.C:3705-3745) from the step's
// edge fluxes (recomputed from the previous state buffer and the step's k act/pass), and the
// pile-contour tests of H_adapt (Element::if_pile_boundary, element2.C:4020-4065, at GEOFLOW_TINY
// x 1, 5, 15, 40, hadpt.C:46-48,139-149) on the new state: flag bits 0-3.  Bit 4 (weight above the
// mean) is set by the second kernel once the mean is known.  Per-block partial sums of the weight
// over cells with hu > GEOFLOW_TINY (element_weight.C:36-79) in a fixed order.
__device__ __forceinline__ int pile_boundary(const MeshArgs &m, const double *hnew_d, const float *hnew_f, int i,
                                             double contour) {
    auto hv = [&](int k) { return hnew_d ? hnew_d[k] : double(hnew_f[k]); };
    const uint8_t bf = m.bflag[i];
    const bool in = hv(i) >= contour;
    for (int s = 0; s < 4; ++s) {
        if (bf & (1 << s)) continue;  // outside the map
        const int ne = (bf & (0x10 << s)) ? 2 : 1;  // a duplicate second slot is skipped
        for (int q = 0; q < ne; ++q) {
            const double hk = hv(m.nbr[(size_t)(s + 4 * q) * m.n + i]);
            if (in && hk < contour) return 2;
            if (!in && hk >= contour) return 1;
        }
    }
    return 0;
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_refine_info(MeshArgs m, StateRef<R> Uprev, StateRef<R> Unew,
                                                        const R *kact, double *el_error, uint8_t *flags,
                                                        double *parts) {
    __shared__ double s_sum[kBlock], s_cnt[kBlock];
    const int per = (m.n + kVolParts - 1) / kVolParts;
    const int i0 = blockIdx.x * per, i1 = min(m.n, i0 + per);
    double sum = 0.0, cnt = 0.0;
    const double *hd = sizeof(R) == 8 ? (const double *)Unew.h : nullptr;
    const float *hf = sizeof(R) == 8 ? nullptr : (const float *)Unew.h;
    for (int i = i0 + threadIdx.x; i < i1; i += kBlock) {
        const R prev[3] = {Uprev.h[i], Uprev.hu[i], Uprev.hv[i]};
        R div[2][3];
        flux_div<R>(global_view<R>(m, Uprev, kact), i, m.bflag[i], prev, div);
        double f = 0.0;
        for (int v = 0; v < 3; ++v) f += fabs(double(div[0][v])) + fabs(double(div[1][v]));
        const double dxc = double(cell_dx<R>(m, i)), dyc = double(cell_dy<R>(m, i));
        const double e = 2. * f * f / (dxc + dyc) + 1.0;  // WEIGHT_ADJUSTER (geoflow.h:22)
        el_error[i] = e;
        uint8_t fl = 0;
        const double contours[4] = {DA_TINY, 5 * DA_TINY, 15 * DA_TINY, 40 * DA_TINY};
        for (int c = 0; c < 4; ++c)
            if (pile_boundary(m, hd, hf, i, contours[c]) > 0) fl |= uint8_t(1u << c);
        flags[i] = fl;
        if (double(Unew.hu[i]) > DA_TINY) {
            sum += e;
            cnt += 1.0;
        }
    }
    s_sum[threadIdx.x] = sum;
    s_cnt[threadIdx.x] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int t = 0; t < kBlock; ++t) {
            a += s_sum[t];
            b += s_cnt[t];
        }
        parts[2 * blockIdx.x] = a;
        parts[2 * blockIdx.x + 1] = b;
    }
}

__global__ void __launch_bounds__(kBlock) k_refine_flag(int n, const double *el_error, uint8_t *flags,
                                                        const double *parts, double *target) {
    __shared__ double t;
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < kVolParts; ++k) {
            a += parts[2 * k];
            b += parts[2 * k + 1];
        }
        t = b > 0.0 ? a / b : 1.0;  // element_weight.C:72-76
        if (blockIdx.x == 0) *target = t;
    }
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (el_error[i] > t) flags[i] |= uint8_t(16);
}

template <class R>
int refine_info_t(da_ctx *ctx, double *el_error, uint8_t *flags, double *parts, double *target) {
    const MeshArgs m = mesh_args(ctx);
    const int c = ctx->cur, p = 1 - c;
    StateRef<R> Un{(const R *)ctx->U[c][0], (const R *)ctx->U[c][1], (const R *)ctx->U[c][2]};
    StateRef<R> Up{(const R *)ctx->U[p][0], (const R *)ctx->U[p][1], (const R *)ctx->U[p][2]};
    k_refine_info<R><<<kVolParts, kBlock, 0, ctx->stream>>>(m, Up, Un, (const R *)ctx->kact, el_error, flags, parts);
    k_refine_flag<<<(ctx->sm_count > 0 ? ctx->sm_count : 148) * 4, kBlock, 0, ctx->stream>>>(m.n, el_error, flags,
                                                                                            parts, target);
    return cuda_check(ctx, cudaGetLastError(), "refine info launch");
}

}  // namespace
}  // namespace fwd
}  // namespace da
