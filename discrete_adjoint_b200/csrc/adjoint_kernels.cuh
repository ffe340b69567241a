// Launchers of the adjoint kernels for one precision (included by adjoint_fp64.cu / _fp32.cu).
#pragma once
#include <algorithm>

#include "adjoint_impl.cuh"
#include "forward_impl.cuh"
#include "adjoint_staged.cuh"

namespace da {
namespace adj {
namespace {

template <class R>
AdjArgs adj_args(da_ctx *ctx, const double *sec2, double cos_int) {
    AdjArgs a;
    a.mask = ctx->mask;
    a.tile_epoch = ctx->tile_epoch;
    a.seg_act = ctx->seg_act;
    a.lam_clean = ctx->lam_clean;
    a.rec_id = ctx->rec_id;
    a.ntiles = ctx->ntiles;
    a.A = ctx->adjA;
    a.B = ctx->adjB;
    a.gbed = ctx->gbed;
    a.gint = ctx->gint;
    a.dk_dbed = ctx->dk_tab;
    a.dk_dint = ctx->dk_tab + DA_MAX_MATERIALS * 3;
    for (int m = 0; m < DA_MAX_MATERIALS; ++m) a.sec2_bed[m] = sec2[m];
    a.cos_int = cos_int;
    return a;
}

template <class R>
int step_t(da_ctx *ctx, int lam_in, int lam_out, const double *sec2, double cos_int) {
    // the forward step of U^n has just been replayed: U^n is in buffer 1 - cur, its codes in mask
    const MeshArgs m = mesh_args(ctx);
    const int un = 1 - ctx->cur;
    StateRef<R> U{(const R *)ctx->U[un][0], (const R *)ctx->U[un][1], (const R *)ctx->U[un][2]};
    StateRef<R> Ln{(const R *)ctx->lam[lam_in][0], (const R *)ctx->lam[lam_in][1], (const R *)ctx->lam[lam_in][2]};
    StateOut<R> Lo{(R *)ctx->lam[lam_out][0], (R *)ctx->lam[lam_out][1], (R *)ctx->lam[lam_out][2]};
    const AdjArgs aa = adj_args<R>(ctx, sec2, cos_int);
    const int grid = ctx->grid;
    const R floor = R(ctx->mc.sign_floor);
    trace_begin(ctx, TR_ADJ_SRC);
    k_adj_src<R><<<grid, kBlock, 0, ctx->stream>>>(m, U, Ln, ctx->mc, aa, ctx->dsc, floor);
    trace_end(ctx);
    trace_begin(ctx, TR_ADJ_GATHER);
    k_adj_gather<R><<<grid, kBlock, 0, ctx->stream>>>(m, U, Ln, Lo, ctx->mc, aa, ctx->dsc);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "adjoint step launch");
}

template <class R>
int reduce_t(da_ctx *ctx, int lam0, int n_piles) {
    const MeshArgs m = mesh_args(ctx);
    StateRef<R> L{(const R *)ctx->lam[lam0][0], (const R *)ctx->lam[lam0][1], (const R *)ctx->lam[lam0][2]};
    const int nout = ctx->p.n_materials + 1 + n_piles;
    trace_begin(ctx, TR_ADJ_REDUCE);
    k_adj_reduce<R><<<dim3(kReduceParts, nout), kBlock, 0, ctx->stream>>>(m, L, ctx->gbed, ctx->gint, ctx->dh0,
                                                                           ctx->p.n_materials, n_piles, ctx->red_part);
    k_adj_reduce_final<<<nout, kReduceParts, 0, ctx->stream>>>(ctx->red_part, ctx->red_out);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "adjoint reduce launch");
}

// Ensemble gradients: (n_mat + 2) outputs per member into red_out, n_mat the largest material
// count of the members.
template <class R>
int reduce_inst_t(da_ctx *ctx, int lam0) {
    const MeshArgs m = mesh_args(ctx);
    StateRef<R> L{(const R *)ctx->lam[lam0][0], (const R *)ctx->lam[lam0][1], (const R *)ctx->lam[lam0][2]};
    trace_begin(ctx, TR_ADJ_REDUCE);
    k_adj_reduce_inst<R><<<dim3(ctx->ninst, ctx->p.n_materials + 2), kBlock, 0, ctx->stream>>>(
        m, L, ctx->gbed, ctx->gint, ctx->dh0, ctx->p.n_materials, ctx->ia.seg0, ctx->red_out);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "ensemble reduce launch");
}

// The gather shares its work out by quarter tiles when four times the tiles the recording update
// listed fit in the grid (a flow over few tiles), else by tiles; every block reads the same count
// after the barrier that ends the update.
// split: 0 by that rule, 1 tiles, 2 quarters (da_params.tile_staging 1, 2, 3).
__device__ __forceinline__ bool gather_quarters(const DevScalars *sc, int split) {
    if (split) return split == 2;
    return 4ull * __ldcg(&sc->listed) <= gridDim.x;
}

// ------------------------------------------------------------------------ k_youturn
// One whole reverse step in one cooperative launch: the forward step of U^n replayed with its
// branch codes recorded (coefficient phase, barrier, dt, update phase), a barrier, the source
// adjoint, a barrier and the gather, i.e. the four launches of the separate path with grid
// barriers instead of kernel boundaries.  U^n stays in buffer cur; U^{n+1} goes to cur ^ 1.
// SEED (the last step of the horizon): lambda^N is seeded from the U^N just produced before the
// adjoint phases, with each segment's part of J.  BATCH: every member with its own constants and
// dt (the members' dt pass between two barriers).  Block 0 writes the step's scalars at the end,
// as the separate kernels do.  pre (mode NONE when unused): a checkpoint restore before the step,
// followed by a barrier.  STAGED: the replayed forward phases stage tiles and halos in shared
// memory (staged_impl.cuh).
template <class R, bool BATCH, bool SEED, int OCC, bool STAGED>
__global__ void __launch_bounds__(kBlock, OCC) k_youturn(MeshArgs m, fwd::StatePair<R> S, int cur, R *kact, unsigned *active,
                                                    uint8_t *seg_clean, uint8_t *seg_wet, double *seg_vol,
                                                    uint8_t *seg_dirty, int ntiles, int cull, MatConsts mc,
                                                    TimeConsts tc, DevScalars *sc, uint8_t *mask, int *tile_epoch,
                                                    uint8_t *seg_act, int rec_id, StateRef<R> Ln, StateOut<R> Lseed,
                                                    StateOut<R> Lo, AdjArgs aa, InstArgs ia, Box box, double *seg_J,
                                                    snap::SnapArgs<R> pre, fwd::HaloArgs ha, int gsplit) {
    __shared__ int list[kBlock];
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    fwd::StageSmem<R> &stg = *reinterpret_cast<fwd::StageSmem<R> *>(dyn_smem);
    // the recording update counts its listed tiles from zero (the adds follow a barrier)
    if (blockIdx.x == 0 && threadIdx.x == 0) sc->listed = 0u;
    if (pre.mode != snap::NONE) {
        snap::snap_segments<R>(pre);
        snap::snap_scalars<R>(pre);
        if (!fwd::grid_sync(sc)) return;
    }
    const double time = __ldcg(&sc->time);
    const long long iter = __ldcg(&sc->iter);
    const StateRef<R> U{S.h[cur], S.hu[cur], S.hv[cur]};
    const StateOut<R> O{S.h[cur ^ 1], S.hu[cur ^ 1], S.hv[cur ^ 1]};
    unsigned long long my_min = 0x7FF0000000000000ull, my_max = 0ull;
    if (STAGED)
        fwd::coef_phase_staged<R, true, BATCH>(m, ha, U, kact, active, seg_wet, ntiles, cull, mc, sc, mask, list, my_min,
                                               my_max, ia, stg);
    else
        fwd::coef_phase<R, true, BATCH>(m, U, kact, active, seg_wet, ntiles, cull, mc, sc, mask, list, my_min, my_max,
                                        ia);
    if (!BATCH) fwd::push_minmax(my_min, my_max, &sc->acc_min_dxe, &sc->acc_hmax);
    if (!fwd::grid_sync(sc)) return;
    double dt = 0.0, ft, min_dxe = 0.0, hmax = 0.0;
    if (BATCH) {
        ft = iter < tc.frict_tiny_iters ? tc.frict_tiny_early : tc.frict_tiny_late;
        fwd::inst_dt_pass(ia, iter, tc, sc);
        if (!fwd::grid_sync(sc)) return;
    } else {
        min_dxe = __longlong_as_double(__ldcg(&sc->acc_min_dxe));
        hmax = __longlong_as_double(__ldcg(&sc->acc_hmax));
        fwd::step_dt(min_dxe, hmax, time, iter, tc, dt, ft);
        if (blockIdx.x == 0 && threadIdx.x == 0 && !isfinite(dt)) raise_err(sc, DA_ERR_NAN);
    }
    const R ftr = R(ft) > R(mc.sign_floor) ? R(ft) : R(mc.sign_floor);
    if (STAGED && !SEED) {
        // the source adjoint of each wet cell right after its update, from the tile and halo
        // staged for it (its own branches and lambda^{n+1}, U^n around it: nothing another cell
        // writes in this phase), so the reverse step needs no source phase of its own
        const SrcEpilogue<R, BATCH> src{m, Ln, mc, aa, ia, R(dt), ftr};
        fwd::update_phase_staged<R, true, BATCH>(m, ha, U, O, kact, active, seg_clean, seg_wet, seg_vol, seg_dirty,
                                                 ntiles, cull, mc, sc, R(dt), ftr, mask, tile_epoch, seg_act, rec_id,
                                                 list, ia, stg, src);
        if (!fwd::grid_sync(sc)) return;
        adj_gather_phase_staged<R, BATCH>(m, ha, U, Ln, Lo, mc, aa, R(dt), list, ia,
                                          *reinterpret_cast<GatherSmem<R> *>(dyn_smem), gather_quarters(sc, gsplit));
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            sc->iter = iter + 1;
            sc->frict_tiny = ft;
            if (!BATCH) {
                sc->time = time + dt;
                sc->dt = dt;
                sc->min_dxe = min_dxe;
                sc->hmax = hmax;
                sc->acc_min_dxe = fwd::kMinDxeStart;
                sc->acc_hmax = 0ull;
            }
        }
        fwd::grid_exit(sc);
        return;
    }
    if (STAGED)
        fwd::update_phase_staged<R, true, BATCH>(m, ha, U, O, kact, active, seg_clean, seg_wet, seg_vol, seg_dirty,
                                                 ntiles, cull, mc, sc, R(dt), ftr, mask, tile_epoch, seg_act, rec_id,
                                                 list, ia, stg);
    else
        fwd::update_phase<R, true, BATCH>(m, U, O, kact, active, seg_clean, seg_wet, seg_vol, seg_dirty, ntiles, cull,
                                          mc, sc, R(dt), ftr, mask, tile_epoch, seg_act, rec_id, list, ia);
    if (!fwd::grid_sync(sc)) return;
    if (SEED) {
        seed_phase<R, BATCH>(m, StateRef<R>{O.h, O.hu, O.hv}, Lseed, box, seg_J, ntiles * (kBlock / 32), ia);
        if (!fwd::grid_sync(sc)) return;
    }
    adj_src_phase<R, BATCH>(m, U, Ln, mc, aa, R(dt), ftr, list, ia);
    if (!fwd::grid_sync(sc)) return;
    if (STAGED)
        adj_gather_phase_staged<R, BATCH>(m, ha, U, Ln, Lo, mc, aa, R(dt), list, ia,
                                          *reinterpret_cast<GatherSmem<R> *>(dyn_smem), gather_quarters(sc, gsplit));
    else
        adj_gather_phase<R, BATCH>(m, U, Ln, Lo, mc, aa, R(dt), list, ia);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->iter = iter + 1;
        sc->frict_tiny = ft;
        if (!BATCH) {
            sc->time = time + dt;
            sc->dt = dt;
            sc->min_dxe = min_dxe;
            sc->hmax = hmax;
            sc->acc_min_dxe = fwd::kMinDxeStart;
            sc->acc_hmax = 0ull;
        }
    }
    fwd::grid_exit(sc);
}

// The k_youturn instantiation for the launch's flags.
template <class R>
const void *youturn_kernel(bool batch, bool seed, bool occ3, bool staged) {
#define DA_YT(B, S, O, G) (const void *)k_youturn<R, B, S, O, G>
#define DA_YT_OCC(B, S, G) (occ3 ? DA_YT(B, S, 3, G) : DA_YT(B, S, 2, G))
#define DA_YT_SEED(B, G) (seed ? DA_YT_OCC(B, true, G) : DA_YT_OCC(B, false, G))
#define DA_YT_BATCH(G) (batch ? DA_YT_SEED(true, G) : DA_YT_SEED(false, G))
    return staged ? DA_YT_BATCH(true) : DA_YT_BATCH(false);
#undef DA_YT_BATCH
#undef DA_YT_SEED
#undef DA_YT_OCC
#undef DA_YT
}

// The live state is U^n in buffer cur; afterwards U^{n+1} is (cur flips) and lambda^n is in
// lam_out.  seed: lambda^N goes into lam_in first (from U^{n+1} = U^N) with J's segment parts.
// pre_slot (or null): a checkpoint slot restored first, in the same launch (the live state is then
// the restored one).
template <class R>
int youturn_t(da_ctx *ctx, int lam_in, int lam_out, const double *sec2, double cos_int, bool seed,
              const double *box4, void *pre_slot) {
    const int pi = sizeof(R) == 8;
    const bool batch = ctx->ninst > 0;
    const int occ3 = ctx->p.blocks_per_sm == 3;
    const bool staged = fwd::staged_ok(ctx);
    const void *kern = youturn_kernel<R>(batch, seed, occ3, staged);
    // the staged phases and the staged gather use the same dynamic shared memory in turn
    const size_t smem = staged ? std::max(fwd::stage_smem_bytes<R>(), gather_smem_bytes<R>()) : 0;
    int &cap_ref = ctx->coop_cap_yt[pi + 2 * batch + 4 * seed + 8 * occ3 + 16 * staged];
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
    if (cap <= 0) return set_error(ctx, DA_ERR_UNSUPPORTED, "reverse-step kernel cannot be resident");
    // FP64: every co-resident block, at most four per tile, whatever the forward steps' tuned grid:
    // the gather spreads a sparse flow's quarter tiles over them, which outweighs the dearer
    // barriers (the forward phases split no tile and keep the tuned grid; in FP32 the shorter
    // gather gains less than the barriers cost).  FP32: the tuned grid, but never below one block
    // per SM (a forward grid of half the SMs leaves the reverse step short of memory parallelism).
    // Results do not depend on it.
    int want = ctx->grid;
    const int per_sm1 = ctx->sm_count > 0 ? ctx->sm_count : 148;
    if (want < per_sm1) want = per_sm1 < ctx->ntiles ? per_sm1 : ctx->ntiles;
    if (sizeof(R) == 8 && want < 4 * ctx->ntiles) want = 4 * ctx->ntiles;
    const int grid = want < cap ? want : cap;
    ++ctx->rec_id;
    MeshArgs m = mesh_args(ctx);
    fwd::StatePair<R> S;
    for (int b = 0; b < 2; ++b) {
        S.h[b] = (R *)ctx->U[b][0];
        S.hu[b] = (R *)ctx->U[b][1];
        S.hv[b] = (R *)ctx->U[b][2];
    }
    int cur = ctx->cur, ntiles = ctx->ntiles, cull = ctx->p.tile_culling, rec_id = ctx->rec_id;
    R *kact = (R *)ctx->kact;
    unsigned *active = ctx->active;
    uint8_t *seg_clean = ctx->seg_clean, *seg_wet = ctx->seg_wet, *mask = ctx->mask, *seg_act = ctx->seg_act;
    int *tile_epoch = ctx->tile_epoch;
    double *seg_vol = ctx->seg_vol, *seg_J = ctx->seg_J;
    uint8_t *seg_dirty = ctx->seg_dirty;
    MatConsts mc = ctx->mc;
    TimeConsts tc = ctx->tc;
    DevScalars *sc = ctx->dsc;
    StateRef<R> Ln{(const R *)ctx->lam[lam_in][0], (const R *)ctx->lam[lam_in][1], (const R *)ctx->lam[lam_in][2]};
    StateOut<R> Ls{(R *)ctx->lam[lam_in][0], (R *)ctx->lam[lam_in][1], (R *)ctx->lam[lam_in][2]};
    StateOut<R> Lo{(R *)ctx->lam[lam_out][0], (R *)ctx->lam[lam_out][1], (R *)ctx->lam[lam_out][2]};
    AdjArgs aa = adj_args<R>(ctx, sec2, cos_int);
    InstArgs ia = ctx->ia;
    Box box{};
    if (box4)
        for (int q = 0; q < 4; ++q) box.v[q] = box4[q];
    if (seed) {
        // lambda^N is written everywhere: the two adjoint buffers differ on every segment
        int st = cuda_check(ctx, cudaMemsetAsync(ctx->lam_clean, 0, ctx->nseg, ctx->stream), "memset");
        if (st) return st;
    }
    snap::SnapArgs<R> pre = pre_slot ? snap::snap_args<R>(ctx, pre_slot, false, cur) : snap::no_snap<R>();
    fwd::HaloArgs ha = fwd::halo_args(ctx);
    int gsplit = ctx->p.tile_staging >= 2 ? ctx->p.tile_staging - 1 : 0;
    void *args[] = {&m,      &S,    &cur, &kact, &active, &seg_clean, &seg_wet,    &seg_vol, &seg_dirty,
                    &ntiles, &cull, &mc,  &tc,   &sc,     &mask,      &tile_epoch, &seg_act, &rec_id,
                    &Ln,     &Ls,   &Lo,  &aa,   &ia,     &box,       &seg_J,      &pre,     &ha,      &gsplit};
    trace_begin(ctx, TR_YOUTURN);
    const cudaError_t e = cudaLaunchCooperativeKernel(kern, grid, kBlock, args, smem, ctx->stream);
    trace_end(ctx);
    if (e != cudaSuccess) return cuda_check(ctx, e, "reverse-step launch");
    ctx->cur = cur ^ 1;
    return DA_OK;
}

// Per-member J (or the single J) from the segments' parts, fixed order; one block per member.
template <class R>
int functional_t(da_ctx *ctx, double *out) {
    const int nm = ctx->ninst > 0 ? ctx->ninst : 1;
    trace_begin(ctx, TR_ADJ_SEED);
    k_inst_sum<<<nm, kBlock, 0, ctx->stream>>>(ctx->seg_J, ctx->ninst > 0 ? ctx->ia.seg0 : nullptr, ctx->nseg, out);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "functional launch");
}

}  // namespace
}  // namespace adj
}  // namespace da
