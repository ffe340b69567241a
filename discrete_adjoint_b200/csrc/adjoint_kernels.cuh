// Launchers of the adjoint kernels for one precision (included by adjoint_fp64.cu / _fp32.cu).
#pragma once
#include "adjoint_impl.cuh"
#include "forward_impl.cuh"

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
int seed_t(da_ctx *ctx, int lam_out, const double box[4]) {
    const MeshArgs m = mesh_args(ctx);
    const int c = ctx->cur;
    StateRef<R> U{(const R *)ctx->U[c][0], (const R *)ctx->U[c][1], (const R *)ctx->U[c][2]};
    StateOut<R> Lo{(R *)ctx->lam[lam_out][0], (R *)ctx->lam[lam_out][1], (R *)ctx->lam[lam_out][2]};
    // lambda^N is written everywhere: the two adjoint buffers differ on every tile
    cudaMemsetAsync(ctx->lam_clean, 0, ctx->nseg, ctx->stream);
    trace_begin(ctx, TR_ADJ_SEED);
    k_adj_seed<R><<<ctx->nblocks, kBlock, 0, ctx->stream>>>(m, U, Lo, box[0], box[1], box[2], box[3], ctx->seed_part,
                                                             ctx->seed_J, ctx->seed_counter);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "adjoint seed launch");
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

// ------------------------------------------------------------------------ k_youturn
// One whole reverse step in one cooperative launch: the forward step of U^n replayed with its
// branch codes recorded (coefficient phase, barrier, dt, update phase), a barrier, the source
// adjoint, a barrier and the gather, i.e. the four launches of the separate path with grid
// barriers instead of kernel boundaries.  U^n stays in buffer cur; U^{n+1} goes to cur ^ 1.
// Block 0 writes the step's scalars at the end, as the separate kernels do.
template <class R>
__global__ void __launch_bounds__(kBlock) k_youturn(MeshArgs m, fwd::StatePair<R> S, int cur, R *kact, unsigned *active,
                                                    uint8_t *seg_clean, uint8_t *seg_wet, double *seg_vol,
                                                    uint8_t *seg_dirty, int ntiles,
                                                    int cull, MatConsts mc, TimeConsts tc, DevScalars *sc,
                                                    uint8_t *mask, int *tile_epoch, uint8_t *seg_act, int rec_id,
                                                    StateRef<R> Ln, StateOut<R> Lo, AdjArgs aa) {
    __shared__ int list[kBlock];
    const double time = sc->time;
    const long long iter = sc->iter;
    const StateRef<R> U{S.h[cur], S.hu[cur], S.hv[cur]};
    const StateOut<R> O{S.h[cur ^ 1], S.hu[cur ^ 1], S.hv[cur ^ 1]};
    unsigned long long my_min = 0x7FF0000000000000ull, my_max = 0ull;
    fwd::coef_phase<R, true>(m, U, kact, active, seg_wet, ntiles, cull, mc, sc, mask, list, my_min, my_max);
    fwd::push_minmax(my_min, my_max, &sc->acc_min_dxe, &sc->acc_hmax);
    if (!fwd::grid_sync(sc)) return;
    const double min_dxe = __longlong_as_double(__ldcg(&sc->acc_min_dxe));
    const double hmax = __longlong_as_double(__ldcg(&sc->acc_hmax));
    double dt, ft;
    fwd::step_dt(min_dxe, hmax, time, iter, tc, dt, ft);
    const R ftr = R(ft) > R(mc.sign_floor) ? R(ft) : R(mc.sign_floor);
    fwd::update_phase<R, true>(m, U, O, kact, active, seg_clean, seg_wet, seg_vol, seg_dirty, ntiles, cull, mc, sc,
                               R(dt), ftr,
                               mask, tile_epoch, seg_act, rec_id, list);
    if (!fwd::grid_sync(sc)) return;
    adj_src_phase<R>(m, U, Ln, mc, aa, R(dt), ftr, list);
    if (!fwd::grid_sync(sc)) return;
    adj_gather_phase<R>(m, U, Ln, Lo, mc, aa, R(dt), list);
    if (blockIdx.x == 0) {
        if (threadIdx.x == 0) {
            sc->time = time + dt;
            sc->iter = iter + 1;
            sc->dt = dt;
            sc->frict_tiny = ft;
            sc->min_dxe = min_dxe;
            sc->hmax = hmax;
            sc->acc_min_dxe = fwd::kMinDxeStart;
            sc->acc_hmax = 0ull;
        }
    }
}

// The live state is U^n in buffer cur; afterwards U^{n+1} is (cur flips) and lambda^n is in
// lam_out.
template <class R>
int youturn_t(da_ctx *ctx, int lam_in, int lam_out, const double *sec2, double cos_int) {
    const int pi = sizeof(R) == 8;
    if (ctx->coop_cap_yt[pi] <= 0) {
        int per_sm = 0;
        int st = cuda_check(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_youturn<R>, kBlock, 0),
                            "occupancy");
        if (st) return st;
        ctx->coop_cap_yt[pi] = per_sm * (ctx->sm_count > 0 ? ctx->sm_count : 1);
    }
    const int cap = ctx->coop_cap_yt[pi];
    if (cap <= 0) return set_error(ctx, DA_ERR_UNSUPPORTED, "reverse-step kernel cannot be resident");
    const int grid = ctx->grid < cap ? ctx->grid : cap;
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
    double *seg_vol = ctx->seg_vol;
    uint8_t *seg_dirty = ctx->seg_dirty;
    MatConsts mc = ctx->mc;
    TimeConsts tc = ctx->tc;
    DevScalars *sc = ctx->dsc;
    StateRef<R> Ln{(const R *)ctx->lam[lam_in][0], (const R *)ctx->lam[lam_in][1], (const R *)ctx->lam[lam_in][2]};
    StateOut<R> Lo{(R *)ctx->lam[lam_out][0], (R *)ctx->lam[lam_out][1], (R *)ctx->lam[lam_out][2]};
    AdjArgs aa = adj_args<R>(ctx, sec2, cos_int);
    void *args[] = {&m,  &S,    &cur,  &kact, &active,     &seg_clean, &seg_wet, &seg_vol, &seg_dirty, &ntiles, &cull,
                    &mc, &tc,   &sc,   &mask, &tile_epoch, &seg_act,   &rec_id,  &Ln,      &Lo,        &aa};
    trace_begin(ctx, TR_YOUTURN);
    const cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_youturn<R>, grid, kBlock, args, 0, ctx->stream);
    trace_end(ctx);
    if (e != cudaSuccess) return cuda_check(ctx, e, "reverse-step launch");
    ctx->cur = cur ^ 1;
    return DA_OK;
}

}  // namespace
}  // namespace adj
}  // namespace da
