// Launchers of the adjoint kernels for one precision (included by adjoint_fp64.cu / _fp32.cu).
#pragma once
#include "adjoint_impl.cuh"

namespace da {
namespace adj {
namespace {

template <class R>
AdjArgs adj_args(da_ctx *ctx, const double *sec2, double cos_int) {
    AdjArgs a;
    a.mask = ctx->mask;
    a.tile_epoch = ctx->tile_epoch;
    a.tile_act = ctx->tile_act;
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
    const int grid = ctx->nblocks;
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
    cudaMemsetAsync(ctx->lam_clean, 0, ctx->ntiles, ctx->stream);
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
    k_adj_reduce<R><<<nout, kBlock, 0, ctx->stream>>>(m, L, ctx->gbed, ctx->gint, ctx->dh0, ctx->p.n_materials, n_piles,
                                                       ctx->red_out);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "adjoint reduce launch");
}

}  // namespace
}  // namespace adj
}  // namespace da
