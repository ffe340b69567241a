// Host side of the adjoint: workspace, the k act/pass parameter-derivative tables, the optimal
// binomial checkpoint schedule, and the C ABI entry points da_adjoint_run / da_adjoint_step /
// da_set_dt_replay.
//
// The reference's dual_solver (src/adjoint/dual_solver.C:80-273) walks the recorded steps
// backward from gz files written every 50 steps (SolRec, src/datstr/dualmesh.C:82-147).  Here
// the forward states live in HBM only at checkpoints; the reverse sweep recomputes the steps in
// between.  The placement minimises recomputation for the given number of slots: T(l, c), the
// forward steps needed to reverse l steps with c free slots, obeys
//     T(1, c) = 0,  T(l, 0) = l(l-1)/2,  T(l, c) = min_m [ m + T(l-m, c-1) + T(m, c) ],
// the recursion of binomial checkpointing (Griewank's revolve), solved by dynamic programming.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "da_internal.h"

namespace da {

int launch_adjoint_step_fp64(da_ctx *, int, int, const double *, double);
int launch_adjoint_step_fp32(da_ctx *, int, int, const double *, double);
int launch_adjoint_reduce_fp64(da_ctx *, int, int);
int launch_adjoint_reduce_fp32(da_ctx *, int, int);
int launch_functional_fp64(da_ctx *, double *);
int launch_functional_fp32(da_ctx *, double *);
int forward_state_changed(da_ctx *ctx);

int launch_youturn_fp64(da_ctx *, int, int, const double *, double, bool, const double *, void *);
int launch_youturn_fp32(da_ctx *, int, int, const double *, double, bool, const double *, void *);
int launch_youturn(da_ctx *ctx, int a, int b, const double *sec2, double c, bool seed, const double *box,
                   void *pre_slot) {
    return ctx->p.precision == DA_PREC_FP64 ? launch_youturn_fp64(ctx, a, b, sec2, c, seed, box, pre_slot)
                                            : launch_youturn_fp32(ctx, a, b, sec2, c, seed, box, pre_slot);
}
int launch_functional(da_ctx *ctx, double *out) {
    return ctx->p.precision == DA_PREC_FP64 ? launch_functional_fp64(ctx, out) : launch_functional_fp32(ctx, out);
}
int launch_adjoint_reduce_inst_fp64(da_ctx *, int);
int launch_adjoint_reduce_inst_fp32(da_ctx *, int);
int launch_adjoint_reduce_inst(da_ctx *ctx, int lam0) {
    return ctx->p.precision == DA_PREC_FP64 ? launch_adjoint_reduce_inst_fp64(ctx, lam0)
                                            : launch_adjoint_reduce_inst_fp32(ctx, lam0);
}
int launch_adjoint_step(da_ctx *ctx, int a, int b, const double *sec2, double c) {
    return ctx->p.precision == DA_PREC_FP64 ? launch_adjoint_step_fp64(ctx, a, b, sec2, c)
                                            : launch_adjoint_step_fp32(ctx, a, b, sec2, c);
}
int launch_adjoint_reduce(da_ctx *ctx, int a, int np) {
    return ctx->p.precision == DA_PREC_FP64 ? launch_adjoint_reduce_fp64(ctx, a, np)
                                            : launch_adjoint_reduce_fp32(ctx, a, np);
}

namespace {
size_t rsize(const da_ctx *ctx) { return ctx->p.precision == DA_PREC_FP64 ? sizeof(double) : sizeof(float); }
}  // namespace

// d kact / d phi_bed and d phi_int of gmfggetcoef's three signed branches (getcoef.f:19-66):
// k = (2/c^2)(1 - s sqrt|1 - (1 + t^2) c^2|) - 1 with c = cos phi_int, t = tan phi_bed, times
// epsilon; a branch clamped at zero has zero derivative.
void kact_derivatives(const da_params &p, double *dkb, double *dki) {
    for (int m = 0; m < DA_MAX_MATERIALS; ++m)
        for (int k = 0; k < 3; ++k) dkb[m * 3 + k] = dki[m * 3 + k] = 0.0;
    const double c = std::cos(p.intfrict), sn = std::sin(p.intfrict);
    for (int m = 0; m < p.n_materials; ++m) {
        const double t = std::tan(p.bedfrict[m]);
        const double A = 1.0 - (1.0 + t * t) * (c * c);
        const double Q = std::sqrt(std::fabs(A));
        const double sA = A > 0 ? 1.0 : (A < 0 ? -1.0 : 0.0);
        const double dA_db = -(c * c) * 2.0 * t * (1.0 + t * t);
        const double dA_di = 2.0 * (1.0 + t * t) * c * sn;
        const double dQ_db = Q > 0 ? sA * dA_db / (2.0 * Q) : 0.0;
        const double dQ_di = Q > 0 ? sA * dA_di / (2.0 * Q) : 0.0;
        for (int s = -1; s <= 1; ++s) {
            const double k0 = (2.0 / (c * c)) * (1.0 - s * Q) - 1.0;
            if (k0 < 0.0) continue;
            dkb[m * 3 + s + 1] = p.epsilon * (2.0 / (c * c)) * (-s) * dQ_db;
            dki[m * 3 + s + 1] = p.epsilon * ((4.0 * sn / (c * c * c)) * (1.0 - s * Q) + (2.0 / (c * c)) * (-s) * dQ_di);
        }
    }
}

namespace {

int adj_alloc(da_ctx *ctx, int nsnap) {
    const size_t n = (size_t)ctx->mesh.n;
    const size_t rs = rsize(ctx);
    int st = DA_OK;
    const int nouts = (ctx->ninst > 0 ? ctx->ninst : 1) * (DA_MAX_MATERIALS + 1 + DA_MAX_PILES);
    if (ctx->adj_n != (int)n || ctx->adj_ninst != ctx->ninst) {
        auto fr = [](void *p) { if (p) cudaFree(p); };
        fr(ctx->mask); fr(ctx->adjA); fr(ctx->adjB); fr(ctx->gbed); fr(ctx->gint); fr(ctx->dk_tab);
        fr(ctx->red_out); fr(ctx->red_part); fr(ctx->inst_J); fr(ctx->seg_J);
        for (int b = 0; b < 2; ++b)
            for (int v = 0; v < 3; ++v) { fr(ctx->lam[b][v]); ctx->lam[b][v] = nullptr; }
        for (void *s : ctx->snaps) fr(s);
        ctx->snaps.clear();
        ctx->mask = nullptr; ctx->adjA = ctx->adjB = ctx->gbed = ctx->gint = ctx->dk_tab = nullptr;
        ctx->red_out = ctx->red_part = ctx->inst_J = ctx->seg_J = nullptr;
        ctx->adj_n = -1;
        st = cuda_check(ctx, cudaMalloc((void **)&ctx->mask, n), "cudaMalloc(mask)");
        for (int b = 0; b < 2 && !st; ++b)
            for (int v = 0; v < 3 && !st; ++v) st = cuda_check(ctx, cudaMalloc(&ctx->lam[b][v], rs * n), "cudaMalloc(lam)");
        if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->adjA, sizeof(double) * 3 * n), "cudaMalloc(A)");
        if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->adjB, sizeof(double) * 4 * n), "cudaMalloc(B)");
        if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->gbed, sizeof(double) * n), "cudaMalloc(gbed)");
        if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->gint, sizeof(double) * n), "cudaMalloc(gint)");
        if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->dk_tab, sizeof(double) * 2 * DA_MAX_MATERIALS * 3), "cudaMalloc");
        if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->red_out, sizeof(double) * nouts), "cudaMalloc");
        if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->red_part, sizeof(double) * kAdjReduceParts * (DA_MAX_MATERIALS + 1 + DA_MAX_PILES)), "cudaMalloc");
        if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->inst_J, sizeof(double) * (ctx->ninst > 0 ? ctx->ninst : 1)), "cudaMalloc");
        if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->seg_J, sizeof(double) * ctx->nseg), "cudaMalloc");
        if (st) return st;
        ctx->adj_n = (int)n;
        ctx->adj_ninst = ctx->ninst;
    }
    while ((int)ctx->snaps.size() < nsnap && !st) {
        void *p = nullptr;
        st = cuda_check(ctx, cudaMalloc(&p, snapshot_bytes(ctx)), "cudaMalloc(snapshot)");
        if (!st) ctx->snaps.push_back(p);
    }
    return st;
}

// One launch each (csrc/snapshot.cu): the state, the tile wet flags and the step scalars; a
// restore fills both state buffers so that tile culling stays valid.  Inside the reverse sweep the
// same copies run as phases of the cooperative step kernels instead (Runner below).
int store(da_ctx *ctx, int slot) { return launch_snapshot(ctx, ctx->snaps[slot], true); }
int restore(da_ctx *ctx, int slot) { return launch_snapshot(ctx, ctx->snaps[slot], false); }

// The placement is kept in the context and rebuilt only when the horizon or the slot count
// changes (the dynamic programme is O(N^2 C)).
struct Schedule {
    int N = 0, C = 0;
    std::vector<long long> cost;  // [(N+1) x (C+1)]
    std::vector<int> *split = nullptr;
    long long &T(int l, int c) { return cost[(size_t)l * (C + 1) + c]; }
    int &S(int l, int c) { return (*split)[(size_t)l * (C + 1) + c]; }
    void use(da_ctx *ctx, int n, int c) {
        split = &ctx->sched_split;
        N = n;
        C = c;
        if (ctx->sched_n == n && ctx->sched_c == c) return;
        build(n, c);
        ctx->sched_n = n;
        ctx->sched_c = c;
    }
    void build(int n, int c) {
        N = n;
        C = c;
        cost.assign((size_t)(N + 1) * (C + 1), 0);
        split->assign((size_t)(N + 1) * (C + 1), 0);
        for (int l = 1; l <= N; ++l) {
            T(l, 0) = (long long)l * (l - 1) / 2;
            for (int cc = 1; cc <= C; ++cc) {
                if (l == 1) {
                    T(l, cc) = 0;
                    continue;
                }
                long long best = -1;
                int arg = 1;
                for (int m = 1; m < l; ++m) {
                    const long long v = m + T(l - m, cc - 1) + T(m, cc);
                    if (best < 0 || v < best) {
                        best = v;
                        arg = m;
                    }
                }
                T(l, cc) = best;
                S(l, cc) = arg;
            }
        }
    }
};

// DWR indicator along the reverse sweep (da_adjoint_run_dwr): after the reverse step of n -> n+1
// (U^n, U^{n+1} and lambda^{n+1} all resident) the indicator of that step, as the reference's
// dual_solver calls error_compute after each adjoint step (dual_solver.C:206-230).
struct DwrAcc {
    double *cell = nullptr;       // [n] device: el_error per coarse cell, summed over the steps
    double *step_sums = nullptr;  // host [nsteps][2]: total el_error and correction of each step
    long long iter_begin = 0;     // iteration of U^0
    int nsteps = 0;
};

__global__ void k_accumulate(int n, const double *__restrict__ a, double *__restrict__ acc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc[i] += a[i];
}

int dwr_after_reverse_step(da_ctx *ctx, DwrAcc &d, int lam_next) {
    // the reverse step wrote the step's dt, time and iteration like a forward step
    int st = copy_d2h(ctx, ctx->hsc, ctx->dsc, sizeof(DevScalars), "read scalars");
    if (st) return st;
    const double dt = ctx->hsc->dt;
    const long long iter0 = ctx->hsc->iter - 1;
    const double time0 = ctx->hsc->time - dt;  // enters the error grid's step only through clipping
    st = dwr_indicator(ctx, ctx->cur ^ 1, ctx->cur, lam_next, dt, time0, iter0);
    if (st) return st;
    const int n = ctx->mesh.n, grid = (ctx->sm_count > 0 ? ctx->sm_count : 148) * 4;
    k_accumulate<<<grid, 256, 0, ctx->stream>>>(n, ctx->dwr.cell, d.cell);
    st = cuda_check(ctx, cudaGetLastError(), "dwr accumulate");
    const long long k = iter0 - d.iter_begin;
    if (!st && k >= 0 && k < d.nsteps) st = copy_d2h(ctx, d.step_sums + 2 * k, ctx->dwr.sums, 16, "dwr sums");
    return st;
}

struct Runner {
    da_ctx *ctx;
    DwrAcc *dwr = nullptr;
    Schedule sch;
    std::vector<int> free_slots;
    int lam_cur = 0;  // buffer holding lambda^{n+1}
    bool seeded = false;
    double box[4] = {0, 0, 0, 0};
    double sec2[DA_MAX_MATERIALS];
    double cos_int;
    long long fsteps = 0;
    int pos = -1;  // step index of the live forward state; -1 = not a checkpointed state
    int pending = -1;  // checkpoint slot the next launch restores first; -1 = none

    // The live state is already the checkpoint right after a store: no copy back.  Otherwise the
    // restore becomes the first phase of the next step launch (no launch of its own).
    int restore_at(int slot, int step) {
        if (pos == step) return DA_OK;
        const int st = flush();
        pos = step;
        pending = slot;
        return st;
    }
    // Consecutive forward advances (a chain of checkpoint stores between a restore and the next
    // reverse step) go out as one multi-step launch that stores the checkpoints on its way: the
    // advances wait here until a restore, a reverse step or the end of the sweep needs the state.
    int def_k = 0;
    void *def_pre = nullptr;
    MidStoreList def_mid;
    int flush() {
        if (def_k == 0) return DA_OK;
        const int st = launch_forward_steps(ctx, def_k, def_pre, nullptr, &def_mid);
        def_k = 0;
        def_pre = nullptr;
        def_mid.n = 0;
        return st;
    }
    void *take_pending() {
        void *p = pending >= 0 ? ctx->snaps[pending] : nullptr;
        pending = -1;
        return p;
    }
    // k forward steps; store_slot >= 0: the state after them is stored, in the same launch
    int advance(int k, int store_slot = -1) {
        if (k == 0) return DA_OK;  // a pending restore waits for the next launch
        fsteps += k;
        pos += k;
        void *slot = store_slot >= 0 ? ctx->snaps[store_slot] : nullptr;
        if (ctx->ninst > 0) return launch_forward_steps(ctx, k, take_pending(), slot);  // one launch each
        int st = DA_OK;
        if (slot && def_mid.n == kMidStores) st = flush();
        if (def_k == 0) def_pre = take_pending();
        def_k += k;
        if (slot) {
            def_mid.after[def_mid.n] = def_k - 1;
            def_mid.slot[def_mid.n++] = slot;
        }
        return st;
    }
    // every reverse(a, b) ends with a youturn, which takes any restore still pending
    int youturn() {
        ++fsteps;
        pos = -1;  // past the step that is being taken back
        if (const int st = flush()) return st;
        if (ctx->p.jacobian_mode == DA_JAC_REFERENCE) return youturn_reference();
        // the first reverse step (the horizon's last step) also seeds lambda^N from U^N
        int st = launch_youturn(ctx, lam_cur, 1 - lam_cur, sec2, cos_int, !seeded, box, take_pending());
        if (!st && dwr) st = dwr_after_reverse_step(ctx, *dwr, lam_cur);
        seeded = true;
        lam_cur = 1 - lam_cur;
        return st;
    }
    // The reference's dual-solver step instead of the fused exact one: the pending restore, the
    // forward step (its dt and frict_tiny), the seed on the horizon's last step, then the step's
    // adjoint from U^n, which the forward step left in the other state buffer.
    int youturn_reference() {
        void *pre = take_pending();
        int st = pre ? launch_snapshot(ctx, pre, false) : DA_OK;
        if (!st) st = launch_forward_step(ctx, nullptr);
        if (!st && !seeded) st = launch_ref_seed(ctx, lam_cur, box);
        if (!st) st = launch_ref_adjoint_step(ctx, ctx->cur ^ 1, lam_cur, 1 - lam_cur);
        if (!st && dwr) st = dwr_after_reverse_step(ctx, *dwr, lam_cur);
        seeded = true;
        lam_cur = 1 - lam_cur;
        return st;
    }
    int reverse(int a, int b, int slot_a) {
        int st = DA_OK;
        const int l = b - a;
        if (l == 1) {
            st = restore_at(slot_a, a);
            if (!st) st = youturn();
            return st;
        }
        const int c = (int)free_slots.size() < sch.C ? (int)free_slots.size() : sch.C;
        if (c == 0) {
            for (int k = b - 1; k >= a && !st; --k) {
                st = restore_at(slot_a, a);
                if (!st) st = advance(k - a);
                if (!st) st = youturn();
            }
            return st;
        }
        const int m = a + sch.S(l, c);  // a < m < b
        st = restore_at(slot_a, a);
        const int slot_m = free_slots.back();
        free_slots.pop_back();
        if (!st) st = advance(m - a, slot_m);
        if (!st) st = reverse(m, b, slot_m);
        free_slots.push_back(slot_m);
        if (!st) st = reverse(a, m, slot_a);
        return st;
    }
};

int sync_check(da_ctx *ctx) {
    int st = cuda_check(ctx, cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream),
                        "read scalars");
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (!st) st = device_error(ctx, "adjoint sweep");
    return st;
}

int upload_tables(da_ctx *ctx, double *sec2, double *cos_int) {
    std::vector<double> tab(2 * DA_MAX_MATERIALS * 3);
    kact_derivatives(ctx->p, tab.data(), tab.data() + DA_MAX_MATERIALS * 3);
    for (int m = 0; m < DA_MAX_MATERIALS; ++m) {
        const double t = m < ctx->p.n_materials ? std::tan(ctx->p.bedfrict[m]) : 0.0;
        sec2[m] = 1.0 + t * t;
    }
    *cos_int = std::cos(ctx->p.intfrict);
    int st = copy_h2d(ctx, ctx->dk_tab, tab.data(), sizeof(double) * tab.size(), "upload tables");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->gbed, 0, sizeof(double) * ctx->mesh.n, ctx->stream), "memset");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->gint, 0, sizeof(double) * ctx->mesh.n, ctx->stream), "memset");
    return st;
}

}  // namespace

int copy_lambda_out(da_ctx *ctx, int buf, double *host) {
    const size_t n = (size_t)ctx->mesh.n;
    int st = DA_OK;
    for (int v = 0; v < 3 && !st; ++v) {
        st = download_real(ctx, host + v * n, ctx->lam[buf][v]);
        if (!st && ctx->p.precision != DA_PREC_FP64) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    }
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    return st;
}

namespace {

int fill_gradient(da_ctx *ctx, int lam0, int n_piles, da_gradient *out, bool reduced = false) {
    int st = reduced ? DA_OK : launch_adjoint_reduce(ctx, lam0, n_piles);
    std::vector<double> red(DA_MAX_MATERIALS + 1 + DA_MAX_PILES, 0.0);
    const int nout = ctx->p.n_materials + 1 + n_piles;
    if (!st) st = cuda_check(ctx, cudaMemcpyAsync(red.data(), ctx->red_out, sizeof(double) * nout, cudaMemcpyDeviceToHost,
                                                  ctx->stream), "read gradient");
    double J = 0.0;
    if (!st) st = cuda_check(ctx, cudaMemcpyAsync(&J, ctx->inst_J, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream),
                             "read J");
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (st || !out) return st;
    std::memset(out, 0, sizeof(*out));
    out->J = J;
    for (int m = 0; m < ctx->p.n_materials; ++m) out->dJ_dbedfrict[m] = red[m];
    out->dJ_dintfrict = red[ctx->p.n_materials];
    for (int q = 0; q < n_piles; ++q) out->dJ_dpile[q] = red[ctx->p.n_materials + 1 + q];
    return st;
}

}  // namespace

int adj_alloc_for_dwr(da_ctx *ctx) { return adj_alloc(ctx, 1); }

// Everything the sweep's launches take as arguments, byte for byte: a graph captured from them is
// replayed only for the same key (a different mesh, parameter, buffer, checkpoint slot, horizon,
// launch shape or starting buffer gives a new capture).
std::vector<unsigned char> sweep_key(const da_ctx *ctx, const double *box, int nsteps, int nsnap, int n_piles,
                                     bool seeded, const double *sec2, double cos_int) {
    std::vector<unsigned char> k;
    auto put = [&](const void *p, size_t b) {
        const unsigned char *c = (const unsigned char *)p;
        k.insert(k.end(), c, c + b);
    };
    // structs go in member by member: their padding bytes are not part of the key
    auto val = [&](const auto &v) { put(&v, sizeof(v)); };
    const int ints[] = {nsteps, nsnap, n_piles, seeded ? 1 : 0, ctx->cur, ctx->grid, ctx->ntiles, ctx->nseg,
                        ctx->ninst, ctx->mesh.n, ctx->sm_count};
    put(ints, sizeof(ints));
    double b4[4] = {0, 0, 0, 0};
    if (box) std::memcpy(b4, box, sizeof(b4));
    put(b4, sizeof(b4));
    put(sec2, sizeof(double) * DA_MAX_MATERIALS);
    put(&cos_int, sizeof(cos_int));
    const da_params &p = ctx->p;
    for (const int32_t v : {p.precision, p.device, p.n_materials, p.frict_tiny_iters, p.tile_culling, p.grid_blocks,
                            p.blocks_per_sm, p.tile_staging, p.jacobian_mode})
        val(v);
    for (const double v : {p.epsilon, p.gravity_scale, p.gamma, p.intfrict, p.frict_tiny_early, p.frict_tiny_late,
                           p.max_time, p.next_output, p.next_save, p.influx_dt, p.fp32_sign_floor})
        val(v);
    put(p.bedfrict, sizeof(p.bedfrict));
    const MatConsts &mc = ctx->mc;
    put(mc.kact_sgn, sizeof(mc.kact_sgn));
    put(mc.tan_bed, sizeof(mc.tan_bed));
    for (const double v : {mc.kact_rest, mc.epsilon, mc.sin_int, mc.gamma, mc.sign_floor}) val(v);
    val(mc.n_materials);
    const TimeConsts &tc = ctx->tc;
    for (const double v : {tc.next_output, tc.next_save, tc.max_time, tc.influx_dt, tc.gravity_scale, tc.epsilon,
                           tc.frict_tiny_early, tc.frict_tiny_late})
        val(v);
    for (const long long v : {tc.frict_tiny_iters, tc.iter0, tc.n_replay}) val(v);
    val(tc.dt_replay);
    const DevMesh &dm = ctx->mesh;
    for (const int32_t v : {dm.n, dm.epoch, dm.halo_max}) val(v);
    const void *mptr[] = {dm.nbr, dm.mat, dm.bflag, dm.x, dm.y, dm.dx, dm.dy, dm.g, dm.dg, dm.curv, dm.fdx, dm.fdy,
                          dm.fg, dm.fdg, dm.fcurv, dm.halo_off, dm.halo_idx, dm.nloc};
    put(mptr, sizeof(mptr));
    const InstArgs &ia = ctx->ia;
    val(ia.ninst);
    const void *iptr[] = {ia.tile_inst, ia.mcs, ia.time, ia.dt, ia.min_dxe, ia.hmax, ia.acc_min, ia.acc_max,
                          ia.sec2_bed, ia.cos_int, ia.dk_tab, ia.box, ia.seg0};
    put(iptr, sizeof(iptr));
    const void *ptrs[] = {ctx->U[0][0], ctx->U[0][1], ctx->U[0][2], ctx->U[1][0], ctx->U[1][1], ctx->U[1][2],
                          ctx->lam[0][0], ctx->lam[0][1], ctx->lam[0][2], ctx->lam[1][0], ctx->lam[1][1],
                          ctx->lam[1][2], ctx->kact, ctx->active, ctx->seg_clean, ctx->seg_wet, ctx->seg_vol,
                          ctx->seg_dirty, ctx->mask, ctx->tile_epoch, ctx->seg_act, ctx->lam_clean, ctx->adjA,
                          ctx->adjB, ctx->gbed, ctx->gint, ctx->dk_tab, ctx->red_out, ctx->red_part, ctx->inst_J,
                          ctx->seg_J, ctx->dh0, ctx->dsc};
    put(ptrs, sizeof(ptrs));
    put(ctx->snaps.data(), sizeof(void *) * ctx->snaps.size());
    return k;
}

// The reverse sweep shared by da_adjoint_run and da_ensemble_adjoint: checkpointed forward run
// over nsteps steps from the current state, reverse steps back to step 0, the state put back,
// J and the gradient sums launched (single: red_out[n_mat + 1 + n_piles]; ensemble: per member).
// lam0 receives the buffer that holds lambda^0.
// Without the DWR indicator (which reads every reverse step on the host) and without tracing, the
// sweep's thousand or so launches are captured once as a CUDA graph and replayed while nothing
// they depend on changes: a graph starts its cooperative kernels back to back, without the few
// microseconds of idle GPU between stream launches.  The recording ids the capture gave the
// reverse steps repeat on a replay, so the graph first clears the tiles' recording ids.
int adjoint_sweep(da_ctx *ctx, const double *box, int32_t nsteps, int32_t nsnapshots, int32_t n_piles, int *lam0,
                  long long *fsteps, float *dev_ms, void *dwr_acc, const double *lambda_end) {
    int st = adj_alloc(ctx, nsnapshots + 1);
    Runner r;
    r.ctx = ctx;
    r.dwr = (DwrAcc *)dwr_acc;
    if (box)
        for (int q = 0; q < 4; ++q) r.box[q] = box[q];
    if (!st) st = upload_tables(ctx, r.sec2, &r.cos_int);
    if (!st && lambda_end) {
        // lambda^N given (the adjoint carried back across a later mesh epoch): no functional seed,
        // J = 0 here; the two adjoint buffers differ everywhere
        const size_t n = (size_t)ctx->mesh.n;
        for (int v = 0; v < 3 && !st; ++v) st = upload_real(ctx, ctx->lam[0][v], lambda_end + v * n);
        if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->lam_clean, 0, ctx->nseg, ctx->stream), "memset");
        if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->seg_J, 0, sizeof(double) * ctx->nseg, ctx->stream), "memset");
        if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
        r.lam_cur = 0;
        r.seeded = true;
    }
    if (st) return st;
    // The sweep ends with a restore of the base checkpoint, which writes both ping-pong buffers:
    // afterwards the live buffer is the caller's again, so the next sweep starts from the same one
    // and replays the same captured graph.
    const int cur_in = ctx->cur;
    r.sch.use(ctx, nsteps, nsnapshots);
    for (int s = nsnapshots; s >= 1; --s) r.free_slots.push_back(s);
    // the launches of the sweep, from the base checkpoint to the gradient sums
    auto sweep = [&]() -> int {
        int s = store(ctx, 0);
        r.pos = 0;
        if (!s) s = r.reverse(0, nsteps, 0);
        if (!s) s = r.flush();
        if (!s) s = restore(ctx, 0);
        if (!s) s = launch_functional(ctx, ctx->inst_J);
        if (!s) s = ctx->ninst > 0 ? launch_adjoint_reduce_inst(ctx, r.lam_cur) : launch_adjoint_reduce(ctx, r.lam_cur, n_piles);
        return s;
    };
    bool graph = !r.dwr && !ctx->trace.on && ctx->p.jacobian_mode == DA_JAC_EXACT;
    if (graph) {
        std::vector<unsigned char> key = sweep_key(ctx, box, nsteps, nsnapshots, n_piles, r.seeded, r.sec2, r.cos_int);
        if (!ctx->sweep_graph || key != ctx->sweep_key) {
            if (ctx->sweep_graph) cudaGraphExecDestroy(ctx->sweep_graph);
            ctx->sweep_graph = nullptr;
            ctx->sweep_key.clear();
            // capture: nothing runs; the host-side state the launches leave is kept for replays
            const Runner r0 = r;
            const int cur0 = ctx->cur;
            cudaGraph_t g = nullptr;
            int s = cuda_check(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal),
                               "begin capture");
            if (!s) {
                int s2 = cuda_check(ctx, cudaMemsetAsync(ctx->tile_epoch, 0xff, sizeof(int) * ctx->ntiles, ctx->stream),
                                    "memset");
                if (!s2) s2 = sweep();
                const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
                s = s2 ? s2 : cuda_check(ctx, e, "end capture");
            }
            if (!s) s = cuda_check(ctx, cudaGraphInstantiate(&ctx->sweep_graph, g, 0), "instantiate");
            if (g) cudaGraphDestroy(g);
            if (!s) {
                ctx->sweep_key = key;
                ctx->sweep_lam = r.lam_cur;
                ctx->sweep_fsteps = r.fsteps;
            } else {
                // the launches one by one instead
                if (ctx->sweep_graph) cudaGraphExecDestroy(ctx->sweep_graph);
                ctx->sweep_graph = nullptr;
                cudaGetLastError();
                ctx->err.clear();
                graph = false;
            }
            ctx->cur = cur0;
            r = r0;
        }
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, ctx->stream);
    if (graph) {
        // the gradient sums are in the timed region
        st = cuda_check(ctx, cudaGraphLaunch(ctx->sweep_graph, ctx->stream), "sweep graph launch");
        r.lam_cur = ctx->sweep_lam;
        r.fsteps = ctx->sweep_fsteps;
    } else {
        st = sweep();
    }
    ctx->cur = cur_in;
    cudaEventRecord(e1, ctx->stream);
    if (!st) st = sync_check(ctx);
    float ms = 0.f;
    if (!st) cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!st) st = trace_flush(ctx);
    if (lam0) *lam0 = r.lam_cur;
    if (fsteps) *fsteps = r.fsteps;
    if (dev_ms) *dev_ms = ms;
    return st;
}

}  // namespace da

using namespace da;

extern "C" {

int da_set_dt_replay(da_ctx *ctx, const double *dts, int32_t n, int64_t iter0) {
    if (!ctx || (dts && n <= 0)) return DA_ERR_INVALID;
    cudaSetDevice(ctx->device);
    int st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (ctx->dt_replay) cudaFree(ctx->dt_replay);
    ctx->dt_replay = nullptr;
    ctx->tc.dt_replay = nullptr;
    ctx->tc.n_replay = 0;
    if (!dts || st) return st;
    st = cuda_check(ctx, cudaMalloc((void **)&ctx->dt_replay, sizeof(double) * n), "cudaMalloc(dt replay)");
    if (!st) st = copy_h2d(ctx, ctx->dt_replay, dts, sizeof(double) * n, "copy dts");
    if (st) return st;
    ctx->tc.dt_replay = ctx->dt_replay;
    ctx->tc.iter0 = iter0;
    ctx->tc.n_replay = n;
    for (int b = 0; b < 2; ++b) {
        if (ctx->step_graph[b]) cudaGraphExecDestroy(ctx->step_graph[b]);
        ctx->step_graph[b] = nullptr;
    }
    return DA_OK;
}

int da_adjoint_step(da_ctx *ctx, const double *lambda_next, double *lambda_out, da_gradient *partial) {
    if (!ctx || !lambda_next || !lambda_out) return DA_ERR_INVALID;
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, "da_adjoint_step: ensemble context");
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_adjoint_step: no mesh");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_adjoint_step: no state");
    cudaSetDevice(ctx->device);
    int st = adj_alloc(ctx, 1);
    double sec2[DA_MAX_MATERIALS], cos_int;
    if (!st) st = upload_tables(ctx, sec2, &cos_int);
    const size_t n = (size_t)ctx->mesh.n;
    // lambda_next into buffer 0
    for (int v = 0; v < 3 && !st; ++v) st = upload_real(ctx, ctx->lam[0][v], lambda_next + v * n);
    // the caller's lambda differs from buffer 1 everywhere
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->lam_clean, 0, ctx->nseg, ctx->stream), "memset");
    const bool ref = ctx->p.jacobian_mode == DA_JAC_REFERENCE;
    if (!st) st = store(ctx, 0);
    if (!st) st = launch_forward_step(ctx, ref ? nullptr : ctx->mask);
    if (!st) st = ref ? launch_ref_adjoint_step(ctx, ctx->cur ^ 1, 0, 1) : launch_adjoint_step(ctx, 0, 1, sec2, cos_int);
    if (!st) st = restore(ctx, 0);
    if (!st) st = sync_check(ctx);
    if (!st) st = copy_lambda_out(ctx, 1, lambda_out);
    if (!st && partial) {
        // parameter parts only (the pile term needs lambda^0 of a whole run)
        st = fill_gradient(ctx, 1, 0, partial);
        if (!st) partial->J = 0.0;
    }
    return st;
}

}  // extern "C"

namespace {

int adjoint_run_impl(da_ctx *ctx, const da_functional *f, int32_t nsteps, int32_t nsnapshots, const double *dh0_dpile,
                     int32_t n_piles, da_gradient *out, double *lambda0, DwrAcc *dwr,
                     const double *lambda_end = nullptr) {
    if (!ctx || (!f && !lambda_end) || nsteps <= 0 || nsnapshots < 0 || n_piles < 0 || n_piles > DA_MAX_PILES ||
        (n_piles > 0 && !dh0_dpile) || (f && f->kind != DA_FUNC_H2_BOX))
        return DA_ERR_INVALID;
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_adjoint_run: no mesh");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_adjoint_run: no state");
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, "da_adjoint_run: ensemble context (da_ensemble_adjoint)");
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)ctx->mesh.n;
    int st = DA_OK;
    if (n_piles > 0) {
        // kept between runs (a free synchronises the device)
        const size_t bytes = sizeof(double) * n * n_piles;
        if (ctx->dh0_bytes < bytes) {
            if (ctx->dh0) cudaFree(ctx->dh0);
            ctx->dh0 = nullptr;
            ctx->dh0_bytes = 0;
            st = cuda_check(ctx, cudaMalloc((void **)&ctx->dh0, bytes), "cudaMalloc(dh0)");
            if (!st) ctx->dh0_bytes = bytes;
        }
        if (!st) st = copy_h2d(ctx, ctx->dh0, dh0_dpile, bytes, "copy dh0");
    }
    int lam0 = 0;
    long long fsteps = 0;
    float dev_ms = 0.f;
    if (!st)
        st = adjoint_sweep(ctx, f ? f->box : nullptr, nsteps, nsnapshots, n_piles, &lam0, &fsteps, &dev_ms, dwr,
                           lambda_end);
    if (!st && lambda0) st = copy_lambda_out(ctx, lam0, lambda0);
    if (!st) st = fill_gradient(ctx, lam0, n_piles, out, /*reduced=*/true);
    if (!st && out) {
        out->forward_steps = fsteps;
        out->snapshots = nsnapshots;
        out->device_ms = dev_ms;
    }
    return st;
}

}  // namespace

extern "C" {

int da_adjoint_run(da_ctx *ctx, const da_functional *f, int32_t nsteps, int32_t nsnapshots, const double *dh0_dpile,
                   int32_t n_piles, da_gradient *out, double *lambda0) {
    return adjoint_run_impl(ctx, f, nsteps, nsnapshots, dh0_dpile, n_piles, out, lambda0, nullptr);
}

int da_adjoint_run_seeded(da_ctx *ctx, const double *lambda_end, int32_t nsteps, int32_t nsnapshots,
                          const double *dh0_dpile, int32_t n_piles, da_gradient *out, double *lambda0) {
    if (!lambda_end) return DA_ERR_INVALID;
    return adjoint_run_impl(ctx, nullptr, nsteps, nsnapshots, dh0_dpile, n_piles, out, lambda0, nullptr, lambda_end);
}

int da_adjoint_run_dwr(da_ctx *ctx, const da_functional *f, int32_t nsteps, int32_t nsnapshots,
                       const double *dh0_dpile, int32_t n_piles, da_gradient *out, double *lambda0,
                       double *cell_error, double *step_sums) {
    if (!ctx || !cell_error || !step_sums) return DA_ERR_INVALID;
    if (!ctx->dwr.fine) return set_error(ctx, DA_ERR_INVALID, "da_adjoint_run_dwr: no error grid (da_dwr_setup)");
    if (ctx->mesh.n <= 0 || nsteps <= 0) return da_adjoint_run(ctx, f, nsteps, nsnapshots, dh0_dpile, n_piles, out, lambda0);
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)ctx->mesh.n;
    DwrAcc acc;
    acc.step_sums = step_sums;
    acc.nsteps = nsteps;
    for (int k = 0; k < 2 * nsteps; ++k) step_sums[k] = 0.0;
    int st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (!st) st = copy_d2h(ctx, ctx->hsc, ctx->dsc, sizeof(DevScalars), "read scalars");
    acc.iter_begin = ctx->hsc->iter;
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&acc.cell, sizeof(double) * n), "cudaMalloc(dwr cells)");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(acc.cell, 0, sizeof(double) * n, ctx->stream), "memset");
    if (!st) st = adjoint_run_impl(ctx, f, nsteps, nsnapshots, dh0_dpile, n_piles, out, lambda0, &acc);
    if (!st) st = copy_d2h(ctx, cell_error, acc.cell, sizeof(double) * n, "copy dwr cells");
    if (acc.cell) cudaFree(acc.cell);
    return st;
}

}  // extern "C"
