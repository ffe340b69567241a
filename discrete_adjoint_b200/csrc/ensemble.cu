// Ensembles: many independent instances ("members") on one context, advanced by the same step
// kernels in one cooperative launch.
//
// Layout: member k's cells occupy [cell0[k], cell0[k] + n_k) of the concatenated mesh, cell0[k] a
// multiple of 256 so that every 256-cell tile (and every 32-cell segment) belongs to one member;
// the cells that pad a member to whole tiles have no neighbours, no depth and no box, so they
// stay dry and inert.  Neighbour indices are shifted by cell0[k].  The per-member device tables
// (InstArgs: tile -> member, material constants, time, dt, CFL accumulators, adjoint parameter
// tables, functional box, segment ranges) live in one allocation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "da_internal.h"

namespace da {

void free_members(da_ctx *ctx) {
    if (ctx->inst_mem) cudaFree(ctx->inst_mem);
    if (ctx->inst_vol) cudaFree(ctx->inst_vol);
    ctx->inst_mem = nullptr;
    ctx->inst_vol = nullptr;
    ctx->ninst = 0;
    ctx->ia = InstArgs{};
    ctx->inst_cell0.clear();
    ctx->inst_ncell.clear();
    ctx->inst_nmat.clear();
    ctx->inst_npile.clear();
    ctx->inst_init.clear();
}

namespace {

constexpr int kTile = 256;

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

int member_ok(const da_member &m) {
    const da_mesh_soa &s = m.mesh;
    if (s.n_cells <= 0 || !s.nbr || !s.x || !s.y || !s.dx || !s.dy || !s.gravity || !s.d_gravity || !s.curvature ||
        !s.material || !m.h0 || !m.hu0 || !m.hv0)
        return 0;
    if (m.n_materials < 1 || m.n_materials > DA_MAX_MATERIALS) return 0;
    return 1;
}

// Starting values of a member's step scalars (the same as a fresh single-instance context).
void reset_member_scalars(std::vector<double> &time, std::vector<unsigned long long> &acc_min,
                          std::vector<unsigned long long> &acc_max) {
    const double init = 10000000.0;  // min_dx_dy_evalue start value, get_coef_and_eigen.C:36
    unsigned long long bits;
    std::memcpy(&bits, &init, sizeof(bits));
    std::fill(time.begin(), time.end(), 0.0);
    std::fill(acc_min.begin(), acc_min.end(), bits);
    std::fill(acc_max.begin(), acc_max.end(), 0ull);
}

int upload_member_scalars(da_ctx *ctx) {
    const int nm = ctx->ninst;
    std::vector<double> time(nm);
    std::vector<unsigned long long> amin(nm), amax(nm);
    reset_member_scalars(time, amin, amax);
    int st = copy_h2d(ctx, ctx->ia.time, time.data(), sizeof(double) * nm, "copy");
    // dt, min_dxe, hmax of a member that has not stepped yet: zero
    if (!st) st = copy_h2d(ctx, ctx->ia.dt, time.data(), sizeof(double) * nm, "copy");
    if (!st) st = copy_h2d(ctx, ctx->ia.min_dxe, time.data(), sizeof(double) * nm, "copy");
    if (!st) st = copy_h2d(ctx, ctx->ia.hmax, time.data(), sizeof(double) * nm, "copy");
    if (!st) st = copy_h2d(ctx, ctx->ia.acc_min, amin.data(), sizeof(unsigned long long) * nm, "copy");
    if (!st) st = copy_h2d(ctx, ctx->ia.acc_max, amax.data(), sizeof(unsigned long long) * nm, "copy");
    return st;
}

}  // namespace
}  // namespace da

using namespace da;

extern "C" {

int da_ensemble_upload(da_ctx *ctx, const da_member *members, int32_t n_members) {
    if (!ctx || !members || n_members <= 0) return DA_ERR_INVALID;
    int max_mat = 1;
    size_t total = 0;
    std::vector<int32_t> cell0(n_members + 1);
    for (int k = 0; k < n_members; ++k) {
        if (!member_ok(members[k])) return set_error(ctx, DA_ERR_INVALID, "da_ensemble_upload: invalid member");
        max_mat = std::max(max_mat, (int)members[k].n_materials);
        cell0[k] = (int32_t)total;
        total += ((size_t)members[k].mesh.n_cells + kTile - 1) / kTile * kTile;
        if (total > (size_t)INT32_MAX / 8) return set_error(ctx, DA_ERR_INVALID, "da_ensemble_upload: too many cells");
        for (int i = 0; i < members[k].mesh.n_cells; ++i)
            if (members[k].mesh.material[i] < 0 || members[k].mesh.material[i] >= members[k].n_materials)
                return set_error(ctx, DA_ERR_INVALID, "da_ensemble_upload: material index out of range");
    }
    cell0[n_members] = (int32_t)total;
    const size_t N = total;
    cudaSetDevice(ctx->device);
    int st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (st) return st;
    free_members(ctx);

    // concatenated mesh and state
    std::vector<int32_t> nbr(8 * N, -1), mat(N, 0);
    std::vector<double> x(N, 0.0), y(N, 0.0), dx(N, 1.0), dy(N, 1.0), g(3 * N, 0.0), dg(2 * N, 0.0), cv(2 * N, 0.0);
    std::vector<double> init(3 * N, 0.0), dh0(N, 0.0);
    bool any_pile = false;
    for (size_t i = 0; i < N; ++i) g[2 * N + i] = 1.0;  // padding cells: level ground
    for (int k = 0; k < n_members; ++k) {
        const da_member &mb = members[k];
        const da_mesh_soa &s = mb.mesh;
        const size_t n = (size_t)s.n_cells, o = (size_t)cell0[k];
        for (int q = 0; q < 8; ++q)
            for (size_t i = 0; i < n; ++i) {
                const int32_t e = s.nbr[q * n + i];
                if (e >= (int32_t)n) return set_error(ctx, DA_ERR_INVALID, "da_ensemble_upload: neighbour out of range");
                nbr[q * N + o + i] = e < 0 ? -1 : e + (int32_t)o;
            }
        for (size_t i = 0; i < n; ++i) {
            x[o + i] = s.x[i];
            y[o + i] = s.y[i];
            dx[o + i] = s.dx[i];
            dy[o + i] = s.dy[i];
            mat[o + i] = s.material[i];
            for (int c = 0; c < 3; ++c) g[c * N + o + i] = s.gravity[c * n + i];
            for (int c = 0; c < 2; ++c) {
                dg[c * N + o + i] = s.d_gravity[c * n + i];
                cv[c * N + o + i] = s.curvature[c * n + i];
            }
            init[o + i] = mb.h0[i];
            init[N + o + i] = mb.hu0[i];
            init[2 * N + o + i] = mb.hv0[i];
            if (mb.dh0_dpile) dh0[o + i] = mb.dh0_dpile[i];
        }
        any_pile |= mb.dh0_dpile != nullptr;
    }
    const da_mesh_soa all = {(int32_t)N, nbr.data(), x.data(), y.data(), dx.data(), dy.data(),
                             g.data(), dg.data(), cv.data(), mat.data()};
    da_params p = ctx->p;
    p.n_materials = max_mat;
    for (int m = 0; m < DA_MAX_MATERIALS; ++m) p.bedfrict[m] = members[0].bedfrict[m < members[0].n_materials ? m : 0];
    p.intfrict = members[0].intfrict;
    ctx->p = p;
    fill_consts(ctx->p, &ctx->mc, &ctx->tc);
    st = da_upload_mesh(ctx, &all, 0);
    if (st) return st;

    // member tables: one allocation, 256-byte aligned pieces
    const int nm = n_members, ntiles = ctx->ntiles;
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off = align256(off + bytes); return o; };
    const size_t o_tile = take(sizeof(int32_t) * ntiles), o_mcs = take(sizeof(MatConsts) * nm),
                 o_time = take(sizeof(double) * nm), o_dt = take(sizeof(double) * nm),
                 o_mdx = take(sizeof(double) * nm), o_hmx = take(sizeof(double) * nm),
                 o_amin = take(sizeof(unsigned long long) * nm), o_amax = take(sizeof(unsigned long long) * nm),
                 o_sec2 = take(sizeof(double) * nm * DA_MAX_MATERIALS), o_cos = take(sizeof(double) * nm),
                 o_dk = take(sizeof(double) * nm * 2 * DA_MAX_MATERIALS * 3), o_box = take(sizeof(double) * nm * 4),
                 o_seg0 = take(sizeof(int32_t) * (nm + 1));
    st = cuda_check(ctx, cudaMalloc(&ctx->inst_mem, off), "cudaMalloc(members)");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->inst_vol, sizeof(double) * nm), "cudaMalloc(members)");
    if (st) {
        free_members(ctx);
        return st;
    }
    std::vector<unsigned char> host(off, 0);
    int32_t *tile = (int32_t *)(host.data() + o_tile);
    for (int k = 0; k < nm; ++k)
        for (int t = cell0[k] / kTile; t < cell0[k + 1] / kTile; ++t) tile[t] = k;
    MatConsts *mcs = (MatConsts *)(host.data() + o_mcs);
    double *sec2 = (double *)(host.data() + o_sec2), *cosi = (double *)(host.data() + o_cos);
    double *dk = (double *)(host.data() + o_dk), *box = (double *)(host.data() + o_box);
    int32_t *seg0 = (int32_t *)(host.data() + o_seg0);
    for (int k = 0; k < nm; ++k) {
        da_params pk = ctx->p;
        pk.n_materials = members[k].n_materials;
        for (int m = 0; m < DA_MAX_MATERIALS; ++m) pk.bedfrict[m] = m < pk.n_materials ? members[k].bedfrict[m] : 0.0;
        pk.intfrict = members[k].intfrict;
        TimeConsts tc;
        fill_consts(pk, &mcs[k], &tc);
        for (int m = 0; m < DA_MAX_MATERIALS; ++m) {
            const double t = m < pk.n_materials ? std::tan(pk.bedfrict[m]) : 0.0;
            sec2[k * DA_MAX_MATERIALS + m] = 1.0 + t * t;
        }
        cosi[k] = std::cos(pk.intfrict);
        double *dkk = dk + (size_t)k * 2 * DA_MAX_MATERIALS * 3;
        kact_derivatives(pk, dkk, dkk + DA_MAX_MATERIALS * 3);
        for (int q = 0; q < 4; ++q) box[k * 4 + q] = members[k].box[q];
        seg0[k] = cell0[k] / 32;
    }
    seg0[nm] = cell0[nm] / 32;
    st = copy_h2d(ctx, ctx->inst_mem, host.data(), off, "copy member tables");
    unsigned char *b = (unsigned char *)ctx->inst_mem;
    InstArgs &ia = ctx->ia;
    ia.ninst = nm;
    ia.tile_inst = (const int32_t *)(b + o_tile);
    ia.mcs = (const MatConsts *)(b + o_mcs);
    ia.time = (double *)(b + o_time);
    ia.dt = (double *)(b + o_dt);
    ia.min_dxe = (double *)(b + o_mdx);
    ia.hmax = (double *)(b + o_hmx);
    ia.acc_min = (unsigned long long *)(b + o_amin);
    ia.acc_max = (unsigned long long *)(b + o_amax);
    ia.sec2_bed = (const double *)(b + o_sec2);
    ia.cos_int = (const double *)(b + o_cos);
    ia.dk_tab = (const double *)(b + o_dk);
    ia.box = (const double *)(b + o_box);
    ia.seg0 = (const int32_t *)(b + o_seg0);
    ctx->ninst = nm;
    ctx->inst_cell0 = cell0;
    for (int k = 0; k < nm; ++k) {
        ctx->inst_ncell.push_back(members[k].mesh.n_cells);
        ctx->inst_nmat.push_back(members[k].n_materials);
        ctx->inst_npile.push_back(members[k].dh0_dpile ? 1 : 0);
    }
    ctx->inst_init.swap(init);
    if (!st) st = upload_member_scalars(ctx);
    if (!st && any_pile) {
        st = cuda_check(ctx, cudaMalloc((void **)&ctx->dh0, sizeof(double) * N), "cudaMalloc(dh0)");
        if (!st) ctx->dh0_bytes = sizeof(double) * N;
        if (!st) st = copy_h2d(ctx, ctx->dh0, dh0.data(), sizeof(double) * N, "copy dh0");
    }
    if (!st) st = da_ensemble_restart(ctx);
    if (st) free_members(ctx);
    return st;
}

int da_ensemble_restart(da_ctx *ctx) {
    if (!ctx) return DA_ERR_INVALID;
    if (ctx->ninst <= 0) return set_error(ctx, DA_ERR_INVALID, "da_ensemble_restart: not an ensemble context");
    const size_t N = (size_t)ctx->mesh.n;
    const int nm = ctx->ninst;
    ctx->ninst = 0;  // da_set_state is a single-context call; the layout is unchanged
    int st = da_set_state(ctx, ctx->inst_init.data(), ctx->inst_init.data() + N, ctx->inst_init.data() + 2 * N);
    ctx->ninst = nm;
    if (!st) st = da_set_time(ctx, 0.0, 0);
    if (!st) st = upload_member_scalars(ctx);
    return st;
}

int da_ensemble_forward(da_ctx *ctx, int32_t nsteps, double *device_ms) {
    if (!ctx || nsteps < 0) return DA_ERR_INVALID;
    if (ctx->ninst <= 0) return set_error(ctx, DA_ERR_INVALID, "da_ensemble_forward: not an ensemble context");
    cudaSetDevice(ctx->device);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int st = DA_OK;
    if (device_ms) {
        st = cuda_check(ctx, cudaEventCreate(&e0), "event");
        if (!st) st = cuda_check(ctx, cudaEventCreate(&e1), "event");
        if (!st) st = cuda_check(ctx, cudaEventRecord(e0, ctx->stream), "event record");
    }
    if (!st) st = launch_forward_steps(ctx, nsteps);
    if (!st && device_ms) {
        st = cuda_check(ctx, cudaEventRecord(e1, ctx->stream), "event record");
        if (!st) st = cuda_check(ctx, cudaEventSynchronize(e1), "event sync");
        float ms = 0.f;
        if (!st) st = cuda_check(ctx, cudaEventElapsedTime(&ms, e0, e1), "event time");
        *device_ms = ms;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    // in stream order: the context's stream does not synchronise with the legacy stream
    if (!st) st = cuda_check(ctx, cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost,
                                                  ctx->stream), "scalars");
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (!st) st = device_error(ctx, "ensemble run");
    return st;
}

int da_ensemble_stats(da_ctx *ctx, da_step_stats *out) {
    if (!ctx || !out) return DA_ERR_INVALID;
    if (ctx->ninst <= 0) return set_error(ctx, DA_ERR_INVALID, "da_ensemble_stats: not an ensemble context");
    cudaSetDevice(ctx->device);
    const int nm = ctx->ninst;
    std::vector<double> dt(nm), time(nm), vol(nm), hmax(nm);
    int st = launch_member_volume(ctx, ctx->inst_vol);
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (!st) st = copy_d2h(ctx, dt.data(), ctx->ia.dt, sizeof(double) * nm, "copy");
    if (!st) st = copy_d2h(ctx, time.data(), ctx->ia.time, sizeof(double) * nm, "copy");
    if (!st) st = copy_d2h(ctx, vol.data(), ctx->inst_vol, sizeof(double) * nm, "copy");
    if (!st) st = copy_d2h(ctx, hmax.data(), ctx->ia.hmax, sizeof(double) * nm, "copy");
    if (!st) st = copy_d2h(ctx, ctx->hsc, ctx->dsc, sizeof(DevScalars), "scalars");
    if (st) return st;
    for (int k = 0; k < nm; ++k) out[k] = da_step_stats{dt[k], time[k], vol[k], hmax[k], ctx->hsc->iter};
    return DA_OK;
}

int da_ensemble_get_state(da_ctx *ctx, int32_t member, double *h, double *hu, double *hv) {
    if (!ctx || !h || !hu || !hv) return DA_ERR_INVALID;
    if (ctx->ninst <= 0 || member < 0 || member >= ctx->ninst)
        return set_error(ctx, DA_ERR_INVALID, "da_ensemble_get_state: no such member");
    cudaSetDevice(ctx->device);
    const size_t N = (size_t)ctx->mesh.n;
    std::vector<double> all(3 * N);
    const int nm = ctx->ninst;
    ctx->ninst = 0;
    int st = da_get_state(ctx, all.data(), all.data() + N, all.data() + 2 * N);
    ctx->ninst = nm;
    if (st) return st;
    const size_t o = (size_t)ctx->inst_cell0[member], n = (size_t)ctx->inst_ncell[member];
    std::memcpy(h, all.data() + o, sizeof(double) * n);
    std::memcpy(hu, all.data() + N + o, sizeof(double) * n);
    std::memcpy(hv, all.data() + 2 * N + o, sizeof(double) * n);
    return DA_OK;
}

int da_ensemble_adjoint(da_ctx *ctx, int32_t nsteps, int32_t nsnapshots, da_gradient *out, double *device_ms) {
    if (!ctx || !out || nsteps <= 0 || nsnapshots < 0) return DA_ERR_INVALID;
    if (ctx->ninst <= 0) return set_error(ctx, DA_ERR_INVALID, "da_ensemble_adjoint: not an ensemble context");
    if (ctx->p.jacobian_mode != DA_JAC_EXACT)
        return set_error(ctx, DA_ERR_UNSUPPORTED, "da_ensemble_adjoint: ensembles use the exact adjoint");
    cudaSetDevice(ctx->device);
    const int nm = ctx->ninst, nout = ctx->p.n_materials + 2;
    int lam0 = 0;
    long long fsteps = 0;
    float ms = 0.f;
    int st = adjoint_sweep(ctx, nullptr, nsteps, nsnapshots, 1, &lam0, &fsteps, &ms);
    std::vector<double> red((size_t)nm * nout), J(nm);
    if (!st) st = copy_d2h(ctx, red.data(), ctx->red_out, sizeof(double) * red.size(), "read gradients");
    if (!st) st = copy_d2h(ctx, J.data(), ctx->inst_J, sizeof(double) * nm, "read J");
    if (st) return st;
    for (int k = 0; k < nm; ++k) {
        da_gradient &g = out[k];
        std::memset(&g, 0, sizeof(g));
        g.J = J[k];
        for (int m = 0; m < ctx->inst_nmat[k]; ++m) g.dJ_dbedfrict[m] = red[(size_t)k * nout + m];
        g.dJ_dintfrict = red[(size_t)k * nout + ctx->p.n_materials];
        if (ctx->inst_npile[k]) g.dJ_dpile[0] = red[(size_t)k * nout + ctx->p.n_materials + 1];
        g.forward_steps = fsteps;
        g.snapshots = nsnapshots;
        g.device_ms = ms;
    }
    if (device_ms) *device_ms = ms;
    return DA_OK;
}

}  // extern "C"
