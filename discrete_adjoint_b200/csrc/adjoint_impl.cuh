// Discrete adjoint of one forward step (order_flag = 1), matrix free, for sm_100a.
//
// The reference assembles 9 blocks of 3x3 d R^n / d U^{n-1} per element (calc_jacobian,
// src/adjoint/calc_jacobain.C:40-153; calc_jacobian_elem, compute_jacobian_elem.C:15-121; flux
// Jacobians dual_riemannflux, src/datstr/dualmesh.C:1628-1843) and multiplies their transposes
// into the adjoint (calc_adjoint_elem, src/adjoint/calc_adjoint.C:74-167).  Here the transpose
// of the step is applied without forming blocks:
//   k_adj_src    (one pass over cells i): with lambda_eff_i = lambda^{n+1}_i (depth row dropped
//                where the forward step clamped h at zero), the source terms of update_states
//                (residual.C:162-275) give d(lambda_eff_i . dt S_i)/dU_i (A_i) and the
//                coefficients B_i that the limited depth slopes of cell i pass to its neighbours
//                (the limiter branch is replayed from U^n, as DualElem::get_slopes_prev +
//                hslope_sens do, dualmesh.C:1393-1626);
//   k_adj_gather (one pass over cells j): lambda^n_j = lambda_eff_j + A_j + sum over the
//                Riemann fluxes on j's sides of (dF/dU_j)^T mu, with mu the flux weight of the
//                edge in both cells that use it (hanging sides weigh 1/2, outflow directions 0),
//                plus the slope coefficients B of the neighbours for j.
// k act/pass and the depth clamp come from the branch codes recorded while the forward step was
// replayed; the time step is the forward's (frozen).  Parameter sensitivities (basal friction per
// material, internal friction, through tan/sin in the sources and through k act/pass in fluxes
// and sources) are accumulated per cell in FP64 and reduced at the end.
#pragma once
#include <cuda_runtime.h>

#include "fv_device.cuh"

namespace da {
namespace adj {
namespace {

using namespace fv;

constexpr int kBlock = kTileCells;  // one thread per cell of a tile

// k act/pass of a recorded code (0 rest, 1..3 sgn(vel) = -1, 0, +1)
template <class R>
__device__ __forceinline__ R kact_of(const MatConsts &mc, int mat, uint8_t code) {
    return code == 0 ? R(mc.kact_rest) : R(mc.kact_sgn[mat][code - 1]);
}

// The 8 one-byte segment flags of tile t as one 8-byte load (flag arrays are padded to tiles).
__device__ __forceinline__ unsigned long long seg_flags8(const uint8_t *flags, int t) {
    return *reinterpret_cast<const unsigned long long *>(flags + (size_t)t * 8);
}

// Mask byte of cell i in the current recording step: tiles the step did not list count as zero.
__device__ __forceinline__ uint8_t mask_of(const uint8_t *__restrict__ mask, const int *__restrict__ epoch, int rec_id,
                                           int i) {
    return epoch[i >> 8] == rec_id ? mask[i] : uint8_t(0);
}

template <class R>
__device__ __forceinline__ void lam_eff(const StateRef<R> &L, uint8_t mk, int i, R out[3]) {
    out[0] = (mk & 4) ? R(0) : L.h[i];
    out[1] = L.hu[i];
    out[2] = L.hv[i];
}


// Derivative data of the limited depth slope in one direction (Element::get_slopes for j = 0):
// slope = fac * min(gamma|dp|, gamma|dm|, |dc|); g_dp, g_dm = d slope / d dp, d dm.
template <class R>
struct SlopeD {
    R g_dp, g_dm, dxp, dxm;
};

// v: where the depths, neighbours and centres / sizes come from (global arrays, or a tile staged
// in shared memory with i the cell's slot); the arithmetic is the same either way.
template <class R, class V>
__device__ __forceinline__ void h_slope_deriv(const V &v, int i, uint8_t bf, R gamma, R hi, SlopeD<R> out[2]) {
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
        const int ep = v.nb(dir, i);
        const int em = v.nb(dir + 2, i);
        const bool two_p = bf & (0x10 << dir), two_m = bf & (0x10 << (dir + 2));
        R dxp, dxm, dp, dm;
        if constexpr (sizeof(R) == 8) {
            const double ci = v.coord(dir, i);
            dxp = v.coord(dir, ep) - ci;
            dxm = ci - v.coord(dir, em);
            dp = (v.h(ep) - hi) / dxp;
            if (two_p) dp = .5 * (dp + (v.h(v.nb(dir + 4, i)) - hi) / dxp);
            dm = (hi - v.h(em)) / dxm;
            if (two_m) dm = .5 * (dm + (hi - v.h(v.nb(dir + 6, i))) / dxm);
        } else {
            const float si = v.size(dir, i);
            dxp = 0.5f * (v.size(dir, ep) + si);
            dxm = 0.5f * (v.size(dir, em) + si);
            const float ip = 1.0f / dxp, im = 1.0f / dxm;
            dp = (v.h(ep) - hi) * ip;
            if (two_p) dp = 0.5f * (dp + (v.h(v.nb(dir + 4, i)) - hi) * ip);
            dm = (hi - v.h(em)) * im;
            if (two_m) dm = 0.5f * (dm + (hi - v.h(v.nb(dir + 6, i))) * im);
        }
        const R dc = (dp * dxm + dm * dxp) / (dxm + dxp);
        const R fac = R(.5) * (c_sgn(dp) + c_sgn(dm));
        const R a = gamma * dabs(dp), b = gamma * dabs(dm), c = dabs(dc);
        // selection order of c_dmin1(a, b, c) (geoflow.h:112-120)
        int sel = 0;
        R mn = a;
        if (mn > b) { mn = b; sel = 1; }
        if (mn > c) { mn = c; sel = 2; }
        const auto sgnf = [](R v) { return v > R(0) ? R(1) : (v < R(0) ? R(-1) : R(0)); };
        R gdp = 0, gdm = 0;
        if (sel == 0) gdp = fac * gamma * sgnf(dp);
        else if (sel == 1) gdm = fac * gamma * sgnf(dm);
        else {
            const R gc = fac * sgnf(dc) / (dxm + dxp);
            gdp = gc * dxm;
            gdm = gc * dxp;
        }
        out[dir] = SlopeD<R>{gdp, gdm, dxp, dxm};
    }
}

// Forward pieces of one side's Riemann flux with what the reverse sweep needs.
template <class R>
struct Side {
    R h, hu, hv, k, gz;
    Hfv<R> f;
    R vel, a;
};

template <class R>
__device__ __forceinline__ void make_side(int dir, R h, R hu, R hv, R k, R gz, Side<R> &s) {
    s.h = h; s.hu = hu; s.hv = hv; s.k = k; s.gz = gz;
    dirflux<R>(dir, h, hu, hv, k, gz, s.f);
    if (h < R(DA_TINY)) {
        s.vel = s.a = R(0);
    } else {
        s.a = sqrt(k * h * gz);
        s.vel = (dir == 0 ? hu : hv) / h;
    }
}

// Reverse of dirflux for a wet side: adjoints of (u, f, s) -> adjoints of (h, hu, hv, k).
template <class R>
__device__ __forceinline__ void dirflux_adj(int dir, const Side<R> &s, const R au[3], const R af[3], const R as[3],
                                            R g[3], R &gk) {
    if (s.h < R(DA_TINY)) {
        g[0] = g[1] = g[2] = R(0);
        gk = R(0);
        return;
    }
    // derivatives only (no branch depends on them): one reciprocal of h serves all quotients
    const R vel = s.vel, a = s.a, h = s.h;
    const R ih = R(1) / h;
    const R da_dh = a > R(0) ? R(0.5) * a * ih : R(0);
    const R da_dk = (a > R(0) && s.k > R(0)) ? R(0.5) * a / s.k : R(0);
    const R avel_s = as[0] + as[1] + as[2];
    const R aa = -as[0] + as[2];
    if (dir == 0) {
        const R avel = af[1] * s.hu + af[2] * s.hv + avel_s;
        const R aaa = aa + af[1] * a * h;
        g[0] = au[0] + af[1] * R(0.5) * a * a - avel * vel * ih + aaa * da_dh;
        g[1] = au[1] + af[0] + af[1] * vel + avel * ih;
        g[2] = au[2] + af[2] * vel;
        gk = aaa * da_dk;
    } else {
        const R avel = af[1] * s.hu + af[2] * s.hv + avel_s;
        const R aaa = aa + af[2] * a * h;
        g[0] = au[0] + af[2] * R(0.5) * a * a - avel * vel * ih + aaa * da_dh;
        g[1] = au[1] + af[1] * vel;
        g[2] = au[2] + af[0] + af[2] * vel + avel * ih;
        gk = aaa * da_dk;
    }
}

// mu^T dF/d(left, right) for F = riemannflux(left, right) (element2.C:2228-2264), with the
// branch decisions of the forward evaluation.
template <class R>
__device__ __forceinline__ void riemann_adj(int dir, const Side<R> &L, const Side<R> &Rt, const R mu[3], R gL[3],
                                            R gR[3], R &gkL, R &gkR) {
    gL[0] = gL[1] = gL[2] = gR[0] = gR[1] = gR[2] = R(0);
    gkL = gkR = R(0);
    const Hfv<R> &l = L.f, &r = Rt.f;
    if (l.u[0] == R(0) && r.u[0] == R(0)) return;
    R sl, sr;
    // speed sources: 0 = the zero bound, 1 = wet-wet pick, 2 = dry-side formula
    int which_l = 0, which_r = 0;
    bool l_from_left = false, r_from_left = false;
    if (l.u[0] == R(0)) {
        const R cl = R(2.0) * r.s[0] - r.s[1], cr = R(2.0) * r.s[2] - r.s[1];
        sl = rmin(R(0), cl);
        sr = rmax(R(0), cr);
        which_l = (R(0) > cl) ? 2 : 0;
        which_r = (R(0) > cr) ? 0 : 2;
        l_from_left = r_from_left = false;
    } else if (r.u[0] == R(0)) {
        const R cl = R(2.0) * l.s[0] - l.s[1], cr = R(2.0) * l.s[2] - l.s[1];
        sl = rmin(R(0), cl);
        sr = rmax(R(0), cr);
        which_l = (R(0) > cl) ? 2 : 0;
        which_r = (R(0) > cr) ? 0 : 2;
        l_from_left = r_from_left = true;
    } else {
        const R ml = rmin(l.s[0], r.s[0]);
        l_from_left = !(l.s[0] > r.s[0]);
        const R mr = rmax(l.s[2], r.s[2]);
        r_from_left = l.s[2] > r.s[2];
        sl = rmin(R(0), ml);
        sr = rmax(R(0), mr);
        which_l = (R(0) > ml) ? 1 : 0;
        which_r = (R(0) > mr) ? 0 : 1;
    }
    R afl[3] = {0, 0, 0}, afr[3] = {0, 0, 0}, aul[3] = {0, 0, 0}, aur[3] = {0, 0, 0};
    R asl[3] = {0, 0, 0}, asr[3] = {0, 0, 0};
    if (sl >= R(0)) {
        afl[0] = mu[0]; afl[1] = mu[1]; afl[2] = mu[2];
    } else if (sr <= R(0)) {
        afr[0] = mu[0]; afr[1] = mu[1]; afr[2] = mu[2];
    } else {
        // derivatives of F = (sr fl - sl fr + sl sr du) / D: one reciprocal of D serves them all
        const R iD = R(1) / (sr - sl);
        R a_sr = 0, a_sl = 0;
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const R du = r.u[v] - l.u[v];
            const R F = (sr * l.f[v] - sl * r.f[v] + sl * sr * du) * iD;
            afl[v] = mu[v] * sr * iD;
            afr[v] = -mu[v] * sl * iD;
            aur[v] = mu[v] * sl * sr * iD;
            aul[v] = -aur[v];
            a_sr += mu[v] * (l.f[v] + sl * du - F) * iD;
            a_sl += mu[v] * (-r.f[v] + sr * du + F) * iD;
        }
        // route d/dsl, d/dsr to the Davis speeds they were taken from
        if (which_l == 1) {
            if (l_from_left) asl[0] += a_sl; else asr[0] += a_sl;
        } else if (which_l == 2) {
            if (l_from_left) { asl[0] += R(2) * a_sl; asl[1] -= a_sl; } else { asr[0] += R(2) * a_sl; asr[1] -= a_sl; }
        }
        if (which_r == 1) {
            if (r_from_left) asl[2] += a_sr; else asr[2] += a_sr;
        } else if (which_r == 2) {
            if (r_from_left) { asl[2] += R(2) * a_sr; asl[1] -= a_sr; } else { asr[2] += R(2) * a_sr; asr[1] -= a_sr; }
        }
    }
    // asl/asr above hold the speed adjoints of the left / right side respectively
    dirflux_adj<R>(dir, L, aul, afl, asl, gL, gkL);
    dirflux_adj<R>(dir, Rt, aur, afr, asr, gR, gkR);
}

// Arrays written and read within one launch of the fused step kernel carry no __restrict__
// (coherent loads, no read-only cache).
struct AdjArgs {
    const uint8_t *mask;                // branch codes of the replayed forward step
    const int *tile_epoch;              // recording step that last listed each tile
    const uint8_t *seg_act;             // [nseg] the segment had an active cell in that step
    uint8_t *lam_clean;                 // [nseg] both adjoint buffers hold the same segment
    int rec_id;
    int ntiles;
    double *A;                          // [3][n] source adjoint of each cell (FP64)
    double *B;                          // [4][n] slope coefficients per side
    double *gbed;                       // [n] running d J / d phi_bed of each cell (its material)
    double *gint;                       // [n] running d J / d phi_int of each cell
    const double *__restrict__ dk_dbed; // [DA_MAX_MATERIALS][3] d kact / d phi_bed per sgn branch
    const double *__restrict__ dk_dint; // [DA_MAX_MATERIALS][3]
    double sec2_bed[DA_MAX_MATERIALS];  // 1 + tan^2(phi_bed)
    double cos_int;
};

__device__ __forceinline__ double dk_of(const double *tab, int mat, uint8_t code) {
    return code == 0 ? 0.0 : tab[mat * 3 + (code - 1)];
}

// ------------------------------------------------------------------------- k_adj_src
// Per-member tables of an ensemble tile (BATCH): material constants, dt and the parameter tables.
struct InstTables {
    const double *sec2_bed;
    double cos_int;
    const double *dk_dbed, *dk_dint;
};

template <bool BATCH>
__device__ __forceinline__ InstTables inst_tables(const AdjArgs &aa, const InstArgs &ia, int inst) {
    if (!BATCH) return InstTables{aa.sec2_bed, aa.cos_int, aa.dk_dbed, aa.dk_dint};
    const double *dk = ia.dk_tab + (size_t)inst * 2 * DA_MAX_MATERIALS * 3;
    return InstTables{ia.sec2_bed + (size_t)inst * DA_MAX_MATERIALS, ia.cos_int[inst], dk, dk + DA_MAX_MATERIALS * 3};
}

// The source adjoint of one cell (the body of the source phase): for a wet cell of U^n the
// adjoint of its sources (A), the slope coefficients it passes to its neighbours (B) and its
// parameter sensitivities, from its own recorded branches (mask) and lambda^{n+1}.  Reads U^n
// at the cell and its neighbours; writes only the cell's own entries.
// adj_src_wet: wet cell i with U^n = prev, g_z, branch byte mi, boundary flags bf, lambda^{n+1}
// = lnext and source coefficients cs; v and vi give the neighbour values of the slopes (global
// arrays with vi = i, or the tile staged in shared memory with vi the cell's slot).
// The forward's slopes, velocities and friction signs of wet cell vi (update_cell's arithmetic).
template <class R, class V>
__device__ __forceinline__ SrcFwd<R> src_fwd(const V &v, int vi, uint8_t bf, const R prev[3], R gamma, R ft) {
    SrcFwd<R> f;
    cell_slopes<R>(v, vi, bf, gamma, prev, f.s);
    if constexpr (sizeof(R) == 8) {
        f.vel0 = prev[1] / prev[0];
        f.vel1 = prev[2] / prev[0];
        f.h_inv = 1. / prev[0];
    } else {
        f.h_inv = 1.0f / prev[0];
        f.vel0 = prev[1] * f.h_inv;
        f.vel1 = prev[2] * f.h_inv;
    }
    f.sg0 = tiny_sgn(f.h_inv * (f.s[4] - f.vel0 * f.s[3]), ft);
    f.sg2 = tiny_sgn(f.vel0, ft);
    f.sg1 = tiny_sgn(f.h_inv * (f.s[2] - f.vel1 * f.s[0]), ft);
    f.sg3 = tiny_sgn(f.vel1, ft);
    return f;
}

// get_f() gives the forward's quantities of the cell (computed, or handed over by the update).
template <class R, class V, class GetF>
__device__ __forceinline__ void adj_src_wet(const V &v, int vi, const MeshArgs &m, const R prev[3], R gz,
                                            uint8_t mi, uint8_t bf, const R lnext[3], const CellSrc<R> &cs,
                                            const MatConsts &mc, const AdjArgs &aa, const InstTables &it, R dt, R ft,
                                            int i, const GetF &get_f) {
    double A[3] = {0, 0, 0}, B[4] = {0, 0, 0, 0};
    {
        // lambda_eff: the depth row dropped where the forward step clamped h at zero
        const R le[3] = {(mi & 4) ? R(0) : lnext[0], lnext[1], lnext[2]};
        const R nu_u = dt * le[1], nu_v = dt * le[2];
        if (nu_u != R(0) || nu_v != R(0)) {
            const int mat = cs.mat;
            const uint8_t code = mi & 3;
            const R k = kact_of<R>(mc, mat, code);
            // the parameter tables of the cell's branch, loaded ahead of the arithmetic
            const double sec2 = it.sec2_bed[mat], dkb = dk_of(it.dk_dbed, mat, code),
                         dki = dk_of(it.dk_dint, mat, code);
            const SrcFwd<R> f = get_f();
            const R *s = f.s;
            const R vel0 = f.vel0, vel1 = f.vel1;
            const R sg0 = f.sg0, sg1 = f.sg1, sg2 = f.sg2, sg3 = f.sg3;
            const R h = prev[0];
            const R gx = cs.g[0], gy = cs.g[1];
            const R dgx = cs.dg[0], dgy = cs.dg[1];
            const R kx = cs.cv[0], ky = cs.cv[1];
            const R sin_int = R(mc.sin_int), tan_bed = R(mc.tan_bed[mat]);
            const R Px = gz * h + vel0 * prev[1] * kx, Py = gz * h + vel1 * prev[2] * ky;
            const R px = Px > R(0) ? R(1) : R(0), py = Py > R(0) ? R(1) : R(0);
            const R wx = gz * s[3] + dgy * h, wy = gz * s[0] + dgx * h;
            A[0] = double(nu_u * (gx - sg0 * k * sin_int * (wx + dgy * h) - sg2 * tan_bed * px * (gz - vel0 * vel0 * kx)) +
                          nu_v * (gy - sg1 * k * sin_int * (wy + dgx * h) - sg3 * tan_bed * py * (gz - vel1 * vel1 * ky)));
            A[1] = double(nu_u * (-sg2 * tan_bed * px * R(2) * vel0 * kx));
            A[2] = double(nu_v * (-sg3 * tan_bed * py * R(2) * vel1 * ky));
            // the limited depth slopes of this cell (zero on boundary cells)
            if (!(bf & 0x0F)) {
                SlopeD<R> sd[2];
                h_slope_deriv<R>(v, vi, bf, R(mc.gamma), h, sd);
                const R cx = -nu_v * sg1 * h * k * gz * sin_int;  // on d h / dx
                const R cy = -nu_u * sg0 * h * k * gz * sin_int;  // on d h / dy
                // d slope / d h at the neighbours: g / (centre distance)
                const R qp0 = sd[0].g_dp / sd[0].dxp, qm0 = sd[0].g_dm / sd[0].dxm;
                const R qp1 = sd[1].g_dp / sd[1].dxp, qm1 = sd[1].g_dm / sd[1].dxm;
                A[0] += double(cx * (-qp0 + qm0) + cy * (-qp1 + qm1));
                B[0] = double(cx * qp0);
                B[2] = double(-cx * qm0);
                B[1] = double(cy * qp1);
                B[3] = double(-cy * qm1);
            }
            // parameter sensitivities of the sources
            const double dJ_dk = double(-nu_u * sg0 * h * wx * sin_int - nu_v * sg1 * h * wy * sin_int);
            const double dJ_dsin = double(-nu_u * sg0 * h * k * wx - nu_v * sg1 * h * k * wy);
            const double dJ_dtan = double(-nu_u * sg2 * (Px > R(0) ? Px : R(0)) - nu_v * sg3 * (Py > R(0) ? Py : R(0)));
            const double gb = dJ_dtan * sec2 + dJ_dk * dkb;
            const double gi = dJ_dsin * it.cos_int + dJ_dk * dki;
            if (gb != 0.0) aa.gbed[i] += gb;
            if (gi != 0.0) aa.gint[i] += gi;
        }
    }
    aa.A[i] = A[0];
    aa.A[(size_t)m.n + i] = A[1];
    aa.A[(size_t)2 * m.n + i] = A[2];
#pragma unroll
    for (int s = 0; s < 4; ++s) aa.B[(size_t)s * m.n + i] = B[s];
}

// adj_src_cell: cell i of U^n from global memory (nothing for a dry cell).
template <class R>
__device__ __forceinline__ void adj_src_cell(const MeshArgs &m, const StateRef<R> &U, const StateRef<R> &Lnext,
                                             const MatConsts &mc, const AdjArgs &aa, const InstTables &it, R dt,
                                             R ft, int i) {
    const R h_i = U.h[i];
    // A and B exist for wet cells only; k_adj_gather reads them only there
    if (!(h_i > R(DA_TINY))) return;
    const R prev[3] = {h_i, U.hu[i], U.hv[i]};
    const R lnext[3] = {Lnext.h[i], Lnext.hu[i], Lnext.hv[i]};
    const GlobalView<R> v = global_view<R>(m, U, (const R *)nullptr);
    const uint8_t bf = m.bflag[i];
    adj_src_wet<R>(v, i, m, prev, grav<R>(m, 2, i), aa.mask[i], bf, lnext, cell_src<R>(m, i), mc, aa, it, dt, ft, i,
                   [&]() { return src_fwd<R>(v, i, bf, prev, R(mc.gamma), ft); });
}

template <class R, bool BATCH = false>
__device__ __forceinline__ void adj_src_phase(const MeshArgs &m, const StateRef<R> &U, const StateRef<R> &Lnext,
                                              const MatConsts &mc0, const AdjArgs &aa, R dt0, R ft, int *list,
                                              const InstArgs &ia) {
    for (int round = 0; sched_more(round, aa.ntiles); ++round) {
      const int tq = sched_tile(round);
      // a wet cell is active, so its tile was listed by the recording step and had an active cell
      const bool need = tq < aa.ntiles && aa.tile_epoch[tq] == aa.rec_id && seg_flags8(aa.seg_act, tq) != 0ull;
      const int cnt = compact_tiles(need, tq, list);
      for (int q = 0; q < cnt; ++q) {
        const int t = list[q];
        const int inst = BATCH ? ia.tile_inst[t] : 0;
        const MatConsts &mc = BATCH ? ia.mcs[inst] : mc0;
        const R dt = BATCH ? R(ia.dt[inst]) : dt0;
        const InstTables it = inst_tables<BATCH>(aa, ia, inst);
        const int i = t * kBlock + threadIdx.x;
        if (i >= m.n) continue;
        adj_src_cell<R>(m, U, Lnext, mc, aa, it, dt, ft, i);
      }
    }
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_adj_src(MeshArgs m, StateRef<R> U, StateRef<R> Lnext, MatConsts mc,
                                                    AdjArgs aa, const DevScalars *__restrict__ sc, R sign_floor) {
    __shared__ int list[kBlock];
    const R dt = R(sc->dt);
    const R ft = R(sc->frict_tiny) > sign_floor ? R(sc->frict_tiny) : sign_floor;
    adj_src_phase<R>(m, U, Lnext, mc, aa, dt, ft, list, InstArgs{});
}

// Flux weight of cell c for its side s: -dt/dx on a plus side, +dt/dx on a minus side, halved
// when the side carries two finer neighbours, zero when c's direction has an outflow side.
template <class R>
__device__ __forceinline__ bool side_outflow(uint8_t bf, int s) {
    const int d = s & 1;
    return (bf & ((1 << d) | (1 << (d + 2)))) != 0;
}
// the weight of a side that is not an outflow direction, with dxc the cell's size across it
template <class R>
__device__ __forceinline__ R side_weight_of(R dxc, uint8_t bf, int s, R dt) {
    R w = (s < 2 ? -dt : dt) / dxc;
    if (bf & (0x10 << s)) w = R(0.5) * w;
    return w;
}
template <class R>
__device__ __forceinline__ R side_weight(const MeshArgs &m, int c, uint8_t bf, int s, R dt) {
    if (side_outflow<R>(bf, s)) return R(0);
    const int d = s & 1;
    return side_weight_of<R>(d == 0 ? cell_dx<R>(m, c) : cell_dy<R>(m, c), bf, s, dt);
}

// A side from the cell's values: k act/pass from its material and branch code where it is wet.
template <class R>
__device__ __forceinline__ void side_of(const MatConsts &mc, int dir, R h, R hu, R hv, R gz, int mat, uint8_t mk,
                                        Side<R> &s) {
    const R k = h >= R(DA_TINY) ? kact_of<R>(mc, mat, mk & 3) : R(0);
    make_side<R>(dir, h, hu, hv, k, gz, s);
}
template <class R>
__device__ __forceinline__ void load_side(const MeshArgs &m, const StateRef<R> &U, const MatConsts &mc, uint8_t mk,
                                          int c, int dir, Side<R> &s) {
    side_of<R>(mc, dir, U.h[c], U.hu[c], U.hv[c], grav<R>(m, 2, c), m.mat[c], mk, s);
}

// ---------------------------------------------------------------------- k_adj_gather
template <class R, bool BATCH = false>
__device__ __forceinline__ void adj_gather_phase(const MeshArgs &m, const StateRef<R> &U, const StateRef<R> &Lnext,
                                                 const StateOut<R> &Lout, const MatConsts &mc0, const AdjArgs &aa,
                                                 R dt0, int *list, const InstArgs &ia) {
    for (int round = 0; sched_more(round, aa.ntiles); ++round) {
      const int tq = sched_tile(round);
      bool need = false;
      if (tq < aa.ntiles)
          need = (aa.tile_epoch[tq] == aa.rec_id && seg_flags8(aa.seg_act, tq) != 0ull) ||
                 seg_flags8(aa.lam_clean, tq) != 0x0101010101010101ull;
      const int cnt = compact_tiles(need, tq, list);
      for (int q = 0; q < cnt; ++q) {
        const int t = list[q];
        const int inst = BATCH ? ia.tile_inst[t] : 0;
        const MatConsts &mc = BATCH ? ia.mcs[inst] : mc0;
        const R dt = BATCH ? R(ia.dt[inst]) : dt0;
        const int j = t * kBlock + threadIdx.x;
        const bool recorded = aa.tile_epoch[t] == aa.rec_id;
        const bool seg_active = recorded && aa.seg_act[j >> 5];
        if ((threadIdx.x & 31) == 0) aa.lam_clean[j >> 5] = seg_active ? 0 : 1;
        if (j >= m.n) continue;
        const uint8_t mj = seg_active ? aa.mask[j] : uint8_t(0);
        if (!(mj & 8)) {
            // not active in the forward step: its update was the identity, and no neighbour is wet
            Lout.h[j] = Lnext.h[j];
            Lout.hu[j] = Lnext.hu[j];
            Lout.hv[j] = Lnext.hv[j];
            continue;
        }
        R lj[3];
        lam_eff<R>(Lnext, mj, j, lj);
        double out[3] = {double(lj[0]), double(lj[1]), double(lj[2])};
        const R h_j = U.h[j];
        if (h_j > R(DA_TINY)) {
            out[0] += aa.A[j];
            out[1] += aa.A[(size_t)m.n + j];
            out[2] += aa.A[(size_t)2 * m.n + j];
        }
        const uint8_t bf = m.bflag[j];
        double dJ_dkj = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (bf & (1 << s)) continue;
            const int d = s & 1;
            const bool plus = s < 2;
            const int ne = (bf & (0x10 << s)) ? 2 : 1;
            for (int qq = 0; qq < ne; ++qq) {
                const int k = m.nbr[(size_t)(s + 4 * qq) * m.n + j];
                const uint8_t bk = m.bflag[k];
                const R h_k = U.h[k];
                if (h_k > R(DA_TINY)) {
                    // slope coefficient of neighbour k for j (k's side s^2 faces j)
                    double bk_s = aa.B[(size_t)(s ^ 2) * m.n + k];
                    if (bk & (0x10 << (s ^ 2))) bk_s *= 0.5;
                    out[0] += bk_s;
                }
                if (!(h_k >= R(DA_TINY) || h_j >= R(DA_TINY))) continue;
                const R wj = side_weight<R>(m, j, bf, s, dt);
                const R wk = side_weight<R>(m, k, bk, s ^ 2, dt);
                if (wj == R(0) && wk == R(0)) continue;
                const uint8_t mk = mask_of(aa.mask, aa.tile_epoch, aa.rec_id, k);
                R lk[3];
                lam_eff<R>(Lnext, mk, k, lk);
                const R mu[3] = {wj * lj[0] + wk * lk[0], wj * lj[1] + wk * lk[1], wj * lj[2] + wk * lk[2]};
                if (mu[0] == R(0) && mu[1] == R(0) && mu[2] == R(0)) continue;
                Side<R> sj, sk;
                load_side<R>(m, U, mc, mj, j, d, sj);
                load_side<R>(m, U, mc, mk, k, d, sk);
                R gL[3], gR[3], gkL, gkR;
                if (plus) {
                    riemann_adj<R>(d, sj, sk, mu, gL, gR, gkL, gkR);
                    out[0] += double(gL[0]); out[1] += double(gL[1]); out[2] += double(gL[2]);
                    dJ_dkj += double(gkL);
                } else {
                    riemann_adj<R>(d, sk, sj, mu, gL, gR, gkL, gkR);
                    out[0] += double(gR[0]); out[1] += double(gR[1]); out[2] += double(gR[2]);
                    dJ_dkj += double(gkR);
                }
            }
        }
        Lout.h[j] = R(out[0]);
        Lout.hu[j] = R(out[1]);
        Lout.hv[j] = R(out[2]);
        if (dJ_dkj != 0.0) {
            const uint8_t code = mj & 3;
            const int mat = m.mat[j];
            const InstTables it = inst_tables<BATCH>(aa, ia, inst);
            aa.gbed[j] += dJ_dkj * dk_of(it.dk_dbed, mat, code);
            aa.gint[j] += dJ_dkj * dk_of(it.dk_dint, mat, code);
        }
      }
    }
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_adj_gather(MeshArgs m, StateRef<R> U, StateRef<R> Lnext, StateOut<R> Lout,
                                                       MatConsts mc, AdjArgs aa, const DevScalars *__restrict__ sc) {
    __shared__ int list[kBlock];
    adj_gather_phase<R>(m, U, Lnext, Lout, mc, aa, R(sc->dt), list, InstArgs{});
}

// ------------------------------------------------------------------------ seed
// J = sum over the cells whose centre lies in the box of h^2 dx dy (the member's box in an
// ensemble); lambda^N = dJ/dU^N.  One warp per segment, which stores its part of J; the J of a
// member is the sum of its segments' parts in order (k_inst_sum).
struct Box {
    double v[4];  // xmin, xmax, ymin, ymax
};

template <class R, bool BATCH>
__device__ __forceinline__ void seed_phase(const MeshArgs &m, const StateRef<R> &UN, const StateOut<R> &L,
                                           const Box &box, double *seg_J, int nseg, const InstArgs &ia) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nseg; s += warps) {
        const double *bx = BATCH ? ia.box + (size_t)4 * ia.tile_inst[s >> 3] : box.v;
        const int i = s * 32 + lane;
        double acc = 0.0;
        if (i < m.n) {
            const double xc = m.x[i], yc = m.y[i];
            const bool in = xc >= bx[0] && xc <= bx[1] && yc >= bx[2] && yc <= bx[3];
            const double h = double(UN.h[i]);
            const double area = double(cell_dx<R>(m, i)) * double(cell_dy<R>(m, i));
            L.h[i] = in ? R(2.0 * h * area) : R(0);
            L.hu[i] = R(0);
            L.hv[i] = R(0);
            if (in) acc = h * h * area;
        }
        acc = warp_sum(acc);
        if (lane == 0) seg_J[s] = acc;
    }
}

// Sum of per-segment values over each member's segment range (seg0 == null: one range over all
// segments), thread-strided then block-reduced: a fixed order.
__global__ void __launch_bounds__(kBlock) k_inst_sum(const double *__restrict__ part, const int32_t *__restrict__ seg0,
                                                     int nseg, double *__restrict__ out) {
    __shared__ double red[kBlock / 32];
    const int s0 = seg0 ? seg0[blockIdx.x] : 0, s1 = seg0 ? seg0[blockIdx.x + 1] : nseg;
    double acc = 0.0;
    for (int s = s0 + threadIdx.x; s < s1; s += kBlock) acc += part[s];
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) t += red[w];
        out[blockIdx.x] = t;
    }
}

// Per-material sums of the running per-cell parameter sensitivities, plus the pile-height
// products sum_i lambda_h,i dh0_i/dP_p.  Two launches with a fixed order: block (b, o) sums
// output o over the b-th of kReduceParts contiguous cell ranges, then one block per output adds
// the parts in order.
constexpr int kReduceParts = kAdjReduceParts;

template <class R>
__global__ void __launch_bounds__(kBlock) k_adj_reduce(MeshArgs m, StateRef<R> L0, const double *__restrict__ gbed,
                                                       const double *__restrict__ gint,
                                                       const double *__restrict__ dh0, int n_mat, int n_piles,
                                                       double *__restrict__ part) {
    __shared__ double red[kBlock / 32];
    const int o = blockIdx.y;  // 0..n_mat-1 bed per material, n_mat internal, then piles
    // the owned cells (a subdomain's ghosts are summed by their owner)
    const int per = (m.n_owned + kReduceParts - 1) / kReduceParts;
    const int i0 = blockIdx.x * per, i1 = min(m.n_owned, i0 + per);
    double acc = 0.0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        if (o < n_mat) {
            if (m.mat[i] == o) acc += gbed[i];
        } else if (o == n_mat) {
            acc += gint[i];
        } else {
            acc += double(L0.h[i]) * dh0[(size_t)(o - n_mat - 1) * m.n + i];
        }
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) t += red[w];
        part[(size_t)o * kReduceParts + blockIdx.x] = t;
    }
}

// Ensemble: block (k, o) sums output o of member k over the member's cells, in a fixed order:
// o < n_mat the basal-friction sensitivities of material o, o == n_mat the internal friction,
// o == n_mat + 1 the member's pile height (lambda_h dh0/dP).
template <class R>
__global__ void __launch_bounds__(kBlock) k_adj_reduce_inst(MeshArgs m, StateRef<R> L0, const double *__restrict__ gbed,
                                                            const double *__restrict__ gint,
                                                            const double *__restrict__ dh0, int n_mat,
                                                            const int32_t *__restrict__ seg0, double *__restrict__ out) {
    __shared__ double red[kBlock / 32];
    const int k = blockIdx.x, o = blockIdx.y;
    const int i0 = seg0[k] * 32, i1 = min(m.n, seg0[k + 1] * 32);
    double acc = 0.0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
        if (o < n_mat) {
            if (m.mat[i] == o) acc += gbed[i];
        } else if (o == n_mat) {
            acc += gint[i];
        } else if (dh0) {
            acc += double(L0.h[i]) * dh0[i];
        }
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) t += red[w];
        out[(size_t)k * (n_mat + 2) + o] = t;
    }
}

__global__ void __launch_bounds__(kReduceParts) k_adj_reduce_final(const double *__restrict__ part,
                                                                   double *__restrict__ out) {
    __shared__ double red[kReduceParts / 32];
    double v = warp_sum(part[(size_t)blockIdx.x * kReduceParts + threadIdx.x]);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kReduceParts / 32; ++w) t += red[w];
        out[blockIdx.x] = t;
    }
}

}  // namespace
}  // namespace adj
}  // namespace da
