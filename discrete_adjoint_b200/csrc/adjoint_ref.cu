// The reference's own discrete adjoint of one step, on the device (da_params.jacobian_mode =
// DA_JAC_REFERENCE; FP64 only).
//
// The default adjoint (adjoint_impl.cuh) is the exact transpose of the forward step as it is
// computed here.  The reference's dual solver makes a few approximations of its own (frozen
// records of dry cells, no derivative with respect to void cells, friction-stop gating of the
// neighbours' slope terms, limiter sensitivities without the half-sign factor, the HLL
// state-difference term on dry sides, a flush of entries below 1e-16) and recomputes every branch
// from its records with its own arithmetic (reciprocal products in the slopes and speeds).  This
// mode reproduces that adjoint, structured like the reference:
//   k_ref_prep   per cell: the record of U^n the dual solver reads back (SolRec keeps a zero
//                record where h <= 0, src/datstr/dualmesh.C:35-80), its limited slopes and the
//                depth-slope sensitivities (DualElem::get_slopes_prev, dualmesh.C:1393-1626),
//                k act/pass (gmfggetcoef in update_dual_grid, src/adjoint/dual_grid_routines.C:
//                15-93), and the friction signs and stop flags of update_states
//                (src/adjoint/residual.C:162-275) that calc_jacobian replays;
//   k_ref_faces  per cell and +x/+y side: the flux Jacobians of the side's Riemann fluxes
//                (dual_xdirflux / dual_ydirflux, src/datstr/element2.C:1858-2041;
//                dual_riemannflux, dualmesh.C:1628-1843) stored per cell, direction, side and
//                contributor with the hanging-edge averages of DualElem::calc_flux
//                (dualmesh.C:1853-2239, FluxJac::set, src/header/matrix.h:215-245);
//   k_ref_bcopy  the domain-boundary copies of DualElem::boundary_flux (dualmesh.C:2241-2279);
//   k_ref_gather per cell i: lambda^n_i = -sum over the blocks J_e[which(i)] of the cells whose
//                residual depends on U_i (the cell itself and its up to eight neighbours) of
//                lambda^{n+1}_e J_e, each block formed on the fly as calc_jacobian /
//                set_fluxes_hsens / calc_jacobian_elem form it (src/adjoint/calc_jacobain.C:
//                40-330, src/adjoint/compute_jacobian_elem.C:15-121) and summed in the order of
//                calc_adjoint_elem (src/adjoint/calc_adjoint.C:74-167), entries below 1e-16
//                flushed to zero.
// Neighbour slots follow the reference's absolute side order for an element whose positive-x
// side is side 1 (slot a holds relative side (a + 3) % 4, slots 4..7 the second neighbours), so the
// blocks are summed in the reference's order.  Built with --fmad=false like the other FP64 units.
#include <cuda_runtime.h>

#include <cstring>

#include "da_internal.h"
#include "fv_device.cuh"

namespace da {
namespace refadj {
namespace {

using namespace fv;

constexpr int kBlock = 256;
constexpr int kFJ = 12 * 9;  // flux Jacobian entries per cell: [direction][side][contributor] 3x3

struct Bufs {
    double *S;      // [6][n] limited slopes of the record (d/dx of h, hu, hv, then d/dy)
    double *hs;     // [10][n] d (dh/dx) / d h of self, m1, p1, m2, p2, then the same for y
    double *kact;   // [n]
    int8_t *sgn;    // [4][n] friction signs of update_states
    uint8_t *stop;  // [n] bit 0, 1: s3 of x, y vanished with a nonzero sign
    double *fj;     // [kFJ][n]
};

struct M3 {
    double a[3][3];
};
__device__ __forceinline__ void zero(M3 &m) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) m.a[i][j] = 0.;
}

// flux-Jacobian slot: direction d (0 x, 1 y), side (0 minus, 1 plus), contributor k
__device__ __forceinline__ int fj_slot(int d, int side, int k) { return ((d * 2 + side) * 3 + k) * 9; }
__device__ __forceinline__ void fj_store(const Bufs &b, int n, int c, int slot, const M3 &m) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) b.fj[(size_t)(slot + i * 3 + j) * n + c] = m.a[i][j];
}
__device__ __forceinline__ M3 fj_load(const Bufs &b, int n, int c, int slot) {
    M3 m;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) m.a[i][j] = b.fj[(size_t)(slot + i * 3 + j) * n + c];
    return m;
}
// FluxJac::set(side, dir, index, jac1, jac2) stores (jac1 + jac2) * .5
__device__ __forceinline__ M3 avg(const M3 &x, const M3 &y) {
    M3 m;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) m.a[i][j] = (x.a[i][j] + y.a[i][j]) * .5;
    return m;
}

// The dual solver's record of cell c: the state where h > 0, a zero record otherwise.
struct Rec {
    const double *h, *hu, *hv;
    __device__ __forceinline__ double H(int c) const { return h[c] > 0. ? h[c] : 0.; }
    __device__ __forceinline__ double V(int j, int c) const {
        if (!(h[c] > 0.)) return 0.;
        return j == 0 ? h[c] : (j == 1 ? hu[c] : hv[c]);
    }
};

// neighbour slot a of cell c in the reference's absolute order (relative side (a + 3) % 4)
__device__ __forceinline__ int nb_abs(const MeshArgs &m, int c, int a) {
    const int r = (a + 3) & 3;
    return m.nbr[(size_t)(r + (a & 4)) * m.n + c];
}
// neigh_proc of slot a: -1 domain boundary, -2 a repeated first neighbour, 0 a neighbour
__device__ __forceinline__ int nproc_abs(const MeshArgs &m, int c, int a) {
    const int r = (a + 3) & 3;
    const int e1 = m.nbr[(size_t)r * m.n + c];
    if (a < 4) return e1 < 0 ? -1 : 0;
    const int e2 = m.nbr[(size_t)(r + 4) * m.n + c];
    return (e1 < 0 || e2 == e1) ? -2 : 0;
}
// Element::which_neighbor (element2.C:574-583)
__device__ __forceinline__ int which_neighbor(const MeshArgs &m, int e, int c) {
    for (int a = 0; a < 8; ++a)
        if (nb_abs(m, e, a) == c && nproc_abs(m, e, a) >= 0) return a;
    return 8;
}

// ------------------------------------------------------------------------------ k_ref_prep
__global__ void __launch_bounds__(kBlock) k_ref_prep(MeshArgs m, Rec P, MatConsts mc, const DevScalars *sc, Bufs b) {
    const int n = m.n;
    const double ft = sc->frict_tiny;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint8_t bf = m.bflag[i];
        double d[2][3] = {{0., 0., 0.}, {0., 0., 0.}}, hs[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) hs[k] = 0.;
        if (!(bf & 0x0F)) {
            for (int dir = 0; dir < 2; ++dir) {
                const int ep = m.nbr[(size_t)dir * n + i], em = m.nbr[(size_t)(dir + 2) * n + i];
                const bool two_p = bf & (0x10 << dir), two_m = bf & (0x10 << (dir + 2));
                const int ep2 = two_p ? m.nbr[(size_t)(dir + 4) * n + i] : -1;
                const int em2 = two_m ? m.nbr[(size_t)(dir + 6) * n + i] : -1;
                const double *co = dir == 0 ? m.x : m.y;
                const double dxp = co[ep] - co[i], dxm = co[i] - co[em];
                const double inv_dxp = 1 / dxp, inv_dxm = 1 / dxm, inv_s = 1 / (dxm + dxp);
                for (int j = 0; j < 3; ++j) {
                    const double vi = P.V(j, i);
                    double dp = (P.V(j, ep) - vi) * inv_dxp;
                    if (two_p) dp = .5 * (dp + (P.V(j, ep2) - vi) * inv_dxp);
                    double dm = (vi - P.V(j, em)) * inv_dxm;
                    if (two_m) dm = .5 * (dm + (vi - P.V(j, em2)) * inv_dxm);
                    const double dc = (dp * dxm + dm * dxp) * inv_s;
                    double mn = mc.gamma * dabs(dp);
                    const double bb = mc.gamma * dabs(dm), cc = dabs(dc);
                    if (mn > bb) mn = bb;
                    if (mn > cc) mn = cc;
                    const double fac = .5 * (c_sgn(dp) + c_sgn(dm));
                    d[dir][j] = fac * mn;
                    if (j != 0 || fac == 0) continue;
                    double *s = hs + dir * 5;
                    if (mn == mc.gamma * dabs(dp)) {
                        s[0] = -inv_dxp;
                        s[2] = inv_dxp;
                        if (two_p) s[2] = s[4] = .5 * inv_dxp;
                    } else if (mn == mc.gamma * dabs(dm)) {
                        s[0] = inv_dxm;
                        s[1] = -inv_dxm;
                        if (two_m) s[1] = s[3] = -.5 * inv_dxm;
                    } else {
                        s[0] = inv_dxm - inv_dxp;
                        s[1] = -inv_dxm;
                        s[2] = inv_dxp;
                        if (two_p) s[2] = s[4] = .5 * inv_dxp;
                        if (two_m) s[1] = s[3] = -.5 * inv_dxm;
                        s[1] *= dxp * inv_s;
                        s[2] *= dxm * inv_s;
                        s[3] *= dxp * inv_s;
                        s[4] *= dxm * inv_s;
                    }
                }
            }
        }
        const double U[3] = {P.V(0, i), P.V(1, i), P.V(2, i)};
        const double sl[6] = {d[0][0], d[0][1], d[0][2], d[1][0], d[1][1], d[1][2]};
        const int mat = m.mat[i];
        const double k = U[0] > DA_TINY ? cell_kact<double>(mc, mat, U[0], U[1], U[2], sl) : mc.kact_rest;
        // update_states' friction signs and stop flags (residual.C:196-262)
        int8_t sg[4] = {0, 0, 0, 0};
        uint8_t stop = 0;
        if (U[0] > DA_TINY) {
            const double vel0 = U[1] / U[0], vel1 = U[2] / U[0];
            const double h_inv = 1. / U[0];
            const double s0 = tiny_sgn(h_inv * (sl[4] - vel0 * sl[3]), ft);
            const double s2 = tiny_sgn(vel0, ft);
            const double s1 = tiny_sgn(h_inv * (sl[2] - vel1 * sl[0]), ft);
            const double s3 = tiny_sgn(vel1, ft);
            const double gz = m.g[(size_t)2 * n + i];
            const double cx = m.curv[i], cy = m.curv[(size_t)n + i];
            const double tb = mc.tan_bed[mat];
            const double px = gz * U[0] + vel0 * U[1] * cx, py = gz * U[0] + vel1 * U[2] * cy;
            if (s2 * (px > 0.0 ? px : 0.0) * tb == 0. && s2 != 0.) stop |= 1;
            if (s3 * (py > 0.0 ? py : 0.0) * tb == 0. && s3 != 0.) stop |= 2;
            sg[0] = int8_t(s0); sg[1] = int8_t(s1); sg[2] = int8_t(s2); sg[3] = int8_t(s3);
        }
#pragma unroll
        for (int j = 0; j < 6; ++j) b.S[(size_t)j * n + i] = sl[j];
#pragma unroll
        for (int q = 0; q < 10; ++q) b.hs[(size_t)q * n + i] = hs[q];
        b.kact[i] = k;
#pragma unroll
        for (int q = 0; q < 4; ++q) b.sgn[(size_t)q * n + i] = sg[q];
        b.stop[i] = stop;
    }
}

// --------------------------------------------------------------------------- k_ref_faces
// dual_xdirflux / dual_ydirflux of cell c: hfv (state, flux, speeds), d flux / d U, d speeds / d U
struct DualSide {
    M3 hfv, fj, sj;
};
__device__ __forceinline__ void dual_side(const MeshArgs &m, const Rec &P, const Bufs &b, int c, int dir,
                                          DualSide &o) {
    zero(o.hfv);
    zero(o.fj);
    zero(o.sj);
    const double h = P.H(c);
    if (h < DA_TINY) return;
    const double hu = P.V(1, c), hv = P.V(2, c);
    const double k = b.kact[c], gz = m.g[(size_t)2 * m.n + c];
    o.hfv.a[0][0] = h; o.hfv.a[0][1] = hu; o.hfv.a[0][2] = hv;
    if (dir == 0) {
        const double h_inv = 1. / h;
        const double Vel = hu * h_inv;
        const double a = sqrt(k * h * gz);
        o.hfv.a[1][0] = hu;
        o.hfv.a[1][1] = hu * Vel + 0.5 * a * a * h;
        o.hfv.a[1][2] = hv * Vel;
        o.hfv.a[2][0] = Vel - a; o.hfv.a[2][1] = Vel; o.hfv.a[2][2] = Vel + a;
        o.fj.a[0][1] = 1.;
        o.fj.a[1][0] = a * a - Vel * Vel;
        o.fj.a[1][1] = 2 * Vel;
        o.fj.a[2][0] = -Vel * hv * h_inv;
        o.fj.a[2][1] = hv * h_inv;
        o.fj.a[2][2] = Vel;
        o.sj.a[0][0] = -.5 * a * h_inv - Vel * h_inv;
        o.sj.a[0][1] = h_inv;
        o.sj.a[1][0] = -Vel * h_inv;
        o.sj.a[1][1] = h_inv;
        o.sj.a[2][0] = .5 * a * h_inv - Vel * h_inv;
        o.sj.a[2][1] = h_inv;
    } else {
        const double a = sqrt(k * h * gz);
        const double h_inv = 1. / h;
        const double Vel = hv * h_inv;
        o.hfv.a[1][0] = hv;
        o.hfv.a[1][1] = hu * Vel;
        o.hfv.a[1][2] = hv * Vel + 0.5 * a * a * h;
        o.hfv.a[2][0] = Vel - a; o.hfv.a[2][1] = Vel; o.hfv.a[2][2] = Vel + a;
        o.fj.a[0][2] = 1.;
        o.fj.a[1][0] = -Vel * hu * h_inv;
        o.fj.a[1][1] = Vel;
        o.fj.a[1][2] = hu * h_inv;
        o.fj.a[2][0] = a * a - Vel * Vel;
        o.fj.a[2][2] = 2 * Vel;
        o.sj.a[0][0] = -.5 * a * h_inv - Vel * h_inv;
        o.sj.a[0][2] = h_inv;
        o.sj.a[1][0] = -Vel * h_inv;
        o.sj.a[1][2] = h_inv;
        o.sj.a[2][0] = .5 * a * h_inv - Vel * h_inv;
        o.sj.a[2][2] = h_inv;
    }
}

// dual_riemannflux: d F_HLL / d U_left (jl), d U_right (jr)
__device__ void dual_riemann(const DualSide &L, const DualSide &R, M3 &jl, M3 &jr) {
    zero(jl);
    zero(jr);
    const M3 &hl = L.hfv, &hr = R.hfv;
    if (hl.a[0][0] == 0. && hr.a[0][0] == 0.) return;
    double sl, sr, dsl_l[3], dsl_r[3], dsr_l[3], dsr_r[3];
    if (hl.a[0][0] == 0.) {
        sl = fmin(0., 2. * hr.a[2][0] - hr.a[2][1]);
        sr = fmax(0., 2. * hr.a[2][2] - hr.a[2][1]);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            dsr_l[i] = dsl_l[i] = 0.;
            dsl_r[i] = sl == 0 ? 0. : 2 * R.sj.a[0][i] - R.sj.a[1][i];
            dsr_r[i] = sr == 0 ? 0. : 2 * R.sj.a[2][i] - R.sj.a[1][i];
        }
    } else if (hr.a[0][0] == 0.) {
        sl = fmin(0., 2. * hl.a[2][0] - hl.a[2][1]);
        sr = fmax(0., 2. * hl.a[2][2] - hl.a[2][1]);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            dsr_r[i] = dsl_r[i] = 0.;
            dsl_l[i] = sl == 0 ? 0. : 2 * L.sj.a[0][i] - L.sj.a[1][i];
            dsr_l[i] = sr == 0 ? 0. : 2 * L.sj.a[2][i] - L.sj.a[1][i];
        }
    } else {
        sl = fmin(0., fmin(hl.a[2][0], hr.a[2][0]));
        const int wl = sl == 0 ? 0 : (sl == hl.a[2][0] ? 1 : 2);
        sr = fmax(0., fmax(hl.a[2][2], hr.a[2][2]));
        const int wr = sr == 0 ? 0 : (sr == hl.a[2][2] ? 1 : 2);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            dsl_l[i] = wl == 1 ? L.sj.a[0][i] : 0.;
            dsl_r[i] = wl == 2 ? R.sj.a[0][i] : 0.;
            dsr_l[i] = wr == 1 ? L.sj.a[2][i] : 0.;
            dsr_r[i] = wr == 2 ? R.sj.a[2][i] : 0.;
        }
    }
    if (sl >= 0.) {
        jl = L.fj;
    } else if (sr <= 0.) {
        jr = R.fj;
    } else {
        const double inv = 1. / (sr - sl);
        double vd[3], flux[3], dfsr[3], dfsl[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) vd[i] = hr.a[0][i] - hl.a[0][i];
#pragma unroll
        for (int i = 0; i < 3; ++i) flux[i] = (sr * hl.a[1][i] - sl * hr.a[1][i] + sl * sr * vd[i]) * inv;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            dfsr[i] = (hl.a[1][i] + sl * vd[i] - flux[i]) * inv;
            dfsl[i] = (-hr.a[1][i] + sr * vd[i] + flux[i]) * inv;
        }
        const double dfr = -sl * inv, dfl = sr * inv;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const double vr = i == j ? sr * sl * inv : 0., vl = i == j ? -sr * sl * inv : 0.;
                jr.a[i][j] = dfsr[i] * dsr_r[j] + dfsl[i] * dsl_r[j] + dfr * R.fj.a[i][j] + vr;
                jl.a[i][j] = dfsr[i] * dsr_l[j] + dfsl[i] * dsl_l[j] + dfl * L.fj.a[i][j] + vl;
            }
    }
}

// DualElem::calc_flux of cell i for its + side in direction d.  Every flux-Jacobian entry has one
// writer: a cell its own + side, the cell across it that side's - entries (both fine cells of a
// coarse side give its - entries the same values; the one the coarse cell lists first writes).
__global__ void __launch_bounds__(kBlock) k_ref_faces(MeshArgs m, Rec P, Bufs b) {
    const int n = m.n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * n; t += gridDim.x * blockDim.x) {
        const int i = t >> 1, d = t & 1;
        const int e1 = m.nbr[(size_t)d * n + i];
        if (e1 < 0) continue;
        DualSide si, s1, s2;
        dual_side(m, P, b, i, d, si);
        dual_side(m, P, b, e1, d, s1);
        M3 jc, jn1, jn2, jres, z;
        zero(z);
        dual_riemann(si, s1, jc, jn1);
        const int e2r = m.nbr[(size_t)(d + 4) * n + i];
        const bool coarser = m.nbr[(size_t)(d + 2) * n + e1] != m.nbr[(size_t)(d + 6) * n + e1];
        if (e2r != e1) {
            // two finer neighbours (S_C_CON)
            dual_side(m, P, b, e2r, d, s2);
            dual_riemann(si, s2, jres, jn2);
            fj_store(b, n, i, fj_slot(d, 1, 0), avg(jc, jres));
            fj_store(b, n, i, fj_slot(d, 1, 1), avg(jn1, z));
            fj_store(b, n, i, fj_slot(d, 1, 2), avg(jn2, z));
            fj_store(b, n, e1, fj_slot(d, 0, 0), jn1);
            fj_store(b, n, e1, fj_slot(d, 0, 1), jc);
            fj_store(b, n, e1, fj_slot(d, 0, 2), z);
            fj_store(b, n, e2r, fj_slot(d, 0, 0), jn2);
            fj_store(b, n, e2r, fj_slot(d, 0, 1), jres);
            fj_store(b, n, e2r, fj_slot(d, 0, 2), z);
            continue;
        }
        fj_store(b, n, i, fj_slot(d, 1, 0), jc);
        fj_store(b, n, i, fj_slot(d, 1, 1), jn1);
        fj_store(b, n, i, fj_slot(d, 1, 2), z);
        if (!coarser) {
            fj_store(b, n, e1, fj_slot(d, 0, 0), jn1);
            fj_store(b, n, e1, fj_slot(d, 0, 1), jc);
            fj_store(b, n, e1, fj_slot(d, 0, 2), z);
            continue;
        }
        // one of two finer cells facing e1 (S_S_CON)
        const int zel = which_neighbor(m, e1, i);
        if (zel >= 4) continue;
        const int e2 = nb_abs(m, e1, (zel + 4) & 7);
        dual_side(m, P, b, e2, d, s2);
        dual_riemann(s2, s1, jn2, jres);
        fj_store(b, n, e1, fj_slot(d, 0, 0), avg(jn1, jres));
        fj_store(b, n, e1, fj_slot(d, 0, 1), avg(jc, z));
        fj_store(b, n, e1, fj_slot(d, 0, 2), avg(jn2, z));
    }
}

// DualElem::boundary_flux: a domain-edge side takes the opposite side's Jacobians.
__global__ void __launch_bounds__(kBlock) k_ref_bcopy(MeshArgs m, Bufs b) {
    const int n = m.n;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 2 * n; t += gridDim.x * blockDim.x) {
        const int i = t >> 1, d = t & 1;
        const uint8_t bf = m.bflag[i];
        const int bp = (bf >> d) & 1, bm = (bf >> (d + 2)) & 1;
        for (int rep = 0; rep < bp + bm; ++rep) {
            for (int k = 0; k < 3; ++k) {
                if (bp) fj_store(b, n, i, fj_slot(d, 1, k), fj_load(b, n, i, fj_slot(d, 0, k)));
                if (bm) fj_store(b, n, i, fj_slot(d, 0, k), fj_load(b, n, i, fj_slot(d, 1, k)));
            }
        }
    }
}

// -------------------------------------------------------------------------- k_ref_gather
// Block eff (0 the cell itself, a + 1 its neighbour slot a) of cell c's Jacobian,
// calc_jacobian + set_fluxes_hsens + calc_jacobian_elem.  The caller has ruled out the zero
// blocks (void self or neighbour, repeated or missing neighbour).
__device__ void block_of(const MeshArgs &m, const Rec &P, const Bufs &b, double dt, double sin_int, double tan_bed,
                         int c, int eff, M3 &J) {
    const int n = m.n;
    M3 jnx, jpx, jny, jpy;
    zero(jnx); zero(jpx); zero(jny); zero(jpy);
    double dh[2] = {0., 0.};
    if (eff == 0) {
        jnx = fj_load(b, n, c, fj_slot(0, 0, 0));
        jpx = fj_load(b, n, c, fj_slot(0, 1, 0));
        jny = fj_load(b, n, c, fj_slot(1, 0, 0));
        jpy = fj_load(b, n, c, fj_slot(1, 1, 0));
        dh[0] = b.hs[c];
        dh[1] = b.hs[(size_t)5 * n + c];
    } else {
        const int a = eff - 1, r = (a + 3) & 3, idx = eff <= 4 ? 1 : 2;
        const bool boundary = m.nbr[(size_t)((r + 2) & 3) * n + c] < 0;
        const int hp = eff <= 4 ? 2 : 4, hm = eff <= 4 ? 1 : 3;
        if (r == 0) {
            dh[0] = b.hs[(size_t)hp * n + c];
            jpx = fj_load(b, n, c, fj_slot(0, 1, idx));
            if (boundary) jnx = fj_load(b, n, c, fj_slot(0, 0, idx));
        } else if (r == 2) {
            dh[0] = b.hs[(size_t)hm * n + c];
            jnx = fj_load(b, n, c, fj_slot(0, 0, idx));
            if (boundary) jpx = fj_load(b, n, c, fj_slot(0, 1, idx));
        } else if (r == 1) {
            dh[1] = b.hs[(size_t)(5 + hp) * n + c];
            jpy = fj_load(b, n, c, fj_slot(1, 1, idx));
            if (boundary) jny = fj_load(b, n, c, fj_slot(1, 0, idx));
        } else {
            dh[1] = b.hs[(size_t)(5 + hm) * n + c];
            jny = fj_load(b, n, c, fj_slot(1, 0, idx));
            if (boundary) jpy = fj_load(b, n, c, fj_slot(1, 1, idx));
        }
    }
    const double dtdx = dt / m.dx[c], dtdy = dt / m.dy[c];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j)
            J.a[i][j] = +dtdx * (jpx.a[i][j] - jnx.a[i][j]) + dtdy * (jpy.a[i][j] - jny.a[i][j]);
    if (eff == 0)
#pragma unroll
        for (int i = 0; i < 3; ++i) J.a[i][i] -= 1.;
    const double h = P.H(c);
    if (!(h > DA_TINY)) return;
    const double k = b.kact[c];
    const double sg0 = b.sgn[c], sg1 = b.sgn[(size_t)n + c];
    const double sg2 = b.sgn[(size_t)2 * n + c], sg3 = b.sgn[(size_t)3 * n + c];
    const uint8_t stop = b.stop[c];
    const double alpha = sin_int * sg0 * k;
    const double betta = sin_int * sg1 * k;
    const double gz = m.g[(size_t)2 * n + c];
    if (eff > 0) {
        if (!(stop & 1)) J.a[1][0] -= -dt * h * alpha * gz * dh[1];
        if (!(stop & 2)) J.a[2][0] -= -dt * h * betta * gz * dh[0];
        return;
    }
    const double hu = P.V(1, c), hv = P.V(2, c);
    const double velocity[2] = {hu / h, hv / h};
    const double vx_sq = velocity[0] * velocity[0], vy_sq = velocity[1] * velocity[1];
    const double gx = m.g[c], gy = m.g[(size_t)n + c];
    const double dgx = m.dg[c], dgy = m.dg[(size_t)n + c];
    const double cx = m.curv[c], cy = m.curv[(size_t)n + c];
    const double sx0 = b.S[c], sy0 = b.S[(size_t)3 * n + c];
    J.a[1][0] -= dt * (gx - alpha * h * (2 * dgy + gz * dh[1]) - alpha * gz * sy0);
    if (sg2 != 0. && !(stop & 1)) {
        J.a[1][0] -= -dt * sg2 * tan_bed * (gz - vx_sq * cx);
        J.a[1][1] -= -dt * sg2 * tan_bed * (2 * velocity[0] * cx);
        J.a[1][2] -= 0.;
    }
    J.a[2][0] -= dt * (gy - betta * h * (2 * dgx + gz * dh[0]) - betta * gz * sx0);
    if (sg3 != 0. && !(stop & 2)) {
        J.a[2][0] -= -dt * sg3 * tan_bed * (gz - vy_sq * cy);
        J.a[2][1] -= 0.;
        J.a[2][2] -= -dt * sg3 * tan_bed * (2 * velocity[1] * cy);
    }
}

__global__ void __launch_bounds__(kBlock) k_ref_gather(MeshArgs m, Rec P, Bufs b, MatConsts mc, const DevScalars *sc,
                                                       StateRef<double> Lnext, StateOut<double> Lout) {
    const int n = m.n;
    const double dt = sc->dt;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double ac[3] = {0., 0., 0.};
        // a void cell (zero record): every block that involves it is zero (calc_jacobain.C:109-113)
        if (P.H(i) != 0.) {
            for (int eff = 0; eff < 9; ++eff) {
                int e = i, jacind = 0;
                if (eff > 0) {
                    const int a = eff - 1;
                    if (!(eff <= 4 || nproc_abs(m, i, a) > -2)) continue;
                    e = nb_abs(m, i, a);
                    if (e < 0) continue;
                    jacind = which_neighbor(m, e, i) + 1;
                }
                M3 J;
                block_of(m, P, b, dt, mc.sin_int, mc.tan_bed[m.mat[e]], e, jacind, J);
                const double le[3] = {Lnext.h[e], Lnext.hu[e], Lnext.hv[e]};
#pragma unroll
                for (int k = 0; k < 3; ++k)
#pragma unroll
                    for (int l = 0; l < 3; ++l) ac[k] += le[l] * J.a[l][k];
            }
        }
        double out[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            double v = 0. - ac[j];
            if (fabs(v) < 1e-16) v = 0.;
            out[j] = v;
        }
        Lout.h[i] = out[0];
        Lout.hu[i] = out[1];
        Lout.hv[i] = out[2];
    }
}

// lambda^N = dJ/dU^N of J = sum over the cells whose centre lies in the box of h^2 dx dy, with
// each segment's part of J for the functional's fixed-order sum (the same seed as the exact mode's).
__global__ void __launch_bounds__(kBlock) k_ref_seed(MeshArgs m, StateRef<double> UN, StateOut<double> L, double x0,
                                                     double x1, double y0, double y1, double *seg_J, int nseg) {
    const int lane = threadIdx.x & 31;
    const int warps = (gridDim.x * blockDim.x) >> 5;
    for (int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; s < nseg; s += warps) {
        const int i = s * 32 + lane;
        double acc = 0.0;
        if (i < m.n) {
            const double xc = m.x[i], yc = m.y[i];
            const bool in = xc >= x0 && xc <= x1 && yc >= y0 && yc <= y1;
            const double h = UN.h[i];
            const double area = m.dx[i] * m.dy[i];
            L.h[i] = in ? 2.0 * h * area : 0.0;
            L.hu[i] = 0.0;
            L.hv[i] = 0.0;
            if (in) acc = h * h * area;
        }
        acc = warp_sum(acc);
        if (lane == 0) seg_J[s] = acc;
    }
}

// The neighbour table with each side's two finer neighbours in the reference's order: an element
// keeps them counter-clockwise around its boundary (adapt/refine2.C:590-805), the flattened table
// lists the lower (sides +-x) or left (sides +-y) one first, so the +y and -x pairs swap.  The dual
// solver sums its blocks in slot order; this table gives its sums their order.
__global__ void k_ref_ccw(const int32_t *__restrict__ nbr, int32_t *__restrict__ ccw, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        for (int k = 0; k < 8; ++k) {
            const int r = k & 3;
            const int src = (r == 1 || r == 2) ? (k ^ 4) : k;
            ccw[(size_t)k * n + i] = nbr[(size_t)src * n + i];
        }
}

}  // namespace
}  // namespace refadj

// Workspace of the reference mode: one allocation sized for the mesh (about 1 KB per cell,
// mostly the 108 flux-Jacobian entries), zeroed once so that entries no rule writes read as 0,
// and the counter-clockwise neighbour table.
int ref_adjoint_alloc(da_ctx *ctx) {
    const size_t n = (size_t)ctx->mesh.n;
    if (ctx->refadj_mem && ctx->refadj_n == (int)n) return DA_OK;
    if (ctx->refadj_mem) cudaFree(ctx->refadj_mem);
    ctx->refadj_mem = nullptr;
    ctx->refadj_n = 0;
    const size_t bytes = n * (sizeof(double) * (6 + 10 + 1 + refadj::kFJ) + sizeof(int32_t) * 8 + 4 + 1) + 256;
    int st = cuda_check(ctx, cudaMalloc(&ctx->refadj_mem, bytes), "cudaMalloc(reference-mode adjoint)");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(ctx->refadj_mem, 0, bytes, ctx->stream), "memset");
    if (!st) {
        int32_t *ccw = (int32_t *)((char *)ctx->refadj_mem + sizeof(double) * (6 + 10 + 1 + refadj::kFJ) * n);
        const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
        refadj::k_ref_ccw<<<sms * 4, 256, 0, ctx->stream>>>(ctx->mesh.nbr, ccw, (int)n);
        st = cuda_check(ctx, cudaGetLastError(), "neighbour order launch");
    }
    if (!st) ctx->refadj_n = (int)n;
    return st;
}

// One reverse step of the reference's dual solver: U^n in state buffer un, the step's dt and
// frict_tiny in the device scalars (left there by the replayed forward step), lambda^{n+1} in
// adjoint buffer lam_in, lambda^n into lam_out.
int launch_ref_adjoint_step(da_ctx *ctx, int un, int lam_in, int lam_out) {
    if (ctx->p.precision != DA_PREC_FP64)
        return set_error(ctx, DA_ERR_UNSUPPORTED, "the reference-mode adjoint runs in FP64 only");
    int st = ref_adjoint_alloc(ctx);
    if (st) return st;
    const size_t n = (size_t)ctx->mesh.n;
    char *p = (char *)ctx->refadj_mem;
    refadj::Bufs b;
    b.S = (double *)p; p += sizeof(double) * 6 * n;
    b.hs = (double *)p; p += sizeof(double) * 10 * n;
    b.kact = (double *)p; p += sizeof(double) * n;
    b.fj = (double *)p; p += sizeof(double) * refadj::kFJ * n;
    const int32_t *ccw = (const int32_t *)p; p += sizeof(int32_t) * 8 * n;
    b.sgn = (int8_t *)p; p += 4 * n;
    b.stop = (uint8_t *)p;
    fv::MeshArgs m = fv::mesh_args(ctx);
    m.nbr = ccw;   // the reference's pair order on every side
    const refadj::Rec P{(const double *)ctx->U[un][0], (const double *)ctx->U[un][1], (const double *)ctx->U[un][2]};
    const fv::StateRef<double> Ln{(const double *)ctx->lam[lam_in][0], (const double *)ctx->lam[lam_in][1],
                                  (const double *)ctx->lam[lam_in][2]};
    const fv::StateOut<double> Lo{(double *)ctx->lam[lam_out][0], (double *)ctx->lam[lam_out][1],
                                  (double *)ctx->lam[lam_out][2]};
    const int sms = ctx->sm_count > 0 ? ctx->sm_count : 148;
    const int cells_grid = (int)((n + refadj::kBlock - 1) / refadj::kBlock);
    const int grid = cells_grid < sms * 8 ? (cells_grid > 0 ? cells_grid : 1) : sms * 8;
    const int grid2 = (int)((2 * n + refadj::kBlock - 1) / refadj::kBlock) < sms * 8
                          ? (int)((2 * n + refadj::kBlock - 1) / refadj::kBlock)
                          : sms * 8;
    trace_begin(ctx, TR_ADJ_SRC);
    refadj::k_ref_prep<<<grid, refadj::kBlock, 0, ctx->stream>>>(m, P, ctx->mc, ctx->dsc, b);
    refadj::k_ref_faces<<<grid2, refadj::kBlock, 0, ctx->stream>>>(m, P, b);
    refadj::k_ref_bcopy<<<grid2, refadj::kBlock, 0, ctx->stream>>>(m, b);
    trace_end(ctx);
    trace_begin(ctx, TR_ADJ_GATHER);
    refadj::k_ref_gather<<<grid, refadj::kBlock, 0, ctx->stream>>>(m, P, b, ctx->mc, ctx->dsc, Ln, Lo);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "reference-mode adjoint launch");
}

// The functional's seed from the current state into adjoint buffer lam_out (reference mode).
int launch_ref_seed(da_ctx *ctx, int lam_out, const double box[4]) {
    const fv::MeshArgs m = fv::mesh_args(ctx);
    const int c = ctx->cur;
    const fv::StateRef<double> UN{(const double *)ctx->U[c][0], (const double *)ctx->U[c][1],
                                  (const double *)ctx->U[c][2]};
    const fv::StateOut<double> L{(double *)ctx->lam[lam_out][0], (double *)ctx->lam[lam_out][1],
                                 (double *)ctx->lam[lam_out][2]};
    trace_begin(ctx, TR_ADJ_SEED);
    refadj::k_ref_seed<<<ctx->nblocks > 0 ? ctx->nblocks : 1, refadj::kBlock, 0, ctx->stream>>>(
        m, UN, L, box[0], box[1], box[2], box[3], ctx->seg_J, ctx->nseg);
    trace_end(ctx);
    return cuda_check(ctx, cudaGetLastError(), "reference-mode seed launch");
}

}  // namespace da
