// Forward step kernels (order_flag = 1) for sm_100a -- templates shared by the FP64 and
// FP32-split translation units (forward_fp64.cu is built without FMA contraction).
//
// One step() of the reference (src/geoflow/step.C:29-275) becomes three launches:
//   k_coef    : limited slopes (Element::get_slopes, element2.C:830-939), k act/pass
//               (gmfggetcoef, getcoef.f:19-66), wave speeds (eigen.f:19-49) and the
//               CFL min / hmax reductions of get_coef_and_eigen.C:86-166;
//   k_dt      : dt of get_coef_and_eigen.C:168-179 + TimeProps::incrtime (properties.h:397-410);
//   k_update  : the four side fluxes of every cell (xdirflux/ydirflux/riemannflux with the
//               hanging-node averaging of Element::calc_edge_states, element2.C:2745-3072, and
//               the outflow copy of boundary_flux, element2.C:3374-3411) fused with the
//               corrector update_states (residual.C:162-275) and the FP64 volume partials.
// Each edge flux is evaluated by both cells that share it; the two evaluations run the same
// operations on the same operands, so they agree bit for bit and no edge array is stored.
//
// Two precisions share the code: R = double with centre coordinates (plain FP64 path, built
// without FMA contraction so that it reproduces the CPU reference bit for bit), and R = float
// with centre distances taken from cell sizes (FP32-split path; FP64 for dt and volume).
#pragma once
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>

#include "da_internal.h"

namespace da {
namespace fwd {
namespace {  // internal linkage: each precision TU keeps its own copy

constexpr int kBlock = 256;

template <class R>
struct StateRef {
    const R *__restrict__ h;
    const R *__restrict__ hu;
    const R *__restrict__ hv;
};

// c_sgn (geoflow.h:90-100), c_dmin1 (geoflow.h:103-120), dabs (geoflow.h:143-148)
template <class R>
__device__ __forceinline__ R c_sgn(R zz) {
    return zz > R(DA_TINY) ? R(1) : (zz < -R(DA_TINY) ? R(-1) : R(0));
}
template <class R>
__device__ __forceinline__ R c_dmin1(R d1, R d2) {
    return d1 > d2 ? d2 : d1;
}
template <class R>
__device__ __forceinline__ R dabs(R d) {
    return d < R(0) ? -d : d;
}
// max/min of element2.C:1059-1071
template <class R>
__device__ __forceinline__ R rmax(R x, R y) {
    return x > y ? x : y;
}
template <class R>
__device__ __forceinline__ R rmin(R x, R y) {
    return x > y ? y : x;
}
// sgn(zz, tiny): sgn.f:19-33
template <class R>
__device__ __forceinline__ int fsgn(R zz, R tiny) {
    return dabs(zz) < tiny ? 0 : (zz >= tiny ? 1 : -1);
}
// tiny_sgn: residual.C:153-160
template <class R>
__device__ __forceinline__ R tiny_sgn(R num, R tiny) {
    return dabs(num) < tiny ? R(0) : (num > tiny ? R(1) : R(-1));
}

struct MeshArgs {
    int n;
    const int32_t *__restrict__ nbr;
    const uint8_t *__restrict__ mat;
    const uint8_t *__restrict__ bflag;
    const double *__restrict__ x;
    const double *__restrict__ y;
    const double *__restrict__ dx;
    const double *__restrict__ dy;
    const double *__restrict__ g;
    const double *__restrict__ dg;
    const double *__restrict__ curv;
    const float *__restrict__ fdx;
    const float *__restrict__ fdy;
    const float *__restrict__ fg;
    const float *__restrict__ fdg;
    const float *__restrict__ fcurv;
};

template <class R>
__device__ __forceinline__ R cell_dx(const MeshArgs &m, int i);
template <>
__device__ __forceinline__ double cell_dx<double>(const MeshArgs &m, int i) { return m.dx[i]; }
template <>
__device__ __forceinline__ float cell_dx<float>(const MeshArgs &m, int i) { return m.fdx[i]; }
template <class R>
__device__ __forceinline__ R cell_dy(const MeshArgs &m, int i);
template <>
__device__ __forceinline__ double cell_dy<double>(const MeshArgs &m, int i) { return m.dy[i]; }
template <>
__device__ __forceinline__ float cell_dy<float>(const MeshArgs &m, int i) { return m.fdy[i]; }
template <class R>
__device__ __forceinline__ R grav(const MeshArgs &m, int c, int i);
template <>
__device__ __forceinline__ double grav<double>(const MeshArgs &m, int c, int i) { return m.g[(size_t)c * m.n + i]; }
template <>
__device__ __forceinline__ float grav<float>(const MeshArgs &m, int c, int i) { return m.fg[(size_t)c * m.n + i]; }
template <class R>
__device__ __forceinline__ R dgrav(const MeshArgs &m, int c, int i);
template <>
__device__ __forceinline__ double dgrav<double>(const MeshArgs &m, int c, int i) { return m.dg[(size_t)c * m.n + i]; }
template <>
__device__ __forceinline__ float dgrav<float>(const MeshArgs &m, int c, int i) { return m.fdg[(size_t)c * m.n + i]; }
template <class R>
__device__ __forceinline__ R curvat(const MeshArgs &m, int c, int i);
template <>
__device__ __forceinline__ double curvat<double>(const MeshArgs &m, int c, int i) { return m.curv[(size_t)c * m.n + i]; }
template <>
__device__ __forceinline__ float curvat<float>(const MeshArgs &m, int c, int i) { return m.fcurv[(size_t)c * m.n + i]; }

// Distance between the centres of cell i and its neighbour e along direction dir.
// FP64: difference of stored centres, as the reference does (ep->coord - coord).
// FP32: half the sum of the two sizes, exact for quadtree geometry and free of the
// cancellation that large FP32 coordinates would bring.
template <class R>
__device__ __forceinline__ R centre_dist(const MeshArgs &m, int dir, int from, int to);
template <>
__device__ __forceinline__ double centre_dist<double>(const MeshArgs &m, int dir, int from, int to) {
    const double *co = dir == 0 ? m.x : m.y;
    return co[to] - co[from];
}
template <>
__device__ __forceinline__ float centre_dist<float>(const MeshArgs &m, int dir, int from, int to) {
    const float *sz = dir == 0 ? m.fdx : m.fdy;
    const float d = 0.5f * (sz[to] + sz[from]);
    return d;
}

// Element::get_slopes for one cell (element2.C:830-939); out[0..2] x, out[3..5] y.
template <class R>
__device__ __forceinline__ void cell_slopes(const MeshArgs &m, const StateRef<R> &U, int i, uint8_t bf, R gamma,
                                            R out[6]) {
    if (bf & 0x0F) {
#pragma unroll
        for (int j = 0; j < 6; ++j) out[j] = R(0);
        return;
    }
    const R ui[3] = {U.h[i], U.hu[i], U.hv[i]};
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
        const int ep = m.nbr[(size_t)dir * m.n + i];
        const int em = m.nbr[(size_t)(dir + 2) * m.n + i];
        const bool two_p = bf & (0x10 << dir), two_m = bf & (0x10 << (dir + 2));
        const int ep2 = two_p ? m.nbr[(size_t)(dir + 4) * m.n + i] : ep;
        const int em2 = two_m ? m.nbr[(size_t)(dir + 6) * m.n + i] : em;
        R dxp, dxm;
        if constexpr (sizeof(R) == 8) {
            dxp = centre_dist<R>(m, dir, i, ep);
            dxm = centre_dist<R>(m, dir, em, i);
        } else {
            dxp = centre_dist<R>(m, dir, i, ep);
            dxm = centre_dist<R>(m, dir, i, em);
        }
        const R up[3] = {U.h[ep], U.hu[ep], U.hv[ep]};
        const R um[3] = {U.h[em], U.hu[em], U.hv[em]};
        R up2[3], um2[3];
        if (two_p) { up2[0] = U.h[ep2]; up2[1] = U.hu[ep2]; up2[2] = U.hv[ep2]; }
        if (two_m) { um2[0] = U.h[em2]; um2[1] = U.hu[em2]; um2[2] = U.hv[em2]; }
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            R dp = (up[j] - ui[j]) / dxp;
            if (two_p) dp = R(.5) * (dp + (up2[j] - ui[j]) / dxp);
            R dm = (ui[j] - um[j]) / dxm;
            if (two_m) dm = R(.5) * (dm + (ui[j] - um2[j]) / dxm);
            const R dc = (dp * dxm + dm * dxp) / (dxm + dxp);
            R mn = gamma * dabs(dp);
            const R b = gamma * dabs(dm), c = dabs(dc);
            if (mn > b) mn = b;
            if (mn > c) mn = c;
            out[j + 3 * dir] = R(.5) * (c_sgn(dp) + c_sgn(dm)) * mn;
        }
    }
}

// k act/pass of one cell (gmfggetcoef, getcoef.f:19-66) from the per-material table.
template <class R>
__device__ __forceinline__ R cell_kact(const MatConsts &mc, int mat, R h, R hu, R hv, const R s[6]) {
    if (!(h > R(DA_TINY))) return R(mc.kact_rest);
    const R vel = s[1] / h - hu * s[0] / (h * h) + s[5] / h - hv * s[3] / (h * h);
    const int sg = fsgn(vel, R(DA_TINY));
    R k = R(mc.kact_sgn[mat][sg + 1]);
    if (dabs(hu / h) < R(DA_TINY) && dabs(hv / h) < R(DA_TINY)) k = R(mc.kact_rest);
    return k;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

__device__ __forceinline__ void raise_err(DevScalars *sc, int code) { atomicCAS(&sc->err, 0, code); }

// ----------------------------------------------------------------------------- k_coef
template <class R>
__global__ void __launch_bounds__(kBlock) k_coef(MeshArgs m, StateRef<R> U, R *__restrict__ slopes,
                                                 R *__restrict__ kact, MatConsts mc, DevScalars *sc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long my_min = 0x7FF0000000000000ull;  // +inf
    unsigned long long my_max = 0ull;
    if (i < m.n) {
        const uint8_t bf = m.bflag[i];
        R s[6];
        cell_slopes<R>(m, U, i, bf, R(mc.gamma), s);
#pragma unroll
        for (int j = 0; j < 6; ++j) slopes[(size_t)j * m.n + i] = s[j];
        const R h = U.h[i], hu = U.hu[i], hv = U.hv[i];
        const R k = cell_kact<R>(mc, m.mat[i], h, hu, hv, s);
        kact[i] = k;
        if (h > R(DA_TINY)) {
            const R gz = grav<R>(m, 2, i);
            const R vx = hu / h, vy = hv / h;
            const R c = sqrt(k * gz * h);
            const R evx = dabs(vx) + c, evy = dabs(vy) + c;
            const R ev = evx > evy ? evx : evy;
            if (ev > R(1000000000.)) raise_err(sc, DA_ERR_EIGEN);
            if (!(ev == ev)) raise_err(sc, DA_ERR_NAN);
            const double ratio = double(c_dmin1(cell_dx<R>(m, i), cell_dy<R>(m, i)) / ev);
            my_min = __double_as_longlong(ratio);
            my_max = __double_as_longlong(double(h));
        }
    }
    my_min = warp_min_u64(my_min);
    my_max = warp_max_u64(my_max);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&sc->acc_min_dxe, my_min);
        if (my_max) atomicMax(&sc->acc_hmax, my_max);
    }
}

// ------------------------------------------------------------------------------- k_dt
__global__ void k_dt(DevScalars *sc, TimeConsts tc) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double min_dxe = __longlong_as_double(sc->acc_min_dxe);
    const double hmax = __longlong_as_double(sc->acc_hmax);
    // get_coef_and_eigen.C:168-179 with the single-rank MPI_Allreduce(MIN)
    const double g0 = 0.5 * min_dxe;
    const double g1 = -0.9 * sqrt(hmax * (tc.epsilon) * (tc.gravity_scale) / 9.8);
    double dt = 0.5 * (g0 > -g1 ? -g1 : g0);
    if (dt == 0.0) dt = 0.5 * tc.influx_dt;
    // TimeProps::incrtime
    const double time = sc->time;
    if (time + dt > tc.next_output) dt = tc.next_output - time;
    if (time + dt > tc.next_save) dt = tc.next_save - time;
    if (time + dt > tc.max_time) dt = tc.max_time - time;
    // frict_tiny is chosen from the iteration count before incrtime advances it
    sc->frict_tiny = sc->iter < tc.frict_tiny_iters ? tc.frict_tiny_early : tc.frict_tiny_late;
    sc->dt = dt;
    sc->time = time + dt;
    sc->min_dxe = min_dxe;
    sc->hmax = hmax;
    sc->iter += 1;
    // reset the accumulators for the next coefficient pass (init 1e7: get_coef_and_eigen.C:36)
    sc->acc_min_dxe = __double_as_longlong(10000000.0);
    sc->acc_hmax = 0ull;
}

// Element::xdirflux / ydirflux with dz = 0 (element2.C:1810-1996).
template <class R>
struct Hfv {
    R u[3], f[3], s[3];
};

template <class R>
__device__ __forceinline__ void dirflux(int dir, R h, R hu, R hv, R k, R gz, Hfv<R> &o) {
    if (h < R(DA_TINY)) {
#pragma unroll
        for (int a = 0; a < 3; ++a) o.u[a] = o.f[a] = o.s[a] = R(0);
        return;
    }
    o.u[0] = h; o.u[1] = hu; o.u[2] = hv;
    const R a = sqrt(k * h * gz);
    if (dir == 0) {
        const R vel = hu / h;
        o.f[0] = hu;
        o.f[1] = hu * vel + R(0.5) * a * a * h;
        o.f[2] = hv * vel;
        o.s[0] = vel - a; o.s[1] = vel; o.s[2] = vel + a;
    } else {
        const R vel = hv / h;
        o.f[0] = hv;
        o.f[1] = hu * vel;
        o.f[2] = hv * vel + R(0.5) * a * a * h;
        o.s[0] = vel - a; o.s[1] = vel; o.s[2] = vel + a;
    }
}

// riemannflux (element2.C:2228-2264): HLL with Davis wave speeds.
template <class R>
__device__ __forceinline__ void riemann(const Hfv<R> &l, const Hfv<R> &r, R flux[3]) {
    if (l.u[0] == R(0) && r.u[0] == R(0)) {
        flux[0] = flux[1] = flux[2] = R(0);
        return;
    }
    R sl, sr;
    if (l.u[0] == R(0)) {
        sl = rmin(R(0), R(2.0) * r.s[0] - r.s[1]);
        sr = rmax(R(0), R(2.0) * r.s[2] - r.s[1]);
    } else if (r.u[0] == R(0)) {
        sl = rmin(R(0), R(2.0) * l.s[0] - l.s[1]);
        sr = rmax(R(0), R(2.0) * l.s[2] - l.s[1]);
    } else {
        sl = rmin(R(0), rmin(l.s[0], r.s[0]));
        sr = rmax(R(0), rmax(l.s[2], r.s[2]));
    }
    if (sl >= R(0)) {
        flux[0] = l.f[0]; flux[1] = l.f[1]; flux[2] = l.f[2];
    } else if (sr <= R(0)) {
        flux[0] = r.f[0]; flux[1] = r.f[1]; flux[2] = r.f[2];
    } else {
        const R inv = sr - sl;
#pragma unroll
        for (int v = 0; v < 3; ++v) flux[v] = (sr * l.f[v] - sl * r.f[v] + sl * sr * (r.u[v] - l.u[v])) / inv;
    }
}

template <class R>
__device__ __forceinline__ void nb_hfv(const MeshArgs &m, const StateRef<R> &U, const R *__restrict__ kact, int e,
                                       int dir, Hfv<R> &o) {
    dirflux<R>(dir, U.h[e], U.hu[e], U.hv[e], kact[e], grav<R>(m, 2, e), o);
}

// ---------------------------------------------------------------------------- k_update
template <class R>
__global__ void __launch_bounds__(kBlock) k_update(MeshArgs m, StateRef<R> U, R *__restrict__ oh,
                                                   R *__restrict__ ohu, R *__restrict__ ohv,
                                                   const R *__restrict__ slopes, const R *__restrict__ kact,
                                                   MatConsts mc, DevScalars *sc, double *__restrict__ vol_part) {
    __shared__ double red[kBlock / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double vol = 0.0;
    if (i < m.n) {
        const uint8_t bf = m.bflag[i];
        const R dt = R(sc->dt);
        const R ft = R(sc->frict_tiny);
        const R prev[3] = {U.h[i], U.hu[i], U.hv[i]};
        const R ki = kact[i];
        const R gz = grav<R>(m, 2, i);
        Hfv<R> self[2];
        dirflux<R>(0, prev[0], prev[1], prev[2], ki, gz, self[0]);
        dirflux<R>(1, prev[0], prev[1], prev[2], ki, gz, self[1]);
        R F[4][3];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (bf & (1 << s)) continue;
            const int dir = s & 1;
            const bool plus = s < 2;
            const int e1 = m.nbr[(size_t)s * m.n + i];
            Hfv<R> nb;
            nb_hfv<R>(m, U, kact, e1, dir, nb);
            if (plus) riemann<R>(self[dir], nb, F[s]);
            else riemann<R>(nb, self[dir], F[s]);
            if (bf & (0x10 << s)) {
                // two finer neighbours (node S_C_CON): average of the two fine-side fluxes
                const int e2 = m.nbr[(size_t)(s + 4) * m.n + i];
                R f2[3];
                nb_hfv<R>(m, U, kact, e2, dir, nb);
                if (plus) riemann<R>(self[dir], nb, f2);
                else riemann<R>(nb, self[dir], f2);
#pragma unroll
                for (int v = 0; v < 3; ++v) F[s][v] = R(0.5) * (F[s][v] + f2[v]);
            }
        }
        // boundary_flux: an outflow side takes the flux of the opposite side
#pragma unroll
        for (int s = 0; s < 4; ++s)
            if (bf & (1 << s)) {
                const int o = s ^ 2;
                if (bf & (1 << o)) {
                    F[s][0] = F[s][1] = F[s][2] = R(0);
                } else {
                    F[s][0] = F[o][0]; F[s][1] = F[o][1]; F[s][2] = F[o][2];
                }
            }
        // update_states (residual.C:162-275)
        const R dtdx = dt / cell_dx<R>(m, i);
        const R dtdy = dt / cell_dy<R>(m, i);
        R st[3];
#pragma unroll
        for (int v = 0; v < 3; ++v) st[v] = prev[v] - dtdx * (F[0][v] - F[2][v]) - dtdy * (F[1][v] - F[3][v]);
        if (st[0] < R(0)) st[0] = R(0);
        if (prev[0] > R(DA_TINY)) {
            R sx[3], sy[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                sx[j] = slopes[(size_t)j * m.n + i];
                sy[j] = slopes[(size_t)(j + 3) * m.n + i];
            }
            const R vel0 = prev[1] / prev[0];
            const R vel1 = prev[2] / prev[0];
            const R h_inv = R(1.) / prev[0];
            R tmp = h_inv * (sy[1] - vel0 * sy[0]);
            const R sg0 = tiny_sgn(tmp, ft);
            const R sg2 = tiny_sgn(vel0, ft);
            tmp = h_inv * (sx[2] - vel1 * sx[0]);
            const R sg1 = tiny_sgn(tmp, ft);
            const R sg3 = tiny_sgn(vel1, ft);
            const R sin_int = R(mc.sin_int);
            const R tan_bed = R(mc.tan_bed[m.mat[i]]);
            R s1 = grav<R>(m, 0, i) * prev[0];
            R s2 = sg0 * prev[0] * ki * (gz * sy[0] + dgrav<R>(m, 1, i) * prev[0]) * sin_int;
            R s3 = sg2 * rmax(gz * prev[0] + vel0 * prev[1] * curvat<R>(m, 0, i), R(0.0)) * tan_bed;
            st[1] += dt * (s1 - s2 - s3);
            s1 = grav<R>(m, 1, i) * prev[0];
            s2 = sg1 * prev[0] * ki * (gz * sx[0] + dgrav<R>(m, 0, i) * prev[0]) * sin_int;
            s3 = sg3 * rmax(gz * prev[0] + vel1 * prev[2] * curvat<R>(m, 1, i), R(0.0)) * tan_bed;
            st[2] += dt * (s1 - s2 - s3);
        }
        if (!isfinite(st[0]) || !isfinite(st[1]) || !isfinite(st[2])) raise_err(sc, DA_ERR_NAN);
        oh[i] = st[0];
        ohu[i] = st[1];
        ohv[i] = st[2];
        vol = double(cell_dx<R>(m, i)) * double(cell_dy<R>(m, i)) * double(st[0]);
    }
    // fixed-order block reduction of the volume partial
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) vol += __shfl_xor_sync(0xffffffffu, vol, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vol;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kBlock / 32; ++w) t += red[w];
        vol_part[blockIdx.x] = t;
    }
}

// Sum of the per-block volume partials in a fixed order (one block).
__global__ void __launch_bounds__(1024) k_volume(const double *__restrict__ part, int nparts, DevScalars *sc) {
    __shared__ double red[32];
    double t = 0.0;
    for (int b = threadIdx.x; b < nparts; b += blockDim.x) t += part[b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x < 32) {
        double u = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) u += __shfl_xor_sync(0xffffffffu, u, o);
        if (threadIdx.x == 0) sc->volume = u;
    }
}

inline MeshArgs mesh_args(const da_ctx *ctx) {
    const DevMesh &d = ctx->mesh;
    MeshArgs a;
    a.n = d.n; a.nbr = d.nbr; a.mat = d.mat; a.bflag = d.bflag;
    a.x = d.x; a.y = d.y; a.dx = d.dx; a.dy = d.dy; a.g = d.g; a.dg = d.dg; a.curv = d.curv;
    a.fdx = d.fdx; a.fdy = d.fdy; a.fg = d.fg; a.fdg = d.fdg; a.fcurv = d.fcurv;
    return a;
}

template <class R>
int launch_step_t(da_ctx *ctx, cudaEvent_t *ev = nullptr) {
    const int n = ctx->mesh.n;
    const int nb = (n + kBlock - 1) / kBlock;
    const MeshArgs m = mesh_args(ctx);
    const int c = ctx->cur, o = 1 - c;
    StateRef<R> U{(const R *)ctx->U[c][0], (const R *)ctx->U[c][1], (const R *)ctx->U[c][2]};
    R *kact = (R *)ctx->kact;
    R *slopes = (R *)ctx->slopes;
    if (ev) cudaEventRecord(ev[0], ctx->stream);
    k_coef<R><<<nb, kBlock, 0, ctx->stream>>>(m, U, slopes, kact, ctx->mc, ctx->dsc);
    if (ev) cudaEventRecord(ev[1], ctx->stream);
    k_dt<<<1, 32, 0, ctx->stream>>>(ctx->dsc, ctx->tc);
    if (ev) cudaEventRecord(ev[2], ctx->stream);
    k_update<R><<<nb, kBlock, 0, ctx->stream>>>(m, U, (R *)ctx->U[o][0], (R *)ctx->U[o][1], (R *)ctx->U[o][2],
                                                slopes, kact, ctx->mc, ctx->dsc, ctx->vol_part);
    if (ev) cudaEventRecord(ev[3], ctx->stream);
    k_volume<<<1, 1024, 0, ctx->stream>>>(ctx->vol_part, nb, ctx->dsc);
    if (ev) cudaEventRecord(ev[4], ctx->stream);
    ctx->cur = o;
    return cuda_check(ctx, cudaGetLastError(), "forward step launch");
}

}  // namespace
}  // namespace fwd
}  // namespace da
