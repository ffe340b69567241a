// Device building blocks of the finite-volume step, shared by the forward and adjoint kernels.
// Every function restates one piece of the reference's per-cell numerics; the FP64
// instantiation keeps the reference's operation order (built without FMA contraction) and is
// bit-identical to it, the FP32 instantiation may reassociate (reciprocals, fused multiply-add).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "da_internal.h"

namespace da {
namespace fv {

template <class R>
struct StateRef {  // no __restrict__: the multi-step kernel reads what other blocks wrote
    const R *h;
    const R *hu;
    const R *hv;
};

template <class R>
struct StateOut {
    R *h;
    R *hu;
    R *hv;
};

// c_sgn (src/header/geoflow.h:90-100): zero inside +-GEOFLOW_TINY
template <class R>
__device__ __forceinline__ R c_sgn(R zz) {
    return zz > R(DA_TINY) ? R(1) : (zz < -R(DA_TINY) ? R(-1) : R(0));
}
// dabs (geoflow.h:143-148)
template <class R>
__device__ __forceinline__ R dabs(R d) {
    return d < R(0) ? -d : d;
}
// max/min of src/datstr/element2.C:1059-1071 (first argument wins ties)
template <class R>
__device__ __forceinline__ R rmax(R x, R y) {
    return x > y ? x : y;
}
template <class R>
__device__ __forceinline__ R rmin(R x, R y) {
    return x > y ? y : x;
}
// sgn(zz, tiny) of src/geoflow/sgn.f:19-33
template <class R>
__device__ __forceinline__ int fsgn(R zz, R tiny) {
    return dabs(zz) < tiny ? 0 : (zz >= tiny ? 1 : -1);
}
// tiny_sgn of src/adjoint/residual.C:153-160 (note num == tiny gives -1, as there)
template <class R>
__device__ __forceinline__ R tiny_sgn(R num, R tiny) {
    return dabs(num) < tiny ? R(0) : (num > tiny ? R(1) : R(-1));
}

struct MeshArgs {
    int n;
    int n_owned;  // cells [n_owned, n) are ghost copies of another subdomain's cells (n_owned = n: none)
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

inline MeshArgs mesh_args(const da_ctx *ctx) {
    const DevMesh &d = ctx->mesh;
    MeshArgs a;
    a.n = d.n; a.n_owned = d.n_owned; a.nbr = d.nbr; a.mat = d.mat; a.bflag = d.bflag;
    a.x = d.x; a.y = d.y; a.dx = d.dx; a.dy = d.dy; a.g = d.g; a.dg = d.dg; a.curv = d.curv;
    a.fdx = d.fdx; a.fdy = d.fdy; a.fg = d.fg; a.fdg = d.fdg; a.fcurv = d.fcurv;
    return a;
}

template <class R>
__device__ __forceinline__ R cell_dx(const MeshArgs &m, int i) {
    if constexpr (sizeof(R) == 8) return m.dx[i]; else return m.fdx[i];
}
template <class R>
__device__ __forceinline__ R cell_dy(const MeshArgs &m, int i) {
    if constexpr (sizeof(R) == 8) return m.dy[i]; else return m.fdy[i];
}
template <class R>
__device__ __forceinline__ R grav(const MeshArgs &m, int c, int i) {
    if constexpr (sizeof(R) == 8) return m.g[(size_t)c * m.n + i]; else return m.fg[(size_t)c * m.n + i];
}
template <class R>
__device__ __forceinline__ R dgrav(const MeshArgs &m, int c, int i) {
    if constexpr (sizeof(R) == 8) return m.dg[(size_t)c * m.n + i]; else return m.fdg[(size_t)c * m.n + i];
}
template <class R>
__device__ __forceinline__ R curvat(const MeshArgs &m, int c, int i) {
    if constexpr (sizeof(R) == 8) return m.curv[(size_t)c * m.n + i]; else return m.fcurv[(size_t)c * m.n + i];
}

// A cell's source coefficients: g_x, g_y, the two stored gravity derivatives, the two
// curvatures, and its material.
template <class R>
struct CellSrc {
    R g[2], dg[2], cv[2];
    int mat;
};
template <class R>
__device__ __forceinline__ CellSrc<R> cell_src(const MeshArgs &m, int i) {
    CellSrc<R> s;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        s.g[q] = grav<R>(m, q, i);
        s.dg[q] = dgrav<R>(m, q, i);
        s.cv[q] = curvat<R>(m, q, i);
    }
    s.mat = m.mat[i];
    return s;
}

// What the corrector's source terms form for a wet cell before using them: the limited slopes, the
// velocities, 1/h and the four friction signs (also what the source adjoint needs of the forward).
template <class R>
struct SrcFwd {
    R s[6];
    R vel0, vel1, h_inv;
    R sg0, sg1, sg2, sg3;
};

// No hook (the forward alone).
struct NoSrcHook {
    template <class... A>
    __device__ __forceinline__ void operator()(A &&...) const {}
};

// What the per-cell numerics read about a cell and its neighbours goes through a view: nb(s, c)
// the cell across neighbour entry s of cell c, and the values of a cell.  GlobalView reads the
// mesh table and the global arrays (c, e = cell indices); the step kernels' staged view reads a
// tile and its halo from shared memory (tile-local slots).  The arithmetic is the same either way.
template <class R>
struct GlobalView {
    const MeshArgs &m;
    StateRef<R> U;
    const R *kact;
    __device__ __forceinline__ int nb(int s, int c) const { return m.nbr[(size_t)s * m.n + c]; }
    __device__ __forceinline__ R h(int e) const { return U.h[e]; }
    __device__ __forceinline__ R hu(int e) const { return U.hu[e]; }
    __device__ __forceinline__ R hv(int e) const { return U.hv[e]; }
    __device__ __forceinline__ R k(int e) const { return kact[e]; }
    __device__ __forceinline__ R gz(int e) const { return grav<R>(m, 2, e); }
    __device__ __forceinline__ double coord(int dir, int e) const { return (dir == 0 ? m.x : m.y)[e]; }
    __device__ __forceinline__ float size(int dir, int e) const { return (dir == 0 ? m.fdx : m.fdy)[e]; }
};

template <class R>
__device__ __forceinline__ GlobalView<R> global_view(const MeshArgs &m, const StateRef<R> &U, const R *kact) {
    return GlobalView<R>{m, U, kact};
}

// Element::get_slopes for one interior cell (element2.C:830-939); out[0..2] d/dx, out[3..5] d/dy.
// Boundary cells (any side on the domain edge) have zero slopes.
// FP64: the centre distances are differences of stored centres (ep->coord - coord) and every
// quotient is a true division, as in the reference.  FP32: distances are half sums of cell
// sizes (exact for quadtree geometry) and the three divisors of a direction are inverted once.
template <class R, class V>
__device__ __forceinline__ void cell_slopes(const V &v, int i, uint8_t bf, R gamma, const R ui[3], R out[6]) {
    if (bf & 0x0F) {
#pragma unroll
        for (int j = 0; j < 6; ++j) out[j] = R(0);
        return;
    }
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
        const int ep = v.nb(dir, i);
        const int em = v.nb(dir + 2, i);
        const bool two_p = bf & (0x10 << dir), two_m = bf & (0x10 << (dir + 2));
        const R up[3] = {v.h(ep), v.hu(ep), v.hv(ep)};
        const R um[3] = {v.h(em), v.hu(em), v.hv(em)};
        R up2[3] = {0, 0, 0}, um2[3] = {0, 0, 0};
        if (two_p) {
            const int e = v.nb(dir + 4, i);
            up2[0] = v.h(e); up2[1] = v.hu(e); up2[2] = v.hv(e);
        }
        if (two_m) {
            const int e = v.nb(dir + 6, i);
            um2[0] = v.h(e); um2[1] = v.hu(e); um2[2] = v.hv(e);
        }
        if constexpr (sizeof(R) == 8) {
            const double ci = v.coord(dir, i);
            const double dxp = v.coord(dir, ep) - ci;
            const double dxm = ci - v.coord(dir, em);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                double dp = (up[j] - ui[j]) / dxp;
                if (two_p) dp = .5 * (dp + (up2[j] - ui[j]) / dxp);
                double dm = (ui[j] - um[j]) / dxm;
                if (two_m) dm = .5 * (dm + (ui[j] - um2[j]) / dxm);
                const double dc = (dp * dxm + dm * dxp) / (dxm + dxp);
                double mn = gamma * dabs(dp);
                const double b = gamma * dabs(dm), c = dabs(dc);
                if (mn > b) mn = b;
                if (mn > c) mn = c;
                out[j + 3 * dir] = .5 * (c_sgn(dp) + c_sgn(dm)) * mn;
            }
        } else {
            const float si = v.size(dir, i);
            const float dxp = 0.5f * (v.size(dir, ep) + si), dxm = 0.5f * (v.size(dir, em) + si);
            const float ip = 1.0f / dxp, im = 1.0f / dxm, isum = 1.0f / (dxm + dxp);
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                float dp = (up[j] - ui[j]) * ip;
                if (two_p) dp = 0.5f * (dp + (up2[j] - ui[j]) * ip);
                float dm = (ui[j] - um[j]) * im;
                if (two_m) dm = 0.5f * (dm + (ui[j] - um2[j]) * im);
                const float dc = (dp * dxm + dm * dxp) * isum;
                float mn = gamma * dabs(dp);
                const float b = gamma * dabs(dm), c = dabs(dc);
                if (mn > b) mn = b;
                if (mn > c) mn = c;
                out[j + 3 * dir] = 0.5f * (c_sgn(dp) + c_sgn(dm)) * mn;
            }
        }
    }
}

// k act/pass of a wet cell (h > GEOFLOW_TINY), gmfggetcoef (getcoef.f:19-66), from the table
// of the three sgn(vel) values per material.
// code (optional): 0 for the rest value, 1 + (sgn(vel) + 1) otherwise.
template <class R>
__device__ __forceinline__ R cell_kact(const MatConsts &mc, int mat, R h, R hu, R hv, const R s[6],
                                       uint8_t *code = nullptr) {
    R vel;
    if constexpr (sizeof(R) == 8) {
        vel = s[1] / h - hu * s[0] / (h * h) + s[5] / h - hv * s[3] / (h * h);
    } else {
        const float ih = 1.0f / h;
        vel = (s[1] - hu * ih * s[0] + s[5] - hv * ih * s[3]) * ih;
    }
    const int sg = fsgn(vel, R(DA_TINY));
    R k = R(mc.kact_sgn[mat][sg + 1]);
    uint8_t c = uint8_t(sg + 2);
    if (dabs(hu / h) < R(DA_TINY) && dabs(hv / h) < R(DA_TINY)) {
        k = R(mc.kact_rest);
        c = 0;
    }
    if (code) *code = c;
    return k;
}

// Element::xdirflux / ydirflux with dz = 0 (element2.C:1810-1996): state, physical flux and
// Davis wave speeds of one cell in direction dir; all zero for h < GEOFLOW_TINY.
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

// riemannflux (element2.C:2228-2264): HLL with Davis speeds, dry-side speeds 2*lambda - u.
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
    } else if constexpr (sizeof(R) == 8) {
        const double den = sr - sl;
#pragma unroll
        for (int v = 0; v < 3; ++v) flux[v] = (sr * l.f[v] - sl * r.f[v] + sl * sr * (r.u[v] - l.u[v])) / den;
    } else {
        const float inv = 1.0f / (sr - sl);
#pragma unroll
        for (int v = 0; v < 3; ++v) flux[v] = (sr * l.f[v] - sl * r.f[v] + sl * sr * (r.u[v] - l.u[v])) * inv;
    }
}

// State, flux and speeds of neighbour e; only h is read for a dry neighbour.
template <class R, class V>
__device__ __forceinline__ void nb_hfv(const V &v, int e, int dir, Hfv<R> &o) {
    const R h = v.h(e);
    if (h < R(DA_TINY)) {
#pragma unroll
        for (int a = 0; a < 3; ++a) o.u[a] = o.f[a] = o.s[a] = R(0);
        return;
    }
    dirflux<R>(dir, h, v.hu(e), v.hv(e), v.k(e), v.gz(e), o);
}

// Flux on side s of cell i (the value the reference stores on the side's edge-midpoint node):
// one Riemann flux with a same-size or coarser neighbour, the mean of two with two finer ones.
template <class R, class V>
__device__ __forceinline__ void side_flux(const V &v, int i, uint8_t bf, int s, const Hfv<R> &self, R F[3]) {
    const int dir = s & 1;
    const bool plus = s < 2;
    Hfv<R> nb;
    nb_hfv<R>(v, v.nb(s, i), dir, nb);
    if (plus) riemann<R>(self, nb, F);
    else riemann<R>(nb, self, F);
    if (bf & (0x10 << s)) {
        R f2[3];
        nb_hfv<R>(v, v.nb(s + 4, i), dir, nb);
        if (plus) riemann<R>(self, nb, f2);
        else riemann<R>(nb, self, f2);
#pragma unroll
        for (int v = 0; v < 3; ++v) F[v] = R(0.5) * (F[v] + f2[v]);
    }
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
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void raise_err(DevScalars *sc, int code) { atomicCAS(&sc->err, 0, code); }

// ------------------------------------------------------------------ tile scheduling
// Cells are grouped in tiles of kTileCells consecutive (Morton-ordered) cells, one thread per
// cell.  Round r of block b tests tiles (r * kTileCells + q) * gridDim.x + b, q = thread index:
// consecutive tiles go to consecutive blocks, so the few wet tiles of a compact flow spread over
// the grid instead of queueing in one block.  The tiles that need work are compacted into
// shared memory (increasing order) and processed one after another by the whole block.
__device__ __forceinline__ int sched_tile(int round) {
    return (round * kTileCells + (int)threadIdx.x) * (int)gridDim.x + (int)blockIdx.x;
}

__device__ __forceinline__ bool sched_more(int round, int ntiles) {
    return (long long)round * kTileCells * gridDim.x < ntiles;
}

// Needs blockDim.x == kTileCells; returns the number of tiles listed.
// pa, pb (optional): two values per listed tile stored beside it (pa[k], pb[k] for list[k]).
__device__ __forceinline__ int compact_tiles(bool need, int tile, int *list, int a = 0, int b2 = 0,
                                             int *pa = nullptr, int *pb = nullptr) {
    __shared__ int warp_count[kTileCells / 32];
    __shared__ int total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned b = __ballot_sync(0xffffffffu, need);
    if (lane == 0) warp_count[warp] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int w = 0; w < kTileCells / 32; ++w) {
            const int c = warp_count[w];
            warp_count[w] = acc;
            acc += c;
        }
        total = acc;
    }
    __syncthreads();
    if (need) {
        const int k = warp_count[warp] + __popc(b & ((1u << lane) - 1u));
        list[k] = tile;
        if (pa) {
            pa[k] = a;
            pb[k] = b2;
        }
    }
    __syncthreads();
    return total;
}

}  // namespace fv
}  // namespace da
