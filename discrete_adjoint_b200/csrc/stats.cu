// Flow statistics of the current state (calc_stats, src/geoflow/stats.C:31-360) and the
// discharge through planes (DISCHARGE::update, src/header/properties.h:964-1133), on the device.
//
// One pass over the cells: block b of kParts sums a fixed contiguous range of cells (thread-strided,
// then thread 0 over the threads in order), a final block adds the parts in order: FP64 sums in a
// fixed order (the reference sums in hash-table order, so the two agree to rounding).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "da_internal.h"
#include "fv_device.cuh"

namespace da {
namespace {

using namespace fv;

constexpr int kBlock = 256;
constexpr int kParts = 256;
constexpr int kSums = 14;   // xC yC rC area v_ave vx_ave vy_ave slope_ave energy slopevol testvol xVar yVar u_ave
constexpr int kMax = 3;     // max_height v_max u_max
constexpr int kMin = 4;     // xmin, -xmax, ymin, -ymax (over h >= hxyminmax)
constexpr int kPartLen = kSums + kMax + kMin + 2 + DA_MAX_PLANES;  // + test point (dist2, reach)

struct StatArgs {
    double min_height, hxyminmax, heightifreach, tx, ty;
    int n_planes;
    double planes[DA_MAX_PLANES][10];  // DISCHARGE::init's precomputed rows (properties.h:925-959)
};

// DISCHARGE::update for one cell and one plane (properties.h:965-1133): the plane segment clipped
// to the cell, the flux (hu dy - hv dx) through it.  nodes: 4 corners (SW, SE, NE, NW), 4 edge
// midpoints (S, E, N, W), centre.
__device__ double plane_flux(const double nodes[9][2], double hu, double hv, const double *pl) {
    double nearest[2], ip[2][2];
    double dxn[4], dyn[4];
    const double half = (fabs(nodes[6][0] - nodes[4][0]) + fabs(nodes[6][1] - nodes[4][1]) +
                         fabs(nodes[7][0] - nodes[5][0]) + fabs(nodes[7][1] - nodes[5][1])) *
                        0.25;
    const double half2 = half * half;
    const double err = half / pow(2.0, 19.0);
    for (int c1 = 0; c1 < 4; ++c1) {
        const int c2 = (c1 + 1) % 4;
        dxn[c1] = nodes[c2][0] - nodes[c1][0];
        dyn[c1] = nodes[c2][1] - nodes[c1][1];
    }
    double s1 = nodes[8][1] * pl[5] + nodes[8][0] * pl[4];
    nearest[0] = (-pl[5] * pl[7] + pl[4] * s1) / pl[6];
    nearest[1] = (+pl[4] * pl[7] + pl[5] * s1) / pl[6];
    const double d2 = (nodes[8][0] - nearest[0]) * (nodes[8][0] - nearest[0]) +
                      (nodes[8][1] - nearest[1]) * (nodes[8][1] - nearest[1]);
    if (!(d2 < half2 * pl[8])) return 0.0;
    int ni = 0;
    for (int c1 = 0; c1 < 4; ++c1) {
        s1 = nodes[c1][1] * dxn[c1] - nodes[c1][0] * dyn[c1];
        const double s2 = dxn[c1] * pl[5] - dyn[c1] * pl[4];
        if ((s2 < 0) || (s2 > 0)) {
            ip[ni][0] = (pl[4] * s1 - dxn[c1] * pl[7]) / s2;
            ip[ni][1] = (pl[5] * s1 - dyn[c1] * pl[7]) / s2;
            if (((ip[ni][0] < pl[0] - err) && (pl[0] < pl[1])) || ((ip[ni][0] > pl[0] + err) && (pl[0] > pl[1])) ||
                ((ip[ni][1] < pl[2] - err) && (pl[2] < pl[3])) || ((ip[ni][1] > pl[2] + err) && (pl[2] > pl[3]))) {
                ip[ni][0] = pl[0];
                ip[ni][1] = pl[2];
            } else if (((ip[ni][0] < pl[1] - err) && (pl[1] < pl[0])) ||
                       ((ip[ni][0] > pl[1] + err) && (pl[1] > pl[0])) ||
                       ((ip[ni][1] < pl[3] - err) && (pl[3] < pl[2])) ||
                       ((ip[ni][1] > pl[3] + err) && (pl[3] > pl[2]))) {
                ip[ni][0] = pl[1];
                ip[ni][1] = pl[3];
            }
            if (((((ip[ni][0] - ip[0][0]) * (ip[ni][0] - ip[0][0]) + (ip[ni][1] - ip[0][1]) * (ip[ni][1] - ip[0][1])) >
                  (half / 512.0)) ||
                 (ni == 0)) &&
                (s2 != 0.0))
                ++ni;
            if (ni == 2) {
                if ((ip[1][0] - ip[0][0]) * (pl[1] - pl[0]) + (ip[1][1] - ip[0][1]) * (pl[3] - pl[2]) < 0.0) {
                    double t = ip[0][0];
                    ip[0][0] = ip[1][0];
                    ip[1][0] = t;
                    t = ip[0][1];
                    ip[0][1] = ip[1][1];
                    ip[1][1] = t;
                }
                break;
            }
        }
    }
    if (ni == 1) {
        const double e1 = (nodes[8][0] - pl[0]) * (nodes[8][0] - pl[0]) + (nodes[8][1] - pl[2]) * (nodes[8][1] - pl[2]);
        const double e2 = (nodes[8][0] - pl[1]) * (nodes[8][0] - pl[1]) + (nodes[8][1] - pl[3]) * (nodes[8][1] - pl[3]);
        if (e1 <= e2) {
            ip[1][0] = pl[0];
            ip[1][1] = pl[2];
        } else {
            ip[1][0] = pl[1];
            ip[1][1] = pl[3];
        }
        ni = 2;
    }
    if (ni != 2) return 0.0;
    return hu * (ip[1][1] - ip[0][1]) - hv * (ip[1][0] - ip[0][0]);
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_stats_parts(MeshArgs m, StateRef<R> U, StatArgs a, double *parts) {
    __shared__ double sh[kBlock];
    // the owned cells (a subdomain's ghosts are another subdomain's)
    const int per = (m.n_owned + kParts - 1) / kParts;
    const int i0 = blockIdx.x * per, i1 = min(m.n_owned, i0 + per);
    double s[kSums] = {}, mx[kMax] = {}, mn[kMin], dis[DA_MAX_PLANES] = {};
    for (int q = 0; q < kMin; ++q) mn[q] = HUGE_VAL;
    double tdist = pow(2.0, 30.0), treach = 0.0;  // stats.C:58
    for (int i = i0 + threadIdx.x; i < i1; i += kBlock) {
        const double h = double(U.h[i]), hu = double(U.hu[i]), hv = double(U.hv[i]);
        const double x = m.x[i], y = m.y[i], dx = m.dx ? m.dx[i] : double(m.fdx[i]), dy = m.dy ? m.dy[i] : double(m.fdy[i]);
        if (a.n_planes > 0) {
            double nodes[9][2] = {{x - 0.5 * dx, y - 0.5 * dy}, {x + 0.5 * dx, y - 0.5 * dy}, {x + 0.5 * dx, y + 0.5 * dy},
                                  {x - 0.5 * dx, y + 0.5 * dy}, {x, y - 0.5 * dy},             {x + 0.5 * dx, y},
                                  {x, y + 0.5 * dy},             {x - 0.5 * dx, y},             {x, y}};
            for (int p = 0; p < a.n_planes; ++p) dis[p] += plane_flux(nodes, hu, hv, a.planes[p]);
        }
        if (!(h > a.min_height)) continue;
        mx[0] = h > mx[0] ? h : mx[0];
        if (h >= a.hxyminmax) {
            mn[0] = x < mn[0] ? x : mn[0];
            mn[1] = -x < mn[1] ? -x : mn[1];
            mn[2] = y < mn[2] ? y : mn[2];
            mn[3] = -y < mn[3] ? -y : mn[3];
        }
        const double d2 = (x - a.tx) * (x - a.tx) + (y - a.ty) * (y - a.ty);
        if (d2 < tdist) {
            tdist = d2;
            treach = h >= a.heightifreach ? 1.0 : 0.0;
        }
        const double dA = dx * dy, dV = h * dA;
        s[3] += dA;
        s[10] += dV;
        s[0] += x * dV;
        s[1] += y * dV;
        s[11] += x * x * dV;
        s[12] += y * y * dV;
        s[2] += sqrt((x - 1.2) * (x - 1.2) + (y - 0.3) * (y - 0.3)) * dV;  // xCen, yCen of stats.C:68-69
        const double sp = sqrt(hu * hu + hv * hv) * dA;
        s[4] += sp;
        s[13] += sp;
        double v0 = 0, v1 = 0;
        if (h > DA_TINY) {  // Element::eval_velocity at the centre
            v0 = hu / h;
            v1 = hv / h;
        }
        const double vm = sqrt(v0 * v0 + v1 * v1);
        mx[1] = vm > mx[1] ? vm : mx[1];
        mx[2] = vm > mx[2] ? vm : mx[2];
        s[5] += hu * dA;
        s[6] += hv * dA;
        s[8] += .5 * (9.8 * h * h + h * (v0 * v0 + v1 * v1)) * dA;
        if (vm > DA_TINY) {
            // terrain slope from the gravity vector: (dz/dx, dz/dy) = -(g_x, g_y) / g_z
            const double gz = m.g ? m.g[(size_t)2 * m.n + i] : double(m.fg[(size_t)2 * m.n + i]);
            const double gx = m.g ? m.g[i] : double(m.fg[i]);
            const double gy = m.g ? m.g[(size_t)m.n + i] : double(m.fg[(size_t)m.n + i]);
            const double xs = -gx / gz, ys = -gy / gz;
            s[7] += -(hu * xs + hv * ys) * dA / vm;
            s[9] += dV;
        }
    }
    // the block's values in thread order
    double *out = parts + (size_t)blockIdx.x * kPartLen;
    auto reduce = [&](double v, int slot, int op) {
        __syncthreads();
        sh[threadIdx.x] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = sh[0];
            for (int t = 1; t < kBlock; ++t)
                r = op == 0 ? r + sh[t] : (op == 1 ? (sh[t] > r ? sh[t] : r) : (sh[t] < r ? sh[t] : r));
            out[slot] = r;
        }
    };
    for (int q = 0; q < kSums; ++q) reduce(s[q], q, 0);
    for (int q = 0; q < kMax; ++q) reduce(mx[q], kSums + q, 1);
    for (int q = 0; q < kMin; ++q) reduce(mn[q], kSums + kMax + q, 2);
    for (int p = 0; p < a.n_planes; ++p) reduce(dis[p], kSums + kMax + kMin + 2 + p, 0);
    // test point: the smallest distance; its reach (a tie takes the higher reach)
    __syncthreads();
    sh[threadIdx.x] = tdist;
    __shared__ double rr[kBlock];
    rr[threadIdx.x] = treach;
    __syncthreads();
    if (threadIdx.x == 0) {
        double d = sh[0], r = rr[0];
        for (int t = 1; t < kBlock; ++t)
            if (sh[t] < d || (sh[t] == d && rr[t] > r)) {
                d = sh[t];
                r = rr[t];
            }
        out[kSums + kMax + kMin] = d;
        out[kSums + kMax + kMin + 1] = r;
    }
}

__global__ void k_stats_final(const double *parts, int n_planes, double vslump, double d_time, double *res,
                              double *discharge) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s[kSums] = {}, mx[kMax] = {}, mn[kMin], dis[DA_MAX_PLANES] = {};
    for (int q = 0; q < kMin; ++q) mn[q] = HUGE_VAL;
    double d = pow(2.0, 30.0), reach = 0.0;
    for (int b = 0; b < kParts; ++b) {
        const double *p = parts + (size_t)b * kPartLen;
        for (int q = 0; q < kSums; ++q) s[q] += p[q];
        for (int q = 0; q < kMax; ++q) mx[q] = p[kSums + q] > mx[q] ? p[kSums + q] : mx[q];
        for (int q = 0; q < kMin; ++q) mn[q] = p[kSums + kMax + q] < mn[q] ? p[kSums + kMax + q] : mn[q];
        const double pd = p[kSums + kMax + kMin], pr = p[kSums + kMax + kMin + 1];
        if (pd < d || (pd == d && pr > reach)) {
            d = pd;
            reach = pr;
        }
        for (int q = 0; q < n_planes; ++q) dis[q] += p[kSums + kMax + kMin + 2 + q];
    }
    // stats.C:271-302 with LENGTH_SCALE = HEIGHT_SCALE = velocity scale = 1
    const double tv = s[10];
    res[0] = s[0] / tv;                      // xcen
    res[1] = s[1] / tv;                      // ycen
    res[2] = s[11] / tv - res[0] * res[0];   // xvar
    res[3] = s[12] / tv - res[1] * res[1];   // yvar
    res[4] = s[2] / tv;                      // rmean
    res[5] = s[3];                           // area
    res[6] = s[4] / tv;                      // vmean
    res[7] = s[13] / tv;                     // umean
    res[8] = s[5] / tv;                      // vxmean
    res[9] = s[6] / tv;                      // vymean
    res[10] = s[9] > 0 ? s[7] / s[9] : 0.0;  // slopemean
    res[11] = tv;                            // statvolume
    res[12] = 3.0 * sqrt(res[2] + res[3]);   // piler
    res[13] = mx[0];                         // hmax
    res[14] = mx[1];                         // vmax
    res[15] = mx[2];                         // umax
    res[16] = vslump != 0 ? res[6] / vslump : 0.0;  // vstar
    res[17] = mn[0];
    res[18] = -mn[1];
    res[19] = mn[2];
    res[20] = -mn[3];
    res[21] = reach;
    res[22] = s[8];                          // the energy sum stats.C reduces in its "adjoint" slot
    for (int q = 0; q < n_planes; ++q) discharge[q] += d_time * dis[q];
}

template <class R>
int stats_t(da_ctx *ctx, const StatArgs &a, double vslump, double d_time, double *dev) {
    const MeshArgs m = mesh_args(ctx);
    const int c = ctx->cur;
    StateRef<R> U{(const R *)ctx->U[c][0], (const R *)ctx->U[c][1], (const R *)ctx->U[c][2]};
    double *parts = dev, *res = dev + (size_t)kParts * kPartLen, *dis = res + 32;
    k_stats_parts<R><<<kParts, kBlock, 0, ctx->stream>>>(m, U, a, parts);
    k_stats_final<<<1, 32, 0, ctx->stream>>>(parts, a.n_planes, vslump, d_time, res, dis);
    return cuda_check(ctx, cudaGetLastError(), "stats launch");
}

// OutLine::update (properties.h:726-790) for every cell: the maximum depth so far over the grid
// cells its footprint covers (bit patterns of non-negative doubles order like the values, so an
// integer atomicMax is exact).
template <class R>
__global__ void __launch_bounds__(kBlock) k_outline(MeshArgs m, StateRef<R> U, OutlineGrid g) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.n_owned; i += gridDim.x * blockDim.x) {
        const double height = double(U.h[i]);
        if (!(height > 0.0)) continue;  // the map starts at zero
        const double x = m.x[i], y = m.y[i], dx = m.dx ? m.dx[i] : double(m.fdx[i]), dy = m.dy ? m.dy[i] : double(m.fdy[i]);
        const double xstart = x - 0.5 * dx, xstop = x + 0.5 * dx, ystart = y - 0.5 * dy, ystop = y + 0.5 * dy;
        int ixstart = (int)((xstart - g.x0) / g.dx + 0.5), ixstop = (int)((xstop - g.x0) / g.dx + 0.5);
        int iystart = (int)((ystart - g.y0) / g.dy + 0.5), iystop = (int)((ystop - g.y0) / g.dy + 0.5);
        if (ixstart < 0) ixstart = 0;
        if (ixstop == ixstart) {
            ixstart = (int)((xstart - g.x0) / g.dx);
            ixstop = ixstart + 1;
        }
        if (ixstop > g.nx) ixstop = g.nx;
        if (iystart < 0) iystart = 0;
        if (iystop == iystart) {
            iystart = (int)((ystart - g.y0) / g.dy);
            iystop = iystart + 1;
        }
        if (iystop > g.ny) iystop = g.ny;
        const unsigned long long hb = __double_as_longlong(height);
        for (int iy = iystart; iy < iystop; ++iy)
            for (int ix = ixstart; ix < ixstop; ++ix)
                if (ix >= 0 && iy >= 0) atomicMax(g.map + (size_t)iy * g.nx + ix, hb);
    }
}

}  // namespace
}  // namespace da

using namespace da;

extern "C" {

int da_outline_init(da_ctx *ctx, const double dxy[2], const double xrange[2], const double yrange[2]) {
    if (!ctx || !dxy || !xrange || !yrange || !(dxy[0] > 0) || !(dxy[1] > 0) || !(xrange[1] > xrange[0]) ||
        !(yrange[1] > yrange[0]))
        return DA_ERR_INVALID;
    cudaSetDevice(ctx->device);
    OutlineGrid &g = ctx->outline;
    if (g.map) cudaFree(g.map);
    g = OutlineGrid{};
    // OutLine::init2 (properties.h:702-724)
    g.dx = dxy[0];
    g.dy = dxy[1];
    g.x0 = xrange[0];
    g.y0 = yrange[0];
    g.nx = (int)((xrange[1] - xrange[0]) / g.dx + 0.5);
    g.ny = (int)((yrange[1] - yrange[0]) / g.dy + 0.5);
    if (g.nx <= 0 || g.ny <= 0 || (long long)g.nx * g.ny > (1ll << 28))
        return set_error(ctx, DA_ERR_INVALID, "da_outline_init: grid size");
    int st = cuda_check(ctx, cudaMalloc((void **)&g.map, sizeof(unsigned long long) * (size_t)g.nx * g.ny), "cudaMalloc");
    if (!st) st = cuda_check(ctx, cudaMemsetAsync(g.map, 0, sizeof(unsigned long long) * (size_t)g.nx * g.ny, ctx->stream),
                             "memset");
    return st;
}

int da_outline_update(da_ctx *ctx) {
    if (!ctx) return DA_ERR_INVALID;
    if (!ctx->outline.map) return set_error(ctx, DA_ERR_INVALID, "da_outline_update: no grid (da_outline_init)");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_outline_update: no state");
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, "da_outline_update: ensemble context");
    cudaSetDevice(ctx->device);
    const MeshArgs m = mesh_args(ctx);
    const int c = ctx->cur, grid = (ctx->sm_count > 0 ? ctx->sm_count : 148) * 4;
    if (ctx->p.precision == DA_PREC_FP64) {
        StateRef<double> U{(const double *)ctx->U[c][0], (const double *)ctx->U[c][1], (const double *)ctx->U[c][2]};
        k_outline<double><<<grid, kBlock, 0, ctx->stream>>>(m, U, ctx->outline);
    } else {
        StateRef<float> U{(const float *)ctx->U[c][0], (const float *)ctx->U[c][1], (const float *)ctx->U[c][2]};
        k_outline<float><<<grid, kBlock, 0, ctx->stream>>>(m, U, ctx->outline);
    }
    return cuda_check(ctx, cudaGetLastError(), "outline launch");
}

int da_outline_read(da_ctx *ctx, int32_t *nx, int32_t *ny, double *map) {
    if (!ctx) return DA_ERR_INVALID;
    const OutlineGrid &g = ctx->outline;
    if (!g.map) return set_error(ctx, DA_ERR_INVALID, "da_outline_read: no grid (da_outline_init)");
    if (nx) *nx = g.nx;
    if (ny) *ny = g.ny;
    if (!map) return DA_OK;
    cudaSetDevice(ctx->device);
    int st = cuda_check(ctx, cudaMemcpyAsync(map, g.map, sizeof(double) * (size_t)g.nx * g.ny, cudaMemcpyDeviceToHost,
                                             ctx->stream), "copy");
    return st ? st : cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
}

int da_compute_stats(da_ctx *ctx, const da_stats_props *props, double d_time, da_stats *out, double *discharge) {
    if (!ctx || !props || !out || props->n_planes < 0 || props->n_planes > DA_MAX_PLANES ||
        (props->n_planes > 0 && (!props->planes || !discharge)))
        return DA_ERR_INVALID;
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_compute_stats: no mesh");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_compute_stats: no state");
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, "da_compute_stats: ensemble context");
    cudaSetDevice(ctx->device);
    StatArgs a{};
    a.min_height = props->min_height >= 0 ? props->min_height : ctx->p.epsilon / 10000.0;  // datread.C:210
    a.hxyminmax = props->hxyminmax >= 0 ? props->hxyminmax : 10.0 * a.min_height;     // datread.C:315-316
    a.heightifreach = props->heightifreach;
    a.tx = props->xyifreach[0];
    a.ty = props->xyifreach[1];
    a.n_planes = props->n_planes;
    for (int k = 0; k < props->n_planes; ++k) {
        // DISCHARGE::init (properties.h:925-959)
        double *pl = a.planes[k];
        const double *in = props->planes + 4 * k;
        pl[0] = in[0];
        pl[1] = in[1];
        pl[2] = in[2];
        pl[3] = in[3];
        pl[4] = pl[1] - pl[0];
        pl[5] = pl[3] - pl[2];
        pl[6] = pl[4] * pl[4] + pl[5] * pl[5];
        pl[7] = pl[3] * pl[4] - pl[1] * pl[5];
        pl[8] = ((std::fabs(pl[4]) + std::fabs(pl[5])) * (std::fabs(pl[4]) + std::fabs(pl[5]))) / pl[6];
        pl[9] = 0.0;
        if (!(pl[6] > 0)) return set_error(ctx, DA_ERR_INVALID, "da_compute_stats: degenerate discharge plane");
    }
    const size_t words = (size_t)kParts * kPartLen + 32 + DA_MAX_PLANES;
    double *dev = nullptr;
    int st = cuda_check(ctx, cudaMalloc((void **)&dev, sizeof(double) * words), "cudaMalloc(stats)");
    double *dis = dev + (size_t)kParts * kPartLen + 32;
    // the state the statistics read may still be in flight on the context's stream
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (!st && props->n_planes > 0)
        st = copy_h2d(ctx, dis, discharge, sizeof(double) * props->n_planes, "copy");
    if (!st) st = ctx->p.precision == DA_PREC_FP64 ? stats_t<double>(ctx, a, props->vslump, d_time, dev)
                                                   : stats_t<float>(ctx, a, props->vslump, d_time, dev);
    double res[32];
    // the context's stream does not synchronise with the legacy stream of cudaMemcpy
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (!st) st = copy_d2h(ctx, res, dev + (size_t)kParts * kPartLen, sizeof(res), "copy");
    if (!st && props->n_planes > 0)
        st = copy_d2h(ctx, discharge, dis, sizeof(double) * props->n_planes, "copy");
    if (dev) cudaFree(dev);
    if (st) return st;
    out->xcen = res[0];
    out->ycen = res[1];
    out->xvar = res[2];
    out->yvar = res[3];
    out->rmean = res[4];
    out->area = res[5];
    out->vmean = res[6];
    out->umean = res[7];
    out->vxmean = res[8];
    out->vymean = res[9];
    out->slopemean = res[10];
    out->statvolume = res[11];
    out->piler = res[12];
    out->hmax = res[13];
    out->vmax = res[14];
    out->umax = res[15];
    out->vstar = res[16];
    for (int q = 0; q < 4; ++q) out->xyminmax[q] = res[17 + q];
    out->testpoint_reach = res[21] > 0.5 ? 1 : 0;
    out->pad = 0;
    out->energy = res[22];
    return DA_OK;
}

}  // extern "C"
