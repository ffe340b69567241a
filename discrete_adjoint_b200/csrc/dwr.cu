// Dual-weighted-residual error indicator on the device (error_compute.C:24-119 with the refined
// grid of uniform_refine.C and the reconstruction of bilinear_interp.C).
//
// The context keeps a second context for the error grid (the coarse mesh refined once).  One
// indicator step n -> n+1 from the live state U^n:
//   1. the coarse step U^n -> U^{n+1} (its dt), the state put back afterwards;
//   2. k_dwr_interp: on every fine cell the reconstructed U~^n (written as the error grid's state),
//      U~^{n+1} and lambda~ from the coarse fields through the fixed (cell, weight) pairs;
//   3. one step of the error grid from U~^n with the coarse dt (frozen-dt replay, same iteration);
//   4. k_dwr_residual: r = step(U~^n) - U~^{n+1}; per fine cell |r . (lambda - lambda~)| summed
//      over the three fields (el_error) and r . lambda (correction), lambda the parent's adjoint;
//   5. per coarse cell the sum over its four children (fixed order), and the totals as
//      compensated (Neumaier) FP64 sums in a fixed order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "da_internal.h"

namespace da {
namespace {

constexpr int kBlock = 256;
constexpr int kParts = 256;

template <class R>
struct Fields {
    const R *h, *hu, *hv;
    __device__ R get(int v, int i) const { return v == 0 ? h[i] : (v == 1 ? hu[i] : hv[i]); }
};

template <class R>
__global__ void __launch_bounds__(kBlock) k_dwr_interp(int nf, const int32_t *__restrict__ idx,
                                                       const double *__restrict__ w, Fields<R> un, Fields<R> unext,
                                                       Fields<R> lam, R *fh, R *fhu, R *fhv,
                                                       double *__restrict__ ut_next, double *__restrict__ lamt) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        double a[3] = {0, 0, 0}, b[3] = {0, 0, 0}, c[3] = {0, 0, 0};
        for (int q = 0; q < 4; ++q) {
            const int k = idx[(size_t)q * nf + f];
            if (k < 0) continue;
            const double wq = w[(size_t)q * nf + f];
            for (int v = 0; v < 3; ++v) {
                a[v] += wq * double(un.get(v, k));
                b[v] += wq * double(unext.get(v, k));
                c[v] += wq * double(lam.get(v, k));
            }
        }
        fh[f] = R(a[0]);
        fhu[f] = R(a[1]);
        fhv[f] = R(a[2]);
        for (int v = 0; v < 3; ++v) {
            ut_next[(size_t)v * nf + f] = b[v];
            lamt[(size_t)v * nf + f] = c[v];
        }
    }
}

template <class R>
__global__ void __launch_bounds__(kBlock) k_dwr_residual(int nf, const int32_t *__restrict__ parent, Fields<R> uf,
                                                         const double *__restrict__ ut_next,
                                                         const double *__restrict__ lamt, Fields<R> lam,
                                                         double *__restrict__ err, double *__restrict__ corr) {
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < nf; f += gridDim.x * blockDim.x) {
        const int p = parent[f];
        double e = 0.0, c = 0.0;
        for (int v = 0; v < 3; ++v) {
            const double r = double(uf.get(v, f)) - ut_next[(size_t)v * nf + f];
            const double l = double(lam.get(v, p));
            e += fabs(r * (l - lamt[(size_t)v * nf + f]));
            c += r * l;
        }
        err[f] = e;
        corr[f] = c;
    }
}

// Per coarse cell: the sum of its children's el_error in child order.
__global__ void __launch_bounds__(kBlock) k_dwr_cells(int n, const int32_t *__restrict__ children,
                                                      const double *__restrict__ err, double *__restrict__ cell) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int q = 0; q < 4; ++q) {
            const int f = children[(size_t)q * n + i];
            if (f >= 0) s += err[f];
        }
        cell[i] = s;
    }
}

// Neumaier's compensated addition: (s, c) += x.
__device__ __forceinline__ void neumaier(double &s, double &c, double x) {
    const double t = s + x;
    if (fabs(s) >= fabs(x))
        c += (s - t) + x;
    else
        c += (x - t) + s;
    s = t;
}

// Block b sums its fixed contiguous range of a[] (both arrays) with compensation, thread by
// thread and then thread 0 over the threads in order; then one block adds the parts.
__global__ void __launch_bounds__(kBlock) k_dwr_sum_parts(int nf, const double *__restrict__ a,
                                                          const double *__restrict__ b, double *__restrict__ parts) {
    __shared__ double ss[2][kBlock], cc[2][kBlock];
    const int per = (nf + kParts - 1) / kParts;
    const int f0 = blockIdx.x * per, f1 = min(nf, f0 + per);
    double s0 = 0, c0 = 0, s1 = 0, c1 = 0;
    for (int f = f0 + threadIdx.x; f < f1; f += kBlock) {
        neumaier(s0, c0, a[f]);
        neumaier(s1, c1, b[f]);
    }
    ss[0][threadIdx.x] = s0;
    cc[0][threadIdx.x] = c0;
    ss[1][threadIdx.x] = s1;
    cc[1][threadIdx.x] = c1;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < 2; ++k) {
            double s = 0, c = 0;
            for (int t = 0; t < kBlock; ++t) {
                neumaier(s, c, ss[k][t]);
                neumaier(s, c, cc[k][t]);
            }
            parts[(size_t)4 * blockIdx.x + 2 * k] = s;
            parts[(size_t)4 * blockIdx.x + 2 * k + 1] = c;
        }
    }
}

__global__ void k_dwr_sum_final(const double *__restrict__ parts, double *__restrict__ out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    for (int k = 0; k < 2; ++k) {
        double s = 0, c = 0;
        for (int b = 0; b < kParts; ++b) {
            neumaier(s, c, parts[(size_t)4 * b + 2 * k]);
            neumaier(s, c, parts[(size_t)4 * b + 2 * k + 1]);
        }
        out[k] = s + c;
    }
}

template <class R>
Fields<R> fields(void *const U[3]) {
    return Fields<R>{(const R *)U[0], (const R *)U[1], (const R *)U[2]};
}

template <class R>
int run_t(da_ctx *ctx, DwrState &d, int un, int unext, int lam, double dt, double time0, long long iter0) {
    da_ctx *fc = d.fine;
    const int nf = fc->mesh.n, grid = (ctx->sm_count > 0 ? ctx->sm_count : 148) * 8;
    k_dwr_interp<R><<<grid, kBlock, 0, ctx->stream>>>(nf, d.interp, d.weight, fields<R>(ctx->U[un]),
                                                      fields<R>(ctx->U[unext]), fields<R>(ctx->lam[lam]),
                                                      (R *)fc->U[fc->cur][0], (R *)fc->U[fc->cur][1],
                                                      (R *)fc->U[fc->cur][2], d.ut_next, d.lamt);
    int st = cuda_check(ctx, cudaGetLastError(), "dwr interpolation");
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    // one step of the error grid from U~^n with the coarse dt and iteration
    if (!st) st = forward_state_changed(fc);
    if (!st) st = cuda_check(fc, cudaStreamSynchronize(fc->stream), "sync");
    fc->have_state = true;
    if (!st) st = da_set_time(fc, time0, iter0);
    if (!st) st = da_set_dt_replay(fc, &dt, 1, iter0);
    if (!st) st = launch_forward_step(fc);
    if (!st) st = cuda_check(fc, cudaStreamSynchronize(fc->stream), "sync");
    if (!st) {
        k_dwr_residual<R><<<grid, kBlock, 0, ctx->stream>>>(nf, d.parent, fields<R>(fc->U[fc->cur]), d.ut_next, d.lamt,
                                                            fields<R>(ctx->lam[lam]), d.err, d.corr);
        k_dwr_cells<<<grid, kBlock, 0, ctx->stream>>>(ctx->mesh.n, d.children, d.err, d.cell);
        k_dwr_sum_parts<<<kParts, kBlock, 0, ctx->stream>>>(nf, d.err, d.corr, d.parts);
        k_dwr_sum_final<<<1, 32, 0, ctx->stream>>>(d.parts, d.sums);
        st = cuda_check(ctx, cudaGetLastError(), "dwr residual");
    }
    return st;
}

// The context's scalars in stream order (its stream does not synchronise with the legacy stream).
int read_scalars(da_ctx *ctx) {
    int st = cuda_check(ctx, cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream),
                        "scalars");
    return st ? st : cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
}

void free_dwr(da_ctx *ctx) {
    DwrState &d = ctx->dwr;
    if (d.fine) da_destroy(d.fine);
    if (d.mem) cudaFree(d.mem);
    d = DwrState{};
}

}  // namespace

void dwr_release(da_ctx *ctx) { free_dwr(ctx); }

int dwr_indicator(da_ctx *ctx, int un, int unext, int lam, double dt, double time0, long long iter0) {
    return ctx->p.precision == DA_PREC_FP64 ? run_t<double>(ctx, ctx->dwr, un, unext, lam, dt, time0, iter0)
                                            : run_t<float>(ctx, ctx->dwr, un, unext, lam, dt, time0, iter0);
}

}  // namespace da

using namespace da;

extern "C" {

int da_dwr_setup(da_ctx *ctx, const da_mesh_soa *fine, const int32_t *parent, const int32_t *interp,
                 const double *weight) {
    if (!ctx || !fine || !parent || !interp || !weight) return DA_ERR_INVALID;
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_dwr_setup: no mesh");
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, "da_dwr_setup: ensemble context");
    const int n = ctx->mesh.n, nf = fine->n_cells;
    if (nf <= 0) return set_error(ctx, DA_ERR_INVALID, "da_dwr_setup: empty error grid");
    // host checks: every index in range, every coarse cell with at most four children
    std::vector<int32_t> children((size_t)4 * n, -1);
    std::vector<int> count(n, 0);
    for (int f = 0; f < nf; ++f) {
        const int p = parent[f];
        if (p < 0 || p >= n || count[p] >= 4) return set_error(ctx, DA_ERR_INVALID, "da_dwr_setup: parent map");
        children[(size_t)count[p]++ * n + p] = f;
        for (int q = 0; q < 4; ++q) {
            const int k = interp[(size_t)q * nf + f];
            if (k < -1 || k >= n) return set_error(ctx, DA_ERR_INVALID, "da_dwr_setup: interpolant index");
        }
    }
    cudaSetDevice(ctx->device);
    free_dwr(ctx);
    DwrState &d = ctx->dwr;
    int err = 0;
    d.fine = da_create(&ctx->p, &err);
    if (!d.fine) return set_error(ctx, err, "da_dwr_setup: error-grid context");
    int st = da_upload_mesh(d.fine, fine, 0);
    if (st) {
        set_error(ctx, st, std::string("da_dwr_setup: ") + da_last_error(d.fine));
        free_dwr(ctx);
        return st;
    }
    // device tables: parent, children, interpolants, weights, work arrays
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off = (off + bytes + 255) & ~size_t(255); return o; };
    const size_t o_par = take(4 * (size_t)nf), o_ch = take(4 * (size_t)4 * n), o_idx = take(4 * (size_t)4 * nf),
                 o_w = take(8 * (size_t)4 * nf), o_ut = take(8 * (size_t)3 * nf), o_lt = take(8 * (size_t)3 * nf),
                 o_err = take(8 * (size_t)nf), o_corr = take(8 * (size_t)nf), o_cell = take(8 * (size_t)n),
                 o_parts = take(8 * (size_t)4 * kParts), o_sums = take(8 * 2);
    st = cuda_check(ctx, cudaMalloc(&d.mem, off), "cudaMalloc(dwr)");
    if (st) {
        free_dwr(ctx);
        return st;
    }
    unsigned char *b = (unsigned char *)d.mem;
    d.parent = (int32_t *)(b + o_par);
    d.children = (int32_t *)(b + o_ch);
    d.interp = (int32_t *)(b + o_idx);
    d.weight = (double *)(b + o_w);
    d.ut_next = (double *)(b + o_ut);
    d.lamt = (double *)(b + o_lt);
    d.err = (double *)(b + o_err);
    d.corr = (double *)(b + o_corr);
    d.cell = (double *)(b + o_cell);
    d.parts = (double *)(b + o_parts);
    d.sums = (double *)(b + o_sums);
    d.nf = nf;
    st = copy_h2d(ctx, d.parent, parent, 4 * (size_t)nf, "copy");
    if (!st) st = copy_h2d(ctx, d.children, children.data(), 4 * (size_t)4 * n, "copy");
    if (!st) st = copy_h2d(ctx, d.interp, interp, 4 * (size_t)4 * nf, "copy");
    if (!st) st = copy_h2d(ctx, d.weight, weight, 8 * (size_t)4 * nf, "copy");
    if (st) free_dwr(ctx);
    return st;
}

int da_dwr_step(da_ctx *ctx, const double *lambda_next, double *el_error, double *cell_error, double *sums) {
    if (!ctx || !lambda_next) return DA_ERR_INVALID;
    if (!ctx->dwr.fine) return set_error(ctx, DA_ERR_INVALID, "da_dwr_step: no error grid (da_dwr_setup)");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_dwr_step: no state");
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)ctx->mesh.n;
    int st = adj_alloc_for_dwr(ctx);
    for (int v = 0; v < 3 && !st; ++v) st = upload_real(ctx, ctx->lam[0][v], lambda_next + v * n);
    // the coarse step n -> n+1 from a base checkpoint, put back afterwards
    if (!st) st = launch_snapshot(ctx, ctx->snaps[0], true);
    if (!st) st = read_scalars(ctx);
    const double time0 = ctx->hsc->time;
    const long long iter0 = ctx->hsc->iter;
    if (!st) st = launch_forward_step(ctx);
    if (!st) st = read_scalars(ctx);
    if (!st) st = device_error(ctx, "da_dwr_step: the coarse step");
    const double dt = ctx->hsc->dt;
    if (!st) st = dwr_indicator(ctx, 1 - ctx->cur, ctx->cur, 0, dt, time0, iter0);
    if (!st) st = launch_snapshot(ctx, ctx->snaps[0], false);
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    const int nf = ctx->dwr.nf;
    if (!st && el_error) st = copy_d2h(ctx, el_error, ctx->dwr.err, 8 * (size_t)nf, "copy");
    if (!st && cell_error) st = copy_d2h(ctx, cell_error, ctx->dwr.cell, 8 * n, "copy");
    if (!st && sums) st = copy_d2h(ctx, sums, ctx->dwr.sums, 16, "copy");
    return st;
}

}  // extern "C"
