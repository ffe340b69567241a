// Domain decomposition of one mesh over several contexts (one per GPU, or several on one GPU):
// the reference's only parallel strategy -- weighted Hilbert-curve ranges of elements per MPI
// rank (src/repartition/repartition_BSFC.C:540), ghost elements refreshed every step
// (src/geoflow/move_data.C:28-300), dt from MPI_Allreduce(MIN) (src/geoflow/get_coef_and_eigen.C:173).
//
// A subdomain's context holds its owned cells [0, n_owned) followed by ghost cells (two rings:
// the cells that the step of an owned cell reads).  A step is split at the dt reduction:
//   da_step_bounds  k_coef on every cell; the last block writes the owned cells' CFL bound and
//                   -hmax to a 2-double buffer instead of forming dt
//   (MIN all-reduce of those two doubles over the subdomains: NCCL, or the host)
//   da_step_apply   dt from the reduced pair (the same bits on every subdomain), k_update
//   da_halo_pack / da_halo_unpack
//                   the owners' new values of the cells other subdomains hold as ghosts, gathered
//                   into one contiguous buffer per destination and scattered into the ghost slots
// The ghosts' own updates read domain edges where their neighbours leave the subdomain; the
// exchange overwrites them before the next step reads them, so the owned cells get the bits of
// the undivided mesh's step.
#include <cuda_runtime.h>

#include "da_internal.h"
#include "fv_device.cuh"

namespace da {
int launch_step_half_fp64(da_ctx *ctx, int half, double *bounds);
int launch_step_half_fp32(da_ctx *ctx, int half, double *bounds);

namespace {

constexpr int kBlock = 256;

// Gather: buf[v * n + k] = U_v[cells[k]], cells owned ([0, n_owned)); a bad index is reported
// (DA_ERR_INVALID) and skipped.
template <class R>
__global__ void __launch_bounds__(kBlock) k_halo_pack(const R *__restrict__ h, const R *__restrict__ hu,
                                                      const R *__restrict__ hv, int n_owned,
                                                      const int32_t *__restrict__ cells, int n, R *__restrict__ buf,
                                                      DevScalars *sc) {
    for (int k = blockIdx.x * kBlock + threadIdx.x; k < n; k += gridDim.x * kBlock) {
        const int c = cells[k];
        if (c < 0 || c >= n_owned) {
            fv::raise_err(sc, DA_ERR_INVALID);
            continue;
        }
        buf[k] = h[c];
        buf[(size_t)n + k] = hu[c];
        buf[2 * (size_t)n + k] = hv[c];
    }
}

// Scatter into ghost slots ([n_owned, n_cells)).  The segments written now differ between the two
// state buffers, may hold a wet cell and differ from a checkpoint: their flags say so, so that the
// next coefficient phase lists them and the next update rewrites both buffers' copies.
template <class R>
__global__ void __launch_bounds__(kBlock) k_halo_unpack(R *__restrict__ h, R *__restrict__ hu, R *__restrict__ hv,
                                                        int n_owned, int n_cells, const int32_t *__restrict__ cells,
                                                        int n, const R *__restrict__ buf, uint8_t *__restrict__ seg_clean,
                                                        uint8_t *__restrict__ seg_wet, uint8_t *__restrict__ seg_dirty,
                                                        DevScalars *sc) {
    for (int k = blockIdx.x * kBlock + threadIdx.x; k < n; k += gridDim.x * kBlock) {
        const int c = cells[k];
        if (c < n_owned || c >= n_cells) {
            fv::raise_err(sc, DA_ERR_INVALID);
            continue;
        }
        h[c] = buf[k];
        hu[c] = buf[(size_t)n + k];
        hv[c] = buf[2 * (size_t)n + k];
        const int s = c >> 5;
        seg_clean[s] = 0;
        seg_wet[s] = 1;
        seg_dirty[s] = 1;
    }
}

int halo_grid(const da_ctx *ctx, int n) {
    const int cap = (ctx->sm_count > 0 ? ctx->sm_count : 148) * 4;
    const int g = (n + kBlock - 1) / kBlock;
    return g < 1 ? 1 : (g < cap ? g : cap);
}

bool is_device_pointer(const void *p, int device) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == device;
}

int check_ctx(da_ctx *ctx, const char *what) {
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, std::string(what) + ": ensemble context");
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, std::string(what) + ": no mesh");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, std::string(what) + ": no state");
    return DA_OK;
}

int bounds_alloc(da_ctx *ctx) {
    if (ctx->dd_bounds) return DA_OK;
    return cuda_check(ctx, cudaMalloc((void **)&ctx->dd_bounds, 2 * sizeof(double)), "cudaMalloc(bounds)");
}

int launch_half(da_ctx *ctx, int half, double *bounds) {
    return ctx->p.precision == DA_PREC_FP64 ? launch_step_half_fp64(ctx, half, bounds)
                                            : launch_step_half_fp32(ctx, half, bounds);
}

int read_scalars(da_ctx *ctx, const char *where) {
    int st = cuda_check(ctx, cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost,
                                             ctx->stream), "read scalars");
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "stream sync");
    if (!st) st = device_error(ctx, where);
    return st;
}

}  // namespace
}  // namespace da

using namespace da;

extern "C" {

int da_set_owned(da_ctx *ctx, int32_t n_owned) {
    if (!ctx) return DA_ERR_INVALID;
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, "da_set_owned: ensemble context");
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_set_owned: no mesh");
    if (n_owned < 1 || n_owned > ctx->mesh.n)
        return set_error(ctx, DA_ERR_INVALID, "da_set_owned: n_owned outside [1, n_cells]");
    ctx->mesh.n_owned = n_owned;
    return DA_OK;
}

int da_get_stream(da_ctx *ctx, void **stream) {
    if (!ctx || !stream) return DA_ERR_INVALID;
    *stream = (void *)ctx->stream;
    return DA_OK;
}

int da_step_bounds(da_ctx *ctx, double *bounds) {
    if (!ctx || !bounds) return DA_ERR_INVALID;
    int st = check_ctx(ctx, "da_step_bounds");
    if (st) return st;
    cudaSetDevice(ctx->device);
    if (is_device_pointer(bounds, ctx->device)) return launch_half(ctx, 0, bounds);
    // host pointer: through a device pair of the context, then wait for it
    st = bounds_alloc(ctx);
    if (!st) st = launch_half(ctx, 0, ctx->dd_bounds);
    if (!st) st = copy_d2h(ctx, bounds, ctx->dd_bounds, 2 * sizeof(double), "bounds");
    if (!st) st = read_scalars(ctx, "da_step_bounds");
    return st;
}

int da_step_apply(da_ctx *ctx, const double *bounds, da_step_stats *stats) {
    if (!ctx || !bounds) return DA_ERR_INVALID;
    int st = check_ctx(ctx, "da_step_apply");
    if (st) return st;
    cudaSetDevice(ctx->device);
    double *dev = const_cast<double *>(bounds);
    if (!is_device_pointer(bounds, ctx->device)) {
        st = bounds_alloc(ctx);
        if (st) return st;
        dev = ctx->dd_bounds;
        st = copy_h2d(ctx, dev, bounds, 2 * sizeof(double), "bounds");
        if (st) return st;
    }
    st = launch_half(ctx, 1, dev);
    if (!st && stats) {
        st = launch_volume(ctx);
        if (!st) st = read_scalars(ctx, "da_step_apply");
        stats->dt = ctx->hsc->dt;
        stats->time = ctx->hsc->time;
        stats->volume = ctx->hsc->volume;
        stats->hmax = ctx->hsc->hmax;
        stats->iter = ctx->hsc->iter;
    }
    return st;
}

int da_halo_pack(da_ctx *ctx, const int32_t *cells, int32_t n, void *buf) {
    if (!ctx || n < 0 || (n > 0 && (!cells || !buf))) return DA_ERR_INVALID;
    int st = check_ctx(ctx, "da_halo_pack");
    if (st || n == 0) return st;
    cudaSetDevice(ctx->device);
    if (!is_device_pointer(cells, ctx->device) || !is_device_pointer(buf, ctx->device))
        return set_error(ctx, DA_ERR_INVALID, "da_halo_pack: cells and buf must be device memory of the context's GPU");
    const int c = ctx->cur, g = halo_grid(ctx, n), no = ctx->mesh.n_owned;
    if (ctx->p.precision == DA_PREC_FP64)
        k_halo_pack<double><<<g, kBlock, 0, ctx->stream>>>((const double *)ctx->U[c][0], (const double *)ctx->U[c][1],
                                                           (const double *)ctx->U[c][2], no, cells, n, (double *)buf,
                                                           ctx->dsc);
    else
        k_halo_pack<float><<<g, kBlock, 0, ctx->stream>>>((const float *)ctx->U[c][0], (const float *)ctx->U[c][1],
                                                          (const float *)ctx->U[c][2], no, cells, n, (float *)buf,
                                                          ctx->dsc);
    return cuda_check(ctx, cudaGetLastError(), "halo pack launch");
}

int da_halo_unpack(da_ctx *ctx, const int32_t *cells, int32_t n, const void *buf) {
    if (!ctx || n < 0 || (n > 0 && (!cells || !buf))) return DA_ERR_INVALID;
    int st = check_ctx(ctx, "da_halo_unpack");
    if (st || n == 0) return st;
    cudaSetDevice(ctx->device);
    if (!is_device_pointer(cells, ctx->device) || !is_device_pointer(buf, ctx->device))
        return set_error(ctx, DA_ERR_INVALID, "da_halo_unpack: cells and buf must be device memory of the context's GPU");
    const int c = ctx->cur, g = halo_grid(ctx, n), no = ctx->mesh.n_owned, nc = ctx->mesh.n;
    if (ctx->p.precision == DA_PREC_FP64)
        k_halo_unpack<double><<<g, kBlock, 0, ctx->stream>>>((double *)ctx->U[c][0], (double *)ctx->U[c][1],
                                                             (double *)ctx->U[c][2], no, nc, cells, n,
                                                             (const double *)buf, ctx->seg_clean, ctx->seg_wet,
                                                             ctx->seg_dirty, ctx->dsc);
    else
        k_halo_unpack<float><<<g, kBlock, 0, ctx->stream>>>((float *)ctx->U[c][0], (float *)ctx->U[c][1],
                                                            (float *)ctx->U[c][2], no, nc, cells, n,
                                                            (const float *)buf, ctx->seg_clean, ctx->seg_wet,
                                                            ctx->seg_dirty, ctx->dsc);
    return cuda_check(ctx, cudaGetLastError(), "halo unpack launch");
}

int da_sync(da_ctx *ctx) {
    if (!ctx) return DA_ERR_INVALID;
    cudaSetDevice(ctx->device);
    return read_scalars(ctx, "da_sync");
}

}  // extern "C"
