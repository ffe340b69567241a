// C ABI entry points: context lifecycle, mesh/state transfer and forward stepping.
// Declared in include/discrete_adjoint.h; each replaces a reference call site named there.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <new>
#include <vector>

#include "da_internal.h"

namespace da {

int set_error(da_ctx *ctx, int code, const std::string &msg) {
    if (ctx) ctx->err = msg;
    return code;
}

void trace_begin(da_ctx *ctx, int kind) {
    TraceState &t = ctx->trace;
    if (!t.on) return;
    TraceState::Pending p{kind, 1, nullptr, nullptr};
    for (cudaEvent_t *e : {&p.a, &p.b}) {
        if (!t.pool.empty()) {
            *e = t.pool.back();
            t.pool.pop_back();
        } else if (cudaEventCreate(e) != cudaSuccess) {
            *e = nullptr;
        }
    }
    if (p.a) cudaEventRecord(p.a, ctx->stream);
    t.pending.push_back(p);
}

void trace_end(da_ctx *ctx, int steps) {
    TraceState &t = ctx->trace;
    if (!t.on || t.pending.empty()) return;
    t.pending.back().steps = steps;
    if (t.pending.back().b) cudaEventRecord(t.pending.back().b, ctx->stream);
}

int trace_flush(da_ctx *ctx) {
    TraceState &t = ctx->trace;
    if (t.pending.empty()) return DA_OK;
    int st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "trace sync");
    for (auto &p : t.pending) {
        float ms = 0.f;
        if (!st && p.a && p.b && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            t.total_ms[p.kind] += ms;
            t.launches[p.kind] += 1;
            t.steps[p.kind] += p.steps;
        }
        if (p.a) t.pool.push_back(p.a);
        if (p.b) t.pool.push_back(p.b);
    }
    t.pending.clear();
    return st;
}

int cuda_check(da_ctx *ctx, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return DA_OK;
    const int code = (e == cudaErrorMemoryAllocation) ? DA_ERR_OOM : DA_ERR_CUDA;
    return set_error(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

// gmfggetcoef (src/geoflow/getcoef.f:19-66) depends on the state only through sgn(vel)
// and two guards; the three signed values are formed here once per material.
static double coef_signed(double bedfrict, double intfrict, double s) {
    const double cosphi = std::cos(intfrict);
    const double tandel = std::tan(bedfrict);
    const double ab = 1.0 - (1.0 + tandel * tandel) * (cosphi * cosphi);
    return (2.0 / (cosphi * cosphi)) * (1.0 - s * std::sqrt(ab < 0. ? -ab : ab)) - 1.0;
}

void fill_consts(const da_params &p, MatConsts *mc, TimeConsts *tc) {
    std::memset(mc, 0, sizeof(*mc));
    for (int m = 0; m < p.n_materials; ++m) {
        for (int s = -1; s <= 1; ++s) {
            double k = coef_signed(p.bedfrict[m], p.intfrict, double(s));
            if (k < 0.0) k = 0.0;
            mc->kact_sgn[m][s + 1] = k * p.epsilon;
        }
        mc->tan_bed[m] = std::tan(p.bedfrict[m]);
    }
    mc->kact_rest = 1.0 * p.epsilon;
    mc->epsilon = p.epsilon;
    mc->sin_int = std::sin(p.intfrict);
    mc->gamma = p.gamma;
    mc->sign_floor = p.precision == DA_PREC_FP32_SPLIT ? p.fp32_sign_floor : 0.0;
    mc->n_materials = p.n_materials;
    tc->next_output = p.next_output;
    tc->next_save = p.next_save;
    tc->max_time = p.max_time;
    tc->influx_dt = p.influx_dt;
    tc->gravity_scale = p.gravity_scale;
    tc->epsilon = p.epsilon;
    tc->frict_tiny_early = p.frict_tiny_early;
    tc->frict_tiny_late = p.frict_tiny_late;
    tc->frict_tiny_iters = p.frict_tiny_iters;
}

static bool params_ok(const da_params *p) {
    if (!p) return false;
    if (p->precision != DA_PREC_FP64 && p->precision != DA_PREC_FP32_SPLIT) return false;
    if (p->n_materials < 1 || p->n_materials > DA_MAX_MATERIALS) return false;
    if (!(p->epsilon > 0) || !(p->gravity_scale > 0) || !(p->gamma > 0)) return false;
    if (p->grid_blocks < 0 || p->grid_blocks > (1 << 20)) return false;
    if (p->blocks_per_sm != 0 && p->blocks_per_sm != 2 && p->blocks_per_sm != 3) return false;
    if (p->tile_staging < 0 || p->tile_staging > 3) return false;
    if (p->jacobian_mode != DA_JAC_EXACT && p->jacobian_mode != DA_JAC_REFERENCE) return false;
    return true;
}

template <class T>
static void dfree(T *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}

static void free_mesh(da_ctx *ctx) {
    DevMesh &d = ctx->mesh;
    dfree(d.nbr); dfree(d.mat); dfree(d.bflag);
    dfree(d.x); dfree(d.y); dfree(d.dx); dfree(d.dy);
    dfree(d.g); dfree(d.dg); dfree(d.curv);
    dfree(d.fdx); dfree(d.fdy); dfree(d.fg); dfree(d.fdg); dfree(d.fcurv);
    dfree(d.halo_off); dfree(d.halo_idx); dfree(d.nloc);
    d.halo_max = 0;
    d.n = 0;
    d.n_owned = 0;
    d.epoch = -1;
}

static void free_state(da_ctx *ctx) {
    for (int b = 0; b < 2; ++b)
        for (int v = 0; v < 3; ++v) dfree(ctx->U[b][v]);
    dfree(ctx->kact);
    dfree(ctx->slopes);
    dfree(ctx->seg_vol);
    dfree(ctx->vol_parts);
    dfree(ctx->active);
    dfree(ctx->seg_clean);
    dfree(ctx->seg_wet);
    dfree(ctx->seg_dirty);
    dfree(ctx->stage);
    dfree(ctx->dd_bounds);
    dfree(ctx->tile_epoch);
    dfree(ctx->seg_act);
    dfree(ctx->lam_clean);
    ctx->have_state = false;
}

static void free_adjoint(da_ctx *ctx) {
    auto fr = [](void *p) { if (p) cudaFree(p); };
    fr(ctx->mask); fr(ctx->adjA); fr(ctx->adjB); fr(ctx->gbed); fr(ctx->gint); fr(ctx->dk_tab);
    fr(ctx->red_out); fr(ctx->red_part); fr(ctx->inst_J); fr(ctx->seg_J); fr(ctx->dh0);
    for (int b = 0; b < 2; ++b)
        for (int v = 0; v < 3; ++v) { fr(ctx->lam[b][v]); ctx->lam[b][v] = nullptr; }
    for (void *s : ctx->snaps) fr(s);
    ctx->snaps.clear();
    if (ctx->sweep_graph) cudaGraphExecDestroy(ctx->sweep_graph);
    ctx->sweep_graph = nullptr;
    ctx->sweep_key.clear();
    ctx->mask = nullptr; ctx->adjA = ctx->adjB = ctx->gbed = ctx->gint = ctx->dk_tab = nullptr;
    ctx->red_out = ctx->red_part = ctx->inst_J = ctx->seg_J = ctx->dh0 = nullptr;
    ctx->dh0_bytes = 0;
    fr(ctx->refadj_mem);
    ctx->refadj_mem = nullptr;
    ctx->refadj_n = 0;
    ctx->adj_n = 0;
    ctx->adj_ninst = -1;
}

static void drop_graphs(da_ctx *ctx) {
    for (int b = 0; b < 2; ++b) {
        if (ctx->step_graph[b]) cudaGraphExecDestroy(ctx->step_graph[b]);
        ctx->step_graph[b] = nullptr;
    }
}

template <class T>
static int upload(da_ctx *ctx, T **dst, const T *src, size_t count) {
    int st = cuda_check(ctx, cudaMalloc((void **)dst, sizeof(T) * (count ? count : 1)), "cudaMalloc(mesh)");
    if (st) return st;
    return cuda_check(ctx, cudaMemcpyAsync(*dst, src, sizeof(T) * count, cudaMemcpyHostToDevice, ctx->stream),
                      "copy mesh");
}

// Halo tables of the staged step phases.  For tile t (cells 256 t ... 256 t + 255): its halo, the
// cells outside the tile that its cells name as neighbours (sorted, each once), at
// idx[off[t] .. off[t+1]); for every cell its eight neighbour entries as tile-local slots in
// nloc[i][s]: 0..255 a cell of the same tile, 256 + k the tile's k-th halo cell, -1 no neighbour.
// Built on the host once per mesh; not uploaded when a tile's halo exceeds kHaloMax (the step
// kernels then read neighbours from global memory).
static int build_halo(da_ctx *ctx, const int32_t *nbr, int n) {
    const int nt = (n + kTileCells - 1) / kTileCells;
    std::vector<int32_t> off((size_t)nt + 1), idx, h;
    std::vector<int16_t> nloc((size_t)8 * n);
    idx.reserve((size_t)nt * 96);
    int hmax = 0;
    for (int t = 0; t < nt; ++t) {
        const int a = t * kTileCells, b = std::min(n, a + kTileCells);
        h.clear();
        for (int s = 0; s < 8; ++s)
            for (int i = a; i < b; ++i) {
                const int e = nbr[(size_t)s * n + i];
                if (e >= 0 && (e < a || e >= b)) h.push_back(e);
            }
        std::sort(h.begin(), h.end());
        h.erase(std::unique(h.begin(), h.end()), h.end());
        off[t] = (int32_t)idx.size();
        idx.insert(idx.end(), h.begin(), h.end());
        hmax = std::max(hmax, (int)h.size());
        for (int i = a; i < b; ++i)
            for (int s = 0; s < 8; ++s) {
                const int e = nbr[(size_t)s * n + i];
                int slot = -1;
                if (e >= a && e < b)
                    slot = e - a;
                else if (e >= 0)
                    slot = kTileCells + int(std::lower_bound(h.begin(), h.end(), e) - h.begin());
                nloc[(size_t)i * 8 + s] = (int16_t)slot;
            }
    }
    off[nt] = (int32_t)idx.size();
    DevMesh &d = ctx->mesh;
    d.halo_max = hmax;
    if (hmax > kHaloMax) return DA_OK;
    int st = upload(ctx, &d.halo_off, off.data(), off.size());
    if (!st) st = upload(ctx, &d.halo_idx, idx.data(), idx.size());
    if (!st) st = upload(ctx, &d.nloc, nloc.data(), nloc.size());
    // the host vectors are released on return: the copies must have left them
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    return st;
}

int device_error(da_ctx *ctx, const char *where) {
    const int code = ctx->hsc->err;
    if (!code) return DA_OK;
    if (code == DA_ERR_TIMEOUT) {
        // a cooperative launch gave up at a grid barrier and every block has returned: the next
        // launch starts from a barrier word with no arrivals and generation 0
        cudaMemsetAsync(&ctx->dsc->bar, 0, 2 * sizeof(unsigned long long), ctx->stream);  // bar, bar_exit
        cudaStreamSynchronize(ctx->stream);
    }
    return set_error(ctx, code, std::string(where) + ": " + da_strerror(code));
}

static int sync_scalars(da_ctx *ctx) {
    int st = cuda_check(ctx, cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream),
                        "read scalars");
    if (st) return st;
    st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "stream sync");
    if (st) return st;
    return device_error(ctx, "forward step");
}

void update_grid(da_ctx *ctx) {
    const int per_sm4 = (ctx->sm_count > 0 ? ctx->sm_count : 148) * 4;
    int g = ctx->p.grid_blocks > 0 ? ctx->p.grid_blocks : per_sm4;
    if (ctx->ntiles > 0 && g > ctx->ntiles) g = ctx->ntiles;
    ctx->grid = g > 0 ? g : 1;
}

// FP64 host arrays <-> FP32 device arrays through the FP64 staging buffer: the copy is one DMA
// of the caller's array (fast from pinned memory) and the rounding (to nearest) runs on the device.
__global__ void k_narrow(const double *__restrict__ s, float *__restrict__ d, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = float(s[i]);
}
__global__ void k_widen(const float *__restrict__ s, double *__restrict__ d, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = double(s[i]);
}

static int stage_alloc(da_ctx *ctx) {
    if (ctx->stage) return DA_OK;
    return cuda_check(ctx, cudaMalloc((void **)&ctx->stage, sizeof(double) * (size_t)ctx->mesh.n), "cudaMalloc(stage)");
}

int upload_real(da_ctx *ctx, void *dev, const double *host) {
    const int n = ctx->mesh.n;
    if (ctx->p.precision == DA_PREC_FP64)
        return cuda_check(ctx, cudaMemcpyAsync(dev, host, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream),
                          "copy to device");
    int st = stage_alloc(ctx);
    if (!st) st = cuda_check(ctx, cudaMemcpyAsync(ctx->stage, host, sizeof(double) * n, cudaMemcpyHostToDevice,
                                                  ctx->stream), "copy to device");
    if (!st) k_narrow<<<ctx->sm_count * 4, 256, 0, ctx->stream>>>(ctx->stage, (float *)dev, n);
    return st ? st : cuda_check(ctx, cudaGetLastError(), "narrow");
}

int copy_h2d(da_ctx *ctx, void *dev, const void *host, size_t bytes, const char *what) {
    return cuda_check(ctx, cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, ctx->stream), what);
}

int copy_d2h(da_ctx *ctx, void *host, const void *dev, size_t bytes, const char *what) {
    int st = cuda_check(ctx, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream), what);
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), what);
    return st;
}

int download_real(da_ctx *ctx, double *host, const void *dev) {
    const int n = ctx->mesh.n;
    if (ctx->p.precision == DA_PREC_FP64)
        return cuda_check(ctx, cudaMemcpyAsync(host, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream),
                          "copy to host");
    int st = stage_alloc(ctx);
    if (!st) k_widen<<<ctx->sm_count * 4, 256, 0, ctx->stream>>>((const float *)dev, ctx->stage, n);
    if (!st) st = cuda_check(ctx, cudaGetLastError(), "widen");
    if (!st) st = cuda_check(ctx, cudaMemcpyAsync(host, ctx->stage, sizeof(double) * n, cudaMemcpyDeviceToHost,
                                                  ctx->stream), "copy to host");
    return st;
}

static void fill_stats(const da_ctx *ctx, da_step_stats *out) {
    if (!out) return;
    out->dt = ctx->hsc->dt;
    out->time = ctx->hsc->time;
    out->volume = ctx->hsc->volume;
    out->hmax = ctx->hsc->hmax;
    out->iter = ctx->hsc->iter;
}

}  // namespace da

using namespace da;

extern "C" {

int da_abi_version(void) { return DA_ABI_VERSION; }

const char *da_strerror(int code) {
    switch (code) {
        case DA_OK: return "ok";
        case DA_ERR_INVALID: return "invalid argument or call order";
        case DA_ERR_CUDA: return "CUDA runtime error";
        case DA_ERR_NAN: return "non-finite state or time step";
        case DA_ERR_NEG_DEPTH: return "negative depth";
        case DA_ERR_EIGEN: return "wave speed above 1e9";
        case DA_ERR_TIMEOUT: return "device wait timed out";
        case DA_ERR_NO_MESH: return "no mesh uploaded";
        case DA_ERR_OOM: return "device out of memory";
        case DA_ERR_NO_DEVICE: return "no CUDA device";
        case DA_ERR_UNSUPPORTED: return "unsupported";
        case DA_ERR_IO: return "file could not be opened, read or written";
        default: return "unknown error";
    }
}

void da_params_default(da_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->precision = DA_PREC_FP64;
    p->device = 0;
    p->epsilon = 1.0;
    p->gravity_scale = 1.0;
    p->gamma = 1.0;
    p->intfrict = 30.0 * 3.1415926 / 180.0;  // constant.h:37 PI, datread.C:379-400 deg->rad
    p->n_materials = 1;
    p->bedfrict[0] = 20.0 * 3.1415926 / 180.0;
    p->frict_tiny_iters = 50;
    p->frict_tiny_early = 0.1;
    p->frict_tiny_late = 0.000000001;
    p->max_time = HUGE_VAL;
    p->next_output = HUGE_VAL;
    p->next_save = HUGE_VAL;
    p->influx_dt = HUGE_VAL;
    p->fp32_sign_floor = 0.0;
    p->tile_culling = 1;
    p->grid_blocks = 0;
    p->blocks_per_sm = 0;
    p->tile_staging = 1;
    p->jacobian_mode = DA_JAC_EXACT;
}

da_ctx *da_create(const da_params *p, int *err) {
    int dummy;
    if (!err) err = &dummy;
    if (!params_ok(p)) {
        *err = DA_ERR_INVALID;
        return nullptr;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        *err = DA_ERR_NO_DEVICE;
        return nullptr;
    }
    if (p->device < 0 || p->device >= ndev) {
        *err = DA_ERR_INVALID;
        return nullptr;
    }
    da_ctx *ctx = new (std::nothrow) da_ctx();
    if (!ctx) {
        *err = DA_ERR_OOM;
        return nullptr;
    }
    ctx->p = *p;
    ctx->device = p->device;
    fill_consts(ctx->p, &ctx->mc, &ctx->tc);
    int st = cuda_check(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    if (!st) st = cuda_check(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
    if (!st) st = cuda_check(ctx, cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device),
                             "device attribute");
    if (!st) st = cuda_check(ctx, cudaMalloc((void **)&ctx->dsc, sizeof(DevScalars)), "cudaMalloc(scalars)");
    if (!st) st = cuda_check(ctx, cudaMallocHost((void **)&ctx->hsc, sizeof(DevScalars)), "cudaMallocHost");
    if (st) {
        *err = st;
        da_destroy(ctx);
        return nullptr;
    }
    std::memset(ctx->hsc, 0, sizeof(DevScalars));
    {
        const double init = 10000000.0;  // min_dx_dy_evalue start value, get_coef_and_eigen.C:36
        std::memcpy(&ctx->hsc->acc_min_dxe, &init, sizeof(init));
        std::memcpy(&ctx->hsc->acc_alt_min_dxe, &init, sizeof(init));
    }
    st = copy_h2d(ctx, ctx->dsc, ctx->hsc, sizeof(DevScalars), "init scalars");
    if (st) {
        *err = st;
        da_destroy(ctx);
        return nullptr;
    }
    *err = DA_OK;
    return ctx;
}

void da_destroy(da_ctx *ctx) {
    if (ctx) {
        free_members(ctx);
        dwr_release(ctx);
        if (ctx->outline.map) cudaFree(ctx->outline.map);
        ctx->outline = OutlineGrid{};
    }
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drop_graphs(ctx);
    free_mesh(ctx);
    free_state(ctx);
    free_adjoint(ctx);
    trace_flush(ctx);
    for (cudaEvent_t e : ctx->trace.pool) cudaEventDestroy(e);
    if (ctx->dt_replay) cudaFree(ctx->dt_replay);
    if (ctx->dsc) cudaFree(ctx->dsc);
    if (ctx->hsc) cudaFreeHost(ctx->hsc);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char *da_last_error(const da_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int da_selftest_barrier(da_ctx *ctx, int32_t limit_us) {
    if (!ctx || limit_us <= 0 || limit_us > 4000000) return DA_ERR_INVALID;
    cudaSetDevice(ctx->device);
    int st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (!st) st = launch_barrier_selftest(ctx, 1000ull * (unsigned long long)limit_us);
    if (st) return st;
    st = cuda_check(ctx, cudaMemcpyAsync(ctx->hsc, ctx->dsc, sizeof(DevScalars), cudaMemcpyDeviceToHost, ctx->stream),
                    "read scalars");
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (st) return st;
    const int code = device_error(ctx, "barrier self-test");
    // the context stays usable: the error the test provoked is cleared
    ctx->hsc->err = 0;
    const int st2 = cuda_check(ctx, cudaMemsetAsync(&ctx->dsc->err, 0, sizeof(int), ctx->stream), "memset");
    const int st3 = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    return st2 ? st2 : (st3 ? st3 : code);
}

int da_set_params(da_ctx *ctx, const da_params *p) {
    if (!ctx) return DA_ERR_INVALID;
    if (!params_ok(p) || p->precision != ctx->p.precision || p->device != ctx->p.device ||
        (ctx->mesh.n > 0 && p->tile_culling != ctx->p.tile_culling))
        return set_error(ctx, DA_ERR_INVALID, "da_set_params: invalid parameters or precision/device change");
    ctx->p = *p;
    fill_consts(ctx->p, &ctx->mc, &ctx->tc);
    update_grid(ctx);
    drop_graphs(ctx);
    return DA_OK;
}

int da_set_time(da_ctx *ctx, double time, int64_t iter) {
    if (!ctx) return DA_ERR_INVALID;
    cudaSetDevice(ctx->device);
    int st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (st) return st;
    st = copy_d2h(ctx, ctx->hsc, ctx->dsc, sizeof(DevScalars), "read scalars");
    if (st) return st;
    ctx->hsc->time = time;
    ctx->hsc->iter = iter;
    // a cleared error restarts the grid barrier too (no kernel of the context is running)
    ctx->hsc->err = 0;
    ctx->hsc->bar = 0ull;
    ctx->hsc->bar_exit = 0ull;
    return copy_h2d(ctx, ctx->dsc, ctx->hsc, sizeof(DevScalars), "write scalars");
}

int da_upload_mesh(da_ctx *ctx, const da_mesh_soa *m, int32_t epoch) {
    if (!ctx) return DA_ERR_INVALID;
    if (!m || m->n_cells <= 0 || !m->nbr || !m->x || !m->y || !m->dx || !m->dy || !m->gravity || !m->d_gravity ||
        !m->curvature || !m->material)
        return set_error(ctx, DA_ERR_INVALID, "da_upload_mesh: missing array");
    const int n = m->n_cells;
    // host-side validation: neighbour indices in range, materials in range.  The flag and
    // material bytes are padded with zeros to whole tiles (the staged phases copy a tile's bytes in
    // 16-byte pieces).
    const size_t npad = ((size_t)n + kTileCells - 1) / kTileCells * kTileCells;
    std::vector<uint8_t> bflag(npad, 0), mat(npad, 0);
    for (int i = 0; i < n; ++i) {
        uint8_t b = 0;
        for (int s = 0; s < 4; ++s) {
            const int a = m->nbr[(size_t)s * n + i], c = m->nbr[(size_t)(s + 4) * n + i];
            if (a < -1 || a >= n || c < -1 || c >= n || ((a < 0) != (c < 0)))
                return set_error(ctx, DA_ERR_INVALID, "da_upload_mesh: neighbour index out of range");
            if (a < 0) b |= uint8_t(1u << s);
            else if (c != a) b |= uint8_t(0x10u << s);
        }
        bflag[i] = b;
        if (m->material[i] < 0 || m->material[i] >= ctx->p.n_materials)
            return set_error(ctx, DA_ERR_INVALID, "da_upload_mesh: material index out of range");
        mat[i] = uint8_t(m->material[i]);
        if (!(m->dx[i] > 0) || !(m->dy[i] > 0))
            return set_error(ctx, DA_ERR_INVALID, "da_upload_mesh: non-positive cell size");
    }
    cudaSetDevice(ctx->device);
    int st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (st) return st;
    drop_graphs(ctx);
    free_members(ctx);
    dwr_release(ctx);
    free_mesh(ctx);
    free_state(ctx);
    free_adjoint(ctx);
    DevMesh &d = ctx->mesh;
    d.n = n;
    d.n_owned = n;
    d.epoch = epoch;
    const bool fp64 = ctx->p.precision == DA_PREC_FP64;
    if (!st) st = upload(ctx, &d.nbr, m->nbr, (size_t)8 * n);
    if (!st) st = upload(ctx, &d.bflag, bflag.data(), npad);
    if (!st) st = upload(ctx, &d.mat, mat.data(), npad);
    if (!st) st = build_halo(ctx, m->nbr, n);
    // centres: the FP64 step uses them; both precisions test functional boxes with them
    if (!st) st = upload(ctx, &d.x, m->x, (size_t)n);
    if (!st) st = upload(ctx, &d.y, m->y, (size_t)n);
    if (fp64) {
        if (!st) st = upload(ctx, &d.dx, m->dx, (size_t)n);
        if (!st) st = upload(ctx, &d.dy, m->dy, (size_t)n);
        if (!st) st = upload(ctx, &d.g, m->gravity, (size_t)3 * n);
        if (!st) st = upload(ctx, &d.dg, m->d_gravity, (size_t)2 * n);
        if (!st) st = upload(ctx, &d.curv, m->curvature, (size_t)2 * n);
    } else {
        std::vector<float> tmp((size_t)3 * n);
        auto conv = [&](const double *src, size_t cnt, float **dst) {
            for (size_t k = 0; k < cnt; ++k) tmp[k] = float(src[k]);
            return upload(ctx, dst, tmp.data(), cnt);
        };
        if (!st) st = conv(m->dx, n, &d.fdx);
        if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
        if (!st) st = conv(m->dy, n, &d.fdy);
        if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
        if (!st) st = conv(m->gravity, (size_t)3 * n, &d.fg);
        if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
        if (!st) st = conv(m->d_gravity, (size_t)2 * n, &d.fdg);
        if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
        if (!st) st = conv(m->curvature, (size_t)2 * n, &d.fcurv);
    }
    if (!st) st = forward_alloc(ctx);
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (st) {
        free_mesh(ctx);
        free_state(ctx);
    }
    return st;
}

int da_set_state(da_ctx *ctx, const double *h, const double *hu, const double *hv) {
    if (!ctx || !h || !hu || !hv) return DA_ERR_INVALID;
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_set_state: no mesh");
    cudaSetDevice(ctx->device);
    const double *src[3] = {h, hu, hv};
    int st = DA_OK;
    for (int v = 0; v < 3 && !st; ++v) st = upload_real(ctx, ctx->U[ctx->cur][v], src[v]);
    if (!st) st = forward_state_changed(ctx);
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (!st) ctx->have_state = true;
    return st;
}

int da_get_state(da_ctx *ctx, double *h, double *hu, double *hv) {
    if (!ctx || !h || !hu || !hv) return DA_ERR_INVALID;
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_get_state: no state");
    cudaSetDevice(ctx->device);
    double *dst[3] = {h, hu, hv};
    int st = DA_OK;
    for (int v = 0; v < 3 && !st; ++v) {
        st = download_real(ctx, dst[v], ctx->U[ctx->cur][v]);
        // the staging buffer is reused by the next array
        if (!st && ctx->p.precision != DA_PREC_FP64) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    }
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    return st;
}

int da_forward_step(da_ctx *ctx, da_step_stats *out) {
    if (!ctx) return DA_ERR_INVALID;
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, "da_forward_step: ensemble context (da_ensemble_forward)");
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_forward_step: no mesh");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_forward_step: no state");
    cudaSetDevice(ctx->device);
    int st = launch_forward_step(ctx);
    if (!st) st = launch_volume(ctx);
    if (!st) st = sync_scalars(ctx);
    fill_stats(ctx, out);
    return st;
}

int da_forward_run(da_ctx *ctx, int32_t nsteps, da_step_stats *last) {
    return da_forward_run_timed(ctx, nsteps, last, nullptr);
}

int da_forward_run_timed(da_ctx *ctx, int32_t nsteps, da_step_stats *last, double *device_ms) {
    if (!ctx || nsteps < 0) return DA_ERR_INVALID;
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_forward_run: no mesh");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_forward_run: no state");
    cudaSetDevice(ctx->device);
    int st = DA_OK;
    // the whole run is one cooperative launch of the multi-step kernel
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (device_ms) {
        st = cuda_check(ctx, cudaEventCreate(&e0), "event");
        if (!st) st = cuda_check(ctx, cudaEventCreate(&e1), "event");
        if (!st) st = cuda_check(ctx, cudaEventRecord(e0, ctx->stream), "event record");
    }
    if (!st) st = launch_forward_steps(ctx, nsteps);
    if (device_ms && !st) {
        st = cuda_check(ctx, cudaEventRecord(e1, ctx->stream), "event record");
        if (!st) st = cuda_check(ctx, cudaEventSynchronize(e1), "event sync");
        float ms = 0.f;
        if (!st) st = cuda_check(ctx, cudaEventElapsedTime(&ms, e0, e1), "event time");
        *device_ms = ms;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (!st) st = launch_volume(ctx);
    if (!st) st = sync_scalars(ctx);
    fill_stats(ctx, last);
    return st;
}

const char *da_forward_kernel_name(int32_t k) {
    static const char *names[DA_FWD_KERNELS] = {"k_coef", "k_update"};
    return (k >= 0 && k < DA_FWD_KERNELS) ? names[k] : "";
}

int da_forward_profile(da_ctx *ctx, int32_t nsteps, double *kernel_ms) {
    if (!ctx || nsteps <= 0 || !kernel_ms) return DA_ERR_INVALID;
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, "da_forward_profile: ensemble context");
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_forward_profile: no mesh");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_forward_profile: no state");
    cudaSetDevice(ctx->device);
    TraceState &t = ctx->trace;
    const bool was_on = t.on;
    int st = trace_flush(ctx);
    double tot0[2] = {t.total_ms[TR_COEF], t.total_ms[TR_UPDATE]};
    long long n0[2] = {t.launches[TR_COEF], t.launches[TR_UPDATE]};
    t.on = true;
    for (int s = 0; s < nsteps && !st; ++s) st = launch_forward_step(ctx);
    if (!st) st = trace_flush(ctx);
    if (!st) st = launch_volume(ctx);
    t.on = was_on;
    if (!st) st = sync_scalars(ctx);
    const int kinds[2] = {TR_COEF, TR_UPDATE};
    for (int k = 0; k < DA_FWD_KERNELS; ++k) {
        const long long c = t.launches[kinds[k]] - n0[k];
        kernel_ms[k] = c > 0 ? (t.total_ms[kinds[k]] - tot0[k]) / c : 0.0;
    }
    return st;
}

static const char *kTraceNames[TR_COUNT] = {"k_coef",       "k_update",     "k_coef_record", "k_update_record",
                                            "k_adj_src",    "k_adj_gather", "k_adj_seed",    "k_adj_reduce",
                                            "snapshot_copy", "k_steps", "k_youturn"};

const char *da_trace_name(int32_t k) { return (k >= 0 && k < TR_COUNT) ? kTraceNames[k] : ""; }

int da_set_tracing(da_ctx *ctx, int32_t on) {
    if (!ctx) return DA_ERR_INVALID;
    cudaSetDevice(ctx->device);
    int st = trace_flush(ctx);
    for (int k = 0; k < TR_COUNT; ++k) {
        ctx->trace.total_ms[k] = 0.0;
        ctx->trace.launches[k] = 0;
        ctx->trace.steps[k] = 0;
    }
    ctx->trace.on = on != 0;
    return st;
}

int da_trace_read(da_ctx *ctx, int32_t k, double *total_ms, int64_t *launches) {
    if (!ctx || k < 0 || k >= TR_COUNT || !total_ms || !launches) return DA_ERR_INVALID;
    cudaSetDevice(ctx->device);
    int st = trace_flush(ctx);
    *total_ms = ctx->trace.total_ms[k];
    *launches = ctx->trace.launches[k];
    return st;
}

int da_trace_steps(da_ctx *ctx, int32_t k, int64_t *steps) {
    if (!ctx || k < 0 || k >= TR_COUNT || !steps) return DA_ERR_INVALID;
    cudaSetDevice(ctx->device);
    int st = trace_flush(ctx);
    *steps = ctx->trace.steps[k];
    return st;
}

}  // extern "C"

// ---------------------------------------------------------------------------- autotuner
// Times nsteps forward steps from the current state for each candidate launch shape (register
// budget of 2 or 3 resident blocks per SM x grids of half the SMs and of 1..budget blocks per SM)
// and keeps the fastest.  The state, time and iteration are put back after every trial, so the
// tuning leaves the run where it was.
int da_autotune(da_ctx *ctx, int32_t nsteps, da_tune_result *out) {
    using namespace da;
    if (!ctx || nsteps < 1) return DA_ERR_INVALID;
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_autotune: no mesh");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_autotune: no state");
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)ctx->mesh.n;
    const size_t rs = ctx->p.precision == DA_PREC_FP64 ? sizeof(double) : sizeof(float);
    int st = sync_scalars(ctx);
    if (st) return st;
    const DevScalars saved_sc = *ctx->hsc;
    const int cur0 = ctx->cur;
    // ensemble: the members' times too (their accumulators are at rest between steps)
    std::vector<double> saved_time(ctx->ninst);
    if (ctx->ninst > 0)
        st = copy_d2h(ctx, saved_time.data(), ctx->ia.time, sizeof(double) * ctx->ninst, "save times");
    void *saved[3] = {nullptr, nullptr, nullptr};
    for (int v = 0; v < 3 && !st; ++v) {
        st = cuda_check(ctx, cudaMalloc(&saved[v], rs * n), "cudaMalloc(autotune)");
        if (!st)
            st = cuda_check(ctx, cudaMemcpyAsync(saved[v], ctx->U[cur0][v], rs * n, cudaMemcpyDeviceToDevice, ctx->stream),
                            "save state");
    }
    auto put_back = [&]() -> int {
        ctx->cur = cur0;
        int s = DA_OK;
        for (int v = 0; v < 3 && !s; ++v)
            s = cuda_check(ctx, cudaMemcpyAsync(ctx->U[cur0][v], saved[v], rs * n, cudaMemcpyDeviceToDevice, ctx->stream),
                           "restore state");
        *ctx->hsc = saved_sc;
        if (!s) s = cuda_check(ctx, cudaMemcpyAsync(ctx->dsc, ctx->hsc, sizeof(DevScalars), cudaMemcpyHostToDevice,
                                                    ctx->stream), "restore scalars");
        if (!s && ctx->ninst > 0)
            s = cuda_check(ctx, cudaMemcpyAsync(ctx->ia.time, saved_time.data(), sizeof(double) * ctx->ninst,
                                                cudaMemcpyHostToDevice, ctx->stream), "restore times");
        if (!s) s = forward_state_changed(ctx);
        if (!s) s = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
        return s;
    };
    const int sm = ctx->sm_count > 0 ? ctx->sm_count : 148;
    // (blocks per SM of the register budget, grid): grids of half the SMs, then 1, 2, 3 blocks per
    // SM up to the budget (a sparse flow's few wet tiles can prefer fewer, cheaper barriers)
    int cand_occ[DA_TUNE_MAX], cand[DA_TUNE_MAX], nc = 0;
    for (int occ = 2; occ <= 3; ++occ)
        for (int halves = 1; halves <= 2 * occ; halves = halves == 1 ? 2 : halves + 2) {
            int g = halves * sm / 2;
            if (g > ctx->ntiles) g = ctx->ntiles;
            bool dup = false;
            for (int j = 0; j < nc; ++j) dup |= cand[j] == g && cand_occ[j] == occ;
            if (!dup && nc < DA_TUNE_MAX) {
                cand_occ[nc] = occ;
                cand[nc++] = g;
            }
        }
    const int32_t grid0 = ctx->p.grid_blocks, occ0 = ctx->p.blocks_per_sm;
    double best_ms = HUGE_VAL;
    int best = 0;
    da_tune_result r;
    std::memset(&r, 0, sizeof(r));
    for (int k = 0; k < nc && !st; ++k) {
        ctx->p.grid_blocks = cand[k];
        ctx->p.blocks_per_sm = cand_occ[k];
        update_grid(ctx);
        drop_graphs(ctx);
        // the least of three timings from the same state: a few short steps are noisy, and
        // neighbouring shapes differ by a few per cent
        double ms = HUGE_VAL;
        for (int rep = 0; rep < 3 && !st; ++rep) {
            st = put_back();
            if (!st) st = launch_forward_steps(ctx, 1);  // the first step after a state change sweeps every tile
            double t = 0.0;
            if (!st) st = da_forward_run_timed(ctx, nsteps, nullptr, &t);
            if (!st && t < ms) ms = t;
        }
        r.grid[k] = cand[k];
        r.blocks_per_sm[k] = cand_occ[k];
        r.ms_per_step[k] = ms / nsteps;
        if (!st && ms < best_ms) {
            best_ms = ms;
            best = k;
        }
    }
    r.n = nc;
    r.best = best;
    ctx->p.grid_blocks = st ? grid0 : cand[best];
    ctx->p.blocks_per_sm = st ? occ0 : cand_occ[best];
    update_grid(ctx);
    drop_graphs(ctx);
    const int st2 = put_back();
    for (int v = 0; v < 3; ++v)
        if (saved[v]) cudaFree(saved[v]);
    if (!st) st = st2;
    if (!st && out) *out = r;
    return st;
}

namespace da {
int launch_refine_info_fp64(da_ctx *, double *, uint8_t *, double *, double *);
int launch_refine_info_fp32(da_ctx *, double *, uint8_t *, double *, double *);
}  // namespace da

extern "C" int da_refine_info(da_ctx *ctx, double *el_error, uint8_t *flags, double *geo_target) {
    if (!ctx) return DA_ERR_INVALID;
    if (ctx->mesh.n <= 0) return set_error(ctx, DA_ERR_NO_MESH, "da_refine_info: no mesh");
    if (!ctx->have_state) return set_error(ctx, DA_ERR_INVALID, "da_refine_info: no state");
    if (ctx->ninst > 0) return set_error(ctx, DA_ERR_INVALID, "da_refine_info: ensemble context");
    cudaSetDevice(ctx->device);
    const size_t n = (size_t)ctx->mesh.n;
    unsigned char *mem = nullptr;
    const size_t o_flags = 8 * n, o_parts = (o_flags + n + 255) & ~size_t(255), o_t = o_parts + 8 * 2 * 256;
    int st = cuda_check(ctx, cudaMalloc((void **)&mem, o_t + 8), "cudaMalloc(refine)");
    if (!st) st = ctx->p.precision == DA_PREC_FP64
                      ? launch_refine_info_fp64(ctx, (double *)mem, mem + o_flags, (double *)(mem + o_parts), (double *)(mem + o_t))
                      : launch_refine_info_fp32(ctx, (double *)mem, mem + o_flags, (double *)(mem + o_parts), (double *)(mem + o_t));
    if (!st && el_error)
        st = cuda_check(ctx, cudaMemcpyAsync(el_error, mem, 8 * n, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    if (!st && flags) st = cuda_check(ctx, cudaMemcpyAsync(flags, mem + o_flags, n, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    if (!st && geo_target)
        st = cuda_check(ctx, cudaMemcpyAsync(geo_target, mem + o_t, 8, cudaMemcpyDeviceToHost, ctx->stream), "copy");
    if (!st) st = cuda_check(ctx, cudaStreamSynchronize(ctx->stream), "sync");
    if (mem) cudaFree(mem);
    return st;
}

