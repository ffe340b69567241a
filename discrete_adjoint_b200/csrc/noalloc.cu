// da_forward_step_noalloc: one FP64 step() for callers that cannot allocate device memory.
//
// Some hosts hand this library only device buffers they already own: a plugin inside an
// application whose allocator owns the whole GPU, or a real-time loop in which allocating is not
// allowed.  Such a caller passes the flattened mesh, the state in and the state out as device
// pointers; every temporary the step needs (k act/pass, the active-cell bitmask, tile flags, the
// volume partials and the step scalars) lives in the fixed array below, which each GPU that
// loads the library holds until the process exits.  Nothing here calls cudaMalloc, cudaFree or
// an allocating library routine.
//
// Built without FMA contraction, like the other FP64 kernels: the result is bit-identical to
// da_forward_step on a context.
#include <cuda_runtime.h>

#include <mutex>

#include "forward_impl.cuh"

namespace da {
namespace noalloc {

constexpr size_t kMaxCells = DA_NOALLOC_MAX_CELLS;
constexpr size_t kMaxTiles = (kMaxCells + fwd::kBlock - 1) / fwd::kBlock;
constexpr size_t kMaxGrid = 1024;
constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr size_t kOffKact = 0;
constexpr size_t kOffActive = align256(kOffKact + kMaxCells * sizeof(double));
constexpr size_t kOffBflag = align256(kOffActive + (kMaxCells / 32) * sizeof(unsigned));
constexpr size_t kOffMat = align256(kOffBflag + kMaxCells);
constexpr size_t kMaxSegs = kMaxTiles * (fwd::kBlock / 32);
constexpr size_t kOffClean = align256(kOffMat + kMaxCells);
constexpr size_t kOffSegWet = align256(kOffClean + kMaxSegs);
constexpr size_t kOffSegVol = align256(kOffSegWet + kMaxSegs);
constexpr size_t kOffSegDirty = align256(kOffSegVol + kMaxSegs * sizeof(double));
constexpr size_t kOffVolParts = align256(kOffSegDirty + kMaxSegs);
constexpr size_t kOffScalars = align256(kOffVolParts + fwd::kVolParts * sizeof(double));
constexpr size_t kScratchBytes = align256(kOffScalars + sizeof(DevScalars));

// The scratch of every call.  Host code must not take this name as a device address: the
// address is obtained per device with cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// Per-device set-up: the device address of g_scratch, resolved once with that device current.
std::mutex g_lock;
unsigned char *g_addr[64] = {nullptr};

int scratch_for_current_device(unsigned char **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DA_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> guard(g_lock);
    if (!g_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_scratch) != cudaSuccess || !p) return DA_ERR_CUDA;
        g_addr[dev] = (unsigned char *)p;
    }
    *out = g_addr[dev];
    return DA_OK;
}

__global__ void k_init(DevScalars *sc, double time, long long iter) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    sc->time = time;
    sc->dt = 0.0;
    sc->hmax = 0.0;
    sc->min_dxe = 0.0;
    sc->volume = 0.0;
    sc->frict_tiny = 0.0;
    sc->iter = iter;
    sc->acc_min_dxe = __double_as_longlong(10000000.0);  // get_coef_and_eigen.C:36
    sc->acc_hmax = 0ull;
    sc->err = 0;
    sc->blocks_done[0] = sc->blocks_done[1] = 0u;
    sc->listed = 0;
    sc->acc_alt_min_dxe = __double_as_longlong(10000000.0);
    sc->acc_alt_hmax = 0ull;
    sc->bar = 0ull;
    sc->bar_exit = 0ull;
}

// Boundary / two-neighbour flags and byte materials from the caller's tables; an index out of
// range flags DA_ERR_INVALID and the step is not run.
__global__ void k_prep(int n, const int32_t *__restrict__ nbr, const int32_t *__restrict__ material, int n_mat,
                       uint8_t *__restrict__ bflag, uint8_t *__restrict__ mat8, DevScalars *sc) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint8_t b = 0;
        bool ok = true;
        for (int s = 0; s < 4; ++s) {
            const int a = nbr[(size_t)s * n + i], c = nbr[(size_t)(s + 4) * n + i];
            if (a == -1 && c == -1) b |= uint8_t(1u << s);
            else if (a < 0 || a >= n || c < 0 || c >= n) ok = false;
            else if (c != a) b |= uint8_t(0x10u << s);
        }
        const int m = material[i];
        if (m < 0 || m >= n_mat) ok = false;
        bflag[i] = b;
        mat8[i] = ok ? uint8_t(m) : 0;
        if (!ok) atomicCAS(&sc->err, 0, DA_ERR_INVALID);
    }
}

}  // namespace noalloc
}  // namespace da

using namespace da;

extern "C" int da_forward_step_noalloc(const da_params *p, const da_mesh_soa *mesh, const double *h, const double *hu,
                                       const double *hv, double *h_out, double *hu_out, double *hv_out, double time,
                                       int64_t iter, void *stream, da_step_stats *out) {
    if (!p || !mesh || !h || !hu || !hv || !h_out || !hu_out || !hv_out) return DA_ERR_INVALID;
    if (p->precision != DA_PREC_FP64) return DA_ERR_UNSUPPORTED;
    if (p->n_materials < 1 || p->n_materials > DA_MAX_MATERIALS) return DA_ERR_INVALID;
    if (mesh->n_cells <= 0) return DA_ERR_INVALID;
    if ((size_t)mesh->n_cells > noalloc::kMaxCells) return DA_ERR_UNSUPPORTED;  // beyond the fixed scratch
    if (!mesh->nbr || !mesh->x || !mesh->y || !mesh->dx || !mesh->dy || !mesh->gravity || !mesh->d_gravity ||
        !mesh->curvature || !mesh->material)
        return DA_ERR_INVALID;
    unsigned char *base = nullptr;
    int st = noalloc::scratch_for_current_device(&base);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int n = mesh->n_cells;
    const int ntiles = (n + fwd::kBlock - 1) / fwd::kBlock;
    int sms = 148;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int grid = sms * 4;
    if (grid > (int)noalloc::kMaxGrid) grid = (int)noalloc::kMaxGrid;
    if (grid > ntiles) grid = ntiles;

    double *kact = (double *)(base + noalloc::kOffKact);
    unsigned *active = (unsigned *)(base + noalloc::kOffActive);
    uint8_t *bflag = base + noalloc::kOffBflag;
    uint8_t *mat8 = base + noalloc::kOffMat;
    uint8_t *seg_clean = base + noalloc::kOffClean;
    uint8_t *seg_wet = base + noalloc::kOffSegWet;
    double *seg_vol = (double *)(base + noalloc::kOffSegVol);
    double *vol_parts = (double *)(base + noalloc::kOffVolParts);
    uint8_t *seg_dirty = base + noalloc::kOffSegDirty;
    DevScalars *sc = (DevScalars *)(base + noalloc::kOffScalars);

    MatConsts mc{};
    TimeConsts tc{};  // no frozen time-step sequence
    fill_consts(*p, &mc, &tc);

    // the array keeps the previous call's contents: zero the active bitmask, reset the scalars
    noalloc::k_init<<<1, 32, 0, s>>>(sc, time, (long long)iter);
    if (cudaMemsetAsync(active, 0, sizeof(unsigned) * (size_t)ntiles * (fwd::kBlock / 32), s) != cudaSuccess)
        return DA_ERR_CUDA;
    noalloc::k_prep<<<grid, fwd::kBlock, 0, s>>>(n, mesh->nbr, mesh->material, p->n_materials, bflag, mat8, sc);
    if (cudaGetLastError() != cudaSuccess) return DA_ERR_CUDA;
    DevScalars hs;
    if (cudaMemcpyAsync(&hs, sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s) != cudaSuccess) return DA_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return DA_ERR_CUDA;
    if (hs.err) return hs.err;

    fv::MeshArgs m;
    m.n = n;
    m.n_owned = n;
    m.nbr = mesh->nbr;
    m.mat = mat8;
    m.bflag = bflag;
    m.x = mesh->x;
    m.y = mesh->y;
    m.dx = mesh->dx;
    m.dy = mesh->dy;
    m.g = mesh->gravity;
    m.dg = mesh->d_gravity;
    m.curv = mesh->curvature;
    m.fdx = m.fdy = m.fg = m.fdg = m.fcurv = nullptr;
    fv::StateRef<double> U{h, hu, hv};
    fv::StateOut<double> O{h_out, hu_out, hv_out};
    // every tile is processed (no culling across independent calls)
    fwd::k_coef<double><<<grid, fwd::kBlock, 0, s>>>(m, U, kact, active, seg_wet, ntiles, 0, mc, tc, sc);
    fwd::k_update<double><<<grid, fwd::kBlock, 0, s>>>(m, U, O, kact, active, seg_clean, seg_wet, seg_vol, seg_dirty,
                                                       ntiles, 0, mc, sc);
    fwd::k_volume_parts<<<fwd::kVolParts, fwd::kBlock, 0, s>>>(seg_vol, ntiles * (fwd::kBlock / 32), vol_parts);
    fwd::k_volume_final<<<1, fwd::kVolParts, 0, s>>>(vol_parts, sc);
    if (cudaGetLastError() != cudaSuccess) return DA_ERR_CUDA;
    if (cudaMemcpyAsync(&hs, sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, s) != cudaSuccess) return DA_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return DA_ERR_CUDA;
    if (out) {
        out->dt = hs.dt;
        out->time = hs.time;
        out->volume = hs.volume;
        out->hmax = hs.hmax;
        out->iter = hs.iter;
    }
    return hs.err ? hs.err : DA_OK;
}
