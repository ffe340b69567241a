// Internal declarations shared by the CUDA translation units of libda_b200.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "discrete_adjoint.h"

#define DA_TINY 1.e-4  // GEOFLOW_TINY, src/header/constant.h:68

namespace da {

constexpr int kTileCells = 256;  // cells per tile (Morton-consecutive): one thread each
constexpr int kHaloMax = 192;    // halo cells a staged tile holds in shared memory

// Per-material constants formed on the host once per parameter change (host libm, so the
// device never evaluates a transcendental and the FP64 path matches the CPU bit for bit).
//   kact_sgn[m][s+1]: gmfggetcoef's K_act/pass for sgn(vel) = s, clamped at 0, times epsilon
//   tan_bed[m]     : tan(bedfrict[m])             (residual.C:231)
struct MatConsts {
    double kact_sgn[DA_MAX_MATERIALS][3];
    double tan_bed[DA_MAX_MATERIALS];
    double kact_rest;     // 1 * epsilon: no yield or dry cell (getcoef.f:129-142)
    double epsilon;
    double sin_int;       // sin(intfrict)               (residual.C:227)
    double gamma;
    double sign_floor;    // FP32-split only: lower bound on frict_tiny in the friction sign tests
    int32_t n_materials;
};

// Scalars that live on the device so that whole step loops run without host round trips.
constexpr int kAdjReduceParts = 128;  // cell ranges of the gradient reduction

struct DevScalars {
    double time;          // TimeProps::time
    double dt;            // last dt
    double hmax;          // max h over wet cells (last coef pass)
    double min_dxe;       // min over wet cells of min(dx,dy)/evalue (last coef pass)
    double volume;        // sum dx*dy*h after the last update
    double frict_tiny;    // MatProps::frict_tiny of the current step (hpfem.C:232-235)
    long long iter;       // TimeProps::iter
    unsigned long long acc_min_dxe;  // running min, bit pattern of a positive double
    unsigned long long acc_hmax;     // running max, bit pattern of a non-negative double
    int err;              // sticky DA_ERR_* raised on the device
    unsigned blocks_done[2];  // last-block counters of the coefficient and update kernels
    unsigned listed;      // tiles the reverse step's recording update listed (sets the gather's work split)
    unsigned long long acc_alt_min_dxe;  // the multi-step kernel's second accumulator pair
    unsigned long long acc_alt_hmax;     // (odd steps of a launch), same start values
    unsigned long long bar;       // grid barrier of the cooperative kernels: arrivals since the launch
                                  // began (barrier k of a grid of G blocks opens at G (k + 1))
    unsigned long long bar_exit;  // blocks that have left the launch; the last one restarts both at 0
};

// Time-clipping targets (TimeProps::ndnextoutput / ndnextsave / ndmaxtime) and the
// frict_tiny schedule (hpfem.C:232-235), passed by value to the dt kernel.
struct TimeConsts {
    double next_output, next_save, max_time, influx_dt;
    double gravity_scale, epsilon;
    double frict_tiny_early, frict_tiny_late;
    long long frict_tiny_iters;
    const double *dt_replay;  // when set, step k takes dt_replay[k - iter0] instead of the CFL dt
    long long iter0;
    long long n_replay;
};

// Ensemble (batched) mode: the mesh is the members' meshes one after another, each padded to
// whole tiles, and these device tables give each tile its member and each member its constants
// and step scalars.  All members take the same number of steps (one shared iteration count), each
// with its own dt.  ninst == 0 in a single-instance context.
struct InstArgs {
    int ninst;
    const int32_t *tile_inst;     // [ntiles] member of each tile
    const MatConsts *mcs;         // [ninst]
    double *time;                 // [ninst] TimeProps::time of each member
    double *dt;                   // [ninst] dt of the current step
    double *min_dxe, *hmax;       // [ninst] CFL reductions of the current step
    unsigned long long *acc_min;  // [ninst] running CFL min (bit patterns of positive doubles)
    unsigned long long *acc_max;  // [ninst] running hmax
    const double *sec2_bed;       // [ninst][DA_MAX_MATERIALS] 1 + tan^2(phi_bed)
    const double *cos_int;        // [ninst]
    const double *dk_tab;         // [ninst][2][DA_MAX_MATERIALS][3] d kact / d phi_bed, d phi_int
    const double *box;            // [ninst][4] functional box
    const int32_t *seg0;          // [ninst + 1] first segment of each member
};

// Maximum-depth map (OutLine, properties.h:653-790): depth bit patterns on a regular grid.
struct OutlineGrid {
    int nx = 0, ny = 0;
    double x0 = 0, y0 = 0, dx = 0, dy = 0;
    unsigned long long *map = nullptr;  // [ny][nx]
};

// Dual-weighted-residual indicator: the error grid's own context and the device tables (dwr.cu).
struct DwrState {
    da_ctx *fine = nullptr;      // context of the error grid (the mesh refined once)
    int nf = 0;
    void *mem = nullptr;         // one allocation for the tables below
    int32_t *parent = nullptr;   // [nf]
    int32_t *children = nullptr; // [4][n] fine cells of each coarse cell, -1 unused
    int32_t *interp = nullptr;   // [4][nf] coarse interpolants, -1 unused
    double *weight = nullptr;    // [4][nf]
    double *ut_next = nullptr;   // [3][nf] reconstructed U^{n+1}
    double *lamt = nullptr;      // [3][nf] reconstructed adjoint
    double *err = nullptr;       // [nf] el_error
    double *corr = nullptr;      // [nf] correction
    double *cell = nullptr;      // [n] el_error summed over each coarse cell's children
    double *parts = nullptr;     // compensated partial sums
    double *sums = nullptr;      // [2] total el_error, total correction
};

// Device copy of the flattened mesh.  FP64 path reads the double arrays; the FP32-split
// path reads the float copies.
struct DevMesh {
    int32_t n = 0;
    int32_t n_owned = 0;            // cells [n_owned, n) are ghosts (da_set_owned); n after an upload
    int32_t epoch = -1;
    int32_t *nbr = nullptr;         // [8][n]
    uint8_t *mat = nullptr;         // [n], zero-padded to whole tiles
    uint8_t *bflag = nullptr;       // [n], zero-padded to whole tiles; bit s: side s is a domain boundary; bit 4+s: side s has 2 neighbours
    double *x = nullptr, *y = nullptr, *dx = nullptr, *dy = nullptr;
    double *g = nullptr;            // [3][n]
    double *dg = nullptr;           // [2][n]
    double *curv = nullptr;         // [2][n]
    float *fdx = nullptr, *fdy = nullptr;
    float *fg = nullptr, *fdg = nullptr, *fcurv = nullptr;
    // staged step phases (capi.cu build_halo); null when a tile's halo exceeds kHaloMax
    int32_t *halo_off = nullptr;    // [ntiles + 1]
    int32_t *halo_idx = nullptr;    // halo cells of every tile, tile after tile
    int16_t *nloc = nullptr;        // [n][8] tile-local slot of each neighbour entry
    int32_t halo_max = 0;           // largest halo of a tile
};

// Tracing: CUDA events around every launch of the step and the adjoint, summed per kernel
// (the reference's Timer class, src/header/properties.h:43-71, moved onto the device).
enum TraceKind {
    TR_COEF, TR_UPDATE, TR_COEF_REC, TR_UPDATE_REC, TR_ADJ_SRC, TR_ADJ_GATHER, TR_ADJ_SEED, TR_ADJ_REDUCE,
    TR_SNAPSHOT, TR_STEPS, TR_YOUTURN, TR_COUNT
};

struct TraceState {
    struct Pending {
        int kind;
        int steps;  // time steps the launch covers
        cudaEvent_t a, b;
    };
    bool on = false;
    std::vector<cudaEvent_t> pool;
    std::vector<Pending> pending;
    double total_ms[TR_COUNT] = {};
    long long launches[TR_COUNT] = {};
    long long steps[TR_COUNT] = {};
};

}  // namespace da

struct da_ctx {
    da_params p{};
    da::MatConsts mc{};
    da::TimeConsts tc{};
    int device = 0;
    cudaStream_t stream = nullptr;
    da::DevMesh mesh;
    // state, ping-pong; FP64 or FP32 per precision
    void *U[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    int cur = 0;
    void *kact = nullptr;            // [n] Real
    void *slopes = nullptr;          // [6][n] Real: wet cells' limited slopes from the coefficient phase
    // segments: 32 consecutive cells (one warp), 8 per tile; arrays padded to whole tiles
    int nseg = 0;                    // ntiles * 8
    double *seg_vol = nullptr;       // [nseg] volume partial of each segment after its last update
    double *vol_parts = nullptr;     // [256] partial sums of the volume reduction
    unsigned *active = nullptr;      // [nseg] bit per cell: wet or next to a wet cell
    uint8_t *seg_clean = nullptr;    // [nseg] 1 when both state buffers hold the same segment
    uint8_t *seg_wet = nullptr;      // [nseg] 1 when the segment held a wet cell after the last update
    uint8_t *seg_dirty = nullptr;    // [nseg] 1 when the segment may differ from the base checkpoint
    double *stage = nullptr;         // [n] FP64 staging for host transfers of FP32 arrays
    double *dd_bounds = nullptr;     // [2] a subdomain step's bounds passed by host pointer (domain.cu)
    double *seg_J = nullptr;         // [nseg] functional part of each segment at the final step
    // ensemble mode (ninst > 0): device tables of InstArgs, host copies of the member layout
    int ninst = 0;
    da::InstArgs ia{};
    std::vector<int32_t> inst_cell0;  // [ninst + 1] first cell of each member (multiple of 256)
    std::vector<int32_t> inst_ncell;  // [ninst] cells of each member before padding
    std::vector<int32_t> inst_nmat;   // [ninst] materials of each member
    std::vector<int32_t> inst_npile;  // [ninst] piles of each member (0 or 1)
    void *inst_mem = nullptr;         // one allocation holding every InstArgs table
    double *inst_vol = nullptr;       // [ninst] members' volumes (stats)
    std::vector<double> inst_init;    // [3][n] members' initial states, concatenated (restart)
    da::DwrState dwr;                 // error grid of the DWR indicator (da_dwr_setup)
    da::OutlineGrid outline;          // maximum-depth map (da_outline_init)
    int *tile_epoch = nullptr;       // [ntiles] id of the last recording step that listed the tile
    uint8_t *seg_act = nullptr;      // [nseg] the segment had an active cell in that step
    uint8_t *lam_clean = nullptr;    // [nseg] both adjoint buffers hold the same segment
    int rec_id = 0;                  // id of the current recording step
    int ntiles = 0;                  // tiles of 256 consecutive cells
    int nblocks = 0;                 // grid of the seed kernel (fixed at allocation)
    int grid = 0;                    // grid of the tiled step kernels (da_params.grid_blocks)
    // resident blocks of k_steps [FP32, FP64] x [single, ensemble] x [2, 3 per SM] x [staged] x
    // [checkpoint stores inside the launch]
    int coop_cap[32] = {};
    // of k_youturn [FP32, FP64] x [single, ensemble] x [seed] x [2, 3 per SM] x [staged]
    int coop_cap_yt[32] = {};
    int sm_count = 0;
    da::DevScalars *dsc = nullptr;   // device scalars
    da::DevScalars *hsc = nullptr;   // pinned host mirror
    // graphs of two forward steps, one per starting ping-pong buffer (captured lazily,
    // dropped on mesh or parameter change)
    cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
    std::string err;
    bool have_state = false;
    // adjoint workspace (allocated on first use)
    uint8_t *mask = nullptr;         // [n] branch codes of the replayed forward step
    void *lam[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    double *adjA = nullptr;          // [3][n]
    double *adjB = nullptr;          // [4][n]
    double *gbed = nullptr, *gint = nullptr;  // [n] running parameter sensitivities
    double *dk_tab = nullptr;        // [2][DA_MAX_MATERIALS][3] d kact / d phi_bed, d phi_int
    double *red_out = nullptr;       // [DA_MAX_MATERIALS + 1 + DA_MAX_PILES]
    double *red_part = nullptr;      // [same x kAdjReduceParts] partial sums of the gradient reduction
    double *inst_J = nullptr;        // [max(ninst, 1)] J of each member
    double *dh0 = nullptr;           // [n_piles][n]
    size_t dh0_bytes = 0;            // its allocation
    // the binomial checkpoint placement of the last horizon / slot count (adjoint_host.cu)
    std::vector<int> sched_split;
    int sched_n = -1, sched_c = -1;
    std::vector<void *> snaps;       // checkpoint slots, 3 state arrays each
    // the reverse sweep's launches captured as a CUDA graph (adjoint_host.cu), with the inputs its
    // kernels were given (sweep_key) and the host-side results of building it
    cudaGraphExec_t sweep_graph = nullptr;
    std::vector<unsigned char> sweep_key;
    int sweep_lam = 0;
    long long sweep_fsteps = 0;
    double *dt_replay = nullptr;     // device copy of a frozen time-step sequence
    void *refadj_mem = nullptr;      // workspace of the reference-mode adjoint (adjoint_ref.cu)
    int refadj_n = 0;                // the mesh size it was allocated for
    int adj_n = 0;
    int adj_ninst = -1;
    da::TraceState trace;
};

namespace da {

int set_error(da_ctx *ctx, int code, const std::string &msg);
// capi.cu: the device's sticky error code (already read into ctx->hsc) as a return status; after a
// grid-barrier timeout it also restarts the barrier word
int device_error(da_ctx *ctx, const char *where);
// forward_fp64.cu: a cooperative launch in which block 0 never arrives at the grid barrier, so the
// other blocks' bounded wait runs out after limit_ns (da_selftest_barrier)
int launch_barrier_selftest(da_ctx *ctx, unsigned long long limit_ns);
void trace_begin(da_ctx *ctx, int kind);
void trace_end(da_ctx *ctx, int steps = 1);
int trace_flush(da_ctx *ctx);
int cuda_check(da_ctx *ctx, cudaError_t e, const char *what);
// Host <-> device copies ordered on the context's stream.  That stream is non-blocking, so a
// plain cudaMemcpy (legacy stream) would not wait for the kernels queued on it, and a pageable
// host-to-device cudaMemcpy may return before its data reach the device.  copy_h2d returns once
// the host buffer may be reused (the copy runs before any later work on the stream); copy_d2h
// returns once the data are on the host.
int copy_h2d(da_ctx *ctx, void *dev, const void *host, size_t bytes, const char *what);
int copy_d2h(da_ctx *ctx, void *host, const void *dev, size_t bytes, const char *what);
void fill_consts(const da_params &p, MatConsts *mc, TimeConsts *tc);

// forward_fp64.cu / forward_fp32.cu
// record_mask (optional): branch codes of the step for the adjoint (listed tiles; tile_epoch)
int launch_forward_step(da_ctx *ctx, uint8_t *record_mask = nullptr);
int launch_forward_step_fp64(da_ctx *ctx, uint8_t *record_mask);
int launch_forward_step_fp32(da_ctx *ctx, uint8_t *record_mask);
// the volume (sum dx dy h) of the current state into the device scalars
int launch_volume(da_ctx *ctx);
// nsteps whole steps in one cooperative launch (k_steps); same results as nsteps single steps
// nsteps steps in one cooperative launch; pre_slot / post_slot (checkpoint slots, or null): a
// restore before the first step and a store after the last one inside the same launch.
// Checkpoint stores inside one multi-step launch (single instance): slot[k] receives the state
// after step after[k] of the launch (0-based, increasing), as a store after a launch would.
constexpr int kMidStores = 32;
struct MidStoreList {
    int n = 0;
    int after[kMidStores];
    void *slot[kMidStores];
};
int launch_forward_steps(da_ctx *ctx, int nsteps, void *pre_slot = nullptr, void *post_slot = nullptr,
                         const MidStoreList *mid = nullptr);
int launch_forward_steps_fp64(da_ctx *ctx, int nsteps, void *pre_slot, void *post_slot, const MidStoreList *mid);
int launch_forward_steps_fp32(da_ctx *ctx, int nsteps, void *pre_slot, void *post_slot, const MidStoreList *mid);
int forward_alloc(da_ctx *ctx);
// capi.cu: one FP64 host array to / from a device array of the context's precision (stream-ordered;
// an FP32 download must finish before the next one reuses the staging buffer)
int upload_real(da_ctx *ctx, void *dev, const double *host);
int download_real(da_ctx *ctx, double *host, const void *dev);
// capi.cu: grid of the tiled kernels from da_params.grid_blocks, the SM count and the tile count
void update_grid(da_ctx *ctx);
// adjoint_fp64.cu / adjoint_fp32.cu
int launch_adjoint_step(da_ctx *ctx, int lam_in, int lam_out, const double *sec2, double cos_int);
// replayed forward step + adjoint step in one cooperative launch (k_youturn)
int launch_adjoint_reduce(da_ctx *ctx, int lam0, int n_piles);
// adjoint_ref.cu: one reverse step of the reference's own dual solver (jacobian_mode
// DA_JAC_REFERENCE): U^n in state buffer un, dt and frict_tiny of the step in the device scalars
int launch_ref_adjoint_step(da_ctx *ctx, int un, int lam_in, int lam_out);
int launch_ref_seed(da_ctx *ctx, int lam_out, const double box[4]);
int ref_adjoint_alloc(da_ctx *ctx);
int forward_state_changed(da_ctx *ctx);
// adjoint_host.cu: d kact / d phi_bed and d phi_int of each material's three branches
void kact_derivatives(const da_params &p, double *dkb, double *dki);
// adjoint_host.cu: the checkpointed reverse sweep (see there)
// dwr_acc (or null): accumulate the DWR indicator of every reverse step (adjoint_host.cu DwrAcc)
// lambda_end (or null): lambda^N given instead of the functional's seed (host [3][n])
int adjoint_sweep(da_ctx *ctx, const double *box, int32_t nsteps, int32_t nsnapshots, int32_t n_piles, int *lam0,
                  long long *fsteps, float *dev_ms, void *dwr_acc = nullptr, const double *lambda_end = nullptr);
int copy_lambda_out(da_ctx *ctx, int buf, double *host);
// dwr.cu: the indicator of the step U[un] -> U[unext] with adjoint lam[lam] (coarse dt, time and
// iteration before the step); release of the error grid
int dwr_indicator(da_ctx *ctx, int un, int unext, int lam, double dt, double time0, long long iter0);
void dwr_release(da_ctx *ctx);
// adjoint_host.cu: adjoint buffers and one checkpoint slot
int adj_alloc_for_dwr(da_ctx *ctx);
// ensemble.cu: drop the ensemble tables (back to a single-instance layout)
void free_members(da_ctx *ctx);
// adjoint_fp64.cu: ensemble members' volumes into out[ninst] (device)
int launch_member_volume(da_ctx *ctx, double *out);
// snapshot.cu
size_t snapshot_bytes(const da_ctx *ctx);
int launch_snapshot(da_ctx *ctx, void *slot, bool store);
void forward_free(da_ctx *ctx);

}  // namespace da
