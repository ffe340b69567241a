/*
 * discrete_adjoint.h -- C ABI of the B200 finite-volume step and its discrete adjoint.
 *
 * This is the drop-in boundary that replaces the per-timestep hot path of the
 * TITAN2D-derived solver (haghakhani/discrete_adjoint).  The reference has no
 * plugin or FFI layer; its boundary is a set of C++ call sites, and each entry
 * point below names the call site it replaces:
 *
 *   step()                 src/geoflow/step.C:29-275         (called at src/main/hpfem.C:271)
 *     slopes()             src/geoflow/slopes.C:25-83
 *     get_coef_and_eigen() src/geoflow/get_coef_and_eigen.C:29-180
 *     TimeProps::incrtime  src/header/properties.h:397-410
 *     calc_edge_states<>() src/geoflow/edge_states.C:37-77
 *     correct()            src/geoflow/corrector.C:36-193 -> update_states() src/adjoint/residual.C:162-275
 *   dual_solver()          src/adjoint/dual_solver.C:80-273  (called at src/main/hpfem.C:406)
 *     calc_jacobian()      src/adjoint/calc_jacobain.C:40-153
 *     calc_adjoint()       src/adjoint/calc_adjoint.C:35-167
 *     error_compute()      src/adjoint/error_compute.C:24-119
 *
 * Conventions (the reference's own are printf+exit; here nothing exits):
 *   - every function returns DA_OK (0) or a negative DA_ERR_* code;
 *     da_last_error() gives a one-line message for the last failure on a context;
 *   - host buffers are owned by the caller, device buffers by the context;
 *   - one context per host thread; calls are stream-ordered and not re-entrant.
 *
 * Mesh layout ("flattened quadtree"): cells are in space-filling-curve order.
 * Sides are numbered relative to the cell's positive-x side, as the reference
 * does with Element::positive_x_side (src/datstr/element2.C:694-716):
 *   side 0 = +x (xp), 1 = +y (yp), 2 = -x (xm), 3 = -y (ym).
 * nbr[s*n + i] (s = 0..3) is the first neighbour across side s (Element::neighbor[s]),
 * nbr[(s+4)*n + i] the second one (Element::neighbor[s+4]); the two differ only where
 * the side carries two finer neighbours (edge-midpoint node S_C_CON, constant.h:42), and
 * then the lower one (sides 0 and 2) or the left one (sides 1 and 3) comes first -- the
 * reference keeps the pair counter-clockwise around the element, the other way round on
 * sides 1 and 2 (adapt/refine2.C:590-805);
 * -1 marks the domain boundary (neigh_proc == INIT, constant.h:48).
 */
#ifndef DISCRETE_ADJOINT_H
#define DISCRETE_ADJOINT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DA_ABI_VERSION 2

#define DA_MAX_MATERIALS 16
#define DA_MAX_PILES 8

/* return codes */
#define DA_OK 0
#define DA_ERR_INVALID (-1)     /* bad argument, size or call order */
#define DA_ERR_CUDA (-2)        /* a CUDA runtime call failed */
#define DA_ERR_NAN (-3)         /* NaN/Inf in the state or the time step (residual.C:137-147, :272-273) */
#define DA_ERR_NEG_DEPTH (-4)   /* reserved: negative depth that the clamp could not absorb */
#define DA_ERR_EIGEN (-5)       /* wave speed above 1e9 (get_coef_and_eigen.C:144-156) */
#define DA_ERR_TIMEOUT (-6)     /* a bounded device-side wait gave up */
#define DA_ERR_NO_MESH (-7)     /* no mesh uploaded yet */
#define DA_ERR_OOM (-8)         /* device allocation failed */
#define DA_ERR_NO_DEVICE (-9)   /* no CUDA device visible */
#define DA_ERR_UNSUPPORTED (-10)
#define DA_ERR_IO (-11)         /* a file could not be opened, read or written */

/* adjoint modes (da_params.jacobian_mode) */
#define DA_JAC_EXACT 0          /* the exact transpose of the forward step as computed here */
#define DA_JAC_REFERENCE 1      /* the reference's own dual-solver adjoint, its approximations included
                                 * (calc_jacobian / calc_adjoint, calc_jacobain.C:40-153,
                                 * calc_adjoint.C:35-167); FP64 only */

/* precision modes */
#define DA_PREC_FP64 0          /* plain: every operation in FP64, no contraction, reference order */
#define DA_PREC_FP32_SPLIT 1    /* FP32 state/flux/source; FP64 dt, volume and functional sums */

/* Material and time-stepping properties used on the hot path.
 * Mirrors the fields of MatProps (src/header/properties.h:527-640) and
 * TimeProps (properties.h:321-520) that step() reads.  Angles in radians. */
typedef struct da_params {
    int32_t precision;           /* DA_PREC_* */
    int32_t device;              /* CUDA device ordinal */
    double epsilon;              /* MatProps::epsilon = HEIGHT_SCALE/LENGTH_SCALE */
    double gravity_scale;        /* MatProps::GRAVITY_SCALE */
    double gamma;                /* MatProps::gamma, limiter factor (1 in hpfem.C:82) */
    double intfrict;             /* MatProps::intfrict */
    int32_t n_materials;         /* 1..DA_MAX_MATERIALS */
    int32_t frict_tiny_iters;    /* hpfem.C:232-235: frict_tiny = early while iter < this */
    double bedfrict[DA_MAX_MATERIALS]; /* MatProps::bedfrict, 0-based material index */
    double frict_tiny_early;     /* 0.1 */
    double frict_tiny_late;      /* 1e-9 */
    double max_time;             /* TimeProps::ndmaxtime */
    double next_output;          /* TimeProps::ndnextoutput (clips dt) */
    double next_save;            /* TimeProps::ndnextsave (clips dt) */
    double influx_dt;            /* dt[2] of get_coef_and_eigen.C:49-77; HUGE_VAL when no source is active */
    double fp32_sign_floor;      /* DA_PREC_FP32_SPLIT only: the friction sign tests use
                                  * max(frict_tiny, this); 0 keeps the reference's thresholds */
    int32_t tile_culling;        /* 1: tiles of 256 cells with no wet cell in or next to them are
                                  * not rewritten when both state buffers already hold them
                                  * (results are bit-identical); 0: every cell is rewritten */
    int32_t grid_blocks;         /* blocks of 256 threads per launch of the tiled step kernels
                                  * (each block walks a strided list of 256-cell tiles); 0 = 4 per
                                  * SM.  Results do not depend on it; da_autotune picks it. */
    int32_t blocks_per_sm;       /* register budget of the multi-step and reverse-step kernels:
                                  * compiled for 2 or 3 resident blocks per SM (3: fewer registers,
                                  * more warps to hide latency; pays on dense meshes and ensembles);
                                  * 0 = 2.  Results do not depend on it; da_autotune picks it. */
    int32_t tile_staging;        /* 1: the multi-step and reverse-step kernels copy each 256-cell
                                  * tile and its halo (the outside cells its cells name as
                                  * neighbours) into shared memory one tile ahead, when no tile's
                                  * halo exceeds 192 cells; 0: they read neighbours from global
                                  * memory.  With 1 the reverse step's gather takes a block per
                                  * quarter tile and a thread per cell side when the flow covers
                                  * few tiles, else a block per tile; 2 and 3 fix it to tiles and to
                                  * quarters.  Results do not depend on it.  Default 1. */
    int32_t jacobian_mode;       /* DA_JAC_EXACT (default) or DA_JAC_REFERENCE: which adjoint
                                  * da_adjoint_step / da_adjoint_run apply.  The reference mode
                                  * reproduces the reference's dual solver step for step: it freezes
                                  * dry cells, drops derivatives with respect to cells whose record
                                  * is zero, gates the neighbours' slope terms with the friction-stop
                                  * flags, and flushes adjoint entries below 1e-16, as
                                  * calc_jacobian_elem / calc_adjoint_elem do.  It forms lambda and
                                  * the pile-height gradient; the friction-angle gradients, which the
                                  * reference does not have, are 0 in it.  FP64 contexts only;
                                  * ensembles use the exact mode. */
    int32_t pad_mode;
} da_params;

/* Flattened mesh, host memory, caller-owned.  n = n_cells.  See the file comment. */
typedef struct da_mesh_soa {
    int32_t n_cells;
    const int32_t *nbr;        /* [8][n] neighbour table, -1 = domain boundary */
    const double *x, *y;       /* [n] cell centres (Element::coord) */
    const double *dx, *dy;     /* [n] cell sizes (Element::dx) */
    const double *gravity;     /* [3][n] Element::gravity */
    const double *d_gravity;   /* [2][n] Element::d_gravity (d gz/dx, d gz/dy) */
    const double *curvature;   /* [2][n] Element::curvature */
    const int32_t *material;   /* [n] 0-based material index */
} da_mesh_soa;

/* Per-step scalars (the hot-path parts of get_coef_and_eigen / step / calc_stats). */
typedef struct da_step_stats {
    double dt;                 /* time step taken (after incrtime clipping) */
    double time;               /* TimeProps::time after the step */
    double volume;             /* realvolume of step.C:205, sum dx*dy*h after the update (FP64) */
    double hmax;               /* max h over wet cells before the update */
    int64_t iter;              /* TimeProps::iter after the step */
} da_step_stats;

typedef struct da_ctx da_ctx;

/* ---- context lifecycle ------------------------------------------------------------- */
void da_params_default(da_params *p);
/* Creates a context on p->device.  *err receives the status (may be NULL). */
da_ctx *da_create(const da_params *p, int *err);
void da_destroy(da_ctx *ctx);
const char *da_last_error(const da_ctx *ctx);
const char *da_strerror(int code);
int da_abi_version(void);
/* Replaces the material/time parameters of a live context (MatProps/TimeProps edits between steps). */
int da_set_params(da_ctx *ctx, const da_params *p);
/* TimeProps::time and ::iter (restart, or the adjoint's rewind). */
int da_set_time(da_ctx *ctx, double time, int64_t iter);

/* ---- mesh and state transfer ------------------------------------------------------- */
/* Once per adapt (hpfem.C:243-267): copies the flattened mesh to the device. */
int da_upload_mesh(da_ctx *ctx, const da_mesh_soa *mesh, int32_t epoch);
int da_set_state(da_ctx *ctx, const double *h, const double *hu, const double *hv);
int da_get_state(da_ctx *ctx, double *h, double *hu, double *hv);

/* ---- forward stepping -------------------------------------------------------------- */
/* One step() (order_flag = 1).  DA_ERR_NAN also reports a step whose dt is not finite: with no
 * wet cell, no flux source (da_params.influx_dt infinite) and no output or end time, the CFL rule
 * gives an infinite dt, and the reference's update is then NaN in every cell (its state check at
 * residual.C:272-273 stops the run). */
int da_forward_step(da_ctx *ctx, da_step_stats *out);
/* nsteps step() calls back to back, device-resident, captured in a CUDA graph. */
int da_forward_run(da_ctx *ctx, int32_t nsteps, da_step_stats *last);
/* As da_forward_run; *device_ms receives the time between CUDA events recorded on the
 * context's stream before the first and after the last launch. */
int da_forward_run_timed(da_ctx *ctx, int32_t nsteps, da_step_stats *last, double *device_ms);

/* ---- adjoint ------------------------------------------------------------------------------
 * Replaces dual_solver() (src/adjoint/dual_solver.C:80-273) with calc_jacobian()/calc_adjoint()
 * (calc_jacobain.C:40-153, calc_adjoint.C:35-167) taken over every step, backward in time.
 * By default (DA_JAC_EXACT) the adjoint is the exact transpose of the forward step as it is
 * computed here (k act/pass and all thresholds replayed from recorded branch codes, the time-step
 * sequence frozen), checked against central finite differences of the same forward step;
 * DA_JAC_REFERENCE gives the reference's own adjoint instead (see da_params.jacobian_mode).  Forward states are kept
 * in HBM at nsnapshots checkpoints placed by an optimal binomial schedule and recomputed between
 * them (the reference stores every step to gz files instead, dualmesh.C:82-147). */
#define DA_FUNC_H2_BOX 1          /* J = sum over cells with centre in box of h^2 dx dy, final step */

typedef struct da_functional {
    int32_t kind;                 /* DA_FUNC_H2_BOX */
    int32_t pad;
    double box[4];                /* xmin, xmax, ymin, ymax */
} da_functional;

typedef struct da_gradient {
    double J;                             /* functional value at the final step */
    double dJ_dbedfrict[DA_MAX_MATERIALS];/* per material, radians */
    double dJ_dintfrict;                  /* radians */
    double dJ_dpile[DA_MAX_PILES];        /* per pile height (needs dh0_dpile) */
    int64_t forward_steps;                /* forward steps executed, recomputation included */
    int32_t snapshots;                    /* checkpoints held */
    int32_t pad;
    double device_ms;                     /* device time of the run (CUDA events on its stream) */
} da_gradient;

/* Runs nsteps forward steps from the context's current state and time, then the adjoint back to
 * the start.  dh0_dpile: [n_piles][n] derivative of the initial depth with respect to each pile
 * height (may be NULL when n_piles == 0).  lambda0 (optional, host [3][n]): dJ/dU at the start.
 * The context's state and time are restored to the start on return. */
int da_adjoint_run(da_ctx *ctx, const da_functional *f, int32_t nsteps, int32_t nsnapshots,
                   const double *dh0_dpile, int32_t n_piles, da_gradient *out, double *lambda0);
/* da_adjoint_run from a given lambda^N = dJ/dU^N (host [3][n]) instead of a functional: the
 * reverse sweep of one mesh epoch when the mesh adapts during the horizon (the adjoint of the later
 * epochs carried back through the transpose of the state transfer, as dual_solver moves the adjoint
 * across refinement, dualmesh.C:700-712, 980-995).  out->J is 0; the parameter sums are this
 * epoch's part. */
int da_adjoint_run_seeded(da_ctx *ctx, const double *lambda_end, int32_t nsteps, int32_t nsnapshots,
                          const double *dh0_dpile, int32_t n_piles, da_gradient *out, double *lambda0);
/* One reverse step at the current state U^n: lambda_out = (dU^{n+1}/dU^n)^T lambda_next (host
 * arrays [3][n]).  Replays the forward step to record its branches and time step, then restores
 * the state and time.  The parameter parts of this step are returned in partial (may be NULL). */
int da_adjoint_step(da_ctx *ctx, const double *lambda_next, double *lambda_out, da_gradient *partial);
/* Freezes the time-step sequence: step iter0 + k takes dts[k] (k < n) instead of the CFL dt;
 * dts == NULL clears it.  Used for finite-difference checks of the adjoint. */
int da_set_dt_replay(da_ctx *ctx, const double *dts, int32_t n, int64_t iter0);

/* ---- tracing (the reference's Timer class, properties.h:43-71, moved onto the device) --- */
#define DA_FWD_KERNELS 2  /* coefficients + dt, update + volume */
/* Runs nsteps forward steps with CUDA events around every launch on the context's stream and
 * returns the mean device time of each forward kernel in ms (kernel_ms[DA_FWD_KERNELS]) and
 * the names in kernel order through da_forward_kernel_name().  The state advances. */
int da_forward_profile(da_ctx *ctx, int32_t nsteps, double *kernel_ms);
const char *da_forward_kernel_name(int32_t k);
/* Tracing of every launch of the step and the adjoint (forward runs then skip CUDA graphs):
 * on != 0 starts it with cleared sums, 0 stops it.  da_trace_read returns, for kernel kind k in
 * [0, DA_TRACE_KINDS), the summed device time in ms and the number of launches; da_trace_steps
 * the number of time steps those launches covered (more than the launches only for the
 * multi-step kernel "k_steps"); da_trace_name names the kind. */
#define DA_TRACE_KINDS 11
int da_set_tracing(da_ctx *ctx, int32_t on);
int da_trace_read(da_ctx *ctx, int32_t k, double *total_ms, int64_t *launches);
int da_trace_steps(da_ctx *ctx, int32_t k, int64_t *steps);
const char *da_trace_name(int32_t k);

/* ---- ensembles: many instances in one launch ------------------------------------------------
 * The reference runs the instances of an ensemble (the stochastic module's sampled pile volumes
 * and friction angles) as separate processes, each through step() and dual_solver().  Here the
 * members share one context: their flattened meshes are laid one after another (each padded to
 * whole 256-cell tiles) and every step kernel advances all of them in the same cooperative launch,
 * each member with its own material constants, dt and time; the iteration count (and so
 * frict_tiny) is shared.  A member's state after a run equals its single-instance run bit for bit
 * in FP64 (and its dt and time); J and gradients equal it up to the order of the FP64 sums.  The
 * context's da_params give the precision and every setting but the friction angles and material
 * count, which come from each member.  da_upload_mesh and the single-instance run / adjoint
 * calls are not used on an ensemble context (DA_ERR_INVALID). */
typedef struct da_member {
    da_mesh_soa mesh;                   /* the member's flattened mesh (host arrays) */
    const double *h0, *hu0, *hv0;       /* [n] initial state */
    const double *dh0_dpile;            /* [n] d h0 / d pile height of the member's pile, or NULL */
    int32_t n_materials;
    int32_t pad;
    double bedfrict[DA_MAX_MATERIALS];  /* radians */
    double intfrict;                    /* radians */
    double box[4];                      /* functional box (xmin, xmax, ymin, ymax) */
} da_member;
/* Replaces the context's mesh and state with the members'; time 0, iteration 0. */
int da_ensemble_upload(da_ctx *ctx, const da_member *members, int32_t n_members);
/* Every member back to its initial state, time 0, iteration 0. */
int da_ensemble_restart(da_ctx *ctx);
/* nsteps steps of every member in one cooperative launch; device_ms (optional) its device time. */
int da_ensemble_forward(da_ctx *ctx, int32_t nsteps, double *device_ms);
/* Per-member scalars of the last step (out[n_members]): dt, time, volume, hmax, iteration. */
int da_ensemble_stats(da_ctx *ctx, da_step_stats *out);
/* One member's current state (FP64 host arrays of its own n cells). */
int da_ensemble_get_state(da_ctx *ctx, int32_t member, double *h, double *hu, double *hv);
/* Forward + discrete adjoint of every member over nsteps steps from the current state (binomial
 * checkpoints shared by all members), J = sum of h^2 dx dy over the member's box; out[n_members]
 * gets each member's J and gradients (dJ_dpile[0] for its pile); the state is put back.
 * device_ms (optional): device time of the whole sweep. */
int da_ensemble_adjoint(da_ctx *ctx, int32_t nsteps, int32_t nsnapshots, da_gradient *out, double *device_ms);

/* ---- flow statistics and discharge planes ---------------------------------------------------
 * calc_stats (src/geoflow/stats.C:31-360) of the current state, and DISCHARGE::update
 * (properties.h:964-1133): discharge[k] += d_time * flux of (hu, hv) through plane k (the reference
 * calls calc_stats after every step with that step's dt).  Lengths, heights and velocities are in
 * the mesh's units (the reference's LENGTH/HEIGHT scale factors are 1).  Sums are FP64 in a fixed
 * order (the reference's hash-table order differs, so they agree to rounding).  slopemean uses the
 * terrain slope recovered from the gravity vector, -(g_x, g_y)/g_z, where the reference samples the
 * GIS slope grid. */
#define DA_MAX_PLANES 16
typedef struct da_stats_props {
    double heightifreach;        /* StatProps::heightifreach: depth at the test point that counts as reached */
    double xyifreach[2];         /* StatProps::xyifreach: the test point */
    double hxyminmax;            /* StatProps::hxyminmax (< 0: 10 x min_height, datread.C:315-316) */
    double min_height;           /* MatProps::MAX_NEGLIGIBLE_HEIGHT (< 0: epsilon / 1e4, datread.C:210) */
    double vslump;               /* MatProps::Vslump (vstar = vmean / vslump; 0 gives vstar = 0) */
    int32_t n_planes;            /* discharge planes, <= DA_MAX_PLANES */
    int32_t pad;
    const double *planes;        /* [n_planes][4]: xa, xb, ya, yb */
} da_stats_props;
typedef struct da_stats {
    double xcen, ycen, xvar, yvar, rmean, area;
    double vmean, umean, vxmean, vymean, slopemean;
    double statvolume, piler, hmax, vmax, umax, vstar;
    double xyminmax[4];          /* xmin, xmax, ymin, ymax of the cells with h >= hxyminmax */
    int32_t testpoint_reach;     /* the wet cell nearest the test point is at least heightifreach deep */
    int32_t pad;
    double energy;               /* sum of (g h^2 + h |v|^2) / 2 dA (stats.C's "adjoint" sum) */
} da_stats;
int da_compute_stats(da_ctx *ctx, const da_stats_props *props, double d_time, da_stats *out, double *discharge);
/* Maximum-depth map (OutLine, properties.h:653-790, updated per step at step.C:216-220 under
 * MAX_DEPTH_MAP): a regular grid of cell size dxy over xrange x yrange (OutLine::init2);
 * da_outline_update raises every grid cell covered by a mesh cell to that cell's depth if deeper
 * (call it after each step); da_outline_read gives the grid size and, if map is not NULL, the
 * map [ny][nx]. */
int da_outline_init(da_ctx *ctx, const double dxy[2], const double xrange[2], const double yrange[2]);
int da_outline_update(da_ctx *ctx);
int da_outline_read(da_ctx *ctx, int32_t *nx, int32_t *ny, double *map);

/* ---- adaptation hand-back ---------------------------------------------------------------------
 * After a forward step, what H_adapt reads to pick the cells to refine (hadpt.C:112-151), so the
 * host's adapt needs no state download: per cell the flux-balance weight (el_error[0] of
 * Element::calc_flux_balance, element2.C:3705-3745, from the step's edge fluxes) and flags:
 * bits 0-3 the pile-contour tests Element::if_pile_boundary (element2.C:4020-4065) at GEOFLOW_TINY
 * times 1, 5, 15 and 40 (hadpt.C:46-48) on the new state; bit 4 weight above geo_target, the mean
 * weight of the cells with hu > GEOFLOW_TINY (element_weight.C:36-79; 1 when there is none).  The
 * generation limit and the flux-source test stay with the host.  Outputs may be NULL. */
#define DA_REFINE_CONTOUR_1 1
#define DA_REFINE_CONTOUR_5 2
#define DA_REFINE_CONTOUR_15 4
#define DA_REFINE_CONTOUR_40 8
#define DA_REFINE_WEIGHT 16
int da_refine_info(da_ctx *ctx, double *el_error, uint8_t *flags, double *geo_target);

/* ---- dual-weighted-residual error indicator -------------------------------------------------
 * The reference's estimate (error_compute.C:24-119, called from dual_solver.C:170 and :230):
 * the residual of one step on the mesh refined once, r = update(U~^n) - U~^{n+1}, weighted by the
 * adjoint: el_error = sum_j |r_j (lambda_j - lambda~_j)| and correction = sum_j r_j lambda_j per
 * refined cell, U~ and lambda~ reconstructed from the coarse cell centres (bilinear_interp.C),
 * lambda the coarse adjoint of the parent cell.
 * da_dwr_setup takes the refined grid (every cell of the context's mesh split once, e.g. the
 * mesh builder's extra_level), each fine cell's parent, and the reconstruction as four
 * (coarse cell, weight) pairs per fine cell ([4][nf], -1 = unused).
 * da_dwr_step evaluates the indicator of the step from the context's current state U^n, with
 * lambda_next = dJ/dU^{n+1} (host [3][n]); the coarse step is taken and undone.  Outputs
 * (optional): el_error per fine cell [nf], its sum over each coarse cell's children [n], and
 * sums[2] = total el_error and total correction (compensated FP64 sums in a fixed order). */
int da_dwr_setup(da_ctx *ctx, const da_mesh_soa *fine, const int32_t *parent, const int32_t *interp,
                 const double *weight);
int da_dwr_step(da_ctx *ctx, const double *lambda_next, double *el_error, double *cell_error, double *sums);
/* da_adjoint_run with the DWR indicator of every reverse step, as dual_solver computes
 * error_compute after each adjoint step (src/adjoint/dual_solver.C:206-230): the step n -> n+1 is
 * evaluated right after its reverse step, from U^n, U^{n+1} and lambda^{n+1}.  Needs
 * da_dwr_setup.  cell_error [n]: el_error per coarse cell summed over the steps; step_sums
 * [nsteps][2]: total el_error and total correction of step k (k = 0 the first step of the
 * horizon).  Synchronises with the host once per step. */
int da_adjoint_run_dwr(da_ctx *ctx, const da_functional *f, int32_t nsteps, int32_t nsnapshots,
                       const double *dh0_dpile, int32_t n_piles, da_gradient *out, double *lambda0,
                       double *cell_error, double *step_sums);

/* ---- autotuner (no counterpart in the reference, which has no device launches) ------------
 * Times nsteps forward steps from the current state for each candidate launch shape of the
 * step kernels (register budget of 2 or 3 resident blocks per SM; a block of 256 threads on
 * half the SMs, or 1, 2 or 3 per SM, capped at the resident count and the tile count; the
 * reverse-step kernel keeps at least one block per SM), three times each from the
 * same state, keeps the one with the least time as da_params.blocks_per_sm / grid_blocks and
 * puts the state, time and iteration back after every trial.  Results of later steps do not
 * depend on the choice.  out (optional) receives the candidates and their least mean ms per
 * step. */
#define DA_TUNE_MAX 8
typedef struct da_tune_result {
    int32_t n;                   /* candidates tried */
    int32_t best;                /* index of the one kept */
    int32_t grid[DA_TUNE_MAX];   /* da_params.grid_blocks of each candidate */
    int32_t blocks_per_sm[DA_TUNE_MAX];  /* da_params.blocks_per_sm of each candidate */
    double ms_per_step[DA_TUNE_MAX];
} da_tune_result;
int da_autotune(da_ctx *ctx, int32_t nsteps, da_tune_result *out);

/* ---- diagnostic of the bounded device-side waits ---------------------------------------------
 * No counterpart in the reference (whose only failure handling is exit() on NaN or a runaway wave
 * speed).  The cooperative step kernels synchronise their blocks with a grid barrier whose wait is
 * bounded: after 4 s a waiting block raises DA_ERR_TIMEOUT and every block returns.  This call runs
 * one cooperative launch on the context's stream in which one block never arrives at that barrier,
 * with the wait limited to limit_us microseconds (1 .. 4e6), and returns the status the wait
 * produced (DA_ERR_TIMEOUT when it runs out as designed).  The error is cleared and the barrier
 * restarted afterwards, so the context's next launches run normally. */
int da_selftest_barrier(da_ctx *ctx, int32_t limit_us);

/* ---- domain decomposition: one mesh over several contexts -----------------------------------
 * The reference's only parallel strategy: each MPI rank owns a weighted range of the elements'
 * Hilbert keys (repartition_BSFC.C:540, weights :38-40), refreshes its ghost elements every step
 * (move_data.C:28-300) and takes dt from MPI_Allreduce(MIN) over the ranks
 * (get_coef_and_eigen.C:173).  Here a subdomain is a context whose mesh holds the owned cells
 * first and ghost cells after them: two rings, the cells a step of the owned cells reads (face
 * neighbours, including both fine neighbours of a hanging side, and their face neighbours), with
 * the ghosts' neighbour entries that leave the subdomain set to -1.  discrete_adjoint_b200.domain
 * builds the subdomains and the exchange lists.  One step of all subdomains:
 *   da_step_bounds(ctx_r, b_r)          every subdomain
 *   b = elementwise MIN over r of b_r   (ncclAllReduce(ncclMin, 2 doubles), or on the host)
 *   da_step_apply(ctx_r, b, NULL)       every subdomain: the same dt bits everywhere
 *   da_halo_pack(ctx_r, send cells, n, buf)  ->  transfer  ->  da_halo_unpack(ctx_s, recv cells, n, buf)
 * after which the owned cells hold the undivided mesh's step bit for bit.  Contexts with ghosts
 * refuse the whole-step calls (da_forward_step, da_forward_run, the adjoint: DA_ERR_UNSUPPORTED)
 * unless a dt sequence is replayed (da_set_dt_replay): then dt does not come from their own cells,
 * and da_adjoint_step takes the reverse step of a subdomain -- with four ghost rings (a reverse
 * step of an owned cell reads the forward state four rings out) its owned cells' lambda equals the
 * undivided mesh's, and its parameter partials sum the owned cells only.  Their volume,
 * da_compute_stats and the adjoint's parameter sums cover the owned cells only.
 *
 * da_set_owned: cells [n_owned, n_cells) of the uploaded mesh are ghosts (until the next upload).
 * da_get_stream: the context's cudaStream_t, on which every call below is ordered; a collective
 *   that consumes or produces device buffers of these calls must be ordered on it too.
 * da_step_bounds: the first half of a step (slopes, k act/pass, wave speeds of every cell);
 *   bounds[0] = min over the owned wet cells of min(dx, dy) / wave speed (1e7 when none),
 *   bounds[1] = -(max depth over the owned wet cells), so that one MIN over the pair combines the
 *   subdomains.  bounds: 2 doubles, device memory of the context's GPU (the call returns at once)
 *   or host memory (the call waits for the pair).
 * da_step_apply: dt from the combined pair (get_coef_and_eigen.C:168-179 and
 *   TimeProps::incrtime), then the update of every cell; bounds as above.  stats NULL: returns at
 *   once; otherwise waits and fills stats (volume over the owned cells).
 * da_halo_pack: buf = the current h[cells], hu[cells], hv[cells] (3 n reals of the context's
 *   precision, planar); cells must be owned ([0, n_owned)).
 * da_halo_unpack: the reverse into ghost cells ([n_owned, n_cells)).  cells and buf of both are
 *   device memory of the context's GPU; an index outside its range is skipped and reported as
 *   DA_ERR_INVALID by the next call that waits (da_sync, da_step_apply with stats).
 * da_sync: waits for the context's stream and returns the first error its kernels raised. */
int da_set_owned(da_ctx *ctx, int32_t n_owned);
int da_get_stream(da_ctx *ctx, void **stream);
int da_step_bounds(da_ctx *ctx, double *bounds);
int da_step_apply(da_ctx *ctx, const double *bounds, da_step_stats *stats);
int da_halo_pack(da_ctx *ctx, const int32_t *cells, int32_t n, void *buf);
int da_halo_unpack(da_ctx *ctx, const int32_t *cells, int32_t n, const void *buf);
int da_sync(da_ctx *ctx);

/* ---- one step without any device allocation ------------------------------------------------
 * No counterpart in the reference: an addition for callers that may not allocate device memory
 * themselves or through this library, such as a plugin whose host application owns all of the
 * GPU's memory, or a real-time loop in which allocating is forbidden.  The caller passes device
 * pointers for the flattened mesh (same layout as da_upload_mesh's, FP64), for the state in and
 * for the state out (in and out must not overlap); the step's temporaries live in one fixed
 * array of about 11 MB that every GPU loading this library holds until the process exits.
 * Meshes with more than DA_NOALLOC_MAX_CELLS cells are rejected with DA_ERR_UNSUPPORTED, as is
 * any precision but DA_PREC_FP64; a neighbour or material index out of range gives
 * DA_ERR_INVALID before the step runs.  time/iter are TimeProps::time and ::iter before the
 * step; out receives the step's scalars.  stream is a cudaStream_t of the device that is current
 * when the call is made (NULL: that device's default stream), and the array used is that device's;
 * the call synchronises with the stream and returns after the step has finished on it.
 * The first call on a device resolves the array's device address (cudaGetSymbolAddress) with
 * that device current; make that first call before any stream capture.  All calls share the one
 * array, which keeps the last call's contents: calls that overlap on a GPU (other streams, other
 * host threads) race with each other and must be serialised by the caller.  The result is
 * bit-identical to da_forward_step on a context with the same parameters. */
#define DA_NOALLOC_MAX_CELLS (1 << 20)
int da_forward_step_noalloc(const da_params *p, const da_mesh_soa *dev_mesh, const double *h, const double *hu,
                            const double *hv, double *h_out, double *hu_out, double *hv_out, double time,
                            int64_t iter, void *stream, da_step_stats *out);

#ifdef __cplusplus
}
#endif

#endif /* DISCRETE_ADJOINT_H */
