"""Python mirror of the reference's hot-path call sites over the C ABI.

The reference drives one explicit step per call of
    step(El_Table, NodeTable, myid, nump, matprops, timeprops, pileprops, fluxprops,
         statprops, &order_flag, outline, discharge, adaptflag)      src/geoflow/step.C:29-32
with material data in MatProps (src/header/properties.h:527-640) and time data in
TimeProps (properties.h:321-520).  Here the mesh tables are a flattened Mesh held on the
device by a GeoflowContext; MatProps/TimeProps keep the reference's field names.
Errors that the reference handles with printf+exit raise DAError instead.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _ffi
from .mesh import Mesh

PI_REF = 3.1415926  # src/header/constant.h:37, used for degree -> radian in datread.C:379-400


@dataclass
class MatProps:
    """The fields of MatProps that the step reads.  Angles in degrees as in frict.data."""
    intfrict_deg: float = 30.0
    bedfrict_deg: list = field(default_factory=lambda: [20.0])
    epsilon: float = 1.0
    gravity_scale: float = 1.0
    gamma: float = 1.0
    frict_tiny_iters: int = 50
    frict_tiny_early: float = 0.1
    frict_tiny_late: float = 0.000000001

    @staticmethod
    def rad(deg: float) -> float:
        return deg * PI_REF / 180.0


@dataclass
class TimeProps:
    """TimeProps fields that clip dt (incrtime, properties.h:397-410); nondimensional."""
    maxtime: float = math.inf
    nextoutput: float = math.inf
    nextsave: float = math.inf
    time: float = 0.0
    iter: int = 0


def make_params(mat: MatProps, tp: TimeProps, precision: int = _ffi.DA_PREC_FP64, device: int = 0,
                influx_dt: float = math.inf, fp32_sign_floor: float = 0.0,
                tile_culling: bool = True, grid_blocks: int = 0, blocks_per_sm: int = 0,
                tile_staging: int = 1, jacobian_mode: int = 0) -> _ffi.da_params:
    p = _ffi.da_params()
    _ffi.load().da_params_default(C.byref(p))
    p.precision = precision
    p.device = device
    p.epsilon = mat.epsilon
    p.gravity_scale = mat.gravity_scale
    p.gamma = mat.gamma
    p.intfrict = MatProps.rad(mat.intfrict_deg)
    p.n_materials = len(mat.bedfrict_deg)
    for k, b in enumerate(mat.bedfrict_deg):
        p.bedfrict[k] = MatProps.rad(b)
    p.frict_tiny_iters = mat.frict_tiny_iters
    p.frict_tiny_early = mat.frict_tiny_early
    p.frict_tiny_late = mat.frict_tiny_late
    p.max_time = tp.maxtime
    p.next_output = tp.nextoutput
    p.next_save = tp.nextsave
    p.influx_dt = influx_dt
    p.fp32_sign_floor = fp32_sign_floor
    p.tile_culling = int(tile_culling)
    p.grid_blocks = int(grid_blocks)
    p.blocks_per_sm = int(blocks_per_sm)
    p.tile_staging = int(tile_staging)
    p.jacobian_mode = int(jacobian_mode)
    return p


@dataclass
class StepStats:
    dt: float
    time: float
    volume: float
    hmax: float
    iter: int


class GeoflowContext:
    """One device context: flattened mesh + state resident in HBM."""

    def __init__(self, mat: MatProps, tp: TimeProps | None = None, precision: int = _ffi.DA_PREC_FP64,
                 device: int = 0, influx_dt: float = math.inf, fp32_sign_floor: float = 0.0,
                 tile_culling: bool = True, grid_blocks: int = 0, blocks_per_sm: int = 0,
                 tile_staging: int = 1, jacobian_mode: int = _ffi.DA_JAC_EXACT):
        """jacobian_mode: DA_JAC_EXACT (the exact transpose of this forward step) or DA_JAC_REFERENCE
        (the reference's own dual-solver adjoint, calc_jacobain.C:40-153 and calc_adjoint.C:35-167,
        FP64 only)."""
        self.lib = _ffi.load()
        self.mat = mat
        self.tp = tp or TimeProps()
        self.precision = precision
        self.params = make_params(mat, self.tp, precision, device, influx_dt, fp32_sign_floor, tile_culling,
                                  grid_blocks, blocks_per_sm, tile_staging, jacobian_mode)
        err = C.c_int(0)
        self.ctx = self.lib.da_create(C.byref(self.params), C.byref(err))
        if not self.ctx:
            raise _ffi.DAError(err.value, "da_create failed: " + self.lib.da_strerror(err.value).decode())
        self.mesh: Mesh | None = None
        if self.tp.time or self.tp.iter:
            self.set_time(self.tp.time, self.tp.iter)

    def _check(self, st: int, what: str):
        if st != 0:
            msg = self.lib.da_last_error(self.ctx).decode() if self.ctx else ""
            raise _ffi.DAError(st, f"{what}: {msg}")

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.da_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- mesh / state
    def upload_mesh(self, mesh: Mesh, epoch: int = 0):
        self.mesh = mesh
        self._check(self.lib.da_upload_mesh(self.ctx, C.byref(mesh.soa()), epoch), "da_upload_mesh")

    def set_state(self, h, hu, hv):
        h, hu, hv = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, hu, hv))
        self._check(self.lib.da_set_state(self.ctx, _ffi.dptr(h), _ffi.dptr(hu), _ffi.dptr(hv)), "da_set_state")

    def get_state(self):
        n = self.mesh.n
        h, hu, hv = np.empty(n), np.empty(n), np.empty(n)
        self._check(self.lib.da_get_state(self.ctx, _ffi.dptr(h), _ffi.dptr(hu), _ffi.dptr(hv)), "da_get_state")
        return h, hu, hv

    def set_time(self, time: float, iteration: int):
        self._check(self.lib.da_set_time(self.ctx, time, iteration), "da_set_time")

    # ---- stepping
    def step(self) -> StepStats:
        """One step() (order_flag = 1)."""
        s = _ffi.da_step_stats()
        self._check(self.lib.da_forward_step(self.ctx, C.byref(s)), "da_forward_step")
        return StepStats(s.dt, s.time, s.volume, s.hmax, s.iter)

    def run(self, nsteps: int) -> StepStats:
        s = _ffi.da_step_stats()
        self._check(self.lib.da_forward_run(self.ctx, nsteps, C.byref(s)), "da_forward_run")
        return StepStats(s.dt, s.time, s.volume, s.hmax, s.iter)

    def run_timed(self, nsteps: int):
        """(stats, device ms between events on the context stream around the nsteps steps)."""
        s = _ffi.da_step_stats()
        ms = C.c_double(0.0)
        self._check(self.lib.da_forward_run_timed(self.ctx, nsteps, C.byref(s), C.byref(ms)), "da_forward_run_timed")
        return StepStats(s.dt, s.time, s.volume, s.hmax, s.iter), ms.value

    def set_tracing(self, on: bool):
        self._check(self.lib.da_set_tracing(self.ctx, int(on)), "da_set_tracing")

    def trace(self, with_steps: bool = False) -> dict:
        """{kernel: (total device ms, launches)} since tracing was switched on; with_steps adds
        the time steps those launches covered as a third entry."""
        out = {}
        for k in range(_ffi.DA_TRACE_KINDS):
            ms, n, s = C.c_double(), C.c_int64(), C.c_int64()
            self._check(self.lib.da_trace_read(self.ctx, k, C.byref(ms), C.byref(n)), "da_trace_read")
            self._check(self.lib.da_trace_steps(self.ctx, k, C.byref(s)), "da_trace_steps")
            if n.value:
                name = self.lib.da_trace_name(k).decode()
                out[name] = (ms.value, n.value, s.value) if with_steps else (ms.value, n.value)
        return out

    def stats(self, d_time: float = 0.0, test_point=(0.0, 0.0, 0.0), vslump: float = 0.0, planes=(),
              discharge=None, hxyminmax: float = -1.0, min_height: float = -1.0) -> dict:
        """calc_stats of the current state (da_compute_stats).  test_point = (heightifreach, x, y);
        planes = [(xa, xb, ya, yb), ...]; discharge (float64 array, one per plane) accumulates
        d_time * flux in place.  Returns the StatProps fields by name."""
        pr = _ffi.da_stats_props()
        pr.heightifreach, pr.xyifreach[0], pr.xyifreach[1] = test_point
        pr.hxyminmax, pr.min_height, pr.vslump = hxyminmax, min_height, vslump
        pl = np.ascontiguousarray(np.asarray(planes, dtype=np.float64).reshape(-1, 4)) if len(planes) else None
        pr.n_planes = 0 if pl is None else pl.shape[0]
        pr.planes = _ffi.dptr(pl) if pl is not None else None
        if pl is not None and (discharge is None or len(discharge) != pl.shape[0]):
            raise ValueError("discharge must hold one value per plane")
        out = _ffi.da_stats()
        self._check(self.lib.da_compute_stats(self.ctx, C.byref(pr), d_time, C.byref(out),
                                              _ffi.dptr(discharge) if pl is not None else None), "da_compute_stats")
        res = {k: getattr(out, k) for k, _ in out._fields_ if k not in ("xyminmax", "pad")}
        res["xmin"], res["xmax"], res["ymin"], res["ymax"] = list(out.xyminmax)
        return res

    def refine_info(self):
        """(flux-balance weight per cell, refinement flags per cell, geo_target) after a step
        (da_refine_info)."""
        n = self.mesh.n
        e, f, t = np.empty(n), np.empty(n, dtype=np.uint8), C.c_double()
        self._check(self.lib.da_refine_info(self.ctx, _ffi.dptr(e), f.ctypes.data_as(C.POINTER(C.c_uint8)),
                                            C.byref(t)), "da_refine_info")
        return e, f, t.value

    def outline_init(self, dxy, xrange, yrange):
        """Maximum-depth map on a regular grid (OutLine::init2)."""
        a, b, c = (np.ascontiguousarray(v, dtype=np.float64) for v in (dxy, xrange, yrange))
        self._check(self.lib.da_outline_init(self.ctx, _ffi.dptr(a), _ffi.dptr(b), _ffi.dptr(c)), "da_outline_init")

    def outline_update(self):
        self._check(self.lib.da_outline_update(self.ctx), "da_outline_update")

    def outline(self) -> np.ndarray:
        nx, ny = C.c_int32(), C.c_int32()
        self._check(self.lib.da_outline_read(self.ctx, C.byref(nx), C.byref(ny), None), "da_outline_read")
        out = np.empty((ny.value, nx.value))
        self._check(self.lib.da_outline_read(self.ctx, C.byref(nx), C.byref(ny), _ffi.dptr(out)), "da_outline_read")
        return out

    def autotune(self, nsteps: int = 20) -> dict:
        """Pick the launch shape of the step kernels by timing nsteps steps per candidate
        (da_autotune); the state is left where it was.  Returns {"best": (blocks_per_sm, grid),
        "ms_per_step": {(blocks_per_sm, grid): ms}}."""
        r = _ffi.da_tune_result()
        self._check(self.lib.da_autotune(self.ctx, nsteps, C.byref(r)), "da_autotune")
        self.params.grid_blocks = r.grid[r.best]
        self.params.blocks_per_sm = r.blocks_per_sm[r.best]
        return tune_result(r)

    def profile(self, nsteps: int) -> dict:
        """Mean device ms per forward kernel over nsteps (events around every launch)."""
        out = np.zeros(2)
        self._check(self.lib.da_forward_profile(self.ctx, nsteps, _ffi.dptr(out)), "da_forward_profile")
        return {self.lib.da_forward_kernel_name(k).decode(): float(out[k]) for k in range(2)}


def tune_result(r: _ffi.da_tune_result) -> dict:
    keys = [(r.blocks_per_sm[k], r.grid[k]) for k in range(r.n)]
    return {"best": keys[r.best], "ms_per_step": {keys[k]: r.ms_per_step[k] for k in range(r.n)}}


@dataclass
class Gradient:
    """dJ/d(parameters) of one adjoint run (angles in radians)."""
    J: float
    dJ_dbedfrict: list
    dJ_dintfrict: float
    dJ_dpile: list
    forward_steps: int
    snapshots: int
    device_ms: float = 0.0
    lambda0: np.ndarray | None = None
    dwr_cell: np.ndarray | None = None   # DWR el_error per coarse cell, summed over the steps
    dwr_steps: np.ndarray | None = None  # [nsteps][2] total el_error and correction per step


def _grad(g: _ffi.da_gradient, n_mat: int, n_piles: int, lam0=None) -> Gradient:
    return Gradient(g.J, list(g.dJ_dbedfrict[:n_mat]), g.dJ_dintfrict, list(g.dJ_dpile[:n_piles]),
                    int(g.forward_steps), int(g.snapshots), float(g.device_ms), lam0)


def adjoint_run(ctx: GeoflowContext, box, nsteps: int, nsnapshots: int, dh0_dpile=None,
                want_lambda0: bool = False, lambda0_out: np.ndarray | None = None, dwr: bool = False) -> Gradient:
    """dual_solver() of src/adjoint/dual_solver.C:80 over nsteps steps from the current state, for
    J = sum of h^2 dx dy over the cells whose centre lies in box = (xmin, xmax, ymin, ymax).
    lambda0_out: a caller-owned contiguous float64 array of 3 n values (e.g. in pinned memory)
    that receives lambda^0; want_lambda0 allocates one instead.  dwr: also the DWR indicator of
    every step (da_adjoint_run_dwr; needs dwr.Indicator set up on the context): the Gradient's
    dwr_cell (per coarse cell, summed over the steps) and dwr_steps ([nsteps][2] el_error and
    correction of each step)."""
    f = _ffi.da_functional(_ffi.DA_FUNC_H2_BOX, 0, (C.c_double * 4)(*box))
    n = ctx.mesh.n
    dh = None
    n_piles = 0
    if dh0_dpile is not None and len(dh0_dpile):
        dh = np.ascontiguousarray(dh0_dpile, dtype=np.float64).reshape(-1, n)
        n_piles = dh.shape[0]
    if lambda0_out is not None:
        if lambda0_out.dtype != np.float64 or lambda0_out.size != 3 * n or not lambda0_out.flags.c_contiguous:
            raise ValueError("lambda0_out must be a contiguous float64 array of 3 n values")
        lam0 = lambda0_out.reshape(3 * n)
    else:
        lam0 = np.zeros(3 * n) if want_lambda0 else None
    g = _ffi.da_gradient()
    if dwr:
        cell, steps = np.zeros(n), np.zeros((nsteps, 2))
        ctx._check(ctx.lib.da_adjoint_run_dwr(ctx.ctx, C.byref(f), nsteps, nsnapshots,
                                              _ffi.dptr(dh) if dh is not None else None, n_piles, C.byref(g),
                                              _ffi.dptr(lam0) if lam0 is not None else None, _ffi.dptr(cell),
                                              _ffi.dptr(steps)), "da_adjoint_run_dwr")
        out = _grad(g, len(ctx.mat.bedfrict_deg), n_piles, None if lam0 is None else lam0.reshape(3, n))
        out.dwr_cell, out.dwr_steps = cell, steps
        return out
    ctx._check(ctx.lib.da_adjoint_run(ctx.ctx, C.byref(f), nsteps, nsnapshots,
                                      _ffi.dptr(dh) if dh is not None else None, n_piles, C.byref(g),
                                      _ffi.dptr(lam0) if lam0 is not None else None), "da_adjoint_run")
    return _grad(g, len(ctx.mat.bedfrict_deg), n_piles, None if lam0 is None else lam0.reshape(3, n))


def adjoint_run_seeded(ctx: GeoflowContext, lambda_end, nsteps: int, nsnapshots: int, dh0_dpile=None) -> Gradient:
    """The reverse sweep over nsteps steps from the current state with lambda^N = lambda_end given
    ([3][n], da_adjoint_run_seeded): one mesh epoch of an adjoint across adaptation.  J is 0; the
    gradient is this epoch's part; lambda0 is returned."""
    n = ctx.mesh.n
    le = np.ascontiguousarray(lambda_end, dtype=np.float64).reshape(3 * n)
    dh = None
    n_piles = 0
    if dh0_dpile is not None and len(dh0_dpile):
        dh = np.ascontiguousarray(dh0_dpile, dtype=np.float64).reshape(-1, n)
        n_piles = dh.shape[0]
    lam0 = np.zeros(3 * n)
    g = _ffi.da_gradient()
    ctx._check(ctx.lib.da_adjoint_run_seeded(ctx.ctx, _ffi.dptr(le), nsteps, nsnapshots,
                                             _ffi.dptr(dh) if dh is not None else None, n_piles, C.byref(g),
                                             _ffi.dptr(lam0)), "da_adjoint_run_seeded")
    return _grad(g, len(ctx.mat.bedfrict_deg), n_piles, lam0.reshape(3, n))


def adjoint_step(ctx: GeoflowContext, lam_next) -> tuple:
    """(lambda^n, parameter parts) for one reverse step at the context's current state."""
    n = ctx.mesh.n
    ln = np.ascontiguousarray(lam_next, dtype=np.float64).reshape(3 * n)
    out = np.zeros(3 * n)
    g = _ffi.da_gradient()
    ctx._check(ctx.lib.da_adjoint_step(ctx.ctx, _ffi.dptr(ln), _ffi.dptr(out), C.byref(g)), "da_adjoint_step")
    return out.reshape(3, n), _grad(g, len(ctx.mat.bedfrict_deg), 0)


def set_dt_replay(ctx: GeoflowContext, dts, iter0: int = 0):
    """Freezes the time-step sequence (None clears it)."""
    if dts is None:
        ctx._check(ctx.lib.da_set_dt_replay(ctx.ctx, None, 0, 0), "da_set_dt_replay")
        return
    d = np.ascontiguousarray(dts, dtype=np.float64)
    ctx._check(ctx.lib.da_set_dt_replay(ctx.ctx, _ffi.dptr(d), len(d), iter0), "da_set_dt_replay")


def step(ctx: GeoflowContext) -> StepStats:
    """step() of src/geoflow/step.C:29 on a device-resident context."""
    return ctx.step()
