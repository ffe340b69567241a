"""Oracle: CPU restatement of the reference's hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this package.  It is
the checker for the CUDA path, never the thing measured or shipped.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from discrete_adjoint_b200 import _ffi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libda_oracle.so")

_lib = None

PD = C.POINTER(C.c_double)


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _b
        _b.build()
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER(_ffi.da_params)
    M = C.POINTER(_ffi.da_mesh_soa)
    lib.orc_forward_step.restype = C.c_int
    lib.orc_forward_step.argtypes = [P, M, PD, PD, PD, PD, C.POINTER(C.c_int64), C.POINTER(_ffi.da_step_stats)]
    lib.orc_forward_run.restype = C.c_int
    lib.orc_forward_run.argtypes = [P, M, PD, PD, PD, PD, C.POINTER(C.c_int64), C.c_int, PD,
                                    C.POINTER(_ffi.da_step_stats)]
    lib.orc_slopes.restype = None
    lib.orc_slopes.argtypes = [P, M, PD, PD, PD, PD]
    lib.orc_coef_eigen.restype = C.c_int
    lib.orc_coef_eigen.argtypes = [P, M, PD, PD, PD, PD, PD, PD, PD]
    lib.orc_edge_fluxes.restype = None
    lib.orc_edge_fluxes.argtypes = [P, M, PD, PD, PD, PD, PD]
    lib.orc_adjoint_step_ref.restype = C.c_int
    lib.orc_adjoint_step_ref.argtypes = [P, M, PD, PD, PD, C.c_double, C.c_double, PD, PD]
    lib.orc_forward_step_split.restype = C.c_int
    lib.orc_forward_step_split.argtypes = [P, M, PD, PD, PD, PD, C.POINTER(C.c_int64), PD]
    lib.orc_adjoint_step_var.restype = C.c_int
    lib.orc_adjoint_step_var.argtypes = [P, M, PD, PD, PD, C.c_double, C.c_double, PD, PD, C.c_int]
    lib.orc_step_bounds.restype = C.c_int
    lib.orc_step_bounds.argtypes = [P, M, C.c_int, PD, PD, PD, PD, PD]
    lib.orc_step_frozen.restype = C.c_int
    lib.orc_step_frozen.argtypes = [P, M, C.c_double, PD, PD, PD, C.c_int64]
    lib.orc_step_apply.restype = C.c_int
    lib.orc_step_apply.argtypes = [P, M, PD, PD, PD, PD, PD, PD, C.POINTER(C.c_int64), PD]
    _lib = lib
    return lib


class Oracle:
    """Forward stepping on the host with the restated reference algorithm."""

    def __init__(self, params: _ffi.da_params, mesh):
        self.lib = load()
        self.params = params
        self.mesh = mesh
        self.soa = mesh.soa()
        self.time = C.c_double(0.0)
        self.iter = C.c_int64(0)

    def set_time(self, t: float, it: int):
        self.time.value = t
        self.iter.value = it

    def run(self, h, hu, hv, nsteps: int):
        """Advances (h, hu, hv) in place by nsteps; returns (status, dt history, last stats)."""
        dts = np.zeros(max(nsteps, 1))
        st = _ffi.da_step_stats()
        rc = self.lib.orc_forward_run(C.byref(self.params), C.byref(self.soa), _ffi.dptr(h), _ffi.dptr(hu),
                                      _ffi.dptr(hv), C.byref(self.time), C.byref(self.iter), nsteps,
                                      _ffi.dptr(dts), C.byref(st))
        return rc, dts[:nsteps], st

    def run_split(self, h, hu, hv, nsteps: int):
        """Advances (h, hu, hv) in place by nsteps with FP32 flux and source arithmetic and FP64
        state and corrector accumulation (oracle/da_oracle_split.c); returns the dt history."""
        dts = np.zeros(max(nsteps, 1))
        d = C.c_double()
        for k in range(nsteps):
            rc = self.lib.orc_forward_step_split(C.byref(self.params), C.byref(self.soa), _ffi.dptr(h),
                                                 _ffi.dptr(hu), _ffi.dptr(hv), C.byref(self.time),
                                                 C.byref(self.iter), C.byref(d))
            assert rc == 0
            dts[k] = d.value
        return dts[:nsteps]

    def step_bounds(self, n_owned: int, h, hu, hv, work) -> np.ndarray:
        """First half of a subdomain's step (cells [n_owned, n) are ghosts): fills work (7n) and
        returns [min dx/eigen of the owned wet cells, -hmax]."""
        b = np.zeros(2)
        rc = self.lib.orc_step_bounds(C.byref(self.params), C.byref(self.soa), int(n_owned), _ffi.dptr(h),
                                      _ffi.dptr(hu), _ffi.dptr(hv), _ffi.dptr(work), _ffi.dptr(b))
        assert rc == 0, rc
        return b

    def step_apply(self, bounds, work, h, hu, hv) -> float:
        """Second half: dt from the combined bounds, the update in place; returns dt."""
        b = np.ascontiguousarray(bounds, dtype=np.float64)
        d = C.c_double()
        rc = self.lib.orc_step_apply(C.byref(self.params), C.byref(self.soa), _ffi.dptr(b), _ffi.dptr(work),
                                     _ffi.dptr(h), _ffi.dptr(hu), _ffi.dptr(hv), C.byref(self.time),
                                     C.byref(self.iter), C.byref(d))
        assert rc == 0, rc
        return d.value

    def step_frozen(self, dt: float, h, hu, hv, iteration: int):
        """One step with the given dt in place (no CFL reduction; frict_tiny by `iteration`)."""
        rc = self.lib.orc_step_frozen(C.byref(self.params), C.byref(self.soa), float(dt), _ffi.dptr(h),
                                      _ffi.dptr(hu), _ffi.dptr(hv), int(iteration))
        assert rc == 0, rc

    def slopes(self, h, hu, hv):
        out = np.zeros((6, self.mesh.n))
        self.lib.orc_slopes(C.byref(self.params), C.byref(self.soa), _ffi.dptr(h), _ffi.dptr(hu), _ffi.dptr(hv),
                            _ffi.dptr(out))
        return out

    def coef_eigen(self, h, hu, hv, slopes):
        kact = np.zeros(self.mesh.n)
        mn, hm = C.c_double(), C.c_double()
        rc = self.lib.orc_coef_eigen(C.byref(self.params), C.byref(self.soa), _ffi.dptr(h), _ffi.dptr(hu),
                                     _ffi.dptr(hv), _ffi.dptr(slopes), _ffi.dptr(kact), C.byref(mn), C.byref(hm))
        return rc, kact, mn.value, hm.value

    def adjoint_step_ref(self, h, hu, hv, dt: float, frict_tiny: float, lam_next, keep: int = None):
        """The reference's dual-solver step (restated): lambda of U^{n-1} from lambda of U^n, with
        (h, hu, hv) = U^{n-1}, the step's dt and frict_tiny.  Returns [3][n].  keep: the reference
        approximations to keep (Q_* bits; all by default, 0 gives the exact transpose)."""
        lam_next = np.ascontiguousarray(lam_next, dtype=np.float64).reshape(3, self.mesh.n)
        out = np.zeros((3, self.mesh.n))
        h, hu, hv = (np.ascontiguousarray(a, dtype=np.float64) for a in (h, hu, hv))
        if keep is None:
            rc = self.lib.orc_adjoint_step_ref(C.byref(self.params), C.byref(self.soa), _ffi.dptr(h),
                                               _ffi.dptr(hu), _ffi.dptr(hv), dt, frict_tiny, _ffi.dptr(lam_next),
                                               _ffi.dptr(out))
        else:
            rc = self.lib.orc_adjoint_step_var(C.byref(self.params), C.byref(self.soa), _ffi.dptr(h),
                                               _ffi.dptr(hu), _ffi.dptr(hv), dt, frict_tiny, _ffi.dptr(lam_next),
                                               _ffi.dptr(out), int(keep))
        assert rc == 0
        return out

    def edge_fluxes(self, h, hu, hv, kact):
        F = np.zeros((4, 3, self.mesh.n))
        self.lib.orc_edge_fluxes(C.byref(self.params), C.byref(self.soa), _ffi.dptr(h), _ffi.dptr(hu),
                                 _ffi.dptr(hv), _ffi.dptr(kact), _ffi.dptr(F))
        return F


# the reference's approximations of the exact transpose (oracle/da_oracle_adjoint.c)
Q_RECORD, Q_VOID, Q_STOP, Q_SLOPEFAC, Q_DRYVDIFF, Q_SRTIE, Q_FLUSH = 1, 2, 4, 8, 16, 32, 64
Q_ALL = 127
Q_NAMES = {Q_RECORD: "zero records of dry cells", Q_VOID: "no derivative w.r.t. void cells",
           Q_STOP: "stop-gated neighbour slope terms", Q_SLOPEFAC: "slope sensitivity without sign factor",
           Q_DRYVDIFF: "HLL state-difference term on dry sides", Q_SRTIE: "right-speed ties from the left",
           Q_FLUSH: "flush below 1e-16"}


# ---------------------------------------------------------------- reference harness
REF_EXE = os.path.join(HERE, "_ref", "ref_harness")


def reference_available() -> bool:
    return os.path.exists(REF_EXE)


STAT_FIELDS = ("xcen", "ycen", "xvar", "yvar", "rmean", "area", "vmean", "umean", "vxmean", "vymean", "slopemean",
               "statvolume", "piler", "hmax", "vmax", "umax", "vstar", "xmin", "xmax", "ymin", "ymax", "timereached")


def run_reference(mesh, mat, h, hu, hv, nsteps: int, maxtime: float = float("inf"), ref_static: bool = False,
                  workdir: str | None = None, test_point=(0.0, 0.0, 0.0), vslump: float = 1.0, planes=()) -> dict:
    """Runs the reference's own compiled step() (oracle/_ref/ref_harness) nsteps times.

    mat: MatProps (degrees, as in frict.data).  Returns dt history, time, final state, and the
    per-cell slopes, k act/pass and edge-node fluxes of the last step, plus the gravity and
    d_gravity fields the reference used.
    """
    import struct
    import subprocess
    import tempfile

    from discrete_adjoint_b200.solver import MatProps
    n = mesh.n
    bed = np.zeros(16)
    for k, b in enumerate(mat.bedfrict_deg):
        bed[k] = MatProps.rad(b)
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<6i", 0x31484144, n, mesh.max_level, len(mat.bedfrict_deg), nsteps,
                                int(ref_static)))
            f.write(np.array([MatProps.rad(mat.intfrict_deg), mat.epsilon, mat.gravity_scale, mat.gamma,
                              maxtime], dtype="<f8").tobytes())
            f.write(bed.astype("<f8").tobytes())
            for a in (mesh.nbr, mesh.level, mesh.ix, mesh.iy, mesh.material):
                f.write(np.ascontiguousarray(a, dtype="<i4").tobytes())
            for a in (mesh.x, mesh.y, mesh.dx, mesh.dy, mesh.zeta, mesh.gravity, mesh.d_gravity, mesh.curvature,
                      h, hu, hv):
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
            # calc_stats inputs: test point (height, x, y), Vslump, discharge planes (xa, xb, ya, yb)
            f.write(np.array(list(test_point) + [vslump], dtype="<f8").tobytes())
            f.write(struct.pack("<i", len(planes)))
            for pl in planes:
                f.write(np.array(pl, dtype="<f8").tobytes())
        r = subprocess.run([REF_EXE, fin, fout], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"ref_harness failed ({r.returncode}): {r.stderr[-2000:]}")
        raw = open(fout, "rb").read()
        step_seconds = float("nan")
        for line in r.stderr.splitlines():
            if line.startswith("ref_harness_step_seconds="):
                step_seconds = float(line.split("=", 1)[1])
    magic, n2, ns = struct.unpack_from("<3i", raw, 0)
    assert magic == 0x314F4144 and n2 == n and ns == nsteps
    off = 12
    arr = np.frombuffer(raw, dtype="<f8", offset=off)
    k = 0

    def take(cnt):
        nonlocal k
        v = arr[k:k + cnt].copy()
        k += cnt
        return v

    out = {"dt": take(nsteps), "time": float(take(1)[0]), "step_seconds": step_seconds}
    out["h"], out["hu"], out["hv"] = take(n), take(n), take(n)
    out["slopes"] = take(6 * n).reshape(6, n)
    out["kact"] = take(n)
    out["flux"] = take(12 * n).reshape(4, 3, n)
    out["gravity"] = take(3 * n).reshape(3, n)
    out["d_gravity"] = take(2 * n).reshape(2, n)
    out["stats"] = dict(zip(STAT_FIELDS, take(len(STAT_FIELDS))))
    out["discharge"] = take(len(planes))
    return out


def _harness(payload: bytes, cwd: str) -> bytes:
    import subprocess
    fin, fout = os.path.join(cwd, "in.bin"), os.path.join(cwd, "out.bin")
    with open(fin, "wb") as f:
        f.write(payload)
    r = subprocess.run([REF_EXE, fin, fout], capture_output=True, text=True, cwd=cwd)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness failed ({r.returncode}): {r.stderr[-2000:]}")
    return open(fout, "rb").read()


def ref_hilbert_keys(u, v) -> np.ndarray:
    """The reference's own fhsfc2d_ (src/main/hilbert.C) of normalised points: [n][2] uint32."""
    import struct
    import tempfile
    u = np.ascontiguousarray(u, dtype="<f8")
    v = np.ascontiguousarray(v, dtype="<f8")
    with tempfile.TemporaryDirectory() as td:
        raw = _harness(struct.pack("<2i", 0x314B4144, len(u)) + u.tobytes() + v.tobytes(), td)
    magic, n = struct.unpack_from("<2i", raw, 0)
    assert magic == 0x324B4144 and n == len(u)
    return np.frombuffer(raw, dtype="<u4", offset=8).reshape(n, 2).copy()


def ref_write_solution(directory: str, rank: int, step: int, keys, h, hu, hv):
    """The reference's SolRec writes solution_<rank>_<step> into directory (wrtie_sol_to_disk)."""
    import struct
    k = np.ascontiguousarray(keys, dtype="<u4")
    payload = struct.pack("<4i", 0x31574144, rank, step, len(k)) + k.tobytes()
    for a in (h, hu, hv):
        payload += np.ascontiguousarray(a, dtype="<f8").tobytes()
    raw = _harness(payload, directory)
    assert struct.unpack_from("<i", raw, 0)[0] == 0x32574144


def ref_read_solution(directory: str, rank: int, step: int, keys):
    """The reference's SolRec reads solution_<rank>_<step> from directory (read_sol_from_disk):
    (found [n]: 0 none, 1 zero record, 2 state record; state [n][3])."""
    import struct
    k = np.ascontiguousarray(keys, dtype="<u4")
    raw = _harness(struct.pack("<4i", 0x31524144, rank, step, len(k)) + k.tobytes(), directory)
    magic, n = struct.unpack_from("<2i", raw, 0)
    assert magic == 0x32524144 and n == len(k)
    found = np.frombuffer(raw, dtype="<i4", offset=8, count=n).copy()
    state = np.frombuffer(raw, dtype="<f8", offset=8 + 4 * n).reshape(n, 3).copy()
    return found, state


def run_reference_adjoint(mesh, mat, states, iters, dts, lam_end, workdir: str | None = None) -> dict:
    """The reference's own dual-solver steps (oracle/_ref/ref_harness, mode 'DAJ1').

    Reverse step k takes back the forward step iters[k] (U^{iters[k]-1} -> U^{iters[k]}), with
    states[k] = (h, hu, hv) of U^{iters[k]-1} and dts[k] that step's dt; lam_end ([3][n]) is the
    adjoint of U^{iters[0]}.  Each step runs update_dual_grid, calc_jacobian and calc_adjoint
    (src/adjoint/dual_grid_routines.C:15-93, calc_jacobain.C:40-153, calc_adjoint.C:35-167) with
    a zero functional sensitivity.  Returns {"lam": [K][3][n] the adjoint after each reverse step,
    "seconds": time of the K steps}.
    """
    import struct
    import subprocess
    import tempfile

    from discrete_adjoint_b200.solver import MatProps
    n = mesh.n
    K = len(iters)
    assert len(states) == K and len(dts) == K
    bed = np.zeros(16)
    for k, b in enumerate(mat.bedfrict_deg):
        bed[k] = MatProps.rad(b)
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<6i", 0x314A4144, n, mesh.max_level, len(mat.bedfrict_deg), K, 0))
            f.write(np.array([MatProps.rad(mat.intfrict_deg), mat.epsilon, mat.gravity_scale, mat.gamma,
                              float("inf")], dtype="<f8").tobytes())
            f.write(bed.astype("<f8").tobytes())
            for a in (mesh.nbr, mesh.level, mesh.ix, mesh.iy, mesh.material):
                f.write(np.ascontiguousarray(a, dtype="<i4").tobytes())
            for a in (mesh.x, mesh.y, mesh.dx, mesh.dy, mesh.zeta, mesh.gravity, mesh.d_gravity, mesh.curvature):
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
            f.write(np.asarray(iters, dtype="<i4").tobytes())
            f.write(np.asarray(dts, dtype="<f8").tobytes())
            for (h, hu, hv) in states:
                for a in (h, hu, hv):
                    f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
            f.write(np.ascontiguousarray(lam_end, dtype="<f8").reshape(3, n).tobytes())
        r = subprocess.run([REF_EXE, fin, fout], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"ref_harness failed ({r.returncode}): {r.stderr[-2000:]}")
        raw = open(fout, "rb").read()
    magic, n2, k2 = struct.unpack_from("<3i", raw, 0)
    assert magic == 0x314F4A44 and n2 == n and k2 == K
    arr = np.frombuffer(raw, dtype="<f8", offset=12)
    return {"lam": arr[:K * 3 * n].reshape(K, 3, n).copy(), "seconds": float(arr[K * 3 * n])}


def run_reference_fwdadj(mesh, mat, nsteps: int, warm: int, box, workdir: str | None = None,
                         replicas: int = 1) -> dict:
    """The reference's own forward + adjoint, timed step by step (oracle/_ref/ref_harness, mode 'DAF1'):
    nsteps forward steps from the mesh's initial state with the driver's solution recording, then
    the dual solver's reverse steps back to step `warm` from lambda = dJ/dU of J = sum over the
    cells whose centre lies in box of h^2 dx dy.  Returns {"fwd_seconds": [nsteps],
    "rev_seconds": [nsteps - warm], "lam": [3][n] the adjoint of U^warm}.  replicas > 1: that many
    harness processes run the same input at the same time (one per host core), and
    "replica_seconds" lists each one's timed forward + reverse seconds."""
    import struct
    import subprocess
    import tempfile

    from discrete_adjoint_b200.solver import MatProps
    n = mesh.n
    bed = np.zeros(16)
    for k, b in enumerate(mat.bedfrict_deg):
        bed[k] = MatProps.rad(b)
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<6i", 0x31464144, n, mesh.max_level, len(mat.bedfrict_deg), nsteps, warm))
            f.write(np.array([MatProps.rad(mat.intfrict_deg), mat.epsilon, mat.gravity_scale, mat.gamma,
                              float("inf")], dtype="<f8").tobytes())
            f.write(bed.astype("<f8").tobytes())
            for a in (mesh.nbr, mesh.level, mesh.ix, mesh.iy, mesh.material):
                f.write(np.ascontiguousarray(a, dtype="<i4").tobytes())
            for a in (mesh.x, mesh.y, mesh.dx, mesh.dy, mesh.zeta, mesh.gravity, mesh.d_gravity, mesh.curvature,
                      mesh.h0, mesh.hu0, mesh.hv0):
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
            f.write(np.asarray(box, dtype="<f8").tobytes())
        outs = [fout] + [os.path.join(td, f"out{k}.bin") for k in range(1, max(1, replicas))]
        procs = [subprocess.Popen([REF_EXE, fin, fo], stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, text=True)
                 for fo in outs]
        errs = [p.communicate()[1] for p in procs]
        for p, e in zip(procs, errs):
            if p.returncode != 0:
                raise RuntimeError(f"ref_harness failed ({p.returncode}): {e[-2000:]}")
        raws = [open(fo, "rb").read() for fo in outs]
    nr = nsteps - warm
    arrs = []
    for raw in raws:
        magic, n2, k2, w2 = struct.unpack_from("<4i", raw, 0)
        assert magic == 0x314F4644 and n2 == n and k2 == nsteps and w2 == warm
        arrs.append(np.frombuffer(raw, dtype="<f8", offset=16))
    arr = arrs[0]
    return {"fwd_seconds": arr[:nsteps].copy(), "rev_seconds": arr[nsteps:nsteps + nr].copy(),
            "lam": arr[nsteps + nr:nsteps + nr + 3 * n].reshape(3, n).copy(),
            "replica_seconds": [float(np.sum(a[warm:nsteps]) + np.sum(a[nsteps:nsteps + nr])) for a in arrs]}


def params_for(mat) -> "_ffi.da_params":
    """da_params for the oracle filled here (the values da_params_default and make_params give),
    so that a CPU-only caller does not load the product library."""
    import math

    from discrete_adjoint_b200.solver import MatProps
    p = _ffi.da_params()
    p.precision = _ffi.DA_PREC_FP64
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
    p.max_time = p.next_output = p.next_save = p.influx_dt = math.inf
    p.tile_culling = 1
    p.tile_staging = 1
    return p


def time_port_fwdadj(mesh, mat, warm: int, steps: int, box):
    """Per-step seconds of the restated forward step and reverse step (the oracle), as
    run_reference_fwdadj times the reference: (forward seconds [steps], reverse seconds [steps])."""
    import time
    o = Oracle(params_for(mat), mesh)
    h, hu, hv = mesh.h0.copy(), mesh.hu0.copy(), mesh.hv0.copy()
    o.run(h, hu, hv, warm)
    states, dts, fwd = [], [], []
    for _ in range(steps):
        states.append((h.copy(), hu.copy(), hv.copy()))
        t0 = time.perf_counter()
        rc, dt, _ = o.run(h, hu, hv, 1)
        fwd.append(time.perf_counter() - t0)
        dts.append(float(dt[0]))
    inb = (mesh.x >= box[0]) & (mesh.x <= box[1]) & (mesh.y >= box[2]) & (mesh.y <= box[3])
    lam = np.zeros((3, mesh.n))
    lam[0] = np.where(inb, 2.0 * h * (mesh.dx * mesh.dy), 0.0)
    rev = []
    for k in range(steps - 1, -1, -1):
        it = warm + k + 1
        t0 = time.perf_counter()
        lam = o.adjoint_step_ref(*states[k], dts[k], 0.1 if it < 51 else 1e-9, lam)
        rev.append(time.perf_counter() - t0)
    return np.array(fwd), np.array(rev)


ADAPTER_EXE = os.path.join(HERE, "_ref", "adapter_check")


def adapter_available() -> bool:
    return os.path.exists(ADAPTER_EXE)


def run_adapter_check(mesh, mat, h, hu, hv, nsteps: int = 0, step: bool = False) -> dict:
    """The drop-in adapter (element-table flattening and step() replacement), compiled against the
    reference (oracle/_ref/adapter_check): flattens
    the reference's tables rebuilt from mesh and compares the flattening with mesh; with step=True it
    also takes nsteps steps through the adapter (the device path) and through the reference's step()
    and compares the results.  Returns the mismatch counts."""
    import struct
    import subprocess
    import tempfile

    from discrete_adjoint_b200.solver import MatProps
    n = mesh.n
    bed = np.zeros(16)
    for k, b in enumerate(mat.bedfrict_deg):
        bed[k] = MatProps.rad(b)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("<6i", 0x31494144, n, mesh.max_level, len(mat.bedfrict_deg), nsteps, int(step)))
            f.write(np.array([MatProps.rad(mat.intfrict_deg), mat.epsilon, mat.gravity_scale, mat.gamma,
                              float("inf")], dtype="<f8").tobytes())
            f.write(bed.astype("<f8").tobytes())
            for a in (mesh.nbr, mesh.level, mesh.ix, mesh.iy, mesh.material):
                f.write(np.ascontiguousarray(a, dtype="<i4").tobytes())
            for a in (mesh.x, mesh.y, mesh.dx, mesh.dy, mesh.zeta, mesh.gravity, mesh.d_gravity, mesh.curvature,
                      h, hu, hv):
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
        r = subprocess.run([ADAPTER_EXE, fin, fout], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"adapter_check failed ({r.returncode}): {r.stderr[-2000:]}")
        raw = open(fout, "rb").read()
    v = struct.unpack_from("<7i", raw, 0)
    assert v[0] == 0x314F4944 and v[1] == n
    return {"nbr_mismatch": v[2], "field_mismatch": v[3], "state_mismatch": v[4], "dt_mismatch": v[5],
            "steps": v[6], "max_diff": struct.unpack_from("<d", raw, 28)[0]}


def _mesh_payload(magic: int, mesh, mat, nsteps: int, flag: int, h, hu, hv) -> bytes:
    """The flattened mesh and a state in the harness's 'DAH1' layout (header magic, n, max_level,
    n_materials, nsteps, flag; scalars; tables; fields; h, hu, hv)."""
    import struct

    from discrete_adjoint_b200.solver import MatProps
    bed = np.zeros(16)
    for k, b in enumerate(mat.bedfrict_deg):
        bed[k] = MatProps.rad(b)
    parts = [struct.pack("<6i", magic, mesh.n, mesh.max_level, len(mat.bedfrict_deg), nsteps, flag),
             np.array([MatProps.rad(mat.intfrict_deg), mat.epsilon, mat.gravity_scale, mat.gamma, float("inf")],
                      dtype="<f8").tobytes(), bed.astype("<f8").tobytes()]
    for a in (mesh.nbr, mesh.level, mesh.ix, mesh.iy, mesh.material):
        parts.append(np.ascontiguousarray(a, dtype="<i4").tobytes())
    for a in (mesh.x, mesh.y, mesh.dx, mesh.dy, mesh.zeta, mesh.gravity, mesh.d_gravity, mesh.curvature, h, hu, hv):
        parts.append(np.ascontiguousarray(a, dtype="<f8").tobytes())
    return b"".join(parts)


def _elements_out(raw: bytes, magic: int) -> dict:
    import struct
    m, n, it, ndt = struct.unpack_from("<4i", raw, 0)
    assert m == magic, hex(m)
    arr = np.frombuffer(raw, dtype="<f8", offset=16)
    time_, dts = float(arr[0]), arr[1:1 + ndt].copy()
    rec = np.frombuffer(raw, dtype=np.uint8, offset=16 + 8 * (1 + ndt)).reshape(n, 8 + 16 + 24)
    keys = rec[:, :8].copy().view("<u4").reshape(n, 2)
    xy = rec[:, 8:24].copy().view("<f8").reshape(n, 2)
    st = rec[:, 24:].copy().view("<f8").reshape(n, 3)
    return {"iter": it, "time": time_, "dt": dts, "keys": keys, "x": xy[:, 0], "y": xy[:, 1],
            "h": st[:, 0], "hu": st[:, 1], "hv": st[:, 2]}


def run_reference_save(mesh, mat, h, hu, hv, nsteps: int, outline, directory: str) -> dict:
    """The reference's step() nsteps times from (h, hu, hv) on the mesh's tables, then its
    save_forward (restart.C:21-125): restart_0000 and outline_0000 land in `directory`.
    outline = (dxy, xrange, yrange) of the max-depth grid.  Returns the active elements' keys,
    centres and states and the TimeProps history (harness mode 'DAS1')."""
    import subprocess
    payload = _mesh_payload(0x31534144, mesh, mat, nsteps, 0, h, hu, hv)
    payload += np.concatenate([np.asarray(v, dtype="<f8") for v in outline]).astype("<f8").tobytes()
    fin, fout = os.path.join(directory, "save_in.bin"), os.path.join(directory, "save_out.bin")
    open(fin, "wb").write(payload)
    r = subprocess.run([REF_EXE, fin, fout], capture_output=True, text=True, cwd=directory)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness save failed ({r.returncode}): {r.stderr[-2000:]}")
    return _elements_out(open(fout, "rb").read(), 0x314F5344)


def run_reference_load(mat, nsteps: int, outline, directory: str) -> dict:
    """The reference's loadrun (restart.C:127-239) of restart_0000 / outline_0000 in `directory`,
    then its step() nsteps times (harness mode 'DAL1').  Returns as run_reference_save."""
    import struct
    import subprocess

    from discrete_adjoint_b200.solver import MatProps
    bed = np.zeros(16)
    for k, b in enumerate(mat.bedfrict_deg):
        bed[k] = MatProps.rad(b)
    payload = struct.pack("<3i", 0x314C4144, len(mat.bedfrict_deg), nsteps)
    payload += np.array([MatProps.rad(mat.intfrict_deg), mat.epsilon, mat.gravity_scale, mat.gamma, float("inf")],
                        dtype="<f8").tobytes() + bed.astype("<f8").tobytes()
    payload += np.concatenate([np.asarray(v, dtype="<f8") for v in outline]).astype("<f8").tobytes()
    fin, fout = os.path.join(directory, "load_in.bin"), os.path.join(directory, "load_out.bin")
    open(fin, "wb").write(payload)
    r = subprocess.run([REF_EXE, fin, fout], capture_output=True, text=True, cwd=directory)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness load failed ({r.returncode}): {r.stderr[-2000:]}")
    return _elements_out(open(fout, "rb").read(), 0x314F4C44)


def run_reference_dwr(fine, parent, mat, prev, state, adjoint, dt: float, iteration: int,
                      workdir: str | None = None) -> dict:
    """The reference's DWR estimate of one step on the error grid (harness mode 'DAE1'):
    bilinear_interp, update_bilinear_error_grid and error_compute (dual_solver.C:213-230) on
    `fine` (the coarse mesh refined once, `parent` its coarse cell per fine cell), every fine cell
    starting from its father's prev = U^{iteration-1}, state = U^{iteration} and adjoint (each
    [3][n]); dt the step's.  Returns per fine cell bilin_state, bilin_prev, bilin_adj,
    residual ([3][nf] each), el_error ([2][nf]) and correction ([nf])."""
    import struct
    import subprocess
    import tempfile
    n = np.asarray(prev).shape[-1]
    payload = _mesh_payload(0x31454144, fine, mat, 0, 0, np.zeros(fine.n), np.zeros(fine.n), np.zeros(fine.n))
    # the header's nsteps / flag words carry the iteration and the coarse cell count; the zero
    # state the layout ends with is not part of this mode's input
    payload = bytearray(payload[: len(payload) - 24 * fine.n])
    struct.pack_into("<2i", payload, 16, int(iteration), int(n))
    payload += np.ascontiguousarray(parent, dtype="<i4").tobytes()
    for a in (prev, state, adjoint):
        payload += np.ascontiguousarray(a, dtype="<f8").reshape(3 * n).tobytes()
    payload += struct.pack("<d", float(dt))
    with tempfile.TemporaryDirectory(dir=workdir) as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        open(fin, "wb").write(bytes(payload))
        r = subprocess.run([REF_EXE, fin, fout], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"ref_harness dwr failed ({r.returncode}): {r.stderr[-2000:]}")
        raw = open(fout, "rb").read()
    magic, nf = struct.unpack_from("<2i", raw, 0)
    assert magic == 0x314F4544 and nf == fine.n
    a = np.frombuffer(raw, dtype="<f8", offset=8).reshape(nf, 15)
    return {"bilin_state": a[:, 0:3].T.copy(), "bilin_prev": a[:, 3:6].T.copy(), "bilin_adj": a[:, 6:9].T.copy(),
            "residual": a[:, 9:12].T.copy(), "el_error": a[:, 12:14].T.copy(), "correction": a[:, 14].copy()}
