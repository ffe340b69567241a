"""Ensembles over the C ABI: many independent instances advanced by the same kernels.

The reference runs ensemble members (the stochastic module's sampled pile volumes and friction
angles) as separate processes, each through step() (src/geoflow/step.C:29) and dual_solver()
(src/adjoint/dual_solver.C:80).  Here the members share one device context
(da_ensemble_upload): every launch advances all of them, each with its own material constants,
dt and time, and each member's state equals its own single-instance run.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _ffi
from .mesh import Mesh
from .solver import Gradient, MatProps, StepStats, TimeProps, make_params, tune_result


@dataclass
class Member:
    """One instance: its mesh and initial state (mesh.h0/hu0/hv0), materials, functional box."""
    mesh: Mesh
    mat: MatProps
    box: tuple  # (xmin, xmax, ymin, ymax) of J = sum h^2 dx dy
    pile: int = 0  # which of the mesh's piles the pile-height gradient refers to (-1: none)


class Ensemble:
    def __init__(self, members: list[Member], precision: int = _ffi.DA_PREC_FP64, device: int = 0,
                 tp: TimeProps | None = None, grid_blocks: int = 0, blocks_per_sm: int = 0):
        if not members:
            raise ValueError("empty ensemble")
        self.lib = _ffi.load()
        self.members = members
        self.precision = precision
        self.params = make_params(members[0].mat, tp or TimeProps(), precision, device, grid_blocks=grid_blocks,
                                  blocks_per_sm=blocks_per_sm)
        err = C.c_int(0)
        self.ctx = self.lib.da_create(C.byref(self.params), C.byref(err))
        if not self.ctx:
            raise _ffi.DAError(err.value, "da_create failed: " + self.lib.da_strerror(err.value).decode())
        arr = (_ffi.da_member * len(members))()
        self._keep = []
        for k, mb in enumerate(members):
            m = mb.mesh
            d = _ffi.da_member()
            d.mesh = m.soa()
            h0, hu0, hv0 = (np.ascontiguousarray(a, dtype=np.float64) for a in (m.h0, m.hu0, m.hv0))
            d.h0, d.hu0, d.hv0 = _ffi.dptr(h0), _ffi.dptr(hu0), _ffi.dptr(hv0)
            dh = None
            if mb.pile >= 0 and m.dh0_dpile is not None and len(m.dh0_dpile):
                dh = np.ascontiguousarray(np.asarray(m.dh0_dpile, dtype=np.float64).reshape(-1, m.n)[mb.pile])
                d.dh0_dpile = _ffi.dptr(dh)
            d.n_materials = len(mb.mat.bedfrict_deg)
            for q, b in enumerate(mb.mat.bedfrict_deg):
                d.bedfrict[q] = MatProps.rad(b)
            d.intfrict = MatProps.rad(mb.mat.intfrict_deg)
            for q in range(4):
                d.box[q] = float(mb.box[q])
            arr[k] = d
            self._keep += [h0, hu0, hv0, dh]
        self._check(self.lib.da_ensemble_upload(self.ctx, arr, len(members)), "da_ensemble_upload")
        self._keep = None  # the library copied everything

    def _check(self, st: int, what: str):
        if st != 0:
            msg = self.lib.da_last_error(self.ctx).decode() if self.ctx else ""
            raise _ffi.DAError(st, f"{what}: {msg}")

    def close(self):
        if self.ctx:
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

    def __len__(self):
        return len(self.members)

    @property
    def cells(self) -> int:
        return sum(mb.mesh.n for mb in self.members)

    def restart(self):
        self._check(self.lib.da_ensemble_restart(self.ctx), "da_ensemble_restart")

    def forward(self, nsteps: int) -> float:
        """nsteps steps of every member in one launch; returns the device ms."""
        ms = C.c_double(0.0)
        self._check(self.lib.da_ensemble_forward(self.ctx, nsteps, C.byref(ms)), "da_ensemble_forward")
        return ms.value

    def stats(self) -> list[StepStats]:
        out = (_ffi.da_step_stats * len(self.members))()
        self._check(self.lib.da_ensemble_stats(self.ctx, out), "da_ensemble_stats")
        return [StepStats(s.dt, s.time, s.volume, s.hmax, s.iter) for s in out]

    def get_state(self, k: int):
        n = self.members[k].mesh.n
        h, hu, hv = np.empty(n), np.empty(n), np.empty(n)
        self._check(self.lib.da_ensemble_get_state(self.ctx, k, _ffi.dptr(h), _ffi.dptr(hu), _ffi.dptr(hv)),
                    "da_ensemble_get_state")
        return h, hu, hv

    def adjoint(self, nsteps: int, nsnapshots: int) -> tuple[list[Gradient], float]:
        """Forward + adjoint of every member; (gradients per member, device ms)."""
        out = (_ffi.da_gradient * len(self.members))()
        ms = C.c_double(0.0)
        self._check(self.lib.da_ensemble_adjoint(self.ctx, nsteps, nsnapshots, out, C.byref(ms)), "da_ensemble_adjoint")
        res = []
        for mb, g in zip(self.members, out):
            nm = len(mb.mat.bedfrict_deg)
            res.append(Gradient(g.J, list(g.dJ_dbedfrict[:nm]), g.dJ_dintfrict,
                                [g.dJ_dpile[0]] if mb.pile >= 0 else [], int(g.forward_steps), int(g.snapshots),
                                float(g.device_ms)))
        return res, ms.value

    def autotune(self, nsteps: int = 10) -> dict:
        r = _ffi.da_tune_result()
        self._check(self.lib.da_autotune(self.ctx, nsteps, C.byref(r)), "da_autotune")
        return tune_result(r)



def shard_members(sizes, world: int, rank: int) -> list[int]:
    """Members of one rank under a size-balanced greedy partition: largest first, each to the rank
    with the fewest cells so far (ties to the lower rank).  Every rank computes the same
    partition; the members of a rank keep their ensemble order."""
    load = [0] * world
    owner = [0] * len(sizes)
    for k in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += sizes[k]
    return [k for k in range(len(sizes)) if owner[k] == rank]


def gather_results(local: dict, world: int) -> dict:
    """Member index -> result over all ranks (torch.distributed all_gather_object; the only
    exchange of a sharded ensemble, once per run)."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, local)
    out = {}
    for p in parts:
        out.update(p)
    return out
