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

    def edge_fluxes(self, h, hu, hv, kact):
        F = np.zeros((4, 3, self.mesh.n))
        self.lib.orc_edge_fluxes(C.byref(self.params), C.byref(self.soa), _ffi.dptr(h), _ffi.dptr(hu),
                                 _ffi.dptr(hv), _ffi.dptr(kact), _ffi.dptr(F))
        return F
