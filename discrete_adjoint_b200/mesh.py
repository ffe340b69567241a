"""Flattened quadtree mesh on the host (numpy), built by the native builder in libda_b200.

A Mesh holds the structure-of-arrays the device path consumes (neighbour table in the
layout of include/discrete_adjoint.h, cell geometry and the static per-cell fields) plus
the initial state from the piles.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _ffi

_ARRAYS_F64 = ("x", "y", "dx", "dy", "elevation", "h0", "hu0", "hv0")
_ARRAYS_2D = {"zeta": 2, "curvature": 2, "gravity": 3, "d_gravity": 2}


@dataclass
class Pile:
    """PileProps of one paraboloid pile (src/header/properties.h:199-270)."""
    xc: float
    yc: float
    height: float
    major: float
    minor: float
    rot_deg: float = 0.0
    vx: float = 0.0
    vy: float = 0.0


@dataclass
class DEM:
    """Elevation raster in GRASS layout: row 0 is the northern edge."""
    elev: np.ndarray            # float32 [nrows, ncols]
    xmin: float
    ymin: float
    res: float
    mat: np.ndarray | None = None  # int32 [nrows, ncols], 0-based material ids


@dataclass
class MeshSpec:
    xmin: float
    ymin: float
    dx0: float
    dy0: float
    nx0: int
    ny0: int
    max_level: int
    uniform: bool = False
    refine_margin: float = 0.0
    boxes: list = field(default_factory=list)   # [(xmin, xmax, ymin, ymax), ...]
    random_frac: float = 0.0
    seed: int = 0
    extra_level: bool = False   # split every leaf once more after balancing (DWR error grid)


class Mesh:
    """Host SoA mesh.  Arrays are numpy-owned; soa() gives a C view for da_upload_mesh."""

    def __init__(self, **arrays):
        self.n = int(arrays["n"])
        self.max_level = int(arrays.get("max_level", 0))
        self.nbr = np.ascontiguousarray(arrays["nbr"], dtype=np.int32).reshape(8, self.n)
        self.material = np.ascontiguousarray(arrays["material"], dtype=np.int32)
        self.level = np.ascontiguousarray(arrays.get("level", np.zeros(self.n)), dtype=np.int32)
        self.ix = np.ascontiguousarray(arrays.get("ix", np.zeros(self.n)), dtype=np.int32)
        self.iy = np.ascontiguousarray(arrays.get("iy", np.zeros(self.n)), dtype=np.int32)
        for k in _ARRAYS_F64:
            v = arrays.get(k)
            if v is None:
                v = np.zeros(self.n)
            setattr(self, k, np.ascontiguousarray(v, dtype=np.float64))
        for k, r in _ARRAYS_2D.items():
            v = arrays.get(k)
            if v is None:
                v = np.zeros((r, self.n))
            setattr(self, k, np.ascontiguousarray(v, dtype=np.float64).reshape(r, self.n))
        dp = arrays.get("dh0_dpile")
        self.dh0_dpile = (np.zeros((0, self.n)) if dp is None
                          else np.ascontiguousarray(dp, dtype=np.float64).reshape(-1, self.n))
        self._soa = None

    # ------------------------------------------------------------------ construction
    @classmethod
    def build(cls, spec: MeshSpec, dem: DEM | None = None, piles: list[Pile] | tuple = (),
              length_scale: float = 1.0, gravity_scale: float = 1.0) -> "Mesh":
        lib = _ffi.load()
        boxes = np.ascontiguousarray(np.array(spec.boxes, dtype=np.float64).reshape(-1))
        cs = _ffi.da_mesh_spec(spec.xmin, spec.ymin, spec.dx0, spec.dy0, spec.nx0, spec.ny0, spec.max_level,
                               int(spec.uniform), spec.refine_margin, len(spec.boxes),
                               _ffi.dptr(boxes) if len(spec.boxes) else None, spec.random_frac, spec.seed,
                               int(spec.extra_level), 0)
        cdem = None
        keep = []
        if dem is not None:
            elev = np.ascontiguousarray(dem.elev, dtype=np.float32)
            mat = None if dem.mat is None else np.ascontiguousarray(dem.mat, dtype=np.int32)
            keep += [elev, mat]
            cdem = _ffi.da_dem(elev.shape[0], elev.shape[1], dem.xmin, dem.ymin, dem.res, _ffi.fptr(elev),
                               _ffi.iptr(mat) if mat is not None else None)
        cp = (_ffi.da_pile_spec * max(len(piles), 1))()
        for k, p in enumerate(piles):
            cp[k] = _ffi.da_pile_spec(p.xc, p.yc, p.height, p.major, p.minor, p.rot_deg, p.vx, p.vy)
        out = C.POINTER(_ffi.da_mesh_host)()
        st = lib.da_mesh_build(C.byref(cs), C.byref(cdem) if cdem is not None else None, cp, len(piles),
                               length_scale, gravity_scale, C.byref(out))
        if st != 0:
            raise _ffi.DAError(st, "da_mesh_build failed")
        try:
            h = out.contents
            n = h.n_cells

            def arr(ptr, count, dt):
                return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt, copy=True)

            arrays = dict(n=n, max_level=h.max_level)
            for k in ("level", "ix", "iy", "material"):
                arrays[k] = arr(getattr(h, k), n, np.int32)
            arrays["nbr"] = arr(h.nbr, 8 * n, np.int32)
            for k in _ARRAYS_F64:
                arrays[k] = arr(getattr(h, k), n, np.float64)
            for k, r in _ARRAYS_2D.items():
                arrays[k] = arr(getattr(h, k), r * n, np.float64)
            arrays["dh0_dpile"] = arr(h.dh0_dpile, max(len(piles), 1) * n, np.float64)[: len(piles) * n]
        finally:
            lib.da_mesh_free(out)
        return cls(**arrays)

    # ------------------------------------------------------------------ views
    def soa(self) -> _ffi.da_mesh_soa:
        if self._soa is None:
            self._soa = _ffi.da_mesh_soa(
                self.n, _ffi.iptr(self.nbr), _ffi.dptr(self.x), _ffi.dptr(self.y), _ffi.dptr(self.dx),
                _ffi.dptr(self.dy), _ffi.dptr(self.gravity), _ffi.dptr(self.d_gravity),
                _ffi.dptr(self.curvature), _ffi.iptr(self.material))
        return self._soa

    def arrays(self) -> dict:
        d = dict(n=np.int64(self.n), max_level=np.int64(self.max_level), nbr=self.nbr, material=self.material,
                 level=self.level, ix=self.ix, iy=self.iy, dh0_dpile=self.dh0_dpile)
        for k in _ARRAYS_F64:
            d[k] = getattr(self, k)
        for k in _ARRAYS_2D:
            d[k] = getattr(self, k)
        return d

    def save(self, path: str) -> None:
        np.savez_compressed(path, **self.arrays())

    @classmethod
    def load(cls, path: str) -> "Mesh":
        z = np.load(path)
        return cls(**{k: z[k] for k in z.files})

    def two_neighbour_sides(self) -> int:
        return int(np.sum((self.nbr[4:] != self.nbr[:4]) & (self.nbr[:4] >= 0)))

    def boundary_cells(self) -> np.ndarray:
        return np.any(self.nbr[:4] < 0, axis=0)
