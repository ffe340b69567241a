"""Dual-weighted-residual (DWR) error indicator: the error grid and its interpolation weights.

The reference's estimate (src/adjoint/dual_solver.C:146-170, 213-230) refines every element once
(uniform_refine.C:24-130), reconstructs on the refined grid the previous and current state and the
adjoint from the coarse cell centres (bilinear_interp.C:125-556), takes one step of the refined
grid with the coarse dt (update_bilinear_error_grid, error_grid_routines.C:13-55), and weights
the residual r = update(U~^{n-1}) - U~^n by the adjoint (error_compute.C:24-119):
    el_error = sum_j |r_j (lambda_j - lambda~_j)|,   correction = sum_j r_j lambda_j,
lambda the coarse adjoint carried to the four children, lambda~ its bilinear reconstruction.

Here the error grid is the mesh builder's mesh with one extra level everywhere (da_mesh_spec
extra_level; its terrain data come from the DEM as the reference's refined elements' do), and
the reconstruction is a fixed linear map, so it is computed once per mesh as four (coarse cell,
weight) pairs per fine cell; the device applies it (da_dwr_setup / da_dwr_step).

Interpolants of a fine cell (bilinear_interp.C:125-260, bilinear_interp_elem :424-556): the
centres of its parent, of the parent's neighbour towards the fine cell in x, in y, and of the
diagonal cell between them; the ones missing at domain edges drop out and coincident ones count
once.  Four points: the bilinear polynomial a + b x + c y + d x y through them (the reference
solves the 4 x 4 system with dgesv); three: barycentric weights; two: the reference's
linear_interp (:350-353), which returns (f2 - f1) (x - x1) / (x2 - x1) without the f1 term, is
kept as is; one: the value itself.  Where a neighbour is split in two across the side, the half
nearest the fine cell's centre is taken (the reference walks its hash-table keys to the same
element on regular neighbourhoods).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass

import numpy as np

from .mesh import Mesh


@dataclass
class ErrorGrid:
    fine: Mesh
    parent: np.ndarray   # [nf] coarse cell of each fine cell
    interp: np.ndarray   # [4][nf] coarse cells of the interpolants, -1 unused
    weight: np.ndarray   # [4][nf]


def _keys(level, ix, iy) -> np.ndarray:
    return (level.astype(np.uint64) << np.uint64(58)) | (ix.astype(np.uint64) << np.uint64(29)) | iy.astype(np.uint64)


def _side_pick(m: Mesh, cells: np.ndarray, side: int, fx: np.ndarray, fy: np.ndarray) -> np.ndarray:
    """Neighbour of each cell across side (0 +x, 1 +y, 2 -x, 3 -y) nearest to the points (fx, fy);
    -1 on the domain edge or for cells = -1."""
    out = np.full(cells.shape, -1, dtype=np.int64)
    ok = cells >= 0
    c = cells[ok]
    a = m.nbr[side][c].astype(np.int64)
    b = m.nbr[side + 4][c].astype(np.int64)
    pick = a.copy()
    two = (a != b) & (a >= 0)
    if np.any(two):
        px, py = fx[ok][two], fy[ok][two]
        da = (m.x[a[two]] - px) ** 2 + (m.y[a[two]] - py) ** 2
        db = (m.x[b[two]] - px) ** 2 + (m.y[b[two]] - py) ** 2
        pick[two] = np.where(db < da, b[two], a[two])
    out[ok] = pick
    return out


def weights_for(points_x, points_y, xf, yf) -> np.ndarray:
    """Reconstruction weights of one fine centre from 1-4 distinct coarse centres."""
    k = len(points_x)
    if k == 1:
        return np.array([1.0])
    if k == 2:
        order = sorted(range(2), key=lambda q: (points_x[q], points_y[q]))
        x1, x2 = points_x[order[0]], points_x[order[1]]
        y1, y2 = points_y[order[0]], points_y[order[1]]
        t = (yf - y1) / (y2 - y1) if x2 - x1 < 1e-12 else (xf - x1) / (x2 - x1)
        w = np.zeros(2)
        w[order[0]], w[order[1]] = -t, t
        return w
    if k == 3:
        (x1, x2, x3), (y1, y2, y3) = points_x, points_y
        inv_det = 1.0 / ((y2 - y3) * (x1 - x3) + (x3 - x2) * (y1 - y3))
        l1 = ((y2 - y3) * (xf - x3) + (x3 - x2) * (yf - y3)) * inv_det
        l2 = ((y3 - y1) * (xf - x3) + (x1 - x3) * (yf - y3)) * inv_det
        return np.array([l1, l2, 1.0 - l1 - l2])
    A = np.stack([np.ones(4), np.asarray(points_x), np.asarray(points_y),
                  np.asarray(points_x) * np.asarray(points_y)], axis=1)
    row = np.array([1.0, xf, yf, xf * yf])
    return np.linalg.solve(A.T, row)  # w such that w . f = row . A^-1 f


def error_grid(w) -> ErrorGrid:
    """The error grid of a workload built by inputs.* (it keeps its MeshSpec and DEM)."""
    if w.spec is None:
        raise ValueError("the workload does not carry its mesh spec")
    coarse = w.mesh
    fine = Mesh.build(dataclasses.replace(w.spec, extra_level=True), w.dem, w.piles)
    ck = _keys(coarse.level, coarse.ix, coarse.iy)
    order = np.argsort(ck)
    pk = _keys(fine.level - 1, fine.ix >> 1, fine.iy >> 1)
    pos = np.searchsorted(ck[order], pk)
    parent = order[np.minimum(pos, len(ck) - 1)]
    if not np.array_equal(ck[parent], pk):
        raise ValueError("the fine grid is not the coarse mesh refined once")
    a = fine.ix & 1
    b = fine.iy & 1
    fx, fy = fine.x, fine.y
    nx = _side_pick(coarse, parent.astype(np.int64), 0, fx, fy)
    nx = np.where(a == 1, nx, _side_pick(coarse, parent.astype(np.int64), 2, fx, fy))
    ny = _side_pick(coarse, parent.astype(np.int64), 1, fx, fy)
    ny = np.where(b == 1, ny, _side_pick(coarse, parent.astype(np.int64), 3, fx, fy))
    dy_side = np.where(b == 1, 1, 3)
    dx_side = np.where(a == 1, 0, 2)
    diag = np.full_like(nx, -1)
    for sd in (1, 3):
        sel = (dy_side == sd) & (nx >= 0)
        diag[sel] = _side_pick(coarse, nx[sel], sd, fx[sel], fy[sel])
    for sd in (0, 2):
        sel = (dx_side == sd) & (nx < 0) & (ny >= 0)
        diag[sel] = _side_pick(coarse, ny[sel], sd, fx[sel], fy[sel])
    cand = np.stack([parent.astype(np.int64), nx, ny, diag])
    nf = fine.n
    interp = np.full((4, nf), -1, dtype=np.int32)
    weight = np.zeros((4, nf))
    # the regular case (four distinct interpolants on the corners of an axis-aligned rectangle) in
    # closed form; the rest point by point
    regular = np.all(cand >= 0, axis=0)
    regular &= (cand[0] != cand[1]) & (cand[0] != cand[2]) & (cand[0] != cand[3]) & (cand[1] != cand[2]) & \
        (cand[1] != cand[3]) & (cand[2] != cand[3])
    cx, cy = coarse.x, coarse.y
    rect = regular.copy()
    r = np.where(rect)[0]
    rect[r] = (np.abs(cx[cand[0, r]] - cx[cand[2, r]]) < 1e-12) & (np.abs(cx[cand[1, r]] - cx[cand[3, r]]) < 1e-12) & \
        (np.abs(cy[cand[0, r]] - cy[cand[1, r]]) < 1e-12) & (np.abs(cy[cand[2, r]] - cy[cand[3, r]]) < 1e-12)
    r = np.where(rect)[0]
    x0, x1 = cx[cand[0, r]], cx[cand[1, r]]
    y0, y1 = cy[cand[0, r]], cy[cand[2, r]]
    tx = (fx[r] - x0) / (x1 - x0)
    ty = (fy[r] - y0) / (y1 - y0)
    interp[:, r] = cand[:, r]
    weight[0, r] = (1 - tx) * (1 - ty)
    weight[1, r] = tx * (1 - ty)
    weight[2, r] = (1 - tx) * ty
    weight[3, r] = tx * ty
    for f in np.where(~rect)[0]:
        pts = []
        for c in cand[:, f]:
            if c < 0:
                continue
            if any(abs(cx[c] - cx[q]) < 1e-12 and abs(cy[c] - cy[q]) < 1e-12 for q in pts):
                continue
            pts.append(int(c))
        wv = weights_for([cx[q] for q in pts], [cy[q] for q in pts], fx[f], fy[f])
        interp[: len(pts), f] = pts
        weight[: len(pts), f] = wv
    return ErrorGrid(fine, parent.astype(np.int32), interp, weight)


class Indicator:
    """The DWR indicator of a context's mesh (da_dwr_setup / da_dwr_step)."""

    def __init__(self, ctx, grid: ErrorGrid):
        from . import _ffi
        self.ctx, self.grid = ctx, grid
        self._parent = np.ascontiguousarray(grid.parent, dtype=np.int32)
        self._interp = np.ascontiguousarray(grid.interp, dtype=np.int32)
        self._weight = np.ascontiguousarray(grid.weight, dtype=np.float64)
        ctx._check(ctx.lib.da_dwr_setup(ctx.ctx, _ffi.C.byref(grid.fine.soa()), _ffi.iptr(self._parent),
                                        _ffi.iptr(self._interp), _ffi.dptr(self._weight)), "da_dwr_setup")

    def step(self, lambda_next):
        """(el_error per fine cell, per coarse cell, (total el_error, total correction)) of the step
        from the context's current state; lambda_next = dJ/dU^{n+1} as [3][n]."""
        from . import _ffi
        n, nf = self.ctx.mesh.n, self.grid.fine.n
        lam = np.ascontiguousarray(lambda_next, dtype=np.float64).reshape(3 * n)
        el, cell, sums = np.empty(nf), np.empty(n), np.empty(2)
        self.ctx._check(self.ctx.lib.da_dwr_step(self.ctx.ctx, _ffi.dptr(lam), _ffi.dptr(el), _ffi.dptr(cell),
                                                 _ffi.dptr(sums)), "da_dwr_step")
        return el, cell, (float(sums[0]), float(sums[1]))
