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

Interpolants of a fine cell (bilinear_interp.C:125-290, bilinear_interp_elem :424-556): four
fine cells chosen around its family (the four sons of its father) by the reference's own walk
over neighbour slots -- Element::get_side_neighbor (element2.C:4224-4330) with the side pairs in the
element's counter-clockwise order, and the equality tests of bilinear_interp -- each standing for
its father (centre and values); missing ones at domain edges drop out and fathers met twice count
once.  Four points: the bilinear polynomial a + b x + c y + d x y through them (the reference
solves the 4 x 4 system with dgesv); three: barycentric weights; two: the reference's
linear_interp (:350-353), which returns (f2 - f1) (x - x1) / (x2 - x1) without the f1 term, is
kept as is; one: the value itself.
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


def _ccw_pairs(m: Mesh):
    """First and second neighbour of every cell across each relative side (0 +x, 1 +y, 2 -x, 3 -y)
    in the order an element keeps them: counter-clockwise around its boundary
    (adapt/refine2.C:590-805) -- +x lower then upper, +y right then left, -x upper then lower,
    -y left then right -- where the table lists the lower / left one first.  -1 at a domain edge."""
    nb = m.nbr.astype(np.int64)
    first = np.stack([nb[0], nb[5], nb[6], nb[3]])
    second = np.stack([nb[4], nb[1], nb[2], nb[7]])
    return first, second


def _side_neighbor(first, second, cells: np.ndarray, k: int) -> np.ndarray:
    """Element::get_side_neighbor (src/datstr/element2.C:4224-4330) for every cell of `cells`
    (-1 = none): 0-3 the first neighbour across +x, +y, -x, -y; 4-6 the second one across +x, +y,
    -x when the side has two, else the first; 7 always the second across -y (its test,
    neigh_proc[ym] < INIT, never holds, and a side with one neighbour stores it twice); 8-11 the
    diagonal cells reached through +y then +x, -x then +y, -y then -x, +x then -y."""
    ok = cells >= 0
    c = np.where(ok, cells, 0)
    if k < 4:
        out = first[k][c]
    elif k < 7:
        r = k - 4
        out = np.where(first[r][c] != second[r][c], second[r][c], first[r][c])
    elif k == 7:
        out = second[3][c]
    else:
        via, then = {8: (1, 0), 9: (2, 1), 10: (3, 2), 11: (0, 3)}[k]
        out = _side_neighbor(first, second, _side_neighbor(first, second, cells, via), then)
    return np.where(ok, out, -1)


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
    # the four sons of every father, counter-clockwise from the lower left (which_son 0..3)
    fk = _keys(fine.level, fine.ix, fine.iy)
    forder = np.argsort(fk)
    s0 = np.flatnonzero(((fine.ix & 1) == 0) & ((fine.iy & 1) == 0))
    sons = [s0]
    for dx, dy in ((1, 0), (1, 1), (0, 1)):
        k = _keys(fine.level[s0], fine.ix[s0] + dx, fine.iy[s0] + dy)
        sons.append(forder[np.searchsorted(fk[forder], k)])
    first, second = _ccw_pairs(fine)

    def nb(cells, k):
        return _side_neighbor(first, second, cells, k)

    def two(cells, r):   # the side carries two finer neighbours (neigh_proc[side + 4] >= 0)
        return first[r][cells] != second[r][cells]

    # the twelve cells around a family (bilinear_interp.C:140-180)
    N = {3: nb(sons[0], 3), 6: nb(sons[0], 6), 10: nb(sons[0], 10), 0: nb(sons[1], 0), 7: nb(sons[1], 7),
         11: nb(sons[1], 11), 8: nb(sons[2], 8), 4: nb(sons[2], 4), 1: nb(sons[2], 1), 5: nb(sons[3], 5),
         9: nb(sons[3], 9), 2: nb(sons[3], 2)}

    def same(a, b):
        return (N[a] >= 0) & (N[b] >= 0) & (N[a] == N[b])

    def pick(cond, x, y):
        return [np.where(cond, p, q) for p, q in zip(x, y)]

    # the four elements bilinear_interp_elem receives for each son (bilinear_interp.C:182-270)
    S = sons
    args = [None] * 4
    a0 = pick(~two(S[0], 2), [N[10], N[3], N[9], S[0]], [N[10], N[3], N[2], S[0]])
    b0 = pick(~two(S[0], 3), [N[10], N[11], N[6], S[0]], [N[10], N[7], N[6], S[0]])
    args[0] = pick(same(6, 10), a0, pick(same(3, 10), b0, [N[10], N[3], N[6], S[0]]))
    a1 = pick(~two(S[1], 0), [N[7], N[11], S[1], N[8]], [N[7], N[11], S[1], N[4]])
    b1 = pick(~two(S[1], 3), [N[10], N[11], S[1], N[0]], [N[3], N[11], S[1], N[0]])
    args[1] = pick(same(11, 0), a1, pick(same(7, 11), b1, [N[7], N[11], S[1], N[0]]))
    a2 = pick(~two(S[2], 0), [S[2], N[11], N[1], N[8]], [S[2], N[0], N[1], N[8]])
    b2 = pick(~two(S[2], 1), [S[2], N[4], N[9], N[8]], [S[2], N[4], N[5], N[8]])
    args[2] = pick(same(4, 8), a2, pick(same(8, 1), b2, [S[2], N[4], N[1], N[8]]))
    a3 = pick(~two(S[3], 2), [N[10], S[3], N[9], N[5]], [N[6], S[3], N[9], N[5]])
    b3 = pick(~two(S[3], 1), [N[2], S[3], N[9], N[8]], [N[2], S[3], N[9], N[1]])
    args[3] = pick(same(9, 2), a3, pick(same(9, 5), b3, [N[2], S[3], N[9], N[5]]))
    nf = fine.n
    cand = np.full((4, nf), -1, dtype=np.int64)
    for j in range(4):
        for q in range(4):
            el = args[j][q]
            cand[q, S[j]] = np.where(el >= 0, parent[np.maximum(el, 0)], -1)   # the element's father
    interp = np.full((4, nf), -1, dtype=np.int32)
    weight = np.zeros((4, nf))
    # the regular case (four distinct fathers on the corners of an axis-aligned rectangle, in the
    # order lower left, lower right, upper left, upper right) in closed form; the rest point by point
    cx, cy = coarse.x, coarse.y
    fx, fy = fine.x, fine.y
    rect = np.all(cand >= 0, axis=0)
    r = np.flatnonzero(rect)
    c0, c1, c2, c3 = (cand[q, r] for q in range(4))
    rect[r] = (cx[c0] == cx[c2]) & (cx[c1] == cx[c3]) & (cy[c0] == cy[c1]) & (cy[c2] == cy[c3]) & \
        (cx[c1] > cx[c0]) & (cy[c2] > cy[c0])
    r = np.flatnonzero(rect)
    x0, x1 = cx[cand[0, r]], cx[cand[1, r]]
    y0, y1 = cy[cand[0, r]], cy[cand[2, r]]
    tx = (fx[r] - x0) / (x1 - x0)
    ty = (fy[r] - y0) / (y1 - y0)
    interp[:, r] = cand[:, r]
    weight[0, r] = (1 - tx) * (1 - ty)
    weight[1, r] = tx * (1 - ty)
    weight[2, r] = (1 - tx) * ty
    weight[3, r] = tx * ty
    for f in np.flatnonzero(~rect):
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
