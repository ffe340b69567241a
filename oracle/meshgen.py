"""Inputs for the reference arm of bench.py without the product library -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of what the product's mesh builder (discrete_adjoint_b200/csrc/mesh_host.cpp,
da_mesh_build) produces for a uniform mesh: Morton order, neighbour table, cell geometry, the
terrain fields sampled from a DEM (Sobel slopes and curvatures on the posts in float32, bilinear
sampling), the gravity vector and its derivatives (Element::calc_gravity_vector / calc_d_gravity,
src/datstr/element2.C:3545-3653) and the paraboloid piles (elliptical_pile_height,
src/main/init_piles.C:167-277).  It lets the reference arm build the headline workload's mesh
without loading libda_b200.so; tests/test_meshgen.py checks it against the product builder bit
for bit.  Transcendental functions go through Python's math module (the C library), as the
builder's do.
"""
from __future__ import annotations

import math

import numpy as np

TINY = 1.e-4


def _spread(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint64) & np.uint64(0x1FFFFFFF)
    for s, m in ((16, 0x0000FFFF0000FFFF), (8, 0x00FF00FF00FF00FF), (4, 0x0F0F0F0F0F0F0F0F),
                 (2, 0x3333333333333333), (1, 0x5555555555555555)):
        v = (v | (v << np.uint64(s))) & np.uint64(m)
    return v


def _sobel(g: np.ndarray, res: float):
    """Sobel gradient (float32, the builder's operation order), edges replicated from inside."""
    f = np.float32
    inv = f(8.0) * f(res)
    gx = np.zeros_like(g)
    gy = np.zeros_like(g)
    a = g
    gx[1:-1, 1:-1] = (((a[:-2, 2:] - a[:-2, :-2]) + f(2.0) * (a[1:-1, 2:] - a[1:-1, :-2])) +
                      (a[2:, 2:] - a[2:, :-2])) / inv
    gy[1:-1, 1:-1] = (((a[:-2, :-2] - a[2:, :-2]) + f(2.0) * (a[:-2, 1:-1] - a[2:, 1:-1])) +
                      (a[:-2, 2:] - a[2:, 2:])) / inv
    for o in (gx, gy):
        o[0, 1:-1] = o[1, 1:-1]
        o[-1, 1:-1] = o[-2, 1:-1]
        o[:, 0] = o[:, 1]
        o[:, -1] = o[:, -2]
    return gx, gy


def _bilinear(g: np.ndarray, x: np.ndarray, y: np.ndarray) -> np.ndarray:
    nrows, ncols = g.shape
    x = np.clip(x, 0, ncols - 1)
    y = np.clip(y, 0, nrows - 1)
    c = np.minimum(x.astype(np.int64), ncols - 2)
    r = np.minimum(y.astype(np.int64), nrows - 2)
    fx, fy = x - c, y - r
    gd = g.astype(np.float64)
    p1 = gd[r, c] * (1.0 - fy) + gd[r + 1, c] * fy
    p2 = gd[r, c + 1] * (1.0 - fy) + gd[r + 1, c + 1] * fy
    return p1 * (1.0 - fx) + p2 * fx


def uniform_mesh(xmin, ymin, dx0, dy0, nx0, ny0, max_level, elev, dem_xmin, dem_ymin, dem_res, piles,
                 gravity_scale: float = 1.0) -> dict:
    """Arrays of the uniform mesh (every leaf at max_level) in the layout of Mesh.arrays().
    elev: float32 DEM posts, row 0 the northern edge; piles: (xc, yc, height, major, minor)."""
    L = max_level
    nxl, nyl = nx0 << L, ny0 << L
    dx, dy = math.ldexp(dx0, -L), math.ldexp(dy0, -L)
    J, I = np.meshgrid(np.arange(nyl, dtype=np.int64), np.arange(nxl, dtype=np.int64), indexing="ij")
    I, J = I.ravel(), J.ravel()
    key = _spread(I) | (_spread(J) << np.uint64(1))
    order = np.argsort(key, kind="stable")
    I, J = I[order], J[order]
    n = I.size
    index = np.empty(nxl * nyl, dtype=np.int64)
    index[J * nxl + I] = np.arange(n)
    nbr = np.full((8, n), -1, dtype=np.int32)
    for s, (di, dj) in enumerate(((1, 0), (0, 1), (-1, 0), (0, -1))):
        ni, nj = I + di, J + dj
        ok = (ni >= 0) & (nj >= 0) & (ni < nxl) & (nj < nyl)
        nbr[s, ok] = index[nj[ok] * nxl + ni[ok]]
        nbr[s + 4] = nbr[s]
    x = xmin + (I.astype(np.float64) + 0.5) * dx
    y = ymin + (J.astype(np.float64) + 0.5) * dy
    # terrain: Sobel slopes and curvatures of the posts, bilinear at the cell centres
    e32 = np.ascontiguousarray(elev, dtype=np.float32)
    nrows = e32.shape[0]
    xs, ys = _sobel(e32, dem_res)
    kx, _ = _sobel(xs, dem_res)
    _, ky = _sobel(ys, dem_res)
    ymax = dem_ymin + (nrows - 1) * dem_res
    px, py = (x - dem_xmin) / dem_res, (ymax - y) / dem_res
    elevation = _bilinear(e32, px, py)
    zx, zy = _bilinear(xs, px, py), _bilinear(ys, px, py)
    cx, cy = _bilinear(kx, px, py), _bilinear(ky, px, py)
    # Element::calc_gravity_vector
    slope = np.sqrt(zx * zx + zy * zy)
    ang = np.array([math.atan(v) for v in slope])
    down = 9.8 * np.array([math.sin(v) for v in ang])
    cosa = np.array([math.cos(v) for v in ang])
    steep = np.abs(down) > TINY
    with np.errstate(invalid="ignore", divide="ignore"):
        g0 = np.where(steep, -down * zx / slope, 0.0)
        g1 = np.where(steep, -down * zy / slope, 0.0)
    g2 = np.where(steep, 9.8 * cosa, 9.8)
    grav = np.stack([g0 / gravity_scale, g1 / gravity_scale, g2 / gravity_scale])
    # Element::calc_d_gravity: weighted central difference of g_z, one-sided at the edges
    gz = grav[2]
    dgrav = np.zeros((2, n))
    for d, co in ((0, x), (1, y)):
        ep, em = nbr[d], nbr[d + 2]
        both, onlym, onlyp = (ep >= 0) & (em >= 0), (ep < 0) & (em >= 0), (ep >= 0) & (em < 0)
        epc, emc = np.maximum(ep, 0), np.maximum(em, 0)
        dxp = co[epc] - co
        dxm = co - co[emc]
        with np.errstate(invalid="ignore", divide="ignore"):
            dp = (gz[epc] - gz) / dxp
            dm = (gz - gz[emc]) / dxm
            v = np.where(both, (dp * dxm + dm * dxp) / (dxm + dxp), 0.0)
            v = np.where(onlym, (gz - gz[emc]) / (co - co[emc]), v)
            v = np.where(onlyp, (gz[epc] - gz) / (co[epc] - co), v)
        dgrav[d] = v
    # piles: the 9-node weighted paraboloid
    NX = (-0.5, 0.5, 0.5, -0.5, 0.0, 0.5, 0.0, -0.5, 0.0)
    NY = (-0.5, -0.5, 0.5, 0.5, -0.5, 0.0, 0.5, 0.0, 0.0)
    W = (1, 1, 1, 1, 2, 2, 2, 2, 4)
    hn, dP = [], np.zeros((len(piles), 9, n))
    for q in range(9):
        ndx, ndy = x + NX[q] * dx, y + NY[q] * dy
        node_h = np.zeros(n)
        arg = np.full(n, -1)
        for p, (xc, yc, hgt, major_r, minor_r) in enumerate(piles):
            major = (ndx - xc) * 1.0 + (ndy - yc) * 0.0
            sw = major / major_r
            minor = (-(ndx - xc) * 0.0 + (ndy - yc) * 1.0) / minor_r
            height = hgt * (1. - sw * sw - minor * minor)
            height = np.where(height >= 0.0, height, 0.0)
            up = node_h < height
            node_h = np.where(up, height, node_h)
            arg = np.where(up, p, arg)
        for p, (xc, yc, hgt, major_r, minor_r) in enumerate(piles):
            sw = ((ndx - xc) * 1.0 + (ndy - yc) * 0.0) / major_r
            minor = (-(ndx - xc) * 0.0 + (ndy - yc) * 1.0) / minor_r
            dP[p, q] = np.where(arg == p, 1. - sw * sw - minor * minor, 0.0)
        hn.append(node_h)
    h0 = (hn[0] + hn[1] + hn[2] + hn[3] + 2.0 * (hn[4] + hn[5] + hn[6] + hn[7]) + 4.0 * hn[8]) / 16.0
    dh0 = np.zeros((len(piles), n))
    for p in range(len(piles)):
        acc = np.zeros(n)
        for q in range(9):
            acc = acc + W[q] * dP[p, q]
        dh0[p] = acc / 16.0
    return dict(n=np.int64(n), max_level=np.int64(L), nbr=nbr, material=np.zeros(n, dtype=np.int32),
                level=np.full(n, L, dtype=np.int32), ix=I.astype(np.int32), iy=J.astype(np.int32), x=x, y=y,
                dx=np.full(n, dx), dy=np.full(n, dy), elevation=elevation, zeta=np.stack([zx, zy]), curvature=np.stack([cx, cy]),
                gravity=grav, d_gravity=dgrav, h0=h0, hu0=np.zeros(n), hv0=np.zeros(n), dh0_dpile=dh0)


def headline_mesh(cells_per_side: int = 1024) -> dict:
    """The headline workload's mesh (the plane-and-runout terrain on 5 km x 5 km, uniform at
    cells_per_side^2, the 30 m x 100 m pile 300 m downslope of the top) -- the same arrays as
    discrete_adjoint_b200.inputs.workload3(cells_per_side).mesh."""
    from discrete_adjoint_b200.inputs import inclined_plane
    L = 5000.0
    dem = inclined_plane(L, L, 5.0, 30.0, 3000.0)
    base = cells_per_side // 16
    return uniform_mesh(0.0, 0.0, L / base, L / base, base, base, 4, dem.elev, dem.xmin, dem.ymin, dem.res,
                        [(300.0, 2500.0, 30.0, 100.0, 100.0)])
