"""Seeded synthetic inputs (terrain rasters, piles, mesh specs) for the benchmark workloads.

The reference runs on GIS rasters (the Colima DEM its driver points at is not available);
these generators stand in with the shapes, sizes and value ranges of each workload:
  inclined_plane : a plane of given slope meeting a flat runout (workloads 1, 3, 4)
  hill_noise     : Gaussian hill plus seeded 1/f^2 spectral noise (workload 2)
  fractal        : seeded fractal (spectral, Hurst exponent H) terrain (workload 5)
All generators use numpy.random.default_rng(seed).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .mesh import DEM, Mesh, MeshSpec, Pile
from .solver import MatProps


def _posts(xmin, ymin, lx, ly, res):
    ncols = int(round(lx / res)) + 1
    nrows = int(round(ly / res)) + 1
    xs = xmin + res * np.arange(ncols)
    ys = ymin + res * np.arange(nrows)[::-1]  # row 0 = north edge
    return np.meshgrid(xs, ys)


def analytic_dem(fn, xmin: float, ymin: float, lx: float, ly: float, res: float, mat=None) -> DEM:
    X, Y = _posts(xmin, ymin, lx, ly, res)
    return DEM(elev=fn(X, Y).astype(np.float32), xmin=xmin, ymin=ymin, res=res, mat=mat)


def inclined_plane(lx: float, ly: float, res: float, slope_deg: float, x_break: float) -> DEM:
    """Plane descending in +x at slope_deg until x_break, flat beyond."""
    t = math.tan(math.radians(slope_deg))
    return analytic_dem(lambda X, Y: np.where(X < x_break, (x_break - X) * t, 0.0), 0.0, 0.0, lx, ly, res)


def spectral_noise(shape, beta: float, rms: float, rng) -> np.ndarray:
    """Gaussian random field with power spectrum ~ 1/f^beta, scaled to the given RMS."""
    ny, nx = shape
    fy = np.fft.fftfreq(ny)[:, None]
    fx = np.fft.rfftfreq(nx)[None, :]
    f = np.sqrt(fx * fx + fy * fy)
    f[0, 0] = 1.0
    amp = f ** (-beta / 2.0)
    amp[0, 0] = 0.0
    spec = amp * (rng.standard_normal(amp.shape) + 1j * rng.standard_normal(amp.shape))
    z = np.fft.irfft2(spec, s=(ny, nx))
    z *= rms / max(z.std(), 1e-30)
    return z


def hill_noise(lx: float, ly: float, res: float, relief: float, noise_rms: float, seed: int,
               n_zones: int = 4) -> DEM:
    rng = np.random.default_rng(seed)
    X, Y = _posts(0.0, 0.0, lx, ly, res)
    cx, cy = 0.5 * lx, 0.5 * ly
    sig = 0.22 * min(lx, ly)
    z = relief * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * sig * sig))
    z += spectral_noise(z.shape, 2.0, noise_rms, rng)
    mat = None
    if n_zones > 1:
        mat = ((X > cx).astype(np.int32) + 2 * (Y > cy).astype(np.int32)) % n_zones
    return DEM(elev=z.astype(np.float32), xmin=0.0, ymin=0.0, res=res, mat=mat)


def fractal(lx: float, ly: float, res: float, hurst: float, relief: float, seed: int) -> DEM:
    """Seeded fractal (fractional Brownian) surface of Hurst exponent hurst: power spectrum
    ~ 1/f^(2H + 2), scaled to the given relief."""
    rng = np.random.default_rng(seed)
    shape = (int(round(ly / res)) + 1, int(round(lx / res)) + 1)
    z = spectral_noise(shape, 2.0 * hurst + 2.0, 1.0, rng)
    z = (z - z.min()) / max(np.ptp(z), 1e-30) * relief
    return DEM(elev=z.astype(np.float32), xmin=0.0, ymin=0.0, res=res)


@dataclass
class Workload:
    name: str
    mesh: Mesh
    mat: MatProps
    piles: list
    nsteps: int
    spec: MeshSpec | None = None  # how the mesh was built (the DWR error grid rebuilds it one level finer)
    dem: DEM | None = None


def workload1(seed: int = 0) -> Workload:
    """2 km x 2 km, 10 m posts, 30 deg plane meeting a flat runout at x = 1.2 km; one 30 m x 100 m
    paraboloid pile 300 m downslope of the top; phi_bed 20, phi_int 30; ~40k active cells."""
    dem = inclined_plane(2000.0, 2000.0, 10.0, 30.0, 1200.0)
    piles = [Pile(300.0, 1000.0, 30.0, 100.0, 100.0)]
    spec = MeshSpec(xmin=0.0, ymin=0.0, dx0=40.0, dy0=40.0, nx0=50, ny0=50, max_level=2,
                    refine_margin=60.0, boxes=[(0.0, 2000.0, 100.0, 1900.0)])
    mesh = Mesh.build(spec, dem, piles)
    return Workload("inclined-plane 2km x 2km, 1 pile, adaptive (~40k cells)", mesh,
                    MatProps(intfrict_deg=30.0, bedfrict_deg=[20.0]), piles, 200, spec, dem)


def workload3(cells_per_side: int = 1024, seed: int = 0) -> Workload:
    """The plane-and-runout terrain (30 deg plane meeting a flat runout) on 5 km x 5 km at uniform
    resolution (1024^2 ~ 1M cells, 4.9 m), the 30 m x 100 m paraboloid pile 300 m downslope of the
    top, phi_bed 20, phi_int 30; 512 steps; J = sum of h^2 dx dy over a 500 m x 500 m box."""
    L = 5000.0
    dem = inclined_plane(L, L, 5.0, 30.0, 3000.0)
    piles = [Pile(300.0, 2500.0, 30.0, 100.0, 100.0)]
    base = cells_per_side // 16
    spec = MeshSpec(xmin=0.0, ymin=0.0, dx0=L / base, dy0=L / base, nx0=base, ny0=base, max_level=4, uniform=True)
    mesh = Mesh.build(spec, dem, piles)
    return Workload(f"inclined-plane 5km x 5km uniform {cells_per_side}^2, 1 pile", mesh,
                    MatProps(intfrict_deg=30.0, bedfrict_deg=[20.0]), piles, 512, spec, dem)


WORKLOAD3_BOX = (350.0, 850.0, 2250.0, 2750.0)


@dataclass
class MemberSpec:
    slope_deg: float
    volume: float      # pile volume, m^3
    bedfrict_deg: float
    side: int          # cells across (side^2 cells)


def ensemble_specs(n: int, seed: int = 4, min_side: int = 128, max_side: int = 512) -> list:
    """Seeded draws for an ensemble of inclined-plane runs: slope U(20, 35) deg, pile volume
    U(1e4, 1e6) m^3, basal friction U(12, 28) deg, uneven meshes of side U{min_side..max_side}
    (a multiple of 16) cells."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        out.append(MemberSpec(float(rng.uniform(20.0, 35.0)), float(rng.uniform(1.0e4, 1.0e6)),
                              float(rng.uniform(12.0, 28.0)), int(16 * rng.integers(min_side // 16, max_side // 16 + 1))))
    return out


def ensemble_member(spec: MemberSpec, intfrict_deg: float = 30.0):
    """(mesh, MatProps, pile, box) of one ensemble member: a plane of the drawn slope meeting a flat
    runout at mid-domain, a paraboloid pile (height 0.3 R, volume pi/2 H R^2, so R scales with
    volume^(1/3)) a fifth of the way down, a uniform mesh of side^2 cells over 24 R x 24 R, and the
    functional box from the pile's centre to 6 R downslope (where the flow's front is after a few
    hundred steps), 4.8 R wide."""
    R = (spec.volume / (0.15 * math.pi)) ** (1.0 / 3.0)
    L = 24.0 * R
    res = L / spec.side
    dem = inclined_plane(L, L, res, spec.slope_deg, 0.5 * L)
    pile = Pile(0.2 * L, 0.5 * L, 0.3 * R, R, R)
    base = spec.side // 16
    mesh_spec = MeshSpec(xmin=0.0, ymin=0.0, dx0=L / base, dy0=L / base, nx0=base, ny0=base, max_level=4, uniform=True)
    mesh = Mesh.build(mesh_spec, dem, [pile])
    mat = MatProps(intfrict_deg=intfrict_deg, bedfrict_deg=[spec.bedfrict_deg])
    box = (0.2 * L, 0.45 * L, 0.4 * L, 0.6 * L)
    return mesh, mat, pile, box


def test_case(seed: int = 1, nx0: int = 24, ny0: int = 16, max_level: int = 2, random_frac: float = 0.35,
              n_materials: int = 2) -> Workload:
    """Small seeded case with hanging nodes everywhere: bumpy slope, two piles, two materials."""
    rng = np.random.default_rng(seed)
    lx, ly = 40.0 * nx0, 40.0 * ny0
    amp = rng.uniform(5.0, 15.0, size=4)
    kx = rng.uniform(1.0, 3.0, size=4) * 2 * math.pi / lx
    ky = rng.uniform(1.0, 3.0, size=4) * 2 * math.pi / ly
    t = math.tan(math.radians(25.0))

    def z(X, Y):
        out = (lx - X) * t * 0.6
        for a, p, q in zip(amp, kx, ky):
            out = out + a * np.sin(p * X) * np.cos(q * Y)
        return out

    res = 10.0
    X, Y = _posts(0.0, 0.0, lx, ly, res)
    mat = ((X > 0.55 * lx).astype(np.int32) % n_materials) if n_materials > 1 else None
    dem = analytic_dem(z, 0.0, 0.0, lx, ly, res, mat=mat)
    piles = [Pile(0.3 * lx, 0.45 * ly, 25.0, 120.0, 90.0, rot_deg=20.0),
             Pile(0.45 * lx, 0.7 * ly, 15.0, 80.0, 80.0)]
    spec = MeshSpec(xmin=0.0, ymin=0.0, dx0=40.0, dy0=40.0, nx0=nx0, ny0=ny0, max_level=max_level,
                    refine_margin=40.0, random_frac=random_frac, seed=seed)
    mesh = Mesh.build(spec, dem, piles)
    bed = [20.0, 16.0][:n_materials]
    return Workload(f"test case seed {seed}", mesh, MatProps(intfrict_deg=32.0, bedfrict_deg=bed), piles, 50, spec, dem)


def workload2(seed: int = 2, target_cells: float = 4.0e6, res: float = 5.0) -> Workload:
    """20 km x 20 km at 5 m posts: 1.2 km Gaussian hill + seeded 1/f^2 noise (20 m RMS); three
    paraboloid piles (heights U(20,60) m, radii U(80,300) m); basal friction 15-25 deg over a
    4-zone material map; adaptive mesh refined to 5 m around the piles (~4M active cells)."""
    rng = np.random.default_rng(seed)
    L = 20000.0
    dem = hill_noise(L, L, res, 1200.0, 20.0, seed)
    piles = []
    for k in range(3):
        ang = 2 * math.pi * (k / 3.0) + rng.uniform(-0.3, 0.3)
        rr = rng.uniform(0.12, 0.2) * L
        r = rng.uniform(80.0, 300.0)
        piles.append(Pile(0.5 * L + rr * math.cos(ang), 0.5 * L + rr * math.sin(ang), rng.uniform(20.0, 60.0), r, r))
    max_level = 4
    base = 250  # 80 m base cells -> 5 m at level 4
    fine = (L / base / 2 ** max_level) ** 2
    # refinement disc radius such that three discs of finest cells hold ~target_cells
    radius = math.sqrt(target_cells * fine / (3 * math.pi))
    margin = max(radius - max(p.major for p in piles), 0.0)
    spec = MeshSpec(xmin=0.0, ymin=0.0, dx0=L / base, dy0=L / base, nx0=base, ny0=base, max_level=max_level,
                    refine_margin=margin)
    mesh = Mesh.build(spec, dem, piles)
    bed = [float(b) for b in rng.uniform(15.0, 25.0, size=4)]
    return Workload("hill+noise 20km x 20km, 3 piles, 4 materials, adaptive to 5 m", mesh,
                    MatProps(intfrict_deg=30.0, bedfrict_deg=bed), piles, 1000, spec, dem)


WORKLOAD5_SIDE = 8192


def workload5(seed: int = 5, crop: int | None = None, dem: DEM | None = None) -> Workload:
    """Large single instance: 40 km x 40 km of seeded fractal terrain (H = 0.8, 2 km relief) at
    5 m posts, uniform at the finest level (8192^2 = 67M cells of 4.88 m); two paraboloid piles
    near the centre (seeded heights and radii); phi_bed 20, phi_int 30; 2000 steps.  The flux
    source of the workload (1e3 m^3/s for 60 s) does not change the state in the reference
    (corrector.C:136-140) and enters dt only while no cell is wet, which never happens with two
    piles: it is carried as influx_dt (influx5_dt).

    crop: build only the crop x crop cells centred on the domain (same cell positions, same
    terrain, same piles).  Away from its edges a crop's cells have the same static fields as the
    full mesh's, so a flow that stays inside evolves identically on both.  dem: the terrain of an
    earlier call with the same seed (it takes a while to generate)."""
    rng = np.random.default_rng(seed)
    L = 40000.0
    if dem is None:
        dem = fractal(L, L, 5.0, 0.8, 2000.0, seed)
    d = L / WORKLOAD5_SIDE
    piles = []
    for k in range(2):
        ang = math.pi * k + rng.uniform(-0.4, 0.4)
        r = rng.uniform(80.0, 300.0)
        piles.append(Pile(0.5 * L + 900.0 * math.cos(ang), 0.5 * L + 900.0 * math.sin(ang), rng.uniform(20.0, 60.0),
                          r, r))
    side = WORKLOAD5_SIDE if crop is None else int(crop)
    if side % 16 or side > WORKLOAD5_SIDE:
        raise ValueError("crop must be a multiple of 16 up to the full side")
    x0 = 0.5 * L - 0.5 * side * d
    spec = MeshSpec(xmin=x0, ymin=x0, dx0=16 * d, dy0=16 * d, nx0=side // 16, ny0=side // 16, max_level=4,
                    uniform=True)
    mesh = Mesh.build(spec, dem, piles)
    name = f"fractal 40km x 40km (H 0.8, 2 km relief), uniform {side}^2" + ("" if crop is None else " crop")
    return Workload(name, mesh, MatProps(intfrict_deg=30.0, bedfrict_deg=[20.0]), piles, 2000, spec, dem)


def influx5_dt(mesh: Mesh, gravity_scale: float = 1.0, epsilon: float = 1.0, rate_m3s: float = 1.0e3,
               area_m2: float = 1.0e4) -> float:
    """dt[2] of get_coef_and_eigen.C:48-77 for the large workload's flux source while it is active:
    min(min_dx / influx, 0.81 influx g_s / 9.8) with influx = rate / area * epsilon (m/s)."""
    influx = rate_m3s / area_m2 * epsilon
    mindx = float(min(mesh.dx.min(), mesh.dy.min()))
    return min(mindx / influx, 0.81 * influx * gravity_scale / 9.8)
