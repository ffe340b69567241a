"""Properties of the CPU oracle (restated reference step) that hold by construction."""
import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import TimeProps, inputs, make_params
from discrete_adjoint_b200.mesh import Mesh, MeshSpec
from discrete_adjoint_b200.solver import MatProps


def run(w, nsteps, h=None, hu=None, hv=None, tp=None):
    p = make_params(w.mat, tp or TimeProps())
    o = oracle.Oracle(p, w.mesh)
    m = w.mesh
    h = m.h0.copy() if h is None else h.copy()
    hu = m.hu0.copy() if hu is None else hu.copy()
    hv = m.hv0.copy() if hv is None else hv.copy()
    rc, dts, st = o.run(h, hu, hv, nsteps)
    return rc, h, hu, hv, dts, st


def test_runs_and_stays_finite():
    w = inputs.test_case(seed=1)
    rc, h, hu, hv, dts, st = run(w, 60)
    assert rc == 0
    assert np.all(np.isfinite(h)) and np.all(h >= 0)
    assert np.all(dts > 0)
    assert st.iter == 60


def test_mass_conserved_away_from_outflow_boundary():
    # a pile far from the domain edge, few steps: the update is conservative (shared edge fluxes,
    # averaged hanging fluxes) so the volume changes only by rounding
    w = inputs.test_case(seed=2)
    m = w.mesh
    rc, h, hu, hv, dts, st = run(w, 15)
    assert rc == 0
    assert h[m.boundary_cells()].max() == 0.0
    v0 = (m.h0 * m.dx * m.dy).sum()
    assert abs(st.volume - v0) / v0 < 1e-12


def test_lake_at_rest_flat_terrain():
    # flat bed, uniform depth, no velocity: fluxes balance, sources vanish -> state unchanged
    m = Mesh.build(MeshSpec(0, 0, 20.0, 20.0, 6, 5, 2, random_frac=0.4, seed=3))
    w = inputs.Workload("flat", m, MatProps(), [], 10)
    h = np.full(m.n, 2.0)
    rc, h1, hu1, hv1, dts, st = run(w, 10, h=h, hu=np.zeros(m.n), hv=np.zeros(m.n))
    assert rc == 0
    assert np.allclose(h1, 2.0, rtol=0, atol=1e-12)
    assert np.allclose(hu1, 0.0, atol=1e-12) and np.allclose(hv1, 0.0, atol=1e-12)


def test_mirror_symmetry():
    # uniform mesh, terrain and pile symmetric about y = ly/2: hv is odd, h and hu even
    spec = MeshSpec(0, 0, 40.0, 40.0, 12, 8, 1, uniform=True)
    lx, ly = 480.0, 320.0
    dem = inputs.analytic_dem(lambda X, Y: (lx - X) * 0.4 + 5 * np.cos(2 * np.pi * (Y - ly / 2) / ly),
                              0, 0, lx, ly, 10.0)
    from discrete_adjoint_b200.mesh import Pile
    m = Mesh.build(spec, dem, [Pile(150.0, 160.0, 20.0, 60.0, 60.0)])
    w = inputs.Workload("sym", m, MatProps(), [], 30)
    rc, h, hu, hv, dts, st = run(w, 30)
    assert rc == 0
    key = {(round(x, 6), round(y, 6)): i for i, (x, y) in enumerate(zip(m.x, m.y))}
    mirror = np.array([key[(round(x, 6), round(ly - y, 6))] for x, y in zip(m.x, m.y)])
    assert np.allclose(h, h[mirror], rtol=1e-9, atol=1e-12)
    assert np.allclose(hu, hu[mirror], rtol=1e-9, atol=1e-12)
    assert np.allclose(hv, -hv[mirror], rtol=1e-9, atol=1e-12)


def test_time_clipping_hits_maxtime():
    w = inputs.test_case(seed=1)
    rc, h, hu, hv, dts, st = run(w, 40, tp=TimeProps(maxtime=1.0))
    assert rc == 0
    assert st.time == 1.0
    assert dts[-1] == 0.0  # once time reached maxtime every further dt is clipped to zero


def test_dry_domain_dt_is_half_influx_dt():
    w = inputs.test_case(seed=1)
    p = make_params(w.mat, TimeProps(), influx_dt=3.0)
    o = oracle.Oracle(p, w.mesh)
    z = np.zeros(w.mesh.n)
    rc, dts, st = o.run(z.copy(), z.copy(), z.copy(), 1)
    assert rc == 0 and dts[0] == 1.5


def test_edge_fluxes_hanging_average():
    # the coarse side of a hanging edge carries the average of the two fine-side fluxes
    w = inputs.test_case(seed=3)
    m = w.mesh
    p = make_params(w.mat, TimeProps())
    o = oracle.Oracle(p, m)
    h, hu, hv = m.h0.copy(), m.hu0 + 0.3 * m.h0, m.hv0 - 0.2 * m.h0
    s = o.slopes(h, hu, hv)
    rc, kact, _, _ = o.coef_eigen(h, hu, hv, s)
    F = o.edge_fluxes(h, hu, hv, kact)
    checked = 0
    for side in range(4):
        two = np.nonzero((m.nbr[side + 4] != m.nbr[side]) & (m.nbr[side] >= 0))[0]
        for i in two:
            a, b = m.nbr[side][i], m.nbr[side + 4][i]
            exp = 0.5 * (F[side ^ 2, :, a] + F[side ^ 2, :, b])
            assert np.array_equal(F[side, :, i], exp)
            checked += 1
    assert checked > 50


def test_fp32_state_storage_diverges_after_friction_threshold_switch():
    # Property of the reference model behind the FP32-split error budget: FP64 arithmetic with
    # the state rounded to FP32 after every step tracks FP64 to rounding level while
    # frict_tiny = 0.1, and departs from it once frict_tiny drops to 1e-9 (step 50), whereas a
    # one-off 1e-8 perturbation of the initial depth stays at the 1e-9 level.
    w = inputs.test_case(seed=1)
    m = w.mesh
    p = make_params(w.mat, TimeProps())

    def run(h, hu, hv, steps, round32):
        o = oracle.Oracle(p, m)
        out = {}
        for k in range(1, max(steps) + 1):
            o.run(h, hu, hv, 1)
            if round32:
                for a in (h, hu, hv):
                    a[:] = np.float32(a)
            if k in steps:
                out[k] = h.copy()
        return out

    steps = (50, 120)
    ref = run(m.h0.copy(), m.hu0.copy(), m.hv0.copy(), steps, False)
    r32 = run(*[np.float64(np.float32(a)) for a in (m.h0, m.hu0, m.hv0)], steps, True)
    rng = np.random.default_rng(0)
    pert = run(m.h0 * (1 + 1e-8 * rng.standard_normal(m.n)), m.hu0.copy(), m.hv0.copy(), steps, False)
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)  # noqa: E731
    assert rel(r32[50], ref[50]) < 1e-6
    assert rel(r32[120], ref[120]) > 1e-4
    assert rel(pert[120], ref[120]) < 1e-7


def test_fp32_flux_and_source_arithmetic_with_fp64_state_also_diverges():
    # The other precision split (oracle/da_oracle_split.c): FP64 state and FP64 corrector
    # accumulation, FP32 slopes, k act/pass, wave speeds, fluxes, sources and sign tests.  It tracks
    # FP64 to ~1e-7 while frict_tiny = 0.1 and for a while after the switch, then departs: the
    # basal-friction sign test at 1e-9 m/s sees FP32 flux noise (the hydrostatic pressure terms of
    # the two sides cancel to ~1e-7 of their size) in cells coming to rest.
    w = inputs.test_case(seed=1)
    m = w.mesh
    p = make_params(w.mat, TimeProps())
    ref = oracle.Oracle(p, m)
    spl = oracle.Oracle(p, m)
    A = [m.h0.copy(), m.hu0.copy(), m.hv0.copy()]
    B = [m.h0.copy(), m.hu0.copy(), m.hv0.copy()]
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)  # noqa: E731
    errs = {}
    for k in range(1, 131):
        ref.run(*A, 1)
        spl.run_split(*B, 1)
        if k in (50, 90, 130):
            errs[k] = rel(B[0], A[0])
    print(errs)
    assert errs[50] < 1e-6 and errs[90] < 1e-6
    assert errs[130] > 1e-4
