"""DWR error indicator on the device against the same steps assembled on the host."""
import numpy as np
import pytest

from discrete_adjoint_b200 import GeoflowContext, MatProps, TimeProps, _ffi, adjoint_step, inputs, set_dt_replay
from discrete_adjoint_b200.dwr import Indicator, error_grid
from discrete_adjoint_b200.mesh import Mesh, MeshSpec

pytestmark = pytest.mark.gpu


def ctx_for(w, mesh=None):
    c = GeoflowContext(w.mat, TimeProps())
    m = mesh or w.mesh
    c.upload_mesh(m)
    c.set_state(m.h0, m.hu0, m.hv0)
    return c


def reconstruct(g, field):
    out = np.zeros(g.fine.n)
    for q in range(4):
        k = g.interp[q]
        out += np.where(k >= 0, g.weight[q] * field[np.maximum(k, 0)], 0.0)
    return out


@pytest.mark.parametrize("seed", [1, 3])
def test_indicator_matches_host_assembly(seed):
    w = inputs.test_case(seed=seed)
    m = w.mesh
    g = error_grid(w)
    with ctx_for(w) as c:
        c.run(4)
        un = np.stack(c.get_state())
        # an adjoint field with structure: one reverse step of a seeded lambda
        rng = np.random.default_rng(seed)
        lam_next = np.stack([rng.standard_normal(m.n) * (un[0] > 1e-4), rng.standard_normal(m.n) * 0.1,
                             rng.standard_normal(m.n) * 0.1])
        ind = Indicator(c, g)
        el, cell, sums = ind.step(lam_next)
        # the context is where it was
        assert np.array_equal(np.stack(c.get_state()), un)
        s_before = c.step()
        unext = np.stack(c.get_state())
        dt, time0, iter0 = s_before.dt, s_before.time - s_before.dt, s_before.iter - 1
    # host assembly: reconstructions, one step of the error grid with the coarse dt, residual
    ut_n = np.stack([reconstruct(g, un[v]) for v in range(3)])
    ut_next = np.stack([reconstruct(g, unext[v]) for v in range(3)])
    lamt = np.stack([reconstruct(g, lam_next[v]) for v in range(3)])
    with GeoflowContext(w.mat, TimeProps()) as f:
        f.upload_mesh(g.fine)
        f.set_state(*ut_n)
        f.set_time(time0, iter0)
        set_dt_replay(f, [dt], iter0)
        f.step()
        uf = np.stack(f.get_state())
    r = uf - ut_next
    lam = lam_next[:, g.parent]
    e_ref = np.abs(r * (lam - lamt)).sum(0)
    c_ref = (r * lam).sum(0)
    # FP64 on both sides; the device fuses multiply-adds in the reconstruction and r cancels, so
    # the bound is relative to the largest cell value
    tol = 1e-12 * e_ref.max()
    np.testing.assert_allclose(el, e_ref, rtol=1e-10, atol=tol)
    cell_ref = np.zeros(m.n)
    np.add.at(cell_ref, g.parent, e_ref)
    np.testing.assert_allclose(cell, cell_ref, rtol=1e-10, atol=4 * tol)
    assert abs(sums[0] - e_ref.sum()) <= 1e-10 * abs(e_ref.sum())
    assert abs(sums[1] - c_ref.sum()) <= 1e-11 * np.abs(r * lam).sum()
    assert e_ref.sum() > 0


def test_indicator_vanishes_for_a_lake_at_rest():
    # level ground, uniform depth, no motion: every step is the identity, so the residual is zero
    # wherever the reconstruction is exact (away from the domain edges, where the reference's
    # two-point formula drops the f1 term)
    from discrete_adjoint_b200.inputs import Workload, analytic_dem
    dem = analytic_dem(lambda X, Y: 0.0 * X, 0.0, 0.0, 640.0, 640.0, 10.0)
    spec = MeshSpec(xmin=0.0, ymin=0.0, dx0=40.0, dy0=40.0, nx0=16, ny0=16, max_level=1, random_frac=0.3, seed=5)
    mesh = Mesh.build(spec, dem, [])
    w = Workload("lake", mesh, MatProps(), [], 1, spec, dem)
    g = error_grid(w)
    with GeoflowContext(w.mat, TimeProps()) as c:
        c.upload_mesh(mesh)
        c.set_state(np.full(mesh.n, 2.0), np.zeros(mesh.n), np.zeros(mesh.n))
        ind = Indicator(c, g)
        el, cell, sums = ind.step(np.ones((3, mesh.n)))
    fx, fy = g.fine.x, g.fine.y
    inner = (fx > 100.0) & (fx < 540.0) & (fy > 100.0) & (fy < 540.0)
    # rounding only: the reconstruction weights at hanging nodes sum to one within 1e-16
    assert el[inner].max() < 1e-25 and el[inner].max() >= 0.0


def test_adjoint_run_accumulates_the_step_indicators():
    # the indicator of every reverse step of the checkpointed sweep (da_adjoint_run_dwr) against the
    # same steps one by one: forward states U^n, lambda^N = dJ/dU^N, lambda^n by single reverse
    # steps, and da_dwr_step at each U^n with lambda^{n+1}
    from discrete_adjoint_b200 import adjoint_run
    w = inputs.test_case(seed=1)
    m = w.mesh
    g = error_grid(w)
    N = 6
    wet = m.h0 > 1.0
    box = (0.5 * (m.x[wet].min() + m.x[wet].max()), m.x[wet].max() + 100.0, m.y[wet].min(), m.y[wet].max())
    with ctx_for(w) as c:
        Indicator(c, g)
        res = adjoint_run(c, box, N, 2, dwr=True)
    with ctx_for(w) as c:
        states, times = [np.stack(c.get_state())], [(0.0, 0)]
        for k in range(N):
            s = c.step()
            states.append(np.stack(c.get_state()))
            times.append((s.time, s.iter))
        hN = states[N][0]
        inb = (m.x >= box[0]) & (m.x <= box[1]) & (m.y >= box[2]) & (m.y <= box[3])
        lam = np.stack([np.where(inb, 2.0 * hN * (m.dx * m.dy), 0.0), np.zeros(m.n), np.zeros(m.n)])
        ind = Indicator(c, g)
        sums, cells = np.zeros((N, 2)), np.zeros(m.n)
        for k in range(N - 1, -1, -1):
            c.set_state(*states[k])
            c.set_time(*times[k])
            _, cell, sk = ind.step(lam)
            sums[k] = sk
            cells += cell
            lam, _ = adjoint_step(c, lam)
    assert np.all(sums[:, 0] > 0)
    np.testing.assert_allclose(res.dwr_steps, sums, rtol=1e-12, atol=1e-14 * np.abs(sums).max())
    np.testing.assert_allclose(res.dwr_cell, cells, rtol=1e-12, atol=1e-14 * cells.max())


def test_indicator_matches_the_reference_estimate_fixture():
    # the reference's own estimate of the step n0 -> n0 + 1 (bilinear_interp, update_bilinear_error_grid,
    # error_compute through the harness), committed as tests/golden/dwr_s11_55.npz
    import os
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "dwr_s11_55.npz"))
    w = inputs.test_case(seed=11, nx0=12, ny0=8, max_level=2, random_frac=0.4)
    g = error_grid(w)
    assert np.array_equal(g.parent, z["parent"])
    with GeoflowContext(w.mat, TimeProps()) as c:
        c.upload_mesh(w.mesh)
        c.set_state(*z["un"])
        c.set_time(0.0, int(z["n0"]))
        el, cell, sums = Indicator(c, g).step(z["lam_next"])
    ref = z["ref_el_error"]
    assert np.abs(el - ref).max() <= 1e-10 * np.abs(ref).max()
    assert abs(sums[0] - ref.sum()) <= 1e-12 * ref.sum()
    assert abs(sums[1] - z["ref_correction"].sum()) <= 1e-10 * np.abs(z["ref_correction"]).sum()
    assert np.allclose(cell, np.bincount(g.parent, weights=el, minlength=w.mesh.n), rtol=1e-12, atol=0)
