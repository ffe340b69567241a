"""The DWR error indicator against the reference's own estimate (bilinear_interp,
update_bilinear_error_grid, error_compute; src/adjoint/dual_solver.C:213-230): the error grid's
reconstruction weights (the reference's choice of interpolants, hanging sides included), the
error grid's one-step residual and the per-cell indicator.  The weights and the oracle's
frozen-dt step of the error grid are checked against the committed fixture and against live
harness runs.  Tolerances: the reference solves a 4 x 4 system per value where the weights here
are precomputed, so the reconstructions agree to rounding (1e-11 of the field's largest value),
and what follows from them to 1e-10."""
import os

import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import MatProps, TimeProps, inputs, make_params
from discrete_adjoint_b200.dwr import error_grid
from discrete_adjoint_b200.mesh import Mesh

HERE = os.path.dirname(os.path.abspath(__file__))
RECON_TOL = 1e-11
DWR_TOL = 1e-10
needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")


def reconstruct(g, field):
    out = np.zeros(g.fine.n)
    for q in range(4):
        k = g.interp[q]
        out += np.where(k >= 0, g.weight[q] * field[np.maximum(k, 0)], 0.0)
    return out


def indicator_on_host(w, g, un, unext, lam, dt, n0):
    """Reconstructions, the error grid's step with the coarse dt, residual and indicator
    (el_error = sum_j |r_j (lambda_j - lambda~_j)|, correction = sum_j r_j lambda_j)."""
    rec = lambda f: np.stack([reconstruct(g, f[v]) for v in range(3)])  # noqa: E731
    ut_n, ut_next, lamt = rec(un), rec(unext), rec(lam)
    of = oracle.Oracle(make_params(w.mat, TimeProps()), g.fine)
    u = [ut_n[v].copy() for v in range(3)]
    of.step_frozen(dt, *u, n0)
    res = np.stack(u) - ut_next
    lam_f = lam[:, g.parent]
    return {"bilin_prev": ut_n, "bilin_adj": lamt, "residual": res, "el_error": np.abs(res * (lam_f - lamt)).sum(0),
            "correction": (res * lam_f).sum(0)}


def close(a, b, tol):
    scale = max(float(np.abs(b).max()), 1e-300)
    return float(np.abs(a - b).max()) <= tol * scale


def test_fixture_reconstruction_residual_and_indicator():
    z = np.load(os.path.join(HERE, "golden", "dwr_s11_55.npz"))
    w = inputs.test_case(seed=11, nx0=12, ny0=8, max_level=2, random_frac=0.4)
    m = Mesh(**{k[5:]: z[k] for k in z.files if k.startswith("mesh_")})
    assert np.array_equal(m.nbr, w.mesh.nbr) and np.array_equal(m.x, w.mesh.x)
    g = error_grid(w)
    assert np.array_equal(g.parent, z["parent"])
    # the fixture's mesh has hanging sides, and interpolants of every count occur
    assert m.two_neighbour_sides() > 0
    counts = (g.interp >= 0).sum(0)
    assert set(np.unique(counts)) >= {2, 3, 4}
    un, lam, dt, n0 = z["un"], z["lam_next"], float(z["dt"]), int(z["n0"])
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    u = [un[v].copy() for v in range(3)]
    o.set_time(0.0, n0)
    rc, dts, _ = o.run(*u, 1)
    assert rc == 0 and dts[0] == dt
    r = indicator_on_host(w, g, un, np.stack(u), lam, dt, n0)
    assert close(r["bilin_prev"], z["ref_bilin_prev"], RECON_TOL)
    assert close(r["bilin_adj"], z["ref_bilin_adj"], RECON_TOL)
    assert close(r["residual"], z["ref_residual"], DWR_TOL)
    assert close(r["el_error"], z["ref_el_error"], DWR_TOL)
    assert close(r["correction"], z["ref_correction"], DWR_TOL)
    assert abs(r["el_error"].sum() - z["ref_el_error"].sum()) <= 1e-12 * z["ref_el_error"].sum()


@needs_ref
@pytest.mark.parametrize("seed,n0,frac", [(1, 4, None), (3, 49, None), (3, 50, None), (21, 60, 0.5), (13, 12, 0.0)])
def test_live_reference_estimate(seed, n0, frac):
    # n0 = 49 / 50 straddle the frict_tiny switch: the reference's error step tests iter < 51 with
    # iter = n0 + 1, the forward step iter < 50 with iter = n0
    w = inputs.test_case(seed=seed) if frac is None else \
        inputs.test_case(seed=seed, nx0=12, ny0=8, max_level=2 if frac > 0 else 1, random_frac=frac)
    m = w.mesh
    g = error_grid(w)
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    u = [m.h0.copy(), m.hu0.copy(), m.hv0.copy()]
    o.run(*u, n0)
    un = np.stack(u).copy()
    rc, dts, _ = o.run(*u, 1)
    unext = np.stack(u)
    rng = np.random.default_rng(seed)
    lam = rng.standard_normal((3, m.n))
    ref = oracle.run_reference_dwr(g.fine, g.parent, w.mat, un, unext, lam, dts[0], n0 + 1)
    r = indicator_on_host(w, g, un, unext, lam, dts[0], n0)
    assert close(r["bilin_prev"], ref["bilin_prev"], RECON_TOL)
    assert close(r["bilin_adj"], ref["bilin_adj"], RECON_TOL)
    assert close(r["residual"], ref["residual"], DWR_TOL)
    assert close(r["el_error"], ref["el_error"][1], DWR_TOL)
    assert close(r["correction"], ref["correction"], DWR_TOL)
