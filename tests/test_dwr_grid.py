"""The DWR error grid and its reconstruction weights (host side, no GPU)."""
import numpy as np

from discrete_adjoint_b200 import inputs
from discrete_adjoint_b200.dwr import error_grid, weights_for


def test_error_grid_is_the_mesh_refined_once():
    w = inputs.test_case(seed=2)
    g = error_grid(w)
    m, f = w.mesh, g.fine
    assert f.n == 4 * m.n
    assert np.array_equal(np.bincount(g.parent, minlength=m.n), np.full(m.n, 4))
    assert np.all(f.level == m.level[g.parent] + 1)
    assert np.allclose(f.dx, 0.5 * m.dx[g.parent]) and np.allclose(f.dy, 0.5 * m.dy[g.parent])
    # children tile their parent: centres at the parent's centre +- a quarter of its size
    assert np.allclose(np.abs(f.x - m.x[g.parent]), 0.25 * m.dx[g.parent])
    assert np.allclose(np.abs(f.y - m.y[g.parent]), 0.25 * m.dy[g.parent])


def test_reconstruction_is_exact_for_linear_fields_away_from_edges():
    w = inputs.test_case(seed=1)
    g = error_grid(w)
    m = w.mesh
    fld = 2.0 + 3.0 * m.x - 0.5 * m.y
    val = sum(np.where(g.interp[q] >= 0, g.weight[q] * fld[np.maximum(g.interp[q], 0)], 0.0) for q in range(4))
    k = (g.interp >= 0).sum(0)
    exact = 2.0 + 3.0 * g.fine.x - 0.5 * g.fine.y
    assert np.abs(val - exact)[k >= 3].max() < 1e-9
    assert np.all(k >= 1)


def test_two_point_formula_is_the_references():
    # linear_interp (bilinear_interp.C:350-353): (f2 - f1) / (x2 - x1) * (x - x1), no f1 term
    w = weights_for([0.0, 2.0], [5.0, 5.0], 0.5, 5.0)
    f1, f2 = 7.0, 11.0
    assert abs(w[0] * f1 + w[1] * f2 - (f2 - f1) / 2.0 * 0.5) < 1e-15
    # sorted by x: the order of the points does not matter
    w2 = weights_for([2.0, 0.0], [5.0, 5.0], 0.5, 5.0)
    assert abs(w2[1] * f1 + w2[0] * f2 - (f2 - f1) / 2.0 * 0.5) < 1e-15
    # same x: along y
    w3 = weights_for([1.0, 1.0], [0.0, 4.0], 1.0, 1.0)
    assert abs(w3[0] * f1 + w3[1] * f2 - (f2 - f1) / 4.0 * 1.0) < 1e-15
