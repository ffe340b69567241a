"""State transfer between the meshes of two epochs (host): the reference's refine / unrefine rules
and their transposes."""
import dataclasses

import numpy as np
import pytest

from discrete_adjoint_b200 import inputs
from discrete_adjoint_b200.epochs import transfer_between
from discrete_adjoint_b200.mesh import Mesh


def meshes():
    w = inputs.test_case(seed=1)
    a = dataclasses.replace(w.spec, max_level=1, uniform=True, random_frac=0.0, refine_margin=0.0)
    b = dataclasses.replace(w.spec, max_level=2, random_frac=0.0, refine_margin=40.0)
    return Mesh.build(a, w.dem, w.piles), Mesh.build(b, w.dem, w.piles)


def test_transfer_rules_and_transposes():
    A, B = meshes()
    assert set(np.unique(B.level)) == {0, 1, 2}  # both refinement and unrefinement against A
    T, U = transfer_between(A, B), transfer_between(B, A)
    rng = np.random.default_rng(0)
    u = rng.standard_normal(A.n)
    tu = T.apply(u)
    # a son copies its father, an unchanged cell is copied, a father is the mean of its sons
    for c in range(B.n):
        if T.src[1][c] < 0:
            assert tu[c] == u[T.src[0][c]]
        else:
            s = T.src[:, c]
            assert tu[c] == ((((0.0 + u[s[0]] * 0.25) + u[s[1]] * 0.25) + u[s[2]] * 0.25) + u[s[3]] * 0.25)
    # transposes
    lam = rng.standard_normal(B.n)
    assert abs(np.dot(tu, lam) - np.dot(u, T.adjoint(lam))) <= 1e-12 * np.abs(tu * lam).sum()
    v, mu = rng.standard_normal(B.n), rng.standard_normal(A.n)
    assert abs(np.dot(U.apply(v), mu) - np.dot(v, U.adjoint(mu))) <= 1e-12 * np.abs(v).sum() * np.abs(mu).max()
    # the volume is kept by unrefinement (four sons of a quarter area each)
    h = rng.random(B.n)
    assert abs(np.sum(h * B.dx * B.dy) - np.sum(U.apply(h) * A.dx * A.dy)) <= 1e-12 * np.sum(h * B.dx * B.dy)


def test_meshes_two_levels_apart_are_rejected():
    w = inputs.test_case(seed=1)
    a = dataclasses.replace(w.spec, max_level=0, uniform=True, random_frac=0.0, refine_margin=0.0)
    b = dataclasses.replace(w.spec, max_level=2, uniform=True, random_frac=0.0, refine_margin=0.0)
    with pytest.raises(ValueError):
        transfer_between(Mesh.build(a, w.dem, w.piles), Mesh.build(b, w.dem, w.piles))
