"""Adjoint across mesh adaptation: a horizon of three epochs (uniform mesh, a refined and
unrefined one, the uniform mesh again), gradients against central finite differences of the same
epochs with the time steps frozen."""
import dataclasses

import numpy as np
import pytest

from discrete_adjoint_b200 import MatProps, inputs
from discrete_adjoint_b200.epochs import Epoch, adjoint, forward
from discrete_adjoint_b200.mesh import Mesh

pytestmark = pytest.mark.gpu

TOL_GRAD = 1e-4


def setup():
    w = inputs.test_case(seed=1)
    a = dataclasses.replace(w.spec, max_level=1, uniform=True, random_frac=0.0, refine_margin=0.0)
    b = dataclasses.replace(w.spec, max_level=2, random_frac=0.0, refine_margin=40.0)
    A, B = Mesh.build(a, w.dem, w.piles), Mesh.build(b, w.dem, w.piles)
    epochs = [Epoch(A, 10), Epoch(B, 12), Epoch(A, 10)]
    wet = A.h0 > 1.0
    box = (0.5 * (A.x[wet].min() + A.x[wet].max()), A.x[wet].max() + 100.0, A.y[wet].min(), A.y[wet].max())
    return w, A, epochs, box


def J_of(m, h, box):
    inb = (m.x >= box[0]) & (m.x <= box[1]) & (m.y >= box[2]) & (m.y <= box[3])
    return float(np.sum(h[inb] ** 2 * m.dx[inb] * m.dy[inb]))


def test_gradients_across_refinement_against_central_differences():
    w, A, epochs, box = setup()
    state0 = (A.h0, A.hu0, A.hv0)
    _, _, _, dts = forward(w.mat, epochs, state0)
    g = adjoint(w.mat, epochs, state0, box, 4, A.dh0_dpile, dts=dts)

    def J(mat=None, h0=None):
        _, _, fin, _ = forward(mat or w.mat, epochs, (A.h0 if h0 is None else h0, A.hu0, A.hv0), dts=dts)
        return J_of(A, fin[0], box)

    assert abs(g.J - J()) <= 1e-12 * abs(g.J)
    assert g.J > 0
    checks = []
    for p in range(A.dh0_dpile.shape[0]):
        fds = [(J(h0=A.h0 + e * A.dh0_dpile[p]) - J(h0=A.h0 - e * A.dh0_dpile[p])) / (2 * e) for e in (1e-5, 1e-6)]
        checks.append((f"pile{p}", g.dJ_dpile[p], fds))

    def angle_fd(k):
        fds = []
        for e_deg in (1e-6, 1e-7):
            e_rad = MatProps.rad(e_deg)
            if k < 0:
                mp = MatProps(intfrict_deg=w.mat.intfrict_deg + e_deg, bedfrict_deg=list(w.mat.bedfrict_deg))
                mm = MatProps(intfrict_deg=w.mat.intfrict_deg - e_deg, bedfrict_deg=list(w.mat.bedfrict_deg))
            else:
                bp = [b + (e_deg if q == k else 0) for q, b in enumerate(w.mat.bedfrict_deg)]
                bm = [b - (e_deg if q == k else 0) for q, b in enumerate(w.mat.bedfrict_deg)]
                mp = MatProps(intfrict_deg=w.mat.intfrict_deg, bedfrict_deg=bp)
                mm = MatProps(intfrict_deg=w.mat.intfrict_deg, bedfrict_deg=bm)
            fds.append((J(mat=mp) - J(mat=mm)) / (2 * e_rad))
        return fds

    for k in range(len(w.mat.bedfrict_deg)):
        checks.append((f"bed{k}", g.dJ_dbedfrict[k], angle_fd(k)))
    checks.append(("int", g.dJ_dintfrict, angle_fd(-1)))
    scale = max(abs(v) for _, v, _ in checks)
    for name, ad, fds in checks:
        best = min(abs(ad - fd) for fd in fds)
        print(f"{name}: adjoint {ad:.10e} fd {fds}")
        assert best <= TOL_GRAD * max(abs(ad), 1e-3 * scale), name
