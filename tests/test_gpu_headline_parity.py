"""Parity on the benchmark meshes themselves, through the C ABI with the default launch path
(staged tiles, tile culling, the multi-step kernel under a CUDA graph): the 1M-cell uniform
plane-and-runout mesh of the forward + adjoint headline (20 forward steps, then 5 reverse steps of
the reference's own adjoint) and the 3.75M-cell adaptive hill mesh of the forward-only workload
(5 steps), against the oracle (pinned bit for bit to the reference's step() and dual solver)."""
import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import GeoflowContext, TimeProps, _ffi, adjoint_run, inputs, make_params

pytestmark = pytest.mark.gpu


def _forward_bit_exact(w, nsteps):
    m = w.mesh
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    rc, dts, st = o.run(h, hu, hv, nsteps)
    assert rc == 0
    with GeoflowContext(w.mat, TimeProps()) as c:
        c.upload_mesh(m)
        c.set_state(m.h0, m.hu0, m.hv0)
        s = c.run(nsteps)
        gh, ghu, ghv = c.get_state()
    assert s.time == st.time and s.iter == nsteps
    assert np.array_equal(gh, h) and np.array_equal(ghu, hu) and np.array_equal(ghv, hv)
    return o, (h, hu, hv), dts


def test_headline_mesh_forward_and_reference_adjoint():
    w = inputs.workload3()
    m = w.mesh
    N = 20
    _forward_bit_exact(w, N)
    # the reference's own adjoint over the last 5 steps of those 20 (device reference mode vs the
    # oracle's restatement, both from the same states)
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    states = []
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    dts = []
    for _ in range(N):
        states.append((h.copy(), hu.copy(), hv.copy()))
        rc, dt, _ = o.run(h, hu, hv, 1)
        dts.append(float(dt[0]))
    box = inputs.WORKLOAD3_BOX
    inb = (m.x >= box[0]) & (m.x <= box[1]) & (m.y >= box[2]) & (m.y <= box[3])
    K = 5
    with GeoflowContext(w.mat, TimeProps(), jacobian_mode=_ffi.DA_JAC_REFERENCE) as c:
        c.upload_mesh(m)
        c.set_state(*states[N - K])
        c.set_time(float(np.sum(dts[:N - K])), N - K)
        g = adjoint_run(c, box, K, 2, want_lambda0=True)
    lam = np.zeros((3, m.n))
    lam[0] = np.where(inb, 2.0 * h * (m.dx * m.dy), 0.0)
    for it in range(N, N - K, -1):
        lam = o.adjoint_step_ref(*states[it - 1], dts[it - 1], 0.1 if it < 51 else 1e-9, lam)
    rel = np.linalg.norm(g.lambda0 - lam) / np.linalg.norm(lam)
    print(f"headline mesh, reference-mode adjoint over {K} steps: rel {rel:.3e}")
    assert rel <= 1e-12


def test_adaptive_hill_mesh_forward():
    w = inputs.workload2()
    assert w.mesh.two_neighbour_sides() > 0
    _forward_bit_exact(w, 5)
