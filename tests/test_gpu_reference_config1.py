"""The device against the reference's own compiled code (oracle/_ref/ref_harness, run live) on the
CPU-runnable configuration: the 36,400-cell adaptive plane-and-runout mesh.  step() over 200 steps
(FP64 state and dt history bit for bit, through the multi-step kernel and through single steps),
calc_stats and the discharge planes over the same run, and reverse steps of the reference's own
dual solver."""
import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import GeoflowContext, TimeProps, inputs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")]

NSTEPS = 200


def probes(m):
    """A test point (not equidistant from two cell centres) and two discharge planes, one slanted,
    placed around the pile."""
    wet = m.h0 > 1.0
    cx, cy = float(m.x[wet].mean()), float(m.y[wet].mean())
    return (0.5, cx + 97.3, cy + 11.1), [(cx + 61.7, cx + 61.7, cy - 250.0, cy + 230.0),
                                         (cx - 180.0, cx + 260.0, cy + 131.0, cy + 57.0)]


@pytest.fixture(scope="module")
def reference_run():
    w = inputs.workload1()
    m = w.mesh
    test_point, planes = probes(m)
    return w, oracle.run_reference(m, w.mat, m.h0, m.hu0, m.hv0, NSTEPS, test_point=test_point, vslump=2.0,
                                   planes=planes)


@pytest.mark.parametrize("how", ["multi-step", "single steps"])
def test_device_equals_the_reference_step_on_config1(reference_run, how):
    w, ref = reference_run
    m = w.mesh
    with GeoflowContext(w.mat, TimeProps()) as c:
        c.upload_mesh(m)
        c.set_state(m.h0, m.hu0, m.hv0)
        if how == "multi-step":
            dts = [c.step().dt]           # the two-launch path's first step, then one launch of the rest
            st = c.run(NSTEPS - 1)
        else:
            dts = []
            for _ in range(NSTEPS):
                st = c.step()
                dts.append(st.dt)
        h, hu, hv = c.get_state()
    assert np.array_equal(h, ref["h"]) and np.array_equal(hu, ref["hu"]) and np.array_equal(hv, ref["hv"])
    if how == "single steps":
        assert np.array_equal(np.array(dts), ref["dt"][:NSTEPS])
    else:
        assert dts[0] == ref["dt"][0]
    assert st.time == ref["time"] and st.iter == NSTEPS


def test_stats_and_discharge_on_config1(reference_run):
    # calc_stats after every step, as the reference's step() calls it (step.C:248): its StatProps
    # after the last step and its discharge through two planes over all steps, with the tolerances
    # of the fixture test in test_gpu_golden.py (sums in another order)
    w, ref = reference_run
    m = w.mesh
    test_point, planes = probes(m)
    discharge = np.zeros(len(planes))
    reached = -1.0
    with GeoflowContext(w.mat, TimeProps()) as c:
        c.upload_mesh(m)
        c.set_state(m.h0, m.hu0, m.hv0)
        for _ in range(NSTEPS):
            s = c.step()
            st = c.stats(d_time=s.dt, test_point=test_point, vslump=2.0, planes=planes, discharge=discharge)
            if st["testpoint_reach"] and reached < 0:
                reached = s.time
    rs = ref["stats"]
    scale2 = rs["xcen"] ** 2 + rs["ycen"] ** 2
    for k, v in rs.items():
        if k == "slopemean":
            continue  # the harness has no GIS slope grid (zero there); this build uses the terrain slope
        if k == "timereached":
            assert reached == v
            continue
        if k in ("xvar", "yvar"):
            tol = 1e-9 * scale2
        elif k in ("vxmean", "vymean"):
            tol = 1e-12 * max(abs(v), rs["vmean"])  # vymean cancels to ~1e-17 on this symmetric flow
        else:
            tol = 1e-12 * max(abs(v), 1e-300)
        assert abs(st[k] - v) <= tol, (k, st[k], v)
    np.testing.assert_allclose(discharge, ref["discharge"], rtol=1e-10)
    assert st["statvolume"] > 0 and np.all(discharge != 0.0)


def test_reference_adjoint_steps_on_config1(reference_run):
    # the reference's own dual-solver steps (harness mode 'DAJ1', run live) against the device's
    # reverse steps in reference mode, on the same mesh: chained from lambda^N of J = sum h^2 dx dy
    # over the wet cells' box, back across the frict_tiny switch at step 50; 1e-12 relative, the
    # tolerance of the fixture-mesh tests in test_gpu_adjoint_ref.py
    from discrete_adjoint_b200 import _ffi, adjoint_step, make_params
    from test_oracle_adjoint import forward_states
    w, _ = reference_run
    m = w.mesh
    N, K = 56, 10
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    states, dts = forward_states(o, m, N)
    wet = states[N][0] > 0
    box = (m.x[wet].min(), m.x[wet].max(), m.y[wet].min(), m.y[wet].max())
    inb = (m.x >= box[0]) & (m.x <= box[1]) & (m.y >= box[2]) & (m.y <= box[3])
    lam_end = np.zeros((3, m.n))
    lam_end[0] = np.where(inb, 2.0 * states[N][0] * (m.dx * m.dy), 0.0)
    iters = [N - k for k in range(K)]
    ref = oracle.run_reference_adjoint(m, w.mat, [states[it - 1] for it in iters], iters,
                                       [dts[it - 1] for it in iters], lam_end)
    times = np.concatenate([[0.0], np.cumsum(dts)])
    with GeoflowContext(w.mat, TimeProps(), jacobian_mode=_ffi.DA_JAC_REFERENCE) as c:
        c.upload_mesh(m)
        lam = lam_end.copy()
        for k, it in enumerate(iters):
            c.set_state(*states[it - 1])
            c.set_time(float(times[it - 1]), it - 1)
            lam, _ = adjoint_step(c, lam)
            r = np.linalg.norm(lam - ref["lam"][k]) / np.linalg.norm(ref["lam"][k])
            assert r <= 1e-12, (k, it, r)
