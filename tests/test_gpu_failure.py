"""Failure detection on the device without a GPU fault: the bounded wait of the cooperative
kernels' grid barrier is made to run out (a launch in which one block never arrives,
da_selftest_barrier), the status comes back as DA_ERR_TIMEOUT within the limit, and the same
context then runs the multi-step forward kernel and the checkpointed adjoint sweep (both
synchronised by that barrier) bit for bit like a fresh context."""
import time

import numpy as np
import pytest

from discrete_adjoint_b200 import GeoflowContext, TimeProps, _ffi, adjoint_run, inputs

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_the_context_recovers():
    w = inputs.test_case(seed=2)
    m = w.mesh
    wet = m.h0 > 1.0
    box = (float(m.x[wet].min()), float(m.x[wet].max()) + 100.0, float(m.y[wet].min()), float(m.y[wet].max()))
    with GeoflowContext(w.mat, TimeProps()) as c, GeoflowContext(w.mat, TimeProps()) as ref:
        for x in (c, ref):
            x.upload_mesh(m)
            x.set_state(m.h0, m.hu0, m.hv0)
        for limit_us in (20000, 2000):
            t0 = time.perf_counter()
            st = c.lib.da_selftest_barrier(c.ctx, limit_us)
            elapsed = time.perf_counter() - t0
            assert st == _ffi.DA_ERR_TIMEOUT, st
            assert elapsed < 2.0
            assert "barrier" in c.lib.da_last_error(c.ctx).decode()
        # forward: one cooperative launch per horizon, grid barriers between its phases
        s1, s2 = c.run(40), ref.run(40)
        assert s1.time == s2.time and s1.iter == s2.iter
        for a, b in zip(c.get_state(), ref.get_state()):
            assert np.array_equal(a, b)
        # adjoint: the checkpointed sweep (fused reverse steps, also barrier-synchronised)
        g1 = adjoint_run(c, box, 30, 6, m.dh0_dpile, want_lambda0=True)
        g2 = adjoint_run(ref, box, 30, 6, m.dh0_dpile, want_lambda0=True)
        assert g1.J == g2.J and np.array_equal(g1.lambda0, g2.lambda0)
        assert g1.dJ_dbedfrict == g2.dJ_dbedfrict and g1.dJ_dpile == g2.dJ_dpile
        # and once more after a further timeout
        assert c.lib.da_selftest_barrier(c.ctx, 1000) == _ffi.DA_ERR_TIMEOUT
        s1, s2 = c.run(5), ref.run(5)
        for a, b in zip(c.get_state(), ref.get_state()):
            assert np.array_equal(a, b)
