"""The device step against the reference's own compiled step() (oracle/_ref/ref_harness) on the
CPU-runnable configuration: the 36,400-cell adaptive plane-and-runout mesh, 200 steps.  FP64
state and dt history bit for bit, through the multi-step kernel and through single steps."""
import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import GeoflowContext, TimeProps, inputs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")]

NSTEPS = 200


@pytest.fixture(scope="module")
def reference_run():
    w = inputs.workload1()
    m = w.mesh
    return w, oracle.run_reference(m, w.mat, m.h0, m.hu0, m.hv0, NSTEPS)


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
