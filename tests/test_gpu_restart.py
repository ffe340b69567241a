"""A run the reference saved (save_forward) resumes on the device from this package's reader of
restart_<rank> and continues bit for bit as the reference's own loadrun + step() continue it."""
import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import GeoflowContext, TimeProps, inputs, records

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")]


@pytest.mark.parametrize("seed,first,then", [(11, 30, 40), (2, 45, 30)])
def test_device_resumes_a_reference_restart(tmp_path, seed, first, then):
    w = inputs.test_case(seed=seed, nx0=12, ny0=8, max_level=2, random_frac=0.4) if seed == 11 else \
        inputs.test_case(seed=seed)
    m = w.mesh
    ol = ((10.0, 10.0), (float(m.x.min()) - 50.0, float(m.x.max()) + 50.0),
          (float(m.y.min()) - 50.0, float(m.y.max()) + 50.0))
    oracle.run_reference_save(m, w.mat, m.h0, m.hu0, m.hv0, first, ol, str(tmp_path))
    r = records.read_restart(str(tmp_path / "restart_0000"))
    ref = oracle.run_reference_load(w.mat, then, ol, str(tmp_path))   # the reference continues
    rm = r["mesh"]
    with GeoflowContext(w.mat, TimeProps()) as c:
        c.upload_mesh(rm)
        c.set_state(r["h"], r["hu"], r["hv"])
        c.set_time(r["time"], r["iter"])
        dts = [c.step().dt for _ in range(then // 2)]
        st = c.run(then - then // 2)      # the rest in one multi-step launch
        h, hu, hv = c.get_state()
    key_of = {(int(a), int(b)): i for i, (a, b) in enumerate(r["keys"])}
    p = np.array([key_of[(int(a), int(b))] for a, b in ref["keys"]])
    assert np.array_equal(h[p], ref["h"]) and np.array_equal(hu[p], ref["hu"]) and np.array_equal(hv[p], ref["hv"])
    assert np.array_equal(np.array(dts), ref["dt"][first:first + then // 2])
    assert st.time == ref["time"] and st.iter == first + then
