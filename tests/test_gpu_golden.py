"""The device FP64 path against the reference's own step() (golden fixtures), through the C ABI."""
import os

import numpy as np
import pytest

from discrete_adjoint_b200 import GeoflowContext, TimeProps
from golden_util import fixtures, load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("path", fixtures(), ids=os.path.basename)
def test_device_fp64_matches_reference_fixture_bit_for_bit(path):
    mesh, mat, nsteps, ref = load(path)
    with GeoflowContext(mat, TimeProps()) as ctx:
        ctx.upload_mesh(mesh)
        ctx.set_state(mesh.h0, mesh.hu0, mesh.hv0)
        dts = [ctx.step().dt for _ in range(nsteps)]
        h, hu, hv = ctx.get_state()
    assert np.array_equal(np.array(dts), ref["dt"])
    assert np.array_equal(h, ref["h"]) and np.array_equal(hu, ref["hu"]) and np.array_equal(hv, ref["hv"])
