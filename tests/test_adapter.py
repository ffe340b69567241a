"""The drop-in adapter (element-table flattening, step() replacement) compiled against the reference (oracle/ref/adapter_check.cpp, linked with
the reference's objects and libda_b200.so): it flattens the reference's own element tables
(positive_x_side, neighbour keys, neigh_proc; src/datstr/element2.C:694-716) into exactly the
integer neighbour table and fields of this repository's flattening, and, on a GPU, replaces step()
(src/main/hpfem.C:271) by da_forward_step with results equal to the reference's step() bit for bit."""
import os

import pytest

import oracle
from discrete_adjoint_b200 import inputs
from golden_util import fixtures, load

needs_adapter = pytest.mark.skipif(not oracle.adapter_available(), reason="adapter_check not built")


@needs_adapter
@pytest.mark.parametrize("path", fixtures(), ids=os.path.basename)
def test_adapter_flattening_of_the_reference_tables_is_exact(path):
    mesh, mat, _, _ = load(path)
    r = oracle.run_adapter_check(mesh, mat, mesh.h0, mesh.hu0, mesh.hv0)
    assert r["nbr_mismatch"] == 0 and r["field_mismatch"] == 0


@needs_adapter
@pytest.mark.gpu
@pytest.mark.parametrize("seed,nsteps", [(11, 60), (2, 80)])
def test_adapter_step_equals_the_reference_step(seed, nsteps):
    w = inputs.test_case(seed=seed, nx0=12, ny0=8, max_level=2, random_frac=0.4) if seed == 11 else \
        inputs.test_case(seed=seed)
    m = w.mesh
    r = oracle.run_adapter_check(m, w.mat, m.h0, m.hu0, m.hv0, nsteps, step=True)
    print(r)
    assert r["steps"] == nsteps
    assert r["nbr_mismatch"] == 0 and r["field_mismatch"] == 0
    assert r["state_mismatch"] == 0 and r["dt_mismatch"] == 0
