"""The reference arm's input builder (oracle/meshgen.py, numpy, no product library) against the
product's mesh builder (da_mesh_build in libda_b200.so): the headline workload's uniform mesh, bit
for bit, at a reduced and at the full size."""
import numpy as np
import pytest

from discrete_adjoint_b200 import inputs
from oracle import meshgen


@pytest.mark.parametrize("side", [256, 1024])
def test_headline_mesh_equals_the_product_builder(side):
    ref = inputs.workload3(side).mesh.arrays()
    got = meshgen.headline_mesh(side)
    for k, v in got.items():
        assert np.array_equal(np.asarray(v), np.asarray(ref[k])), k
