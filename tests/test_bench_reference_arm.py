"""The reference arm of bench.py: it times the reference's own forward + adjoint (or the oracle's
restatement) on the headline workload without ever loading the product library, and the oracle's
library-free parameters equal the library's defaults."""
import os
import subprocess
import sys

import pytest

import oracle
from discrete_adjoint_b200 import TimeProps, make_params
from discrete_adjoint_b200.solver import MatProps

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_oracle_params_equal_the_library_defaults():
    mat = MatProps(intfrict_deg=30.0, bedfrict_deg=[20.0, 17.5])
    a, b = oracle.params_for(mat), make_params(mat, TimeProps())
    for name, _ in a._fields_:
        va, vb = getattr(a, name), getattr(b, name)
        if hasattr(va, "__len__"):
            assert list(va) == list(vb), name
        else:
            assert va == vb, name


@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")
def test_reference_arm_runs_the_reference_without_the_product_library():
    code = (
        "import sys, json; sys.path.insert(0, %r)\n"
        "import bench\n"
        "r = bench.reference_fwdadj(1, 1, side=128)\n"
        "maps = open('/proc/self/maps').read()\n"
        "print(json.dumps({'kind': r['kind'], 'value': r['value'], 'loaded': 'libda_b200' in maps}))\n" % ROOT)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    import json
    res = json.loads(out.stdout.strip().splitlines()[-1])
    assert res["kind"] == "reference" and res["value"] > 0
    assert not res["loaded"]


@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")
def test_reference_arm_runs_one_harness_per_core():
    # side-by-side harness processes on the same input: each one's lambda is the single run's,
    # the rate is their total work over the slowest one's timed seconds, and the replica count
    # follows the usable cores and the memory they would take
    import numpy as np

    import bench
    from discrete_adjoint_b200.inputs import WORKLOAD3_BOX
    from discrete_adjoint_b200.mesh import Mesh
    from oracle import meshgen
    m = Mesh(**meshgen.headline_mesh(64))
    mat = MatProps(intfrict_deg=30.0, bedfrict_deg=[20.0])
    one = oracle.run_reference_fwdadj(m, mat, 3, 1, WORKLOAD3_BOX)
    two = oracle.run_reference_fwdadj(m, mat, 3, 1, WORKLOAD3_BOX, replicas=2)
    assert len(one["replica_seconds"]) == 1 and len(two["replica_seconds"]) == 2
    assert np.array_equal(one["lam"], two["lam"])
    r = bench.reference_fwdadj(1, 1, side=64, replicas=2)
    assert r["cores"] == 2 and r["value"] > 0 and "2 harness processes" in r["sample"]
    cores = len(os.sched_getaffinity(0))
    assert 1 <= bench.reference_replicas(64 * 64) <= cores
    assert bench.reference_replicas(10 ** 12) == 1
