"""The reference's element keys and forward solution records (host, no GPU): the keys against its
own fhsfc2d_, the gz records read and written by its own SolRec (the compiled reference, when the
harness is built) and by this library."""
import os
import tempfile

import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import inputs, records
from golden_util import GOLDEN

needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")


def test_keys_match_the_reference_fixture():
    z = np.load(os.path.join(GOLDEN, "hilbert_keys.npz"))
    assert np.array_equal(records.cell_keys(z["u"], z["v"], (0.0, 1.0), (0.0, 1.0)), z["keys"])


@needs_ref
def test_keys_match_the_reference_live():
    rng = np.random.default_rng(5)
    x, y = rng.uniform(-100.0, 2100.0, 3000), rng.uniform(50.0, 1950.0, 3000)
    xr, yr = (0.0, 2000.0), (100.0, 1900.0)
    ref = oracle.ref_hilbert_keys((x - xr[0]) / (xr[1] - xr[0]), (y - yr[0]) / (yr[1] - yr[0]))
    assert np.array_equal(records.cell_keys(x, y, xr, yr), ref)


def state(m, seed):
    rng = np.random.default_rng(seed)
    h = np.where(rng.random(m.n) < 0.3, rng.random(m.n), 0.0)
    return h, rng.standard_normal(m.n) * (h > 0), rng.standard_normal(m.n) * (h > 0)


def test_record_round_trip_and_missing_cells():
    m = inputs.test_case(seed=1).mesh
    k = records.mesh_keys(m)
    assert len(np.unique(k.view(np.uint64))) == m.n
    h, hu, hv = state(m, 0)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, records.solution_name(0, 3))
        records.write_solution(p, k, h, hu, hv)
        h2, hu2, hv2, miss = records.read_solution(p, k)
        assert miss == 0 and np.array_equal(h2, h) and np.array_equal(hu2, hu) and np.array_equal(hv2, hv)
        # a mesh with extra cells: those have no record
        extra = np.concatenate([k, np.array([[1, 2], [3, 4]], dtype=np.uint32)])
        h3, _, _, miss = records.read_solution(p, extra)
        assert miss == 2 and np.array_equal(h3[: m.n], h) and not h3[m.n:].any()
        # a record for a cell the mesh does not have is an error
        with pytest.raises(Exception):
            records.read_solution(p, k[: m.n - 5])


@needs_ref
def test_records_interoperate_with_the_reference_solrec():
    m = inputs.test_case(seed=2).mesh
    k = records.mesh_keys(m)
    h, hu, hv = state(m, 1)
    with tempfile.TemporaryDirectory() as d:
        # written here, read by the reference's read_sol_from_disk
        records.write_solution(os.path.join(d, records.solution_name(0, 7)), k, h, hu, hv)
        found, st = oracle.ref_read_solution(d, 0, 7, k)
        assert np.array_equal(found, np.where(h > 0, 2, 1))
        assert np.array_equal(st[:, 0], h) and np.array_equal(st[:, 1], hu) and np.array_equal(st[:, 2], hv)
    with tempfile.TemporaryDirectory() as d:
        # written by the reference's wrtie_sol_to_disk, read here
        oracle.ref_write_solution(d, 3, 12, k, h, hu, hv)
        h2, hu2, hv2, miss = records.read_solution(os.path.join(d, records.solution_name(3, 12)), k)
        assert miss == 0 and np.array_equal(h2, h) and np.array_equal(hu2, hu) and np.array_equal(hv2, hv)
