"""The oracle against the reference's own step(): committed golden fixtures (always) and the
compiled reference harness run live on fresh seeds (when oracle/_ref/ref_harness exists)."""
import os

import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import TimeProps, inputs, make_params
from golden_util import fixtures, load


@pytest.mark.parametrize("path", fixtures(), ids=os.path.basename)
def test_oracle_matches_reference_fixture_bit_for_bit(path):
    mesh, mat, nsteps, ref = load(path)
    o = oracle.Oracle(make_params(mat, TimeProps()), mesh)
    h, hu, hv = mesh.h0.copy(), mesh.hu0.copy(), mesh.hv0.copy()
    rc, dts, st = o.run(h, hu, hv, nsteps - 1)
    assert rc == 0
    # the last step's intermediate fields, from the state entering it
    s = o.slopes(h, hu, hv)
    rc, kact, _, _ = o.coef_eigen(h, hu, hv, s)
    F = o.edge_fluxes(h, hu, hv, kact)
    assert np.array_equal(s, ref["slopes"])
    assert np.array_equal(kact, ref["kact"])
    assert np.array_equal(F, ref["flux"])
    rc, dt_last, st = o.run(h, hu, hv, 1)
    assert np.array_equal(np.concatenate([dts, dt_last]), ref["dt"])
    assert st.time == ref["time"]
    assert np.array_equal(h, ref["h"]) and np.array_equal(hu, ref["hu"]) and np.array_equal(hv, ref["hv"])


@pytest.mark.parametrize("path", fixtures(), ids=os.path.basename)
def test_host_static_fields_match_reference(path):
    mesh, mat, nsteps, ref = load(path)
    import numpy as _np
    z = _np.load(path)
    assert np.array_equal(mesh.gravity, z["ref_static_gravity"])
    assert np.array_equal(mesh.d_gravity, z["ref_static_d_gravity"])


def test_fixtures_exercise_every_case():
    kinds = set()
    for p in fixtures():
        m, mat, n, ref = load(p)
        two = (m.nbr[4:] != m.nbr[:4]) & (m.nbr[:4] >= 0)
        if two.any():
            kinds.add("S_C_CON")
            kinds.add("S_S_CON")
        if (m.nbr[:4] < 0).any():
            kinds.add("boundary")
        if len(mat.bedfrict_deg) > 1:
            kinds.add("materials")
        if n > 50:
            kinds.add("frict_tiny switch")
        if (ref["h"] > 0).any() and (ref["h"] == 0).any():
            kinds.add("dry/wet front")
    assert kinds == {"S_C_CON", "S_S_CON", "boundary", "materials", "frict_tiny switch", "dry/wet front"}


needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")


@needs_ref
@pytest.mark.parametrize("seed,frac,L", [(21, 0.35, 2), (22, 0.5, 3), (23, 0.0, 2)])
def test_oracle_matches_live_reference(seed, frac, L):
    w = inputs.test_case(seed=seed, random_frac=frac, max_level=L, nx0=16, ny0=12)
    m = w.mesh
    ref = oracle.run_reference(m, w.mat, m.h0, m.hu0, m.hv0, 80)
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    rc, dts, st = o.run(h, hu, hv, 80)
    assert np.array_equal(dts, ref["dt"]) and st.time == ref["time"]
    assert np.array_equal(h, ref["h"]) and np.array_equal(hu, ref["hu"]) and np.array_equal(hv, ref["hv"])


@needs_ref
def test_oracle_matches_live_reference_time_clipping():
    w = inputs.test_case(seed=24)
    m = w.mesh
    ref = oracle.run_reference(m, w.mat, m.h0, m.hu0, m.hv0, 40, maxtime=1.7)
    o = oracle.Oracle(make_params(w.mat, TimeProps(maxtime=1.7)), m)
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    rc, dts, st = o.run(h, hu, hv, 40)
    assert np.array_equal(dts, ref["dt"]) and st.time == ref["time"] == 1.7
    assert np.array_equal(h, ref["h"])


def test_stats_fixture_matches_a_live_reference_run():
    # the committed calc_stats / DISCHARGE fixture still matches the reference when it can be run
    import numpy as np
    import pytest

    import oracle
    from golden_util import GOLDEN, load_stats
    if not oracle.reference_available():
        pytest.skip("reference harness not built")
    import os
    mesh, mat, nsteps, z = load_stats(os.path.join(GOLDEN, "stats_s12_80.npz"))
    r = oracle.run_reference(mesh, mat, mesh.h0, mesh.hu0, mesh.hv0, nsteps, test_point=tuple(z["test_point"]),
                             vslump=float(z["vslump"]), planes=[tuple(p) for p in z["planes"]])
    assert np.array_equal(r["h"], z["ref_h"])
    assert np.array_equal(np.array([r["stats"][k] for k in oracle.STAT_FIELDS]), z["stat_values"])
    assert np.array_equal(r["discharge"], z["discharge"])
