"""The reference's restart files (save_forward / loadrun, src/main/restart.C:21-239): this package's
reader on files the reference wrote, the reference's loadrun on files this package wrote, and
the round trip.  The reference side runs in oracle/_ref/ref_harness (modes 'DAS1' and 'DAL1')."""
import os

import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import MatProps, TimeProps, _ffi, inputs, make_params, records

needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")


def cases():
    return {
        "s11": inputs.test_case(seed=11, nx0=12, ny0=8, max_level=2, random_frac=0.4),
        "s2": inputs.test_case(seed=2),
    }


def outline_of(m):
    return ((10.0, 10.0), (float(m.x.min()) - 50.0, float(m.x.max()) + 50.0),
            (float(m.y.min()) - 50.0, float(m.y.max()) + 50.0))


def oracle_steps(w, h, hu, hv, nsteps, time=0.0, it=0):
    o = oracle.Oracle(make_params(w.mat, TimeProps()), w.mesh)
    o.set_time(time, it)
    rc, dts, st = o.run(h, hu, hv, nsteps)
    assert rc == 0
    return dts, st


def perm_by_centre(m, x, y):
    idx = {(a, b): i for i, (a, b) in enumerate(zip(m.x, m.y))}
    return np.array([idx[(a, b)] for a, b in zip(x, y)])


@needs_ref
@pytest.mark.parametrize("name,nsteps", [("s11", 30), ("s2", 60)])
def test_reader_takes_the_reference_save_forward(tmp_path, name, nsteps):
    w = cases()[name]
    m = w.mesh
    ref = oracle.run_reference_save(m, w.mat, m.h0, m.hu0, m.hv0, nsteps, outline_of(m), str(tmp_path))
    r = records.read_restart(str(tmp_path / "restart_0000"))
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    dts, st = oracle_steps(w, h, hu, hv, nsteps)
    rm = r["mesh"]
    assert rm.n == m.n and r["n_unresolved"] == 0 and r["n_elements"] == m.n
    p = perm_by_centre(m, rm.x, rm.y)
    assert sorted(p.tolist()) == list(range(m.n))
    # cells in key order, the reference's own keys
    k64 = (r["keys"][:, 0].astype(np.uint64) << np.uint64(32)) | r["keys"][:, 1]
    assert np.all(np.diff(k64.astype(np.float64)) > 0)
    rk = {(int(a), int(b)): i for i, (a, b) in enumerate(ref["keys"])}
    assert all((int(a), int(b)) in rk for a, b in r["keys"])
    # neighbour table, static fields, state, time history
    for k in range(8):
        g = np.where(rm.nbr[k] >= 0, p[np.maximum(rm.nbr[k], 0)], -1)
        assert np.array_equal(g, m.nbr[k][p])
    for f in ("dx", "dy", "material", "level"):
        assert np.array_equal(getattr(rm, f), getattr(m, f)[p])
    for f in ("gravity", "d_gravity", "curvature", "zeta"):
        assert np.array_equal(getattr(rm, f), getattr(m, f)[:, p])
    assert np.array_equal(r["h"], h[p]) and np.array_equal(r["hu"], hu[p]) and np.array_equal(r["hv"], hv[p])
    assert np.array_equal(r["dt"], dts) and r["time"] == st.time and r["iter"] == nsteps
    assert r["iter"] == ref["iter"] and np.array_equal(r["dt"], ref["dt"])


@needs_ref
@pytest.mark.parametrize("name,first,then", [("s11", 30, 40), ("s2", 20, 50)])
def test_reference_loadrun_continues_a_written_restart(tmp_path, name, first, then):
    # this package writes the restart of a run at step `first`; the reference's loadrun rebuilds its
    # tables from it and its step() continues: the state and the dt history equal the oracle's
    # uninterrupted run (past the frict_tiny switch at step 50)
    w = cases()[name]
    m = w.mesh
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    dts, st = oracle_steps(w, h, hu, hv, first)
    bed = [MatProps.rad(b) for b in w.mat.bedfrict_deg]
    records.write_restart(str(tmp_path / "restart_0000"), m, h, hu, hv, time=st.time, iteration=first,
                          dt_hist=dts, bedfrict=bed)
    ol = outline_of(m)
    nx, ny = int(round((ol[1][1] - ol[1][0]) / 10)), int(round((ol[2][1] - ol[2][0]) / 10))
    records.write_outline(str(tmp_path / "outline_0000"), *ol, np.zeros((ny, nx)))
    ref = oracle.run_reference_load(w.mat, then, ol, str(tmp_path))
    dts2, st2 = oracle_steps(w, h, hu, hv, then, st.time, first)
    p = perm_by_centre(m, ref["x"], ref["y"])
    assert len(p) == m.n
    assert np.array_equal(ref["h"], h[p]) and np.array_equal(ref["hu"], hu[p]) and np.array_equal(ref["hv"], hv[p])
    assert np.array_equal(ref["dt"], np.concatenate([dts, dts2])) and ref["iter"] == first + then
    assert ref["time"] == st2.time


def test_round_trip_keeps_mesh_state_and_header(tmp_path):
    w = cases()["s11"]
    m = w.mesh
    rng = np.random.default_rng(3)
    h = np.abs(rng.normal(size=m.n))
    hu, hv = rng.normal(size=m.n), rng.normal(size=m.n)
    dts = rng.uniform(0.01, 0.1, size=17)
    path = str(tmp_path / "restart_0003")
    records.write_restart(path, m, h, hu, hv, time=1.25, iteration=17, dt_hist=dts, adjiter=4, min_dx=(2.5, 3.5),
                          min_gen=1.0, maxh=(12, 7.5), solrec_last_step=16)
    r = records.read_restart(path)
    rm = r["mesh"]
    p = perm_by_centre(m, rm.x, rm.y)
    for k in range(8):
        g = np.where(rm.nbr[k] >= 0, p[np.maximum(rm.nbr[k], 0)], -1)
        assert np.array_equal(g, m.nbr[k][p])
    assert np.array_equal(r["h"], h[p]) and np.array_equal(r["hu"], hu[p]) and np.array_equal(r["hv"], hv[p])
    assert np.array_equal(r["dt"], dts) and r["time"] == 1.25 and r["iter"] == 17 and r["adjiter"] == 4
    assert r["min_dx"] == (2.5, 3.5) and r["min_gen"] == 1.0 and r["maxh"] == (12, 7.5)
    assert r["solrec_last_step"] == 16
    # keys: the Hilbert keys of the centres in the element table's range (da_cell_keys)
    keys = records.cell_keys(rm.x, rm.y, r["xrange"], r["yrange"])
    assert np.array_equal(keys, r["keys"])


def test_bad_files_and_arguments_are_errors(tmp_path):
    with pytest.raises(_ffi.DAError) as e:
        records.read_restart(str(tmp_path / "missing"))
    assert e.value.code == _ffi.DA_ERR_IO
    w = cases()["s11"]
    m = w.mesh
    path = str(tmp_path / "restart_0000")
    records.write_restart(path, m, m.h0, m.hu0, m.hv0)
    import gzip
    raw = gzip.open(path).read()
    gzip.open(str(tmp_path / "cut"), "wb").write(raw[: len(raw) // 2])
    with pytest.raises(_ffi.DAError) as e:
        records.read_restart(str(tmp_path / "cut"))
    assert e.value.code == _ffi.DA_ERR_IO
    with pytest.raises(_ffi.DAError) as e:
        records.write_restart(path, m, -np.ones(m.n), m.hu0, m.hv0)   # negative depth
    assert e.value.code == _ffi.DA_ERR_INVALID
