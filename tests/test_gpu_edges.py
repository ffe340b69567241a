"""Edge cases of the device step against the oracle: meshes smaller than a tile, exactly one tile,
a last tile left ragged, every side of every cell on the domain edge (one and two cells); a dry
mesh (no wet cell: dt is half the flux source's time scale when there is one and the state stays
put; with none, dt is infinite and the step is reported as DA_ERR_NAN, as by the restatement and
as the reference's own step stops at its state check); an empty mesh and missing arguments
refused with DA_ERR_INVALID."""
import ctypes as C
import math

import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import GeoflowContext, TimeProps, _ffi, inputs, make_params

pytestmark = pytest.mark.gpu

# (nx0, ny0, max_level, random_frac): 1, 2, 12, 36, 256, 272 and 876 cells
SHAPES = [(1, 1, 0, 0.0), (2, 1, 0, 0.0), (1, 3, 1, 0.0), (3, 3, 1, 0.5), (16, 16, 0, 0.0), (16, 17, 0, 0.0),
          (9, 7, 2, 0.4)]


@pytest.mark.parametrize("shape", SHAPES, ids=lambda s: "x".join(map(str, s[:3])))
def test_small_and_ragged_meshes_match_the_oracle(shape):
    nx, ny, lev, rf = shape
    w = inputs.test_case(seed=5, nx0=nx, ny0=ny, max_level=lev, random_frac=rf)
    m = w.mesh
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    rc, dts, st = o.run(h, hu, hv, 60)
    assert rc == 0
    for staging in (0, 1):
        with GeoflowContext(w.mat, TimeProps(), tile_staging=staging) as c:
            c.upload_mesh(m)
            c.set_state(m.h0, m.hu0, m.hv0)
            c.run(25)
            d = [c.step().dt for _ in range(5)]   # the two-launch path between multi-step launches
            s = c.run(30)
            H, HU, HV = c.get_state()
        assert np.array_equal(H, h) and np.array_equal(HU, hu) and np.array_equal(HV, hv)
        assert d == list(dts[25:30]) and s.time == st.time and s.iter == 60
        # the volume is a sum in another order (segment partials, then the partials in order)
        assert abs(s.volume - st.volume) <= 1e-12 * st.volume


def test_dry_mesh():
    w = inputs.test_case(seed=5, nx0=6, ny0=5, max_level=1, random_frac=0.3)
    m = w.mesh
    z = np.zeros(m.n)
    # a flux source's time scale: dt = influx_dt / 2 while nothing is wet, the state stays zero
    o = oracle.Oracle(make_params(w.mat, TimeProps(), influx_dt=3.0), m)
    h, hu, hv = z.copy(), z.copy(), z.copy()
    rc, dts, st = o.run(h, hu, hv, 4)
    assert rc == 0 and list(dts) == [1.5] * 4
    with GeoflowContext(w.mat, TimeProps(), influx_dt=3.0) as c:
        c.upload_mesh(m)
        c.set_state(z, z, z)
        s = c.run(4)
        H, HU, HV = c.get_state()
    assert s.time == st.time == 6.0 and s.iter == 4 and s.volume == 0.0
    assert not H.any() and not HU.any() and not HV.any()
    # no flux source: an infinite dt, a non-finite update, reported rather than taken
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    rc, dts, _ = o.run(z.copy(), z.copy(), z.copy(), 1)
    assert rc == _ffi.DA_ERR_NAN and math.isinf(dts[0])
    for run in (lambda c: c.run(1), lambda c: c.step()):   # the multi-step kernel, the two launches
        with GeoflowContext(w.mat, TimeProps()) as c:
            c.upload_mesh(m)
            c.set_state(z, z, z)
            with pytest.raises(_ffi.DAError) as e:
                run(c)
            assert e.value.code == _ffi.DA_ERR_NAN


def test_empty_mesh_and_missing_arguments_are_refused():
    w = inputs.test_case(seed=5, nx0=3, ny0=3, max_level=1, random_frac=0.5)
    with GeoflowContext(w.mat, TimeProps()) as c:
        lib, ctx = c.lib, c.ctx
        soa = w.mesh.soa()
        empty = _ffi.da_mesh_soa()
        C.memmove(C.byref(empty), C.byref(soa), C.sizeof(soa))
        empty.n_cells = 0
        assert lib.da_upload_mesh(ctx, C.byref(empty), 0) == _ffi.DA_ERR_INVALID
        assert lib.da_upload_mesh(ctx, None, 0) == _ffi.DA_ERR_INVALID
        s = _ffi.da_step_stats()
        assert lib.da_forward_run(ctx, 2, C.byref(s)) == _ffi.DA_ERR_NO_MESH
        c.upload_mesh(w.mesh)
        assert lib.da_set_state(ctx, None, None, None) == _ffi.DA_ERR_INVALID
        h = np.ascontiguousarray(w.mesh.h0)
        assert lib.da_set_state(ctx, _ffi.dptr(h), None, _ffi.dptr(h)) == _ffi.DA_ERR_INVALID
        assert lib.da_get_state(ctx, None, None, None) == _ffi.DA_ERR_INVALID
        c.set_state(w.mesh.h0, w.mesh.hu0, w.mesh.hv0)
        f = _ffi.da_functional(_ffi.DA_FUNC_H2_BOX, 0, (C.c_double * 4)(0.0, 1e9, 0.0, 1e9))
        g = _ffi.da_gradient()
        assert lib.da_adjoint_run(ctx, C.byref(f), 0, 4, None, 0, C.byref(g), None) == _ffi.DA_ERR_INVALID
        assert lib.da_adjoint_run(ctx, C.byref(f), 5, -1, None, 0, C.byref(g), None) == _ffi.DA_ERR_INVALID
        assert lib.da_adjoint_run(ctx, C.byref(f), 5, 2, None, 1, C.byref(g), None) == _ffi.DA_ERR_INVALID
        # the context is still usable after the refusals
        s0 = c.run(3)
        assert s0.iter == 3


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


@pytest.mark.parametrize("shape", [SHAPES[1], SHAPES[2], SHAPES[5], SHAPES[6]], ids=lambda s: "x".join(map(str, s[:3])))
def test_small_and_ragged_meshes_adjoint(shape):
    # the reference's adjoint (jacobian_mode = reference) as a checkpointed sweep against the
    # oracle's chained dual-solver steps, 1e-12; the exact transpose, one reverse step at a time,
    # against the oracle's dual-solver step without the reference's approximations, 1e-9 (the
    # tolerances of the fixture-mesh tests in test_gpu_adjoint_ref.py)
    from discrete_adjoint_b200 import adjoint_run, adjoint_step
    from test_oracle_adjoint import forward_states, frict_tiny
    nx, ny, lev, rf = shape
    w = inputs.test_case(seed=5, nx0=nx, ny0=ny, max_level=lev, random_frac=rf)
    m = w.mesh
    N = 30
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    states, dts = forward_states(o, m, N)
    box = (float(m.x.min()) - 1.0, float(m.x.max()) + 1.0, float(m.y.min()) - 1.0, float(m.y.max()) + 1.0)
    lam = np.zeros((3, m.n))
    lam[0] = 2.0 * states[N][0] * (m.dx * m.dy)
    for it in range(N, 0, -1):
        lam = o.adjoint_step_ref(*states[it - 1], dts[it - 1], frict_tiny(it), lam)
    dh0 = (m.h0 > 0).astype(np.float64).reshape(1, m.n)
    with GeoflowContext(w.mat, TimeProps(), jacobian_mode=_ffi.DA_JAC_REFERENCE) as c:
        c.upload_mesh(m)
        c.set_state(m.h0, m.hu0, m.hv0)
        g = adjoint_run(c, box, N, 4, dh0_dpile=dh0, want_lambda0=True)
    assert rel(g.lambda0, lam) <= 1e-12
    rng = np.random.default_rng(7)
    with GeoflowContext(w.mat, TimeProps()) as c:
        c.upload_mesh(m)
        for it in (N, 17, 1):
            lam_next = rng.standard_normal((3, m.n))
            c.set_state(*states[it - 1])
            c.set_time(float(np.sum(dts[:it - 1])), it - 1)
            lam_dev, _ = adjoint_step(c, lam_next)
            ex = o.adjoint_step_ref(*states[it - 1], dts[it - 1], frict_tiny(it), lam_next, keep=0)
            assert rel(lam_dev, ex) <= 1e-9, it
