"""Ensembles (da_ensemble_*): every member of a batched run against its own single-instance run."""
import numpy as np
import pytest

from discrete_adjoint_b200 import (Ensemble, GeoflowContext, MatProps, Member, TimeProps, _ffi, adjoint_run,
                                   inputs)

pytestmark = pytest.mark.gpu


def members():
    """Uneven small members: hanging nodes everywhere, different sizes, materials and angles."""
    out = []
    for seed, (nx0, ny0), bed, phi_int in ((1, (24, 16), [20.0, 16.0], 32.0), (2, (12, 10), [18.0, 14.0], 30.0),
                                           (3, (30, 8), [24.0, 17.0], 34.0), (7, (16, 16), [15.0, 21.0], 28.0)):
        w = inputs.test_case(seed=seed, nx0=nx0, ny0=ny0)
        m = w.mesh
        wet = m.h0 > 1.0
        x0, x1, y0, y1 = m.x[wet].min(), m.x[wet].max(), m.y[wet].min(), m.y[wet].max()
        out.append(Member(m, MatProps(intfrict_deg=phi_int, bedfrict_deg=bed), (0.5 * (x0 + x1), x1 + 100.0, y0, y1)))
    return out


def single(mb, precision):
    c = GeoflowContext(mb.mat, TimeProps(), precision=precision)
    c.upload_mesh(mb.mesh)
    c.set_state(mb.mesh.h0, mb.mesh.hu0, mb.mesh.hv0)
    return c


@pytest.mark.parametrize("precision", [_ffi.DA_PREC_FP64, _ffi.DA_PREC_FP32_SPLIT])
def test_ensemble_forward_equals_single_runs(precision):
    mbs = members()
    with Ensemble(mbs, precision=precision) as ens:
        ens.forward(40)
        ens.forward(25)
        st = ens.stats()
        for k, mb in enumerate(mbs):
            with single(mb, precision) as c:
                s = c.run(65)
                ref = c.get_state()
            got = ens.get_state(k)
            for a, b in zip(got, ref):
                assert np.array_equal(a, b)
            assert st[k].dt == s.dt and st[k].time == s.time and st[k].iter == s.iter == 65
            assert abs(st[k].volume - s.volume) <= 1e-12 * s.volume


def test_ensemble_restart_and_autotune_keep_results():
    mbs = members()
    with Ensemble(mbs) as ens:
        ens.forward(30)
        a = [ens.get_state(k) for k in range(len(mbs))]
        ens.restart()
        ens.forward(10)
        ens.autotune(5)
        ens.forward(20)
        for k in range(len(mbs)):
            for u, v in zip(ens.get_state(k), a[k]):
                assert np.array_equal(u, v)


def test_ensemble_adjoint_equals_single_runs():
    mbs = members()
    with Ensemble(mbs) as ens:
        ens.forward(3)
        before = [ens.get_state(k) for k in range(len(mbs))]
        grads, ms = ens.adjoint(30, 4)
        assert ms > 0
        for k, mb in enumerate(mbs):
            for u, v in zip(ens.get_state(k), before[k]):
                assert np.array_equal(u, v)
            with single(mb, _ffi.DA_PREC_FP64) as c:
                c.run(3)
                g = adjoint_run(c, mb.box, 30, 4, mb.mesh.dh0_dpile[0])
            e = grads[k]
            assert e.forward_steps == g.forward_steps
            for x, y in [(e.J, g.J), (e.dJ_dintfrict, g.dJ_dintfrict), (e.dJ_dpile[0], g.dJ_dpile[0])] + \
                    list(zip(e.dJ_dbedfrict, g.dJ_dbedfrict)):
                assert abs(x - y) <= 1e-12 * max(abs(y), 1e-30), (k, x, y)
