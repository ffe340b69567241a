"""The large single-instance workload at full size (67M cells, 40 km x 40 km of fractal terrain,
uniform 8192^2), checked through a size-independent property: its cells and static fields are
those of a centred crop of the same terrain, so a flow that stays well inside the crop evolves
bit for bit as on the 4M-cell crop alone (the same wet cells give the same dt), forward and
adjoint.  This exercises indexing, tiling, halo tables and checkpoints at 67M cells against a mesh
size the other tests cover.  Also one full-horizon forward + adjoint run (2000 steps, FP32-split,
64 checkpoints) whose J and gradients must be finite and whose state must be put back."""
import numpy as np
import pytest

from discrete_adjoint_b200 import GeoflowContext, TimeProps, _ffi, adjoint_run, inputs

pytestmark = pytest.mark.gpu

CROP = 2048
MARGIN = 64  # cells: the flow must stay this far inside the crop
FWD_STEPS = 400
ADJ_STEPS = 160


@pytest.fixture(scope="module")
def meshes():
    big = inputs.workload5()
    crop = inputs.workload5(crop=CROP, dem=big.dem)
    # crop cell -> full-mesh cell, by the finest-level integer coordinates
    off = (inputs.WORKLOAD5_SIDE - CROP) // 2
    side = inputs.WORKLOAD5_SIDE
    inv = np.empty(side * side, dtype=np.int64)
    inv[big.mesh.iy.astype(np.int64) * side + big.mesh.ix] = np.arange(big.mesh.n)
    idx = inv[(crop.mesh.iy.astype(np.int64) + off) * side + crop.mesh.ix + off]
    return big, crop, idx


def _inside(crop_mesh, h):
    """The crop's wet cells keep MARGIN cells away from its edges."""
    wet = h >= 1e-4
    lo, hi = MARGIN, CROP - MARGIN
    return bool(np.all((crop_mesh.ix[wet] >= lo) & (crop_mesh.ix[wet] < hi) &
                       (crop_mesh.iy[wet] >= lo) & (crop_mesh.iy[wet] < hi)))


def _run(w, precision, nsteps):
    with GeoflowContext(w.mat, TimeProps(), precision=precision) as c:
        c.upload_mesh(w.mesh)
        c.set_state(w.mesh.h0, w.mesh.hu0, w.mesh.hv0)
        s = c.run(nsteps)
        return c.get_state(), s


@pytest.mark.parametrize("precision", [_ffi.DA_PREC_FP64, _ffi.DA_PREC_FP32_SPLIT])
def test_full_size_forward_equals_the_crop(meshes, precision):
    big, crop, idx = meshes
    (hb, hub, hvb), sb = _run(big, precision, FWD_STEPS)
    (hc, huc, hvc), sc = _run(crop, precision, FWD_STEPS)
    assert _inside(crop.mesh, hc)
    # nothing wet outside the crop region of the full mesh
    outside = np.ones(big.mesh.n, dtype=bool)
    outside[idx] = False
    assert not np.any(hb[outside] >= 1e-4)
    assert sb.dt == sc.dt and sb.time == sc.time
    assert np.array_equal(hb[idx], hc) and np.array_equal(hub[idx], huc) and np.array_equal(hvb[idx], hvc)


def test_full_size_adjoint_equals_the_crop(meshes):
    big, crop, idx = meshes
    p = big.piles[0]
    box = (p.xc - 400.0, p.xc + 400.0, p.yc - 400.0, p.yc + 400.0)
    out = []
    for w in (big, crop):
        with GeoflowContext(w.mat, TimeProps()) as c:
            c.upload_mesh(w.mesh)
            c.set_state(w.mesh.h0, w.mesh.hu0, w.mesh.hv0)
            out.append(adjoint_run(c, box, ADJ_STEPS, 12, w.mesh.dh0_dpile, want_lambda0=True))
    gb, gc = out
    assert gc.J > 0
    assert gb.J == gc.J and gb.dJ_dintfrict == gc.dJ_dintfrict
    assert np.array_equal(gb.dJ_dbedfrict, gc.dJ_dbedfrict) and np.array_equal(gb.dJ_dpile, gc.dJ_dpile)
    nb, nc = big.mesh.n, crop.mesh.n
    lb, lc = gb.lambda0.reshape(3, nb), gc.lambda0.reshape(3, nc)
    assert np.array_equal(lb[:, idx], lc)


def test_full_horizon_forward_adjoint_fp32_split(meshes):
    big, _, _ = meshes
    m = big.mesh
    p = big.piles[0]
    box = (p.xc - 600.0, p.xc + 600.0, p.yc - 600.0, p.yc + 600.0)
    with GeoflowContext(big.mat, TimeProps(), precision=_ffi.DA_PREC_FP32_SPLIT,
                        influx_dt=inputs.influx5_dt(m)) as c:
        c.upload_mesh(m)
        c.set_state(m.h0, m.hu0, m.hv0)
        g = adjoint_run(c, box, big.nsteps, 64, m.dh0_dpile)
        h = c.get_state()[0]
    assert np.isfinite(g.J) and np.isfinite(g.dJ_dintfrict)
    assert np.all(np.isfinite(g.dJ_dbedfrict)) and np.all(np.isfinite(g.dJ_dpile))
    assert np.array_equal(h, m.h0.astype(np.float32).astype(np.float64))
