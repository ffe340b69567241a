"""Device forward step against the oracle (restated reference), through the C ABI."""
import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import GeoflowContext, TimeProps, _ffi, inputs, make_params
from discrete_adjoint_b200.mesh import Mesh, MeshSpec

pytestmark = pytest.mark.gpu

# FP32-split tolerance against the FP64 oracle (relative L2 over the mesh)
FP32_REL_L2_H = 1e-6
FP32_REL_L2_MOM = 1e-5


def oracle_run(w, nsteps, tp=None):
    m = w.mesh
    o = oracle.Oracle(make_params(w.mat, tp or TimeProps()), m)
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    rc, dts, st = o.run(h, hu, hv, nsteps)
    assert rc == 0
    return h, hu, hv, dts, st


def gpu_ctx(w, precision=_ffi.DA_PREC_FP64, tp=None, tile_culling=True):
    ctx = GeoflowContext(w.mat, tp or TimeProps(), precision=precision, tile_culling=tile_culling)
    ctx.upload_mesh(w.mesh)
    ctx.set_state(w.mesh.h0, w.mesh.hu0, w.mesh.hv0)
    return ctx


def rel_l2(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("seed", [1, 2, 3, 7])
def test_fp64_bit_exact_vs_oracle_100_steps(seed):
    w = inputs.test_case(seed=seed)
    h, hu, hv, dts, st = oracle_run(w, 100)
    with gpu_ctx(w) as ctx:
        gdts = [ctx.step().dt for _ in range(100)]
        gh, ghu, ghv = ctx.get_state()
    assert np.array_equal(np.array(gdts), dts)
    assert np.array_equal(gh, h) and np.array_equal(ghu, hu) and np.array_equal(ghv, hv)


def test_fp64_graph_run_equals_single_steps():
    w = inputs.test_case(seed=4)
    h, hu, hv, dts, st = oracle_run(w, 101)
    with gpu_ctx(w) as ctx:
        s = ctx.run(101)
        gh, ghu, ghv = ctx.get_state()
    assert s.iter == 101 and s.time == st.time and s.dt == dts[-1]
    assert np.array_equal(gh, h) and np.array_equal(ghu, hu) and np.array_equal(ghv, hv)
    assert abs(s.volume - st.volume) <= 1e-12 * st.volume


def test_fp64_workload1_bit_exact_200_steps():
    w = inputs.workload1()
    h, hu, hv, dts, st = oracle_run(w, 200)
    with gpu_ctx(w) as ctx:
        s = ctx.run(200)
        gh, ghu, ghv = ctx.get_state()
    assert s.time == st.time
    assert np.array_equal(gh, h) and np.array_equal(ghu, hu) and np.array_equal(ghv, hv)


def test_fp64_time_clipping_and_schedule():
    w = inputs.test_case(seed=2)
    tp = TimeProps(maxtime=2.5, nextoutput=1.0)
    h, hu, hv, dts, st = oracle_run(w, 60, tp=tp)
    with gpu_ctx(w, tp=tp) as ctx:
        s = ctx.run(60)
        gh, _, _ = ctx.get_state()
    assert s.time == st.time
    assert np.array_equal(gh, h)


@pytest.mark.parametrize("seed", [1, 3])
def test_fp32_split_close_to_fp64_oracle_before_threshold_switch(seed):
    # while frict_tiny = 0.1 (the first 50 steps, hpfem.C:232-235) every sign test is well
    # above FP32 resolution and the split path tracks the FP64 reference to rounding level
    w = inputs.test_case(seed=seed)
    h, hu, hv, dts, st = oracle_run(w, 50)
    with gpu_ctx(w, precision=_ffi.DA_PREC_FP32_SPLIT) as ctx:
        s = ctx.run(50)
        gh, ghu, ghv = ctx.get_state()
    eh, eu, ev = rel_l2(gh, h), rel_l2(ghu, hu), rel_l2(ghv, hv)
    print(f"fp32-split rel L2 after 50 steps: h {eh:.3e} hu {eu:.3e} hv {ev:.3e}")
    assert eh < FP32_REL_L2_H
    assert eu < FP32_REL_L2_MOM and ev < FP32_REL_L2_MOM
    assert abs(s.time - st.time) < 1e-6 * st.time


@pytest.mark.parametrize("precision", [_ffi.DA_PREC_FP64, _ffi.DA_PREC_FP32_SPLIT])
def test_tile_culling_is_bit_identical(precision):
    # a large mostly-dry mesh so that many tiles are culled, long enough for the flow to spread
    w = inputs.workload1()
    out = []
    for cull in (False, True):
        with gpu_ctx(w, precision=precision, tile_culling=cull) as ctx:
            s = ctx.run(150)
            out.append((ctx.get_state(), s))
    (a, sa), (b, sb) = out
    for u, v in zip(a, b):
        assert np.array_equal(u, v)
    assert sa.time == sb.time and sa.volume == sb.volume


@pytest.mark.parametrize("precision", [_ffi.DA_PREC_FP64, _ffi.DA_PREC_FP32_SPLIT])
@pytest.mark.parametrize("layer", [0.0, 0.5])
def test_tile_staging_is_bit_identical(precision, layer):
    # the staged phases (tile and halo in shared memory, activity recomputed from the staged
    # depths) against the phases that read neighbours from global memory: the adaptive mesh with
    # hanging nodes, with its piles alone (culled, sparse) and with a layer on every cell (dense);
    # every staging setting at two launch shapes, with single steps (the two-launch path) between
    # multi-step launches
    w = inputs.workload1()
    out = []
    for staging, occ in ((0, 0), (1, 3), (2, 2), (3, 2), (3, 3)):
        with GeoflowContext(w.mat, TimeProps(), precision=precision, tile_staging=staging,
                            blocks_per_sm=occ) as ctx:
            ctx.upload_mesh(w.mesh)
            ctx.set_state(w.mesh.h0 + layer, w.mesh.hu0, w.mesh.hv0)
            s = ctx.run(45)
            st = [ctx.step() for _ in range(3)]    # single steps between two multi-step launches
            s = ctx.run(42)
            out.append((ctx.get_state(), s, [x.dt for x in st]))
    a, sa, da = out[0]
    for b, sb, db in out[1:]:
        for u, v in zip(a, b):
            assert np.array_equal(u, v)
        assert sa.time == sb.time and sa.volume == sb.volume and sa.dt == sb.dt and da == db


@pytest.mark.parametrize("precision", [_ffi.DA_PREC_FP64, _ffi.DA_PREC_FP32_SPLIT])
def test_grid_size_and_autotune_do_not_change_results(precision):
    # the tiled kernels' results do not depend on the grid (fixed-order volume sum, min for dt),
    # and the autotuner puts the state, time and iteration back after its trials
    w = inputs.workload1()
    out = []
    for grid, occ in ((1, 2), (7, 3), (148, 0), (0, 3), (4096, 2)):
        with GeoflowContext(w.mat, TimeProps(), precision=precision, grid_blocks=grid, blocks_per_sm=occ) as ctx:
            ctx.upload_mesh(w.mesh)
            ctx.set_state(w.mesh.h0, w.mesh.hu0, w.mesh.hv0)
            s = ctx.run(120)
            out.append((ctx.get_state(), s))
    with gpu_ctx(w, precision=precision) as ctx:
        ctx.run(40)
        r = ctx.autotune(10)
        assert r["best"] in r["ms_per_step"] and all(v > 0 for v in r["ms_per_step"].values())
        s = ctx.run(80)
        out.append((ctx.get_state(), s))
    a, sa = out[0]
    for b, sb in out[1:]:
        for u, v in zip(a, b):
            assert np.array_equal(u, v)
        assert sa.time == sb.time and sa.volume == sb.volume and sa.iter == sb.iter


def test_set_state_resets_culling():
    w = inputs.test_case(seed=2)
    h, hu, hv, dts, st = oracle_run(w, 30)
    with gpu_ctx(w) as ctx:
        ctx.run(7)
        ctx.set_state(w.mesh.h0, w.mesh.hu0, w.mesh.hv0)
        ctx.set_time(0.0, 0)
        ctx.run(30)
        gh, ghu, ghv = ctx.get_state()
    assert np.array_equal(gh, h) and np.array_equal(ghu, hu) and np.array_equal(ghv, hv)


def test_errors_are_codes_not_exits():
    w = inputs.test_case(seed=1)
    ctx = GeoflowContext(w.mat, TimeProps())
    with pytest.raises(_ffi.DAError) as e:
        ctx.step()
    assert e.value.code == _ffi.DA_ERR_NO_MESH
    bad = Mesh(**{k: np.copy(v) for k, v in w.mesh.arrays().items()})
    bad.nbr[0, 5] = w.mesh.n + 3
    with pytest.raises(_ffi.DAError) as e:
        ctx.upload_mesh(bad)
    assert e.value.code == _ffi.DA_ERR_INVALID
    ctx.upload_mesh(w.mesh)
    h = w.mesh.h0.copy()
    h[np.argmax(h)] = np.nan
    ctx.set_state(h, w.mesh.hu0, w.mesh.hv0)
    with pytest.raises(_ffi.DAError) as e:
        ctx.run(3)
    assert e.value.code in (_ffi.DA_ERR_NAN,)
    ctx.close()


def outline_host(m, h, g, x0, y0, dx, dy, nx, ny):
    """OutLine::update (properties.h:726-790) of every cell, numpy loops (reference order)."""
    for i in range(m.n):
        xs, xe = m.x[i] - 0.5 * m.dx[i], m.x[i] + 0.5 * m.dx[i]
        ys, ye = m.y[i] - 0.5 * m.dy[i], m.y[i] + 0.5 * m.dy[i]
        ix0, ix1 = int((xs - x0) / dx + 0.5), int((xe - x0) / dx + 0.5)
        iy0, iy1 = int((ys - y0) / dy + 0.5), int((ye - y0) / dy + 0.5)
        ix0 = max(ix0, 0)
        if ix1 == ix0:
            ix0 = int((xs - x0) / dx)
            ix1 = ix0 + 1
        ix1 = min(ix1, nx)
        iy0 = max(iy0, 0)
        if iy1 == iy0:
            iy0 = int((ys - y0) / dy)
            iy1 = iy0 + 1
        iy1 = min(iy1, ny)
        blk = g[iy0:iy1, ix0:ix1]
        np.maximum(blk, h[i], out=blk)


def test_max_depth_map_matches_host_restatement():
    w = inputs.test_case(seed=3)
    m = w.mesh
    x0, y0 = 0.0, 0.0
    xr, yr = (x0, m.x.max() + 20.0), (y0, m.y.max() + 20.0)
    dxy = (15.0, 12.5)  # not aligned with the cells, so footprints cut grid cells
    nx, ny = int((xr[1] - xr[0]) / dxy[0] + 0.5), int((yr[1] - yr[0]) / dxy[1] + 0.5)
    g = np.zeros((ny, nx))
    with gpu_ctx(w) as ctx:
        ctx.outline_init(dxy, xr, yr)
        for _ in range(12):
            ctx.step()
            ctx.outline_update()
            outline_host(m, ctx.get_state()[0], g, x0, y0, dxy[0], dxy[1], nx, ny)
        dev = ctx.outline()
    assert dev.shape == (ny, nx)
    assert np.array_equal(dev, g) and g.max() > 0
