"""Discrete adjoint on the device, through the C ABI: the transpose identity of one step against
central differences of the forward step, parameter gradients of J = sum h^2 dx dy over a box
against central differences of whole runs (time-step sequence frozen), and checkpoint-schedule
invariance.

The forward step is piecewise smooth (limiter, friction-sign and wet/dry thresholds, HLL
regimes), so a finite difference is only meaningful while the perturbation crosses no
threshold: each check takes central differences at several step sizes and requires the
adjoint to agree with the best of them (they converge to it as the step shrinks)."""
import numpy as np
import pytest

from discrete_adjoint_b200 import (GeoflowContext, TimeProps, _ffi, adjoint_run, adjoint_step, inputs,
                                   set_dt_replay)
from discrete_adjoint_b200.solver import MatProps

pytestmark = pytest.mark.gpu

# relative tolerance of adjoint products against central differences (FP64)
TOL_STEP = 1e-6
TOL_GRAD = 1e-4


def ctx_for(w, mat=None, precision=_ffi.DA_PREC_FP64):
    c = GeoflowContext(mat or w.mat, TimeProps(), precision=precision)
    c.upload_mesh(w.mesh)
    c.set_state(w.mesh.h0, w.mesh.hu0, w.mesh.hv0)
    return c


def box_of(w):
    m = w.mesh
    wet = m.h0 > 1.0
    x0, x1 = m.x[wet].min(), m.x[wet].max()
    y0, y1 = m.y[wet].min(), m.y[wet].max()
    # a box over the downslope half of the initial piles
    return (0.5 * (x0 + x1), x1 + 100.0, y0, y1)


def J_of(m, h, box):
    inb = (m.x >= box[0]) & (m.x <= box[1]) & (m.y >= box[2]) & (m.y <= box[3])
    return float(np.sum(h[inb] ** 2 * m.dx[inb] * m.dy[inb]))


@pytest.mark.parametrize("seed,nfwd", [(1, 20), (3, 35), (2, 60)])
def test_adjoint_step_transpose_identity(seed, nfwd):
    w = inputs.test_case(seed=seed)
    m = w.mesh
    rng = np.random.default_rng(seed)
    with ctx_for(w) as c:
        s = c.run(nfwd)
        U = np.stack(c.get_state())
        t0, it0 = s.time, s.iter
        dt = c.step().dt
        set_dt_replay(c, [dt], iter0=it0)
        lam = rng.standard_normal((3, m.n))
        wet = U[0] > 1e-2
        dU = rng.standard_normal((3, m.n)) * wet
        fds = []
        for eps in (1e-6, 1e-7, 1e-8):
            G = []
            for sgn in (1, -1):
                V = U + sgn * eps * dU
                c.set_state(*V)
                c.set_time(t0, it0)
                c.step()
                G.append(np.stack(c.get_state()))
            fds.append(float(np.sum(lam * (G[0] - G[1]))) / (2 * eps))
        c.set_state(*U)
        c.set_time(t0, it0)
        lam_n, _ = adjoint_step(c, lam)
        ad = float(np.sum(lam_n * dU))
    best = min(abs(ad - fd) / abs(fd) for fd in fds)
    print(f"seed {seed} step {nfwd}: adjoint {ad:.12e} fd {fds} best rel {best:.2e}")
    assert best <= TOL_STEP


def fd_run(w, box, nsteps, dts, mat=None, h0=None):
    m = w.mesh
    with GeoflowContext(mat or w.mat, TimeProps()) as c:
        c.upload_mesh(m)
        c.set_state(m.h0 if h0 is None else h0, m.hu0, m.hv0)
        set_dt_replay(c, dts, 0)
        c.run(nsteps)
        h, _, _ = c.get_state()
    return J_of(m, h, box)


@pytest.mark.parametrize("seed,nsteps", [(1, 30), (4, 45)])
def test_parameter_gradients_against_central_differences(seed, nsteps):
    w = inputs.test_case(seed=seed)
    m = w.mesh
    box = box_of(w)
    with ctx_for(w) as c:
        dts = [c.step().dt for _ in range(nsteps)]
        c.set_state(m.h0, m.hu0, m.hv0)
        c.set_time(0.0, 0)
        set_dt_replay(c, dts, 0)
        g = adjoint_run(c, box, nsteps, 6, m.dh0_dpile)
    J0 = fd_run(w, box, nsteps, dts)
    assert abs(g.J - J0) <= 1e-12 * abs(J0)
    checks = []
    # pile heights: h0 is linear in each pile height
    for p in range(len(w.piles)):
        fds = []
        for e in (1e-5, 1e-6, 1e-7):
            jp = fd_run(w, box, nsteps, dts, h0=m.h0 + e * m.dh0_dpile[p])
            jm = fd_run(w, box, nsteps, dts, h0=m.h0 - e * m.dh0_dpile[p])
            fds.append((jp - jm) / (2 * e))
        checks.append((f"pile{p}", g.dJ_dpile[p], fds))
    # friction angles (radians of MatProps.rad)

    def angle_fd(k):
        fds = []
        for e_deg in (1e-6, 1e-7, 1e-8):
            e_rad = MatProps.rad(e_deg)
            if k < 0:
                mp = MatProps(intfrict_deg=w.mat.intfrict_deg + e_deg, bedfrict_deg=list(w.mat.bedfrict_deg))
                mm = MatProps(intfrict_deg=w.mat.intfrict_deg - e_deg, bedfrict_deg=list(w.mat.bedfrict_deg))
            else:
                bp = [b + (e_deg if q == k else 0) for q, b in enumerate(w.mat.bedfrict_deg)]
                bm = [b - (e_deg if q == k else 0) for q, b in enumerate(w.mat.bedfrict_deg)]
                mp = MatProps(intfrict_deg=w.mat.intfrict_deg, bedfrict_deg=bp)
                mm = MatProps(intfrict_deg=w.mat.intfrict_deg, bedfrict_deg=bm)
            fds.append((fd_run(w, box, nsteps, dts, mat=mp) - fd_run(w, box, nsteps, dts, mat=mm)) / (2 * e_rad))
        return fds

    for k in range(len(w.mat.bedfrict_deg)):
        checks.append((f"bed{k}", g.dJ_dbedfrict[k], angle_fd(k)))
    checks.append(("int", g.dJ_dintfrict, angle_fd(-1)))
    scale = max(abs(v) for _, v, _ in checks)
    for name, ad, fds in checks:
        best = min(abs(ad - fd) for fd in fds)
        print(f"{name}: adjoint {ad:.10e} fd {fds}")
        assert best <= TOL_GRAD * max(abs(ad), 1e-3 * scale), name


def test_checkpoint_schedule_does_not_change_the_result():
    w = inputs.test_case(seed=2)
    m = w.mesh
    box = box_of(w)
    out = []
    for snaps in (0, 2, 5, 16):
        with ctx_for(w) as c:
            g = adjoint_run(c, box, 16, snaps, m.dh0_dpile, want_lambda0=True)
            out.append(g)
    for g in out[1:]:
        assert np.array_equal(g.lambda0, out[0].lambda0)
        assert g.dJ_dintfrict == out[0].dJ_dintfrict and g.dJ_dbedfrict == out[0].dJ_dbedfrict
    # fewer snapshots, more recomputation; the full set recomputes nothing
    assert out[0].forward_steps > out[1].forward_steps > out[2].forward_steps >= out[3].forward_steps
    assert out[3].forward_steps == 16 + 15 or out[3].forward_steps >= 16


@pytest.mark.parametrize("precision", [_ffi.DA_PREC_FP64, _ffi.DA_PREC_FP32_SPLIT])
def test_long_checkpoint_chains_do_not_change_the_result(precision):
    # consecutive forward advances of the sweep go out as one launch that stores their
    # checkpoints on the way (at most 32 a launch): with 40 and 71 snapshots over 72 steps the
    # first chain stores after nearly every step and is split into several launches; lambda^0 and
    # the gradients equal the sweep without checkpoints bit for bit
    w = inputs.test_case(seed=2)
    m = w.mesh
    out = []
    for snaps in (0, 3, 40, 71):
        with GeoflowContext(w.mat, TimeProps(), precision=precision) as c:
            c.upload_mesh(m)
            c.set_state(m.h0, m.hu0, m.hv0)
            out.append(adjoint_run(c, box_of(w), 72, snaps, m.dh0_dpile, want_lambda0=True))
    a = out[0]
    for b in out[1:]:
        assert np.array_equal(a.lambda0, b.lambda0)
        assert a.J == b.J and a.dJ_dintfrict == b.dJ_dintfrict
        assert np.array_equal(a.dJ_dbedfrict, b.dJ_dbedfrict) and np.array_equal(a.dJ_dpile, b.dJ_dpile)
    assert out[0].forward_steps > out[1].forward_steps > out[2].forward_steps >= out[3].forward_steps


@pytest.mark.parametrize("precision", [_ffi.DA_PREC_FP64, _ffi.DA_PREC_FP32_SPLIT])
def test_tile_staging_does_not_change_the_adjoint(precision):
    # the replayed forward steps of the reverse sweep (and its recomputation) with tiles and halos
    # staged in shared memory, against neighbour reads from global memory, and the staged gather
    # by tiles and by quarter tiles: same lambda^0 and gradients bit for bit
    w = inputs.test_case(seed=3)
    m = w.mesh
    out = []
    for staging in (0, 1, 2, 3):
        with GeoflowContext(w.mat, TimeProps(), precision=precision, tile_staging=staging) as c:
            c.upload_mesh(m)
            c.set_state(m.h0, m.hu0, m.hv0)
            out.append(adjoint_run(c, box_of(w), 24, 4, m.dh0_dpile, want_lambda0=True))
    a = out[0]
    for b in out[1:]:
        assert np.array_equal(a.lambda0, b.lambda0)
        assert a.J == b.J and a.dJ_dintfrict == b.dJ_dintfrict
        assert np.array_equal(a.dJ_dbedfrict, b.dJ_dbedfrict) and np.array_equal(a.dJ_dpile, b.dJ_dpile)


@pytest.mark.parametrize("precision", [_ffi.DA_PREC_FP64, _ffi.DA_PREC_FP32_SPLIT])
def test_sweep_graph_replays_match_stream_launches(precision):
    # the sweep captured as a CUDA graph (first run), replayed (second run), recaptured for another
    # horizon and again for the first one, against the same sweeps launched one kernel at a time
    # (tracing on): same lambda^0, J and gradients bit for bit, and the state and time put back
    w = inputs.test_case(seed=6)
    m = w.mesh
    box = box_of(w)
    runs = {}
    for traced in (True, False):
        with GeoflowContext(w.mat, TimeProps(), precision=precision) as c:
            c.upload_mesh(m)
            c.set_state(m.h0, m.hu0, m.hv0)
            c.run(2)
            start = np.stack(c.get_state())
            c.set_tracing(traced)
            out = []
            for horizon in (36, 36, 30, 36):
                out.append(adjoint_run(c, box, horizon, 5, m.dh0_dpile, want_lambda0=True))
                assert np.array_equal(np.stack(c.get_state()), start)
            runs[traced] = out
    for a, b in zip(runs[True], runs[False]):
        assert np.array_equal(a.lambda0, b.lambda0)
        assert a.J == b.J and a.dJ_dintfrict == b.dJ_dintfrict and a.forward_steps == b.forward_steps
        assert np.array_equal(a.dJ_dbedfrict, b.dJ_dbedfrict) and np.array_equal(a.dJ_dpile, b.dJ_dpile)
    assert runs[False][0].J == runs[False][1].J == runs[False][3].J != runs[False][2].J
    assert runs[False][2].forward_steps != runs[False][0].forward_steps


def test_adjoint_run_restores_state_and_time():
    w = inputs.test_case(seed=1)
    with ctx_for(w) as c:
        c.run(5)
        before = np.stack(c.get_state())
        adjoint_run(c, box_of(w), 10, 3)
        assert np.array_equal(np.stack(c.get_state()), before)
        s = c.step()
        after = np.stack(c.get_state())
        assert s.iter == 6
        c.set_state(*before)
        c.set_time(s.time - s.dt, 5)
        s2 = c.step()
        assert s2.dt == s.dt
        # the restored checkpoint carries exact culling flags and volume partials
        assert s2.volume == s.volume
        assert np.array_equal(np.stack(c.get_state()), after)


def test_sparse_checkpoints_on_a_mostly_dry_mesh():
    # one pile on a large mesh: most segments never change, so stores and restores copy only the
    # flow's footprint; the result must not depend on the number of checkpoints, and the state
    # and volume after the run must be the starting ones
    w = inputs.workload1()
    m = w.mesh
    box = (w.piles[0].xc - 300.0, w.piles[0].xc + 300.0, w.piles[0].yc - 300.0, w.piles[0].yc + 300.0)
    out = []
    for snaps in (2, 5, 40):
        with ctx_for(w) as c:
            c.run(3)
            start = np.stack(c.get_state())
            g = adjoint_run(c, box, 40, snaps, m.dh0_dpile, want_lambda0=True)
            assert np.array_equal(np.stack(c.get_state()), start)
            s1 = c.step()
            out.append((g, s1))
    (g0, s0), rest = out[0], out[1:]
    for g, s in rest:
        assert g.J == g0.J and g.dJ_dbedfrict == g0.dJ_dbedfrict and g.dJ_dpile == g0.dJ_dpile
        assert np.array_equal(g.lambda0, g0.lambda0)
        assert s.volume == s0.volume and s.time == s0.time


def test_fp32_split_adjoint_close_to_fp64():
    w = inputs.test_case(seed=1)
    m = w.mesh
    box = box_of(w)
    res = {}
    for prec in (_ffi.DA_PREC_FP64, _ffi.DA_PREC_FP32_SPLIT):
        with ctx_for(w, precision=prec) as c:
            res[prec] = adjoint_run(c, box, 40, 5, m.dh0_dpile, want_lambda0=True)
    a, b = res[_ffi.DA_PREC_FP64], res[_ffi.DA_PREC_FP32_SPLIT]
    rel = lambda x, y: abs(x - y) / max(abs(y), 1e-300)  # noqa: E731
    errs = [rel(b.dJ_dintfrict, a.dJ_dintfrict)] + [rel(x, y) for x, y in zip(b.dJ_dbedfrict, a.dJ_dbedfrict)] + \
           [rel(x, y) for x, y in zip(b.dJ_dpile, a.dJ_dpile)]
    lam_err = np.linalg.norm(b.lambda0 - a.lambda0) / np.linalg.norm(a.lambda0)
    print("fp32-split gradient rel errors", errs, "lambda0", lam_err, "J", rel(b.J, a.J))
    assert max(errs) < 1e-4 and lam_err < 1e-4
