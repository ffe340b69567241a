"""The reference's own discrete adjoint on the device (da_params.jacobian_mode = DA_JAC_REFERENCE),
through the C ABI: single reverse steps (da_adjoint_step) and whole checkpointed sweeps
(da_adjoint_run) against the oracle's restatement of the reference's dual solver
(oracle/da_oracle_adjoint.c, pinned bit for bit to the reference's update_dual_grid /
calc_jacobian / calc_adjoint) and against the fixtures made from the reference itself
(tests/golden/adj_*.npz).  Also the default exact mode against the oracle with every one of the
reference's approximations dropped.

Tolerance: FP64, 1e-12 relative (L2 over all cells and components) for the reference mode; the
device sums the same blocks in the same order without contraction, so it is expected to agree to
the last bit or close to it.  The exact mode takes its branch decisions from the replayed forward
step (true divisions) where the oracle takes them from the dual solver's arithmetic (reciprocal
products), so the two agree to rounding: 1e-9."""
import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import GeoflowContext, TimeProps, _ffi, adjoint_run, adjoint_step, inputs, make_params
from test_oracle_adjoint import forward_states, frict_tiny, load_adj

pytestmark = pytest.mark.gpu

TOL_REF = 1e-12
TOL_EXACT = 1e-9


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def device_states(c, mesh, nsteps):
    c.set_state(mesh.h0, mesh.hu0, mesh.hv0)
    c.set_time(0.0, 0)
    states, times = [tuple(c.get_state())], [0.0]
    for _ in range(nsteps):
        s = c.step()
        states.append(tuple(c.get_state()))
        times.append(s.time)
    return states, times


def test_reference_mode_reverse_steps_match_the_reference():
    mesh, mat, z = load_adj("adj_s11_60")
    N = int(z["nsteps"])
    o = oracle.Oracle(make_params(mat, TimeProps()), mesh)
    keep = list(z["keep_steps"])
    worst = 0.0
    with GeoflowContext(mat, TimeProps(), jacobian_mode=_ffi.DA_JAC_REFERENCE) as c:
        c.upload_mesh(mesh)
        states, times = device_states(c, mesh, N)
        ostates, dts = forward_states(o, mesh, N)
        for a, b in zip(states, ostates):
            assert all(np.array_equal(x, y) for x, y in zip(a, b))
        lam_dev = z["lam_end"].copy()
        lam_orc = z["lam_end"].copy()
        for k in range(1, N + 1):
            it = N - k + 1
            c.set_state(*states[it - 1])
            c.set_time(times[it - 1], it - 1)
            lam_dev, part = adjoint_step(c, lam_dev)
            lam_orc = o.adjoint_step_ref(*ostates[it - 1], dts[it - 1], frict_tiny(it), lam_orc)
            r = rel(lam_dev, lam_orc)
            worst = max(worst, r)
            assert r <= TOL_REF, f"reverse step {k}: device vs oracle {r:.3e}"
            if k in keep:
                rr = rel(lam_dev, z["ref_lam"][keep.index(k)])
                assert rr <= TOL_REF, f"after {k} reverse steps: device vs reference fixture {rr:.3e}"
            # no parameter derivatives in the reference
            assert part.dJ_dintfrict == 0.0
    print(f"reference mode, {N} reverse steps: worst device vs oracle {worst:.3e}")


def test_reference_mode_stress_state_matches_the_reference():
    mesh, mat, z = load_adj("adj_stress_s12")
    it = int(z["iter"])
    with GeoflowContext(mat, TimeProps(), jacobian_mode=_ffi.DA_JAC_REFERENCE) as c:
        c.upload_mesh(mesh)
        c.set_state(z["h"], z["hu"], z["hv"])
        c.set_time(0.0, it - 1)
        lam, _ = adjoint_step(c, z["lam_next"])
    r = rel(lam, z["ref_lam"])
    print(f"stress step: device vs reference {r:.3e}, bit-identical {np.array_equal(lam, z['ref_lam'])}")
    assert r <= TOL_REF


@pytest.mark.parametrize("nsnap", [4, 64])
def test_reference_mode_checkpointed_sweep_matches_chained_oracle_steps(nsnap):
    mesh, mat, z = load_adj("adj_s11_60")
    N = int(z["nsteps"])
    box = tuple(float(b) for b in z["box"])
    o = oracle.Oracle(make_params(mat, TimeProps()), mesh)
    ostates, dts = forward_states(o, mesh, N)
    inb = (mesh.x >= box[0]) & (mesh.x <= box[1]) & (mesh.y >= box[2]) & (mesh.y <= box[3])
    lam = np.zeros((3, mesh.n))
    lam[0] = np.where(inb, 2.0 * ostates[N][0] * (mesh.dx * mesh.dy), 0.0)
    J = float(np.sum(np.where(inb, ostates[N][0] ** 2 * (mesh.dx * mesh.dy), 0.0)))
    for it in range(N, 0, -1):
        lam = o.adjoint_step_ref(*ostates[it - 1], dts[it - 1], frict_tiny(it), lam)
    dh0 = np.ones((1, mesh.n)) * (mesh.h0 > 0)
    with GeoflowContext(mat, TimeProps(), jacobian_mode=_ffi.DA_JAC_REFERENCE) as c:
        c.upload_mesh(mesh)
        c.set_state(mesh.h0, mesh.hu0, mesh.hv0)
        g = adjoint_run(c, box, N, nsnap, dh0_dpile=dh0, want_lambda0=True)
        # the state is put back
        assert np.array_equal(c.get_state()[0], mesh.h0)
    r = rel(g.lambda0, lam)
    print(f"sweep with {nsnap} checkpoints: lambda0 device vs chained oracle {r:.3e}")
    assert r <= TOL_REF
    assert abs(g.J - J) <= 1e-12 * abs(J)
    assert abs(g.dJ_dpile[0] - float(np.sum(lam[0] * dh0[0]))) <= 1e-10 * abs(g.dJ_dpile[0])
    assert g.dJ_dbedfrict[0] == 0.0 and g.dJ_dintfrict == 0.0


@pytest.mark.parametrize("fixture", ["adj_s11_60", "adj_stress_s12"])
def test_exact_mode_matches_the_oracle_without_the_reference_approximations(fixture):
    mesh, mat, z = load_adj(fixture)
    o = oracle.Oracle(make_params(mat, TimeProps()), mesh)
    worst = 0.0
    with GeoflowContext(mat, TimeProps()) as c:
        c.upload_mesh(mesh)
        if fixture == "adj_stress_s12":
            it = int(z["iter"])
            c.set_state(z["h"], z["hu"], z["hv"])
            c.set_time(0.0, it - 1)
            lam, _ = adjoint_step(c, z["lam_next"])
            ex = o.adjoint_step_ref(z["h"], z["hu"], z["hv"], float(z["dt"]), frict_tiny(it), z["lam_next"], keep=0)
            worst = rel(lam, ex)
        else:
            N = int(z["nsteps"])
            states, times = device_states(c, mesh, N)
            _, dts = forward_states(o, mesh, N)
            rng = np.random.default_rng(5)
            for it in range(N, 0, -7):
                lam_next = rng.standard_normal((3, mesh.n))
                c.set_state(*states[it - 1])
                c.set_time(times[it - 1], it - 1)
                lam, _ = adjoint_step(c, lam_next)
                ex = o.adjoint_step_ref(*states[it - 1], dts[it - 1], frict_tiny(it), lam_next, keep=0)
                worst = max(worst, rel(lam, ex))
    print(f"{fixture}: exact mode vs oracle without the reference approximations {worst:.3e}")
    assert worst <= TOL_EXACT


def test_reference_mode_is_fp64_only_and_single_instance():
    w = inputs.test_case(seed=1)
    with GeoflowContext(w.mat, TimeProps(), precision=_ffi.DA_PREC_FP32_SPLIT,
                        jacobian_mode=_ffi.DA_JAC_REFERENCE) as c:
        c.upload_mesh(w.mesh)
        c.set_state(w.mesh.h0, w.mesh.hu0, w.mesh.hv0)
        with pytest.raises(_ffi.DAError) as e:
            adjoint_step(c, np.zeros((3, w.mesh.n)))
        assert e.value.code == _ffi.DA_ERR_UNSUPPORTED
