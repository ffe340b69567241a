"""The oracle's restatement of the reference's discrete adjoint (oracle/da_oracle_adjoint.c) against
the reference's own dual solver: committed fixtures made by tests/golden/make_golden.py from the
reference's update_dual_grid / calc_jacobian / calc_adjoint (always), and the compiled harness run
live on fresh meshes and synthetic states (when oracle/_ref/ref_harness exists).  Also: with every
one of the reference's approximations dropped, the restatement is the exact transpose of the
forward step, and converges to central differences of whole runs."""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
from discrete_adjoint_b200 import TimeProps, _ffi, inputs, make_params
from discrete_adjoint_b200.mesh import Mesh
from discrete_adjoint_b200.solver import MatProps
from golden_util import GOLDEN

needs_ref = pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built")


def load_adj(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    mesh = Mesh(**{k[5:]: z[k] for k in z.files if k.startswith("mesh_")})
    mat = MatProps(intfrict_deg=float(z["intfrict_deg"]), bedfrict_deg=[float(b) for b in z["bedfrict_deg"]])
    return mesh, mat, z


def frict_tiny(it):
    # the threshold of the forward step iter - 1 -> iter (hpfem.C:232-235, calc_jacobain.C:82-85)
    return 0.1 if it < 51 else 1e-9


def forward_states(o, mesh, nsteps):
    h, hu, hv = mesh.h0.copy(), mesh.hu0.copy(), mesh.hv0.copy()
    states, dts = [(h.copy(), hu.copy(), hv.copy())], []
    for _ in range(nsteps):
        rc, dt, _ = o.run(h, hu, hv, 1)
        assert rc == 0
        dts.append(float(dt[0]))
        states.append((h.copy(), hu.copy(), hv.copy()))
    return states, dts


def test_reverse_sweep_matches_reference_fixture_bit_for_bit():
    mesh, mat, z = load_adj("adj_s11_60")
    n_steps = int(z["nsteps"])
    o = oracle.Oracle(make_params(mat, TimeProps()), mesh)
    states, dts = forward_states(o, mesh, n_steps)
    assert np.array_equal(np.array(dts), z["dts"])
    keep = list(z["keep_steps"])
    lam = z["lam_end"].copy()
    for k in range(1, n_steps + 1):
        it = n_steps - k + 1
        U = states[it - 1]
        lam = o.adjoint_step_ref(*U, dts[it - 1], frict_tiny(it), lam)
        if k in keep:
            assert np.array_equal(lam, z["ref_lam"][keep.index(k)]), f"after {k} reverse steps"


def test_stress_step_matches_reference_fixture_bit_for_bit():
    mesh, mat, z = load_adj("adj_stress_s12")
    it = int(z["iter"])
    # the state has dry cells with momentum, cells thinner than GEOFLOW_TINY and a random adjoint
    assert ((z["h"] == 0) & (z["hu"] != 0)).any() and ((z["h"] > 0) & (z["h"] < 1e-4)).any()
    o = oracle.Oracle(make_params(mat, TimeProps()), mesh)
    lam = o.adjoint_step_ref(z["h"], z["hu"], z["hv"], float(z["dt"]), frict_tiny(it), z["lam_next"])
    assert np.array_equal(lam, z["ref_lam"])


@needs_ref
@pytest.mark.parametrize("seed,nx0,ny0,L,frac,nsteps", [(12, 12, 8, 2, 0.3, 70), (13, 10, 6, 1, 0.0, 30),
                                                         (21, 16, 10, 2, 0.5, 55)])
def test_reverse_sweep_matches_live_reference(seed, nx0, ny0, L, frac, nsteps):
    w = inputs.test_case(seed=seed, nx0=nx0, ny0=ny0, max_level=L, random_frac=frac)
    m = w.mesh
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    states, dts = forward_states(o, m, nsteps)
    rng = np.random.default_rng(seed)
    lam_end = rng.standard_normal((3, m.n))
    iters = list(range(nsteps, 0, -1))
    r = oracle.run_reference_adjoint(m, w.mat, [states[i - 1] for i in iters], iters, [dts[i - 1] for i in iters],
                                     lam_end)
    lam = lam_end
    for k, it in enumerate(iters):
        lam = o.adjoint_step_ref(*states[it - 1], dts[it - 1], frict_tiny(it), lam)
        assert np.array_equal(lam, r["lam"][k]), f"reverse step {k} (iter {it})"


@needs_ref
@pytest.mark.parametrize("seed,it", [(11, 3), (21, 70), (22, 51)])
def test_stress_states_match_live_reference(seed, it):
    from golden.make_golden import stress_state
    w = inputs.test_case(seed=seed, nx0=12, ny0=8, max_level=2, random_frac=0.4)
    m = w.mesh
    rng = np.random.default_rng(seed)
    h, hu, hv = stress_state(m, rng)
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    o.set_time(0.0, it - 1)
    h2, hu2, hv2 = h.copy(), hu.copy(), hv.copy()
    rc, dts, _ = o.run(h2, hu2, hv2, 1)
    assert rc == 0
    lam = rng.standard_normal((3, m.n))
    r = oracle.run_reference_adjoint(m, w.mat, [(h, hu, hv)], [it], [float(dts[0])], lam)
    assert np.array_equal(o.adjoint_step_ref(h, hu, hv, float(dts[0]), frict_tiny(it), lam), r["lam"][0])


# ------------------------------------------------------------------ the exact transpose (all dropped)
def _frozen_step(o, lib, U, dt, ft):
    h, hu, hv = (np.ascontiguousarray(a) for a in U)
    s = o.slopes(h, hu, hv)
    _, kact, _, _ = o.coef_eigen(h, hu, hv, s)
    F = o.edge_fluxes(h, hu, hv, kact)
    out = [np.zeros_like(h) for _ in range(3)]
    lib.orc_correct(C.byref(o.params), C.byref(o.soa), _ffi.dptr(h), _ffi.dptr(hu), _ffi.dptr(hv), _ffi.dptr(s),
                    _ffi.dptr(kact), _ffi.dptr(F), dt, ft, _ffi.dptr(out[0]), _ffi.dptr(out[1]), _ffi.dptr(out[2]),
                    None, None)
    return out


def test_without_the_reference_approximations_the_adjoint_matches_central_differences():
    lib = oracle.load()
    PD = C.POINTER(C.c_double)
    lib.orc_correct.restype = C.c_int
    lib.orc_correct.argtypes = [C.POINTER(_ffi.da_params), C.POINTER(_ffi.da_mesh_soa), PD, PD, PD, PD, PD, PD,
                                C.c_double, C.c_double, PD, PD, PD, PD, C.c_void_p]
    w = inputs.test_case(seed=12, nx0=12, ny0=8, max_level=2, random_frac=0.3)
    m = w.mesh
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    N = 60
    states, dts = forward_states(o, m, N)
    fts = [frict_tiny(k + 1) for k in range(N)]
    wet = states[N][0] > 1e-4
    cx, cy = m.x[wet].mean(), m.y[wet].mean()
    inb = (m.x >= cx - 150) & (m.x <= cx + 150) & (m.y >= cy - 150) & (m.y <= cy + 150)
    area = m.dx * m.dy

    def J(U):
        return float(np.sum(np.where(inb, U[0] ** 2 * area, 0.0)))

    lam_end = np.zeros((3, m.n))
    lam_end[0] = np.where(inb, 2 * states[N][0] * area, 0.0)

    def sweep(keep):
        lam = lam_end
        for k in range(N - 1, -1, -1):
            lam = o.adjoint_step_ref(*states[k], dts[k], fts[k], lam, keep=keep)
        return lam

    exact, ref = sweep(0), sweep(oracle.Q_ALL)

    def fd_of(d, eps):
        Up = [a + eps * b for a, b in zip(states[0], d)]
        Um = [a - eps * b for a, b in zip(states[0], d)]
        for k in range(N):
            Up = _frozen_step(o, lib, Up, dts[k], fts[k])
            Um = _frozen_step(o, lib, Um, dts[k], fts[k])
        return (J(Up) - J(Um)) / (2 * eps)

    def dot(lam, d):
        return sum(float(np.dot(lam[v], d[v])) for v in range(3))

    rng = np.random.default_rng(3)
    h0 = states[0][0]
    for _ in range(2):
        # wet cells
        d = [1e-3 * rng.standard_normal(m.n) * (h0 > 1e-4) for _ in range(3)]
        fd = fd_of(d, 1e-4)
        assert abs(dot(exact, d) - fd) < 1e-4 * abs(fd)
    # the reference takes no derivative with respect to a cell whose record is zero (h = 0): its
    # lambda is zero on every such cell, where the exact transpose's is not (a dry cell's depth
    # enters its wet neighbours' limited slopes, and its own update is the identity)
    void = states[0][0] == 0
    assert void.any()
    assert (ref[:, void] == 0).all()
    assert (exact[:, void] != 0).any()
