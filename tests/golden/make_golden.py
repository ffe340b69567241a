"""Generates the golden fixtures in this directory from the reference's own compiled step().

Run in a container that has the reference sources (it builds oracle/_ref/ref_harness with
oracle/ref_build.py, then runs it):   python tests/golden/make_golden.py
Each fixture holds a small flattened mesh (seeded, hanging nodes on many sides, two
materials), the initial state, and what the reference's step() produced from it:
dt history, final state, and the slopes, k act/pass and edge-node fluxes of the last step.
Fixture "static_*" also holds gravity and d_gravity from Element::calc_gravity_vector and
Element::calc_d_gravity.  Fixture "stats_*" holds calc_stats' StatProps after the last step and
the discharge through two planes accumulated over all steps (DISCHARGE::update), with the test
point, Vslump and planes it was run with.

Fixtures "adj_*" hold the reference's own discrete adjoint (its dual solver's update_dual_grid,
calc_jacobian and calc_adjoint, run through the harness's 'DAJ1' mode):
  adj_s11_60     the reverse sweep over the 60 steps of fwd_s11_60's mesh and initial state,
                 seeded with lambda^N = dJ/dU^N of J = sum h^2 dx dy over a box, with lambda after
                 1, 10, 30 and 60 reverse steps (the forward states are the oracle's, which equal
                 the reference's step() bit for bit; checked here against a harness run);
  adj_stress_s12 one reverse step from a synthetic state (thin and dry cells, dry cells with
                 momentum, random adjoint) at an iteration past the frict_tiny switch.
Run only these with:   python tests/golden/make_golden.py adj

Fixture "dwr_s11_55" holds the reference's DWR estimate of one step (bilinear_interp,
update_bilinear_error_grid, error_compute through the harness's 'DAE1' mode) on the error grid of
fwd_s11_60's mesh: the reconstructions, the error grid's residual, el_error and correction per
fine cell.  Run only it with:   python tests/golden/make_golden.py dwr
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

import oracle  # noqa: E402
from oracle import ref_build  # noqa: E402
from discrete_adjoint_b200 import inputs  # noqa: E402

CASES = [
    # name, seed, nx0, ny0, max_level, random_frac, nsteps
    ("fwd_s11_60", 11, 12, 8, 2, 0.4, 60),
    ("fwd_s12_120", 12, 12, 8, 2, 0.3, 120),
    ("fwd_s13_uniform_30", 13, 10, 6, 1, 0.0, 30),
]


STATS_CASES = [
    # name, seed, nsteps
    ("stats_s12_80", 12, 80),
]


def stats_case(name, seed, nsteps):
    w = inputs.test_case(seed=seed, nx0=12, ny0=8, max_level=2, random_frac=0.3)
    m = w.mesh
    wet = m.h0 > 1.0
    cx, cy = float(m.x[wet].mean()), float(m.y[wet].mean())
    # a generic test point (not equidistant from two cell centres) and two planes, one slanted
    test_point = (0.5, cx + 97.3, cy + 11.1)
    planes = [(cx + 61.7, cx + 61.7, cy - 250.0, cy + 230.0), (cx - 180.0, cx + 260.0, cy + 131.0, cy + 57.0)]
    r = oracle.run_reference(m, w.mat, m.h0, m.hu0, m.hv0, nsteps, test_point=test_point, vslump=2.0,
                             planes=planes)
    arrs = {("mesh_" + k): v for k, v in m.arrays().items()}
    arrs["ref_dt"] = r["dt"]
    arrs["ref_h"], arrs["ref_hu"], arrs["ref_hv"] = r["h"], r["hu"], r["hv"]
    arrs["stat_names"] = np.array(oracle.STAT_FIELDS)
    arrs["stat_values"] = np.array([r["stats"][k] for k in oracle.STAT_FIELDS])
    arrs["discharge"] = r["discharge"]
    arrs["planes"] = np.array(planes)
    arrs["test_point"] = np.array(test_point)
    arrs["vslump"] = np.float64(2.0)
    arrs["nsteps"] = np.int64(nsteps)
    arrs["intfrict_deg"] = np.float64(w.mat.intfrict_deg)
    arrs["bedfrict_deg"] = np.array(w.mat.bedfrict_deg, dtype=np.float64)
    p = os.path.join(HERE, name + ".npz")
    np.savez_compressed(p, **arrs)
    print(p, m.n, "cells", os.path.getsize(p) // 1024, "KiB")


def hilbert_keys():
    """Element keys of the reference's fhsfc2d_ (src/main/hilbert.C) for seeded points of the unit
    square and its edges."""
    rng = np.random.default_rng(11)
    u = np.concatenate([rng.random(1000), [0.0, 1.0, -0.5, 1.5, 0.5, 1e-12, 1 - 1e-12, 0.25, 0.75]])
    v = np.concatenate([rng.random(1000), [0.0, 1.0, 0.3, 2.0, 0.5, 1 - 1e-12, 1e-12, 0.75, 0.25]])
    p = os.path.join(HERE, "hilbert_keys.npz")
    np.savez_compressed(p, u=u, v=v, keys=oracle.ref_hilbert_keys(u, v))
    print(p)


ADJ_KEEP = (1, 10, 30, 60)


def adjoint_sweep_case(name="adj_s11_60", seed=11, nsteps=60):
    from discrete_adjoint_b200 import TimeProps, make_params
    w = inputs.test_case(seed=seed, nx0=12, ny0=8, max_level=2, random_frac=0.4)
    m = w.mesh
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    states, dts = [(h.copy(), hu.copy(), hv.copy())], []
    for _ in range(nsteps):
        rc, dt, _st = o.run(h, hu, hv, 1)
        assert rc == 0
        dts.append(float(dt[0]))
        states.append((h.copy(), hu.copy(), hv.copy()))
    r = oracle.run_reference(m, w.mat, m.h0, m.hu0, m.hv0, nsteps)
    assert np.array_equal(r["h"], states[-1][0]) and np.array_equal(r["dt"], np.array(dts))
    wet = states[-1][0] > 1e-4
    cx, cy = float(m.x[wet].mean()), float(m.y[wet].mean())
    box = np.array([cx - 150.0, cx + 150.0, cy - 150.0, cy + 150.0])
    inb = (m.x >= box[0]) & (m.x <= box[1]) & (m.y >= box[2]) & (m.y <= box[3])
    lam_end = np.zeros((3, m.n))
    lam_end[0] = np.where(inb, 2.0 * states[-1][0] * m.dx * m.dy, 0.0)
    iters = list(range(nsteps, 0, -1))
    ra = oracle.run_reference_adjoint(m, w.mat, [states[i - 1] for i in iters], iters, [dts[i - 1] for i in iters],
                                      lam_end)
    arrs = {("mesh_" + k): v for k, v in m.arrays().items()}
    arrs["nsteps"] = np.int64(nsteps)
    arrs["dts"] = np.array(dts)
    arrs["box"] = box
    arrs["lam_end"] = lam_end
    arrs["keep_steps"] = np.array(ADJ_KEEP)
    arrs["ref_lam"] = np.stack([ra["lam"][k - 1] for k in ADJ_KEEP])
    arrs["intfrict_deg"] = np.float64(w.mat.intfrict_deg)
    arrs["bedfrict_deg"] = np.array(w.mat.bedfrict_deg, dtype=np.float64)
    p = os.path.join(HERE, name + ".npz")
    np.savez_compressed(p, **arrs)
    print(p, m.n, "cells", os.path.getsize(p) // 1024, "KiB")


def stress_state(m, rng):
    """A synthetic state with deep, thin (below GEOFLOW_TINY) and dry cells, some dry cells
    carrying momentum."""
    n = m.n
    h = np.maximum(0.0, rng.normal(0.6, 1.0, n))
    thin = rng.random(n) < 0.1
    h[thin] = rng.uniform(0.0, 3e-4, thin.sum())
    hu = rng.normal(0, 3.0, n) * np.minimum(h, 1.0)
    hv = rng.normal(0, 3.0, n) * np.minimum(h, 1.0)
    vm = (h == 0) & (rng.random(n) < 0.5)
    hu[vm] = rng.normal(0, 1e-3, vm.sum())
    hv[vm] = rng.normal(0, 1e-3, vm.sum())
    return h, hu, hv


def adjoint_stress_case(name="adj_stress_s12", seed=12, it=70):
    from discrete_adjoint_b200 import TimeProps, make_params
    w = inputs.test_case(seed=seed, nx0=12, ny0=8, max_level=2, random_frac=0.3)
    m = w.mesh
    rng = np.random.default_rng(seed)
    h, hu, hv = stress_state(m, rng)
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    o.set_time(0.0, it - 1)
    h2, hu2, hv2 = h.copy(), hu.copy(), hv.copy()
    rc, dts, _st = o.run(h2, hu2, hv2, 1)
    assert rc == 0
    lam = rng.standard_normal((3, m.n))
    ra = oracle.run_reference_adjoint(m, w.mat, [(h, hu, hv)], [it], [float(dts[0])], lam)
    arrs = {("mesh_" + k): v for k, v in m.arrays().items()}
    arrs.update({"h": h, "hu": hu, "hv": hv, "iter": np.int64(it), "dt": np.float64(dts[0]), "lam_next": lam,
                 "ref_lam": ra["lam"][0]})
    arrs["intfrict_deg"] = np.float64(w.mat.intfrict_deg)
    arrs["bedfrict_deg"] = np.array(w.mat.bedfrict_deg, dtype=np.float64)
    p = os.path.join(HERE, name + ".npz")
    np.savez_compressed(p, **arrs)
    print(p, m.n, "cells", os.path.getsize(p) // 1024, "KiB")


def dwr_case(name="dwr_s11_55", seed=11, n0=55):
    """The reference's DWR estimate (bilinear_interp, update_bilinear_error_grid, error_compute;
    harness mode 'DAE1') of the step n0 -> n0 + 1 on the error grid of fwd_s11_60's mesh, with a
    seeded adjoint lambda^{n0+1}; the forward states are the oracle's (bit for bit the reference's)."""
    from discrete_adjoint_b200 import TimeProps, make_params
    from discrete_adjoint_b200.dwr import error_grid
    w = inputs.test_case(seed=seed, nx0=12, ny0=8, max_level=2, random_frac=0.4)
    m = w.mesh
    g = error_grid(w)
    o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    rc, _dts, _st = o.run(h, hu, hv, n0)
    assert rc == 0
    un = np.stack([h, hu, hv]).copy()
    rc, dts, _st = o.run(h, hu, hv, 1)
    assert rc == 0
    unext = np.stack([h, hu, hv])
    rng = np.random.default_rng(seed)
    wet = unext[0] > 1e-4
    lam = np.stack([rng.standard_normal(m.n) * wet, 0.1 * rng.standard_normal(m.n) * wet,
                    0.1 * rng.standard_normal(m.n) * wet])
    r = oracle.run_reference_dwr(g.fine, g.parent, w.mat, un, unext, lam, float(dts[0]), n0 + 1)
    arrs = {("mesh_" + k): v for k, v in m.arrays().items()}
    arrs.update({"n0": np.int64(n0), "un": un, "dt": np.float64(dts[0]), "lam_next": lam, "parent": g.parent,
                 "ref_bilin_prev": r["bilin_prev"], "ref_bilin_adj": r["bilin_adj"], "ref_residual": r["residual"],
                 "ref_el_error": r["el_error"][1], "ref_correction": r["correction"]})
    arrs["intfrict_deg"] = np.float64(w.mat.intfrict_deg)
    arrs["bedfrict_deg"] = np.array(w.mat.bedfrict_deg, dtype=np.float64)
    p = os.path.join(HERE, name + ".npz")
    np.savez_compressed(p, **arrs)
    print(p, m.n, "cells", g.fine.n, "fine cells", os.path.getsize(p) // 1024, "KiB")


def main():
    ref_build.build()
    if sys.argv[1:] == ["adj"]:
        adjoint_sweep_case()
        adjoint_stress_case()
        return
    if sys.argv[1:] == ["dwr"]:
        dwr_case()
        return
    dwr_case()
    adjoint_sweep_case()
    adjoint_stress_case()
    hilbert_keys()
    for case in STATS_CASES:
        stats_case(*case)
    for name, seed, nx0, ny0, L, frac, nsteps in CASES:
        w = inputs.test_case(seed=seed, nx0=nx0, ny0=ny0, max_level=L, random_frac=frac)
        m = w.mesh
        r = oracle.run_reference(m, w.mat, m.h0, m.hu0, m.hv0, nsteps)
        st = oracle.run_reference(m, w.mat, m.h0, m.hu0, m.hv0, 1, ref_static=True)
        arrs = {("mesh_" + k): v for k, v in m.arrays().items()}
        arrs.update({("ref_" + k): v for k, v in r.items() if k not in ("stats", "discharge")})
        arrs["ref_static_gravity"] = st["gravity"]
        arrs["ref_static_d_gravity"] = st["d_gravity"]
        arrs["nsteps"] = np.int64(nsteps)
        arrs["intfrict_deg"] = np.float64(w.mat.intfrict_deg)
        arrs["bedfrict_deg"] = np.array(w.mat.bedfrict_deg, dtype=np.float64)
        p = os.path.join(HERE, name + ".npz")
        np.savez_compressed(p, **arrs)
        print(p, m.n, "cells", os.path.getsize(p) // 1024, "KiB")


if __name__ == "__main__":
    main()
