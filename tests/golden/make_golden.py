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


def main():
    ref_build.build()
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
