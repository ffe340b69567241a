"""Run one of the synthetic workloads through the C ABI and print a JSON summary.

    python run_case.py --workload 2 --precision fp32 --steps 20 [--full-sweep]
    python run_case.py --workload 3 --precision fp64 --adjoint 64
    python run_case.py --workload 2 --precision fp64 --layer 1 --steps 10
    python run_case.py --workload 3 --precision fp64 --adjoint 512 --grid 74 --blocks-per-sm 2

A fixed, small command line for profilers (ncu -k <kernel> -s <skip> -c <count> python run_case.py ...):
the forward steps go through da_forward_run (CUDA graphs), the adjoint through da_adjoint_run.
Workloads: 1 = 40k-cell plane and runout, 2 = 3.75M-cell adaptive hill + noise, 3 = 1M-cell
uniform plane (the forward + adjoint workload).  --layer adds that many metres of material on
every cell (the dense case: every cell wet and updated every step).
"""
from __future__ import annotations

import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from discrete_adjoint_b200 import _ffi, inputs  # noqa: E402
from discrete_adjoint_b200.solver import GeoflowContext, TimeProps, adjoint_run  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", type=int, default=3, choices=[1, 2, 3])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--steps", type=int, default=20, help="forward steps (ignored with --adjoint)")
    ap.add_argument("--pre-steps", type=int, default=0,
                    help="forward steps taken in a launch of their own before the measured ones (a profiler "
                         "then skips that launch to see the steady flow)")
    ap.add_argument("--full-sweep", action="store_true", help="switch tile culling off")
    ap.add_argument("--layer", type=float, default=0.0, help="metres of material added on every cell")
    ap.add_argument("--adjoint", type=int, default=0, metavar="HORIZON",
                    help="run forward + adjoint over HORIZON steps (32 snapshots) instead")
    ap.add_argument("--grid", type=int, default=0,
                    help="blocks per launch of the step kernels (da_params.grid_blocks; 0 = the default)")
    ap.add_argument("--blocks-per-sm", type=int, default=0, choices=[0, 2, 3],
                    help="register budget of the step kernels (da_params.blocks_per_sm; 0 = 2)")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    w = {1: inputs.workload1, 2: inputs.workload2, 3: inputs.workload3}[a.workload]()
    prec = _ffi.DA_PREC_FP32_SPLIT if a.precision == "fp32" else _ffi.DA_PREC_FP64
    with GeoflowContext(w.mat, TimeProps(), precision=prec, device=a.device, tile_culling=not a.full_sweep,
                        grid_blocks=a.grid, blocks_per_sm=a.blocks_per_sm) as c:
        c.upload_mesh(w.mesh)
        c.set_state(w.mesh.h0 + a.layer, w.mesh.hu0, w.mesh.hv0)
        out = {"workload": w.name, "cells": w.mesh.n, "precision": a.precision, "culling": not a.full_sweep,
               "layer": a.layer, "grid": a.grid, "blocks_per_sm": a.blocks_per_sm}
        if a.adjoint:
            p0 = w.piles[0]
            box = inputs.WORKLOAD3_BOX if a.workload == 3 else (p0.xc - 500.0, p0.xc + 500.0, p0.yc - 500.0, p0.yc + 500.0)
            g = adjoint_run(c, box, a.adjoint, 32, w.mesh.dh0_dpile)
            out.update({"horizon": a.adjoint, "J": g.J, "dJ_dbedfrict": g.dJ_dbedfrict, "dJ_dpile": g.dJ_dpile,
                        "forward_steps": g.forward_steps, "device_ms": g.device_ms})
        else:
            if a.pre_steps:
                c.run(a.pre_steps)
            s, ms = c.run_timed(a.steps)
            out.update({"pre_steps": a.pre_steps, "steps": a.steps, "device_ms": ms, "volume": s.volume,
                        "iter": s.iter})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
