"""Benchmark: cell-updates/s of the finite-volume step on the B200 (see the workload below).

python bench.py --gpus N --steps K --warmup W [--impl ours|reference] [--precision fp32|fp64]

A "step" is one explicit time step (step(), src/geoflow/step.C:29-275) over the whole mesh of
the workload: hill + noise terrain 20 km x 20 km, three piles, four materials, adaptive mesh
refined to 5 m (~3.7M active cells).  value = cells x steps / device seconds (max over ranks);
e2e = the same through the C ABI with host buffers, H2D of the state before and D2H after
every step inside the timed region.

Multi-GPU: the workload is one instance, so N > 1 runs N independent replicas (one per rank,
"weak" scaling, no data-path collective); the barrier and the max over ranks stay.

--impl reference: the reference's CPU algorithm (oracle/_ref when the reference compiled here,
else the oracle restatement) timed on this host's cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "cell-updates/s fwd+adjoint, FP32-split & batched vs plain FP64 GPU at ≤1e-5 rel err"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks sampled during the timed region (every 200 ms)."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 10:
                continue
            try:
                util = float(f[4])
                s = float(f[1])
                smax = float(f[2])
            except ValueError:
                continue
            if util > 0:
                sm.append(s)
                for k, nm in enumerate(names):
                    if f[6 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples_under_load": len(sm)}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def allmax(x: float, ws: int, dev: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{dev}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws: int, dev: int):
    if ws > 1:
        import torch
        import torch.distributed as dist
        dist.barrier(device_ids=[dev])
        torch.cuda.synchronize(dev)


def wet_counts(m, h) -> tuple[int, int]:
    """(cells with h >= GEOFLOW_TINY, cells that are wet or have a wet face neighbour)."""
    wet = h >= 1e-4
    act = wet.copy()
    for k in range(8):
        e = m.nbr[k]
        ok = e >= 0
        act[ok] |= wet[e[ok]]
    return int(wet.sum()), int(act.sum())


def algorithmic_bytes(precision: str, n: int, n_wet: float, n_act: float) -> dict:
    """Algorithmic HBM bytes of one launch of each forward kernel: every array a cell needs is
    touched once (neighbour re-reads are halo traffic, not algorithmic).  Layout of
    csrc/da_internal.h: state r bytes per component, static fields r bytes per component
    (x, y centres only in FP64), nbr 4 x int32 primary neighbours, bflag and material 1 byte.
      k_coef  : every cell reads h; a wet cell reads hu, hv, bflag, mat, nbr, dx, dy, g_z (and
                x, y in FP64) and writes k_act.
      k_update: every cell reads bflag, the state, nbr, dx, dy and writes the state; a cell
                with wet cells around it also reads k_act, g (3), d_gravity (2), curvature (2), mat."""
    r = 8 if precision == "fp64" else 4
    xy = 2 * r if precision == "fp64" else 0
    coef = n * r + n_wet * (2 * r + 1 + 1 + 16 + 2 * r + r + xy + r)
    upd = n * (1 + 3 * r + 16 + 2 * r + 3 * r) + n_act * (r + 3 * r + 2 * r + 2 * r + 1)
    return {"k_coef": coef, "k_update": upd}


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return
    from discrete_adjoint_b200 import TimeProps, inputs, make_params
    import oracle
    w = inputs.workload2()
    m = w.mesh
    p = make_params(w.mat, TimeProps())
    o = oracle.Oracle(p, m)
    h, hu, hv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
    o.run(h, hu, hv, 1)  # warm caches and page in
    t0 = time.perf_counter()
    rc, _, _ = o.run(h, hu, hv, 1)
    one = time.perf_counter() - t0
    per_step = max(1, int(20.0 / max(one, 1e-3)))
    steps = max(1, min(per_step, args.steps))
    t0 = time.perf_counter()
    rc, _, _ = o.run(h, hu, hv, steps)
    dt = time.perf_counter() - t0
    v = m.n * steps / dt
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": 1, "ms_per_step": 1e3 * dt / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": w.name, "cells": m.n, "precision": "fp64"},
            "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": "port",
                             "sample": f"{steps} steps of the {m.n}-cell workload, 1 thread (oracle restatement; "
                                       "the reference itself needs MPI/HDF5/Fortran and is not built here)"},
            "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-clocks", action="store_true", help="skip the clock sampler (profiling runs)")
    ap.add_argument("--sign-floor", type=float, default=0.0,
                    help="FP32-split friction sign threshold floor (0 = the reference's thresholds)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    ws, rank, local = dist_init()
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    from discrete_adjoint_b200 import GeoflowContext, TimeProps, _ffi, inputs

    w = inputs.workload2()
    m = w.mesh
    prec = _ffi.DA_PREC_FP32_SPLIT if args.precision == "fp32" else _ffi.DA_PREC_FP64

    def fresh(precision, cull=True):
        c = GeoflowContext(w.mat, TimeProps(), precision=precision, device=local,
                           fp32_sign_floor=args.sign_floor, tile_culling=cull)
        c.upload_mesh(m)
        c.set_state(m.h0, m.hu0, m.hv0)
        return c

    ctx = fresh(prec)
    ctx.run(args.warmup)
    sampler = ClockSampler(local)
    if not args.no_clocks:
        sampler.start()
        time.sleep(0.4)
    barrier(ws, local)
    stats, ms = ctx.run_timed(args.steps)
    barrier(ws, local)
    if not args.no_clocks:
        # keep the GPU loaded until the sampler has seen a few samples (untimed)
        t_end = time.time() + 1.2
        while time.time() < t_end:
            ctx.run(50)
        clocks = sampler.stop()
    else:
        clocks = {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["not sampled (--no-clocks)"]}
    ms_max = allmax(ms, ws, local)
    value = m.n * args.steps * ws / (ms_max * 1e-3)

    # the same step without tile culling: every cell rewritten every step
    full = fresh(prec, cull=False)
    full.run(args.warmup)
    _, msf = full.run_timed(args.steps)
    msf = allmax(msf, ws, local)
    value_full = m.n * args.steps * ws / (msf * 1e-3)
    w0 = wet_counts(m, full.get_state()[0])
    prof_full = full.profile(20)
    w1 = wet_counts(m, full.get_state()[0])
    n_wet, n_act = 0.5 * (w0[0] + w1[0]), 0.5 * (w0[1] + w1[1])
    full.close()

    # plain FP64 path on the same workload, same step count (the metric's comparison)
    ref64 = fresh(_ffi.DA_PREC_FP64)
    ref64.run(args.warmup)
    _, ms64 = ref64.run_timed(args.steps)
    ms64 = allmax(ms64, ws, local)
    value64 = m.n * args.steps * ws / (ms64 * 1e-3)
    # error of the FP32-split path against the FP64 path after the same number of steps from
    # the same initial state (fresh contexts: the timed contexts ran extra untimed steps)
    e32, e64 = fresh(prec), fresh(_ffi.DA_PREC_FP64)
    nerr = args.warmup + args.steps
    e32.run(nerr)
    e64.run(nerr)
    h32, u32, v32 = e32.get_state()
    h64, u64, v64 = e64.get_state()
    rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))  # noqa: E731
    rel_err = {"steps": nerr, "h": rel(h32, h64), "hu": rel(u32, u64), "hv": rel(v32, v64)}
    e32.close()
    e64.close()

    # per-kernel device times for the roofline (events around each launch); wet / active
    # counts averaged over the profiled steps give the algorithmic bytes of each launch
    # The roofline is taken on the full sweep (tile culling off: every cell read and written),
    # whose algorithmic bytes are defined per cell; the culled step is reported beside it.
    prof = ctx.profile(20)
    dom = max(prof_full, key=prof_full.get)
    alg = algorithmic_bytes(args.precision, m.n, n_wet, n_act)
    hbm, peak_kind = peaks()
    achieved = alg[dom] / (prof_full[dom] * 1e-3) / 1e9

    # e2e through the C ABI with host buffers: H2D state, one step, D2H state, every step
    h, hu, hv = ctx.get_state()
    h, hu, hv = np.ascontiguousarray(h), np.ascontiguousarray(hu), np.ascontiguousarray(hv)
    barrier(ws, local)
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        ctx.set_state(h, hu, hv)
        ctx.run(1)
        h, hu, hv = ctx.get_state()
    e2e_s = time.perf_counter() - t0
    e2e_s = allmax(e2e_s, ws, local)
    e2e_value = m.n * args.e2e_steps * ws / e2e_s
    elt = 8 if args.precision == "fp64" else 4
    h2d = 3 * elt * m.n
    d2h = 3 * elt * m.n

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        import oracle
        from discrete_adjoint_b200 import make_params
        o = oracle.Oracle(make_params(w.mat, TimeProps()), m)
        ch, chu, chv = m.h0.copy(), m.hu0.copy(), m.hv0.copy()
        t0 = time.perf_counter()
        o.run(ch, chu, chv, 1)
        one = time.perf_counter() - t0
        ns = max(1, min(10, int(15.0 / max(one, 1e-3))))
        t0 = time.perf_counter()
        o.run(ch, chu, chv, ns)
        cs = time.perf_counter() - t0
        cpu = {"value": m.n * ns / cs, "unit": "cell-updates/s", "cores": 1, "kind": "port",
               "sample": f"{ns} forward steps of the same {m.n}-cell workload, FP64 oracle restatement, 1 thread"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": w.name + " -- forward step only (adjoint not yet in the timed step)",
                       "cells": m.n, "precision": "fp32-split" if args.precision == "fp32" else "fp64",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
                       "l2": "per-step working set larger than L2 (no flush needed)"},
            "fp64_value": value64, "fp32_over_fp64": value / value64,
            "full_sweep_value": value_full, "full_sweep_kernel_ms": prof_full,
            "rel_err_vs_fp64": rel_err, "fp32_sign_floor": args.sign_floor,
            "roofline": {"bound": "hbm", "kernel": dom + " (full sweep)", "achieved": achieved, "peak": hbm,
                         "unit": "GB/s",
                         "frac": achieved / hbm if hbm else None, "peak_kind": peak_kind,
                         "alg_bytes_per_launch": alg[dom], "wet_cells": n_wet, "active_cells": n_act,
                         "kernel_ms_full_sweep": prof_full, "kernel_ms_culled": prof, "traffic": None},
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": 2 * args.steps,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    ctx.close()
    ref64.close()
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
