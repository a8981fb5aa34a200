"""Batching form: many independent channel/bump cases advanced in one batch.

    python -m myjoe_b200.batch --cases 256 --min-cells 10000 --max-cells 200000
                               [--precision mixed] [--drop 1e-8] [--max-steps 3000]

Cases are seeded: cell counts log-uniform on [min, max] (hex channels, two
cell layers in z), inflow Mach uniform on 0.3-0.8, angle of attack uniform on
+-4 degrees, bump height uniform on 0.05-0.12, inviscid HLLC, far-field
inlet/outlet/top (external flow over the bump).  All cases run
in one jg_batch handle (one launch per stage over all cases, CUDA graph per
step) until every case reaches the residual drop.  Prints one JSON line:
cell-iters/s of the batch, converged solves/hour, per-case steps and
time-to-converge percentiles.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import multiprocessing as mp
import time

import numpy as np


def case_specs(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    cells = np.exp(rng.uniform(math.log(lo), math.log(hi), n))
    specs = []
    for k in range(n):
        ny = max(4, int(round(math.sqrt(cells[k] / 4.0))))
        specs.append(dict(nx=2 * ny, ny=ny, nz=2, mach=float(rng.uniform(0.3, 0.8)),
                          aoa=float(rng.uniform(-4.0, 4.0)), bump=float(rng.uniform(0.05, 0.12)), seed=k))
    return specs


def build_case(spec):
    from myjoe_b200 import case
    _, g, prm = case.bump_case(spec["nx"], spec["ny"], spec["nz"], mach=spec["mach"], aoa_deg=spec["aoa"],
                               bump_h=spec["bump"], seed=spec["seed"], inlet=spec.get("inlet", "FARFIELD"))
    return g, prm


def build_cases(specs, workers):
    if workers <= 1:
        return [build_case(s) for s in specs]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(build_case, specs, chunksize=1)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=256)
    ap.add_argument("--min-cells", type=int, default=10000)
    ap.add_argument("--max-cells", type=int, default=200000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--solver", default="SGS", choices=["SGS", "JACOBI"])
    ap.add_argument("--sweeps", type=int, default=10)
    ap.add_argument("--cfl-ramp", default="10,5,1.2,20",
                    help="CFL_RAMP AFTER_ITER,INTERVAL_ITER,FACTOR_CFL,MAX_CFL")
    ap.add_argument("--under-relax", type=float, default=0.3)
    ap.add_argument("--drop", type=float, default=1e-8)
    ap.add_argument("--max-steps", type=int, default=3000)
    ap.add_argument("--chunk", type=int, default=50)
    ap.add_argument("--workers", type=int, default=min(32, mp.cpu_count()))
    args = ap.parse_args(argv)

    specs = case_specs(args.cases, args.min_cells, args.max_cells, args.seed)
    t0 = time.perf_counter()
    built = build_cases(specs, args.workers)
    t_mesh = time.perf_counter() - t0

    from myjoe_b200 import build, case, solver
    if build.needs_build():
        build.build()
    cases = []
    ra, ri, rf, rm = args.cfl_ramp.split(",")
    ramp = (int(ra), int(ri), float(rf), float(rm))
    for g, prm in built:
        prm = dataclasses.replace(prm, LINEAR_SOLVER_NS=args.solver, LS_MAX_ITER=args.sweeps, CFL=1.0,
                                  CFL_RAMP=ramp, UNDER_RELAXATION=args.under_relax)
        cases.append((g, prm))
    b = solver.JoeGpuBatch(cases, precision=1 if args.precision == "mixed" else 0)
    for k, (g, prm) in enumerate(cases):
        b.set_case_state(k, *case.perturbed_state(g.x_cv, prm, 0.0))
    ncv = b.ncv
    import torch
    stream = torch.cuda.ExternalStream(b.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0 = None
    conv_step = np.full(args.cases, -1)
    failed = np.zeros(args.cases, bool)
    steps = 0
    dev_ms = 0.0
    t_run = time.perf_counter()
    while steps < args.max_steps and ((conv_step < 0) & ~failed).any():
        with torch.cuda.stream(stream):
            e0.record(stream)
        r = b.runBackwardEulerCases(args.chunk)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        dev_ms += e0.elapsed_time(e1)
        if r0 is None:
            r0 = r[0, :, 4].copy()
        drop = r[:, :, 4] / r0[None, :]
        bad = b.status() != 0
        for k in np.nonzero((conv_step < 0) & ~failed)[0]:
            hit = np.nonzero(drop[:, k] <= args.drop)[0]
            if hit.size:
                conv_step[k] = steps + int(hit[0]) + 1
                b.set_active(k, False)      # retire: the converged state stays as it is
            elif bad[k] or not np.isfinite(drop[-1, k]):
                failed[k] = True
                b.set_active(k, False)      # retire the diverged case; the others continue
        steps += args.chunk
    wall = time.perf_counter() - t_run
    step_ms = dev_ms / steps
    done = conv_step > 0
    ttc = conv_step[done] * step_ms / 1000.0  # seconds on the device until each case converged
    out = {
        "form": "batch", "cases": args.cases, "cells": int(ncv), "precision": args.precision,
        "solver": "%s x%d" % (args.solver, args.sweeps), "drop": args.drop,
        "cfl_ramp": list(ramp), "under_relax": args.under_relax,
        "steps": steps, "ms_per_step": step_ms, "cell_iters_per_s": ncv * steps / (dev_ms / 1000.0),
        "converged": int(done.sum()), "failed": int(failed.sum()),
        "failed_cases": [dict(specs[k], cells=int(b.sizes[k])) for k in np.nonzero(failed)[0]][:20],
        "wall_s": wall, "mesh_setup_s": t_mesh,
        "converged_solves_per_hour": float(done.sum()) / wall * 3600.0,
        "steps_to_converge_p50": float(np.percentile(conv_step[done], 50)) if done.any() else None,
        "steps_to_converge_p99": float(np.percentile(conv_step[done], 99)) if done.any() else None,
        "time_to_converge_p50_s": float(np.percentile(ttc, 50)) if done.any() else None,
        "time_to_converge_p99_s": float(np.percentile(ttc, 99)) if done.any() else None,
    }
    print(json.dumps(out))


if __name__ == "__main__":
    main()
