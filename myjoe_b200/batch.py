"""Batching form: many independent channel/bump cases advanced in batches.

    python -m myjoe_b200.batch --cases 256 --min-cells 10000 --max-cells 200000
                               [--sst-fraction 0.5] [--precision mixed] [--drop 1e-8] [--max-steps 3000]

Cases are seeded: cell counts log-uniform on [min, max] (hex channels, two
cell layers in z), inflow Mach uniform on 0.3-0.8, angle of attack uniform on
+-4 degrees, bump height uniform on 0.05-0.12, far-field inlet/outlet/top
(external flow over the bump).  A fraction of the cases are Menter SST RANS
(one fluid: Re on the bump chord 1e6 x Mach / 0.55, rows stretched towards
the wall, 7x7 coupled blocks), the rest inviscid HLLC (5x5).  The cases of each model run in one
jg_batch handle (one launch per stage over all its cases, CUDA graph per
step, launch shapes autotuned on the batch: jg_autotune); the two handles
step concurrently on their own streams until every
case reaches the residual drop.  Prints one JSON line: cell-iters/s over all
cases, converged solves/hour, per-case steps and time-to-converge percentiles,
per model.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import multiprocessing as mp
import time

import numpy as np


# the SST cases' fluid: Sutherland MU_REF giving Re = 1e6 on the bump chord at M 0.55 (p 1e5, T 300)
SST_MU_REF = 1.1628 * 0.55 * math.sqrt(1.4 * 287.0 * 300.0) / 1.0e6 / ((300.0 / 273.15) ** 1.5 * 383.55 / 410.4)


def case_specs(n, lo, hi, seed, sst_fraction=0.0):
    rng = np.random.default_rng(seed)
    cells = np.exp(rng.uniform(math.log(lo), math.log(hi), n))
    sst = rng.uniform(0.0, 1.0, n) < sst_fraction
    specs = []
    for k in range(n):
        ny = max(4, int(round(math.sqrt(cells[k] / 4.0))))
        specs.append(dict(nx=2 * ny, ny=ny, nz=2, mach=float(rng.uniform(0.3, 0.8)),
                          aoa=float(rng.uniform(-4.0, 4.0)), bump=float(rng.uniform(0.05, 0.12)), seed=k,
                          model="SST" if sst[k] else "EULER"))
    return specs


def wall_stretch(ny, first=1.0e-6, height=1.0):
    """Geometric ratio r of ny wall-normal rows over `height` whose first row is `first` high:
    first = height (r - 1) / (r^ny - 1), by bisection (at most 1.1)"""
    lo, hi = 1.0 + 1e-9, 1.1
    if height * (hi - 1.0) / (hi ** ny - 1.0) >= first:
        return hi
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if height * (mid - 1.0) / (mid ** ny - 1.0) > first:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def build_case(spec):
    from myjoe_b200 import case
    if spec.get("model") == "SST":
        # one fluid for every case (a batch shares it): Re on the bump chord grows with the Mach
        # number, about 1e6 at M 0.55; wall-normal rows stretched towards the wall
        _, g, prm = case.sst_bump_case(spec["nx"], spec["ny"], spec["nz"], mach=spec["mach"],
                                       mu_ref=SST_MU_REF,
                                       aoa_deg=spec["aoa"], bump_h=spec["bump"], seed=spec["seed"],
                                       stretch=spec.get("stretch", wall_stretch(spec["ny"])))
        return g, prm
    _, g, prm = case.bump_case(spec["nx"], spec["ny"], spec["nz"], mach=spec["mach"], aoa_deg=spec["aoa"],
                               bump_h=spec["bump"], seed=spec["seed"], inlet=spec.get("inlet", "FARFIELD"))
    return g, prm


def initial_scalars(g, prm):
    if prm.TURB_MODEL == "SA":
        return np.full(g.ncv, prm.NUSA_INITIAL)
    return np.tile([prm.KINE_INITIAL, prm.OMEGA_INITIAL], (g.ncv, 1))


def build_cases(specs, workers):
    if workers <= 1:
        return [build_case(s) for s in specs]
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(build_case, specs, chunksize=1)


class Group:
    """The cases of one model in one batch handle, with their progress."""

    def __init__(self, name, idx, cases, precision, jac_lag=1, renumber=0):
        from myjoe_b200 import case, solver
        self.name, self.idx = name, idx
        self.b = solver.JoeGpuBatch(cases, precision=precision, jac_lag=jac_lag, renumber=renumber)
        for k, (g, prm) in enumerate(cases):
            self.b.set_case_state(k, *case.perturbed_state(g.x_cv, prm, 0.0))
            if prm.TURB_MODEL != "NONE":
                self.b.set_case_scalars(k, initial_scalars(g, prm))
        n = len(cases)
        self.r0 = None
        self.conv_step = np.full(n, -1)
        self.failed = np.zeros(n, bool)
        self.steps = 0
        self.dev_ms = 0.0

    def live(self):
        return ((self.conv_step < 0) & ~self.failed).any()

    def advance(self, chunk, drop):
        import torch
        stream = torch.cuda.ExternalStream(self.b.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = self.b.runBackwardEulerCases(chunk)
        e1.record(stream)
        e1.synchronize()
        self.dev_ms += e0.elapsed_time(e1)
        if self.r0 is None:
            self.r0 = r[0, :, 4].copy()
        d = r[:, :, 4] / self.r0[None, :]
        bad = self.b.status() != 0
        for k in np.nonzero((self.conv_step < 0) & ~self.failed)[0]:
            hit = np.nonzero(d[:, k] <= drop)[0]
            if hit.size:
                self.conv_step[k] = self.steps + int(hit[0]) + 1
                self.b.set_active(k, False)      # retire: the converged state stays as it is
            elif bad[k] or not np.isfinite(d[-1, k]):
                self.failed[k] = True
                self.b.set_active(k, False)      # retire the diverged case; the others continue
        self.steps += chunk


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=256)
    ap.add_argument("--min-cells", type=int, default=10000)
    ap.add_argument("--max-cells", type=int, default=200000)
    ap.add_argument("--sst-fraction", type=float, default=0.5)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--solver", default="SGS", choices=["SGS", "JACOBI"])
    ap.add_argument("--sweeps", type=int, default=10)
    ap.add_argument("--cfl-ramp", default="10,5,1.2,20",
                    help="CFL_RAMP AFTER_ITER,INTERVAL_ITER,FACTOR_CFL,MAX_CFL")
    ap.add_argument("--under-relax", type=float, default=0.3)
    ap.add_argument("--sst-solver", default="LINE", choices=["LINE", "SGS", "JACOBI"],
                    help="relaxation of the SST cases (their wall rows are stretched)")
    ap.add_argument("--sst-cfl-ramp", default="10,5,1.2,200")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--drop", type=float, default=1e-8)
    ap.add_argument("--max-steps", type=int, default=3000)
    ap.add_argument("--chunk", type=int, default=50)
    ap.add_argument("--workers", type=int, default=min(32, mp.cpu_count()))
    ap.add_argument("--jac-lag", type=int, default=4, help="inviscid cases: flux Jacobian every k-th step")
    ap.add_argument("--renumber", type=int, default=2, help="each case's cell order: 0 its own, 1 RCM, 2 RCM by colour")
    args = ap.parse_args(argv)

    specs = case_specs(args.cases, args.min_cells, args.max_cells, args.seed, args.sst_fraction)
    t0 = time.perf_counter()
    built = build_cases(specs, args.workers)
    t_mesh = time.perf_counter() - t0

    from myjoe_b200 import build
    if build.needs_build():
        build.build()
    ra, ri, rf, rm = args.cfl_ramp.split(",")
    ramp = (int(ra), int(ri), float(rf), float(rm))
    precision = 1 if args.precision == "mixed" else 0
    groups = []
    sa, si, sf, sm = args.sst_cfl_ramp.split(",")
    sst_ramp = (int(sa), int(si), float(sf), float(sm))
    for model in ("EULER", "SST"):
        idx = [k for k, sp in enumerate(specs) if sp["model"] == model]
        if not idx:
            continue
        solver_name, r = (args.sst_solver, sst_ramp) if model == "SST" else (args.solver, ramp)
        cases = [(built[k][0], dataclasses.replace(built[k][1], LINEAR_SOLVER_NS=solver_name,
                                                   LS_MAX_ITER=args.sweeps, CFL=1.0, CFL_RAMP=r,
                                                   UNDER_RELAXATION=args.under_relax)) for k in idx]
        gr = Group(model, idx, cases, precision, jac_lag=args.jac_lag if model == "EULER" else 1,
                   renumber=args.renumber)
        gr.shape = None if args.no_autotune else gr.b.autotune(3)
        groups.append(gr)
    # the handles step concurrently: one host thread each (the C calls release the GIL)
    from concurrent.futures import ThreadPoolExecutor
    t_run = time.perf_counter()
    with ThreadPoolExecutor(len(groups)) as pool:
        while True:
            live = [gr for gr in groups if gr.steps < args.max_steps and gr.live()]
            if not live:
                break
            list(pool.map(lambda gr: gr.advance(args.chunk, args.drop), live))
    wall = time.perf_counter() - t_run
    per_model, all_conv, all_ttc = {}, [], []
    cell_iters = 0.0
    for gr in groups:
        done = gr.conv_step > 0
        step_ms = gr.dev_ms / gr.steps
        ttc = gr.conv_step[done] * step_ms / 1000.0
        cell_iters += gr.b.ncv * gr.steps
        all_conv.extend(gr.conv_step[done].tolist())
        all_ttc.extend(ttc.tolist())
        per_model[gr.name] = {
            "cases": len(gr.idx), "cells": int(gr.b.ncv), "steps": gr.steps, "ms_per_step": step_ms,
            "launch_shape": gr.shape,
            "cell_iters_per_s_alone_on_stream": gr.b.ncv / (step_ms / 1000.0),
            "converged": int(done.sum()), "failed": int(gr.failed.sum()),
            "failed_cases": [dict(specs[gr.idx[k]], cells=int(gr.b.sizes[k]))
                             for k in np.nonzero(gr.failed)[0]][:10],
            "steps_to_converge_p50": float(np.percentile(gr.conv_step[done], 50)) if done.any() else None,
            "time_to_converge_p50_s": float(np.percentile(ttc, 50)) if done.any() else None,
            "time_to_converge_p99_s": float(np.percentile(ttc, 99)) if done.any() else None,
        }
    nconv = len(all_conv)
    out = {
        "form": "batch", "cases": args.cases, "cells": int(sum(gr.b.ncv for gr in groups)),
        "precision": args.precision, "solver": "%s x%d" % (args.solver, args.sweeps),
        "sst_solver": "%s x%d" % (args.sst_solver, args.sweeps), "drop": args.drop,
        "cfl_ramp": list(ramp), "sst_cfl_ramp": list(sst_ramp), "under_relax": args.under_relax,
        "sst_fraction": args.sst_fraction, "jac_lag": args.jac_lag, "renumber": args.renumber,
        "cell_iters_per_s": cell_iters / wall, "wall_s": wall, "mesh_setup_s": t_mesh,
        "converged": nconv, "failed": int(sum(gr.failed.sum() for gr in groups)),
        "converged_solves_per_hour": nconv / wall * 3600.0,
        "time_to_converge_p50_s": float(np.percentile(all_ttc, 50)) if nconv else None,
        "time_to_converge_p99_s": float(np.percentile(all_ttc, 99)) if nconv else None,
        "models": per_model,
    }
    print(json.dumps(out))


if __name__ == "__main__":
    main()
