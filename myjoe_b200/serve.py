"""Serving form: a Poisson stream of seed-generated cases through the request loop.

    python -m myjoe_b200.serve --rate 20 --horizon 600 --min-cells 5000 --max-cells 500000
                               [--arms serve,plain] [--max-resident 48]

Requests arrive as a Poisson process (``--rate`` per second for
``--horizon`` seconds).  Each request is an external flow over a channel bump
with cells log-uniform on [min, max] (hex, two cell layers in z), inflow Mach
uniform on 0.3-0.8, angle of attack uniform on +-4 degrees and bump height
uniform on 0.05-0.12 (the batching form's parameters), inviscid HLLC, far-field
inlet/outlet/top.  Meshes are built by a spawn pool of client processes in
arrival order and submitted when they have arrived; a case retires at a 1e-8
drop of its energy residual.

Two arms see the same arrival stream:

* ``serve``: the serving form -- mixed precision (FP32 Jacobian and
  relaxation inside FP64 defect correction) with the flux Jacobian formed every
  ``--jac-lag``-th step, up to ``--max-resident`` cases on the device at once,
  admitted by device-memory footprint (jg_serve_*);
* ``serve-smallest``: the same, admitting the smallest queued footprint first;
* ``plain``: the plain FP64 GPU path, one case at a time in arrival order
  (the same server with one resident case and FP64 throughout).

All arms use the same relaxation (SGS sweeps), CFL ramp, step limit, stall
rule and restart policy.  One JSON line per arm: converged solves/hour over the horizon,
p50/p99 time-to-converge (arrival to retirement) and service time (admission
to retirement), cell-iterations/s, failures and restarts.
"""
from __future__ import annotations

import argparse
import collections
import dataclasses
import json
import math
import multiprocessing as mp
import time

import numpy as np


def request_stream(rate, horizon, lo, hi, seed):
    """Arrival times and case specs of the Poisson stream (seeded)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= horizon:
            break
        cells = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        ny = max(4, int(round(math.sqrt(cells / 4.0))))
        out.append(dict(t=t, nx=2 * ny, ny=ny, nz=2, mach=float(rng.uniform(0.3, 0.8)),
                        aoa=float(rng.uniform(-4.0, 4.0)), bump=float(rng.uniform(0.05, 0.12)),
                        seed=len(out)))
    return out


def case_specs(n, lo, hi, seed):
    """n seeded cases with the stream's distributions (cells log-uniform on [lo, hi], Mach
    U(0.3, 0.8), angle of attack U(+-4 deg), bump height U(0.05, 0.12)), all arriving at t = 0"""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        cells = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        ny = max(4, int(round(math.sqrt(cells / 4.0))))
        out.append(dict(t=0.0, nx=2 * ny, ny=ny, nz=2, mach=float(rng.uniform(0.3, 0.8)),
                        aoa=float(rng.uniform(-4.0, 4.0)), bump=float(rng.uniform(0.05, 0.12)), seed=k))
    return out


def spec_cells(spec):
    return spec["nx"] * spec["ny"] * spec["nz"]


def partition_cases(specs, world, rank):
    """The cases one GPU of `world` runs when a case list is spread over the GPUs of a node: every
    case runs whole on one GPU (no collective on the data path, weak scaling in cases).  Longest
    first by cells, each to the least-loaded GPU (ties: the lower rank), so every rank derives the
    same assignment from the same list; the rank's cases keep their list order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank %d of %d" % (rank, world))
    order = sorted(range(len(specs)), key=lambda k: (-spec_cells(specs[k]), k))
    load = [0] * world
    owner = [0] * len(specs)
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += spec_cells(specs[k])
    return [specs[k] for k in range(len(specs)) if owner[k] == rank]


def merge_rank_results(results):
    """One time-to-converge record from the records of the GPUs of a node (each ran its own share of
    the case list): solves per hour, cases and cells add up, the ratio is of the sums."""
    out = dict(results[0])
    out["solves_per_hour"] = sum(r["solves_per_hour"] for r in results)
    plain = sum(r["plain_fp64"]["solves_per_hour"] for r in results)
    out["ratio_vs_plain_fp64"] = out["solves_per_hour"] / max(1e-300, plain)
    out["cases"] = sum(r.get("cases", 0) for r in results)
    out["cells_total"] = sum(r.get("cells_total", 0) for r in results)
    out["gpus"] = len(results)
    return out


def build_request(spec):
    from myjoe_b200 import case
    _, g, prm = case.bump_case(spec["nx"], spec["ny"], spec["nz"], mach=spec["mach"], aoa_deg=spec["aoa"],
                               bump_h=spec["bump"], seed=spec["seed"], inlet="FARFIELD")
    state = case.perturbed_state(g.x_cv, prm, 0.0)
    return g, prm, state


def solver_params(prm, args):
    ra, ri, rf, rm = args.cfl_ramp.split(",")
    return dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=args.sweeps, CFL=1.0,
                               CFL_RAMP=(int(ra), int(ri), float(rf), float(rm)))


def pct(a, q):
    return float(np.percentile(a, q)) if len(a) else None


@dataclasses.dataclass
class BurstConfig:
    """Settings of a burst: every case submitted at t = 0, the arm runs until all retire."""
    drop: float = 1e-8
    sweeps: int = 10
    cfl_ramp: str = "10,5,1.2,20"
    max_steps: int = 6000
    chunk: int = 25
    max_resident: int = 64
    max_restarts: int = 2
    restart_factor: float = 0.25
    stall_steps: int = 1000
    jac_lag: int = 4          # serving arms: flux Jacobian blocks every jac_lag-th step
    hbm_budget: float = 0.0   # GB; 0: 90% of the free device memory
    renumber: int = 2         # every arm: cells in RCM order grouped by Gauss-Seidel colour


def run_burst(arm, cases, cfg: BurstConfig):
    """One arm over a list of built cases (g, prm, state), all arriving at once.

    * ``plain``: the plain FP64 GPU drop-in, one case at a time in list order, the
      Jacobian formed every step;
    * ``serve``: the serving form, mixed precision with a lagged Jacobian, up to
      ``max_resident`` cases on the device at once, admitted in list order by footprint;
    * ``serve-smallest``: the same, admitting the smallest queued footprint first.

    Time-to-converge is arrival (t = 0) to retirement; solves/hour = converged cases /
    makespan.  Same relaxation, CFL ramp, step limit, stall rule and restart policy in
    every arm."""
    from myjoe_b200 import solver
    serving = arm.startswith("serve")
    srv = solver.JoeServer(max_resident=cfg.max_resident if serving else 1, hbm_budget=cfg.hbm_budget * 1e9,
                           steps_per_poll=cfg.chunk, resid_drop=cfg.drop, max_steps=cfg.max_steps,
                           max_restarts=cfg.max_restarts, restart_cfl_factor=cfg.restart_factor,
                           stall_steps=cfg.stall_steps, admission="smallest" if arm == "serve-smallest" else "fifo")

    class _A:  # solver_params reads these
        sweeps, cfl_ramp = cfg.sweeps, cfg.cfl_ramp
    t0 = srv.now()
    for g, prm, state in cases:
        srv.submit(g, solver_params(prm, _A), state, precision=1 if serving else 0, t_arrival=t0,
                   jac_lag=cfg.jac_lag if serving else 1, renumber=cfg.renumber)
    results = []
    while len(results) < len(cases):
        for r in srv.poll(max_wait=0.05):
            srv.fetch(r["id"])
            results.append(r)
    makespan = max(r["t_done"] for r in results) - t0
    srv.close()
    conv = [r for r in results if r["status"] == 0]
    ttc = [r["t_done"] - t0 for r in conv]
    cell_iters = sum(r["ncv"] * r["steps_total"] for r in results)
    return {"arm": arm, "precision": "mixed" if serving else "fp64", "jac_lag": cfg.jac_lag if serving else 1,
            "max_resident": cfg.max_resident if serving else 1, "cases": len(cases), "converged": len(conv),
            "failed": sum(1 for r in results if r["status"] == 2),
            "max_steps_hit": sum(1 for r in results if r["status"] == 1),
            "stalled": sum(1 for r in results if r["status"] == 3),
            "restarts": sum(r["restarts"] for r in results), "makespan_s": makespan,
            "solves_per_hour": len(conv) / makespan * 3600.0,
            "p50_s": pct(ttc, 50), "p99_s": pct(ttc, 99),
            "steps_to_converge_p50": pct([r["conv_step"] for r in conv], 50),
            "cell_iters_per_s": cell_iters / makespan}


def run_arm(arm, stream, args):
    from myjoe_b200 import solver
    serving = arm.startswith("serve")
    precision = 1 if serving else 0
    resident = args.max_resident if serving else 1
    admission = "smallest" if arm == "serve-smallest" else "fifo"
    srv = solver.JoeServer(max_resident=resident, hbm_budget=args.hbm_budget * 1e9, steps_per_poll=args.chunk,
                           resid_drop=args.drop, max_steps=args.max_steps, max_restarts=args.max_restarts,
                           restart_cfl_factor=args.restart_factor, stall_steps=args.stall_steps,
                           admission=admission)
    pool = mp.get_context("spawn").Pool(args.workers)
    pending = collections.deque()   # mesh builds in flight, in arrival order (bounded lookahead)
    queued = 0                      # next request handed to the pool

    def top_up():
        nonlocal queued
        while queued < len(stream) and len(pending) < args.lookahead:
            pending.append(pool.apply_async(build_request, (stream[queued],)))
            queued += 1

    top_up()
    t0 = srv.now()
    nxt = 0                 # next request to submit
    results = []
    horizon = args.horizon
    while True:
        now = srv.now() - t0
        if now >= horizon:
            break
        st = srv.stats()
        # keep a short server-side queue; the rest wait on the client side
        while nxt < len(stream) and stream[nxt]["t"] <= now and st["queued"] < args.queue:
            if not pending[0].ready():
                break       # the client is still building this mesh: keep the device busy meanwhile
            g, prm, state = pending.popleft().get()
            top_up()
            srv.submit(g, solver_params(prm, args), state, precision=precision, t_arrival=t0 + stream[nxt]["t"],
                       jac_lag=args.jac_lag if serving else 1, renumber=args.renumber)
            nxt += 1
            st["queued"] += 1
        for r in srv.poll(max_wait=0.02):
            srv.fetch(r["id"])
            if r["t_done"] - t0 <= horizon:
                results.append(r)
    arrived = sum(1 for s in stream if s["t"] < horizon)
    srv.close()
    pool.terminate()
    conv = [r for r in results if r["status"] == 0]
    ttc = [r["t_done"] - r["t_arrival"] for r in conv]
    svc = [r["t_done"] - r["t_admit"] for r in conv]
    cell_iters = sum(r["ncv"] * r["steps_total"] for r in results)
    return {
        "form": "serve", "arm": arm, "precision": "mixed" if precision else "fp64", "max_resident": resident,
        "arrived_cells_p50": pct([s["nx"] * s["ny"] * s["nz"] for s in stream if s["t"] < horizon], 50),
        "rate_per_s": args.rate, "horizon_s": horizon, "arrived": arrived, "submitted": nxt,
        "retired": len(results), "converged": len(conv),
        "failed": sum(1 for r in results if r["status"] == 2),
        "max_steps_hit": sum(1 for r in results if r["status"] == 1),
        "stalled": sum(1 for r in results if r["status"] == 3),
        "admission": admission, "stall_steps": args.stall_steps,
        "converged_cells_p50": pct([r["ncv"] for r in conv], 50),
        "restarts": sum(r["restarts"] for r in results),
        "converged_solves_per_hour": len(conv) / horizon * 3600.0,
        "time_to_converge_p50_s": pct(ttc, 50), "time_to_converge_p99_s": pct(ttc, 99),
        "service_time_p50_s": pct(svc, 50), "service_time_p99_s": pct(svc, 99),
        "steps_to_converge_p50": pct([r["conv_step"] for r in conv], 50),
        "cell_iters_per_s": cell_iters / horizon,
        "drop": args.drop, "solver": "SGS x%d" % args.sweeps, "cfl_ramp": args.cfl_ramp,
        "jac_lag": args.jac_lag if serving else 1, "renumber": args.renumber,
        "cells": [args.min_cells, args.max_cells],
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--horizon", type=float, default=600.0)
    ap.add_argument("--min-cells", type=int, default=5000)
    ap.add_argument("--max-cells", type=int, default=500000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--arms", default="serve,plain", help="any of serve, serve-smallest, plain")
    ap.add_argument("--max-resident", type=int, default=48)
    ap.add_argument("--hbm-budget", type=float, default=0.0, help="GB; 0: 90%% of free device memory")
    ap.add_argument("--queue", type=int, default=8, help="server-side queue length")
    ap.add_argument("--chunk", type=int, default=25)
    ap.add_argument("--sweeps", type=int, default=10)
    ap.add_argument("--cfl-ramp", default="10,5,1.2,20")
    ap.add_argument("--drop", type=float, default=1e-8)
    ap.add_argument("--max-steps", type=int, default=6000)
    ap.add_argument("--max-restarts", type=int, default=2)
    ap.add_argument("--restart-factor", type=float, default=0.25)
    ap.add_argument("--stall-steps", type=int, default=1000,
                    help="retire a case whose best residual drop has not halved in this many steps (0: off)")
    ap.add_argument("--workers", type=int, default=min(32, mp.cpu_count()))
    ap.add_argument("--lookahead", type=int, default=48, help="mesh builds in flight")
    ap.add_argument("--jac-lag", type=int, default=4, help="serving arms: flux Jacobian every k-th step")
    ap.add_argument("--renumber", type=int, default=2, help="cell order of every arm (0 none, 1 RCM, 2 RCM by colour)")
    args = ap.parse_args(argv)

    from myjoe_b200 import build
    if build.needs_build():
        build.build()
    stream = request_stream(args.rate, args.horizon, args.min_cells, args.max_cells, args.seed)
    for arm in args.arms.split(","):
        t = time.perf_counter()
        out = run_arm(arm, stream, args)
        out["wall_s"] = time.perf_counter() - t
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
