"""Run a seeded case on the GPU and print its residual history.

    python -m myjoe_b200.run --case plate --steps 50 [--precision mixed] [--sweeps 10]
    python -m myjoe_b200.run --case bump --nx 64 --ny 32 --nz 4 --steps 200 --solver BCGSTAB

Cases: ``bump`` (inviscid channel with a bump, HLLC) and ``plate`` (laminar
flat plate, Roe + Sutherland), from myjoe_b200.case.
"""
from __future__ import annotations

import argparse
import dataclasses
import time

import numpy as np

from . import build, case, solver


def make(args):
    if args.case == "plate":
        _, g, prm = case.plate_case(args.nx or 256, args.ny or 96, args.nz or 2)
    else:
        _, g, prm = case.bump_case(args.nx or 64, args.ny or 32, args.nz or 4, jitter=args.jitter, seed=args.seed)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS=args.solver, LS_MAX_ITER=args.sweeps, CFL=args.cfl,
                              CFL_RAMP=(args.ramp_after, args.ramp_interval, args.ramp_factor, args.cfl_max))
    return g, prm


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="plate", choices=["plate", "bump"])
    ap.add_argument("--nx", type=int, default=0)
    ap.add_argument("--ny", type=int, default=0)
    ap.add_argument("--nz", type=int, default=0)
    ap.add_argument("--jitter", type=float, default=0.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--solver", default="JACOBI", choices=["JACOBI", "SGS", "BCGSTAB", "LUSGS"])
    ap.add_argument("--sweeps", type=int, default=10)
    ap.add_argument("--cfl", type=float, default=1.0)
    ap.add_argument("--cfl-max", type=float, default=100.0)
    ap.add_argument("--ramp-after", type=int, default=10)
    ap.add_argument("--ramp-interval", type=int, default=5)
    ap.add_argument("--ramp-factor", type=float, default=1.2)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    args = ap.parse_args(argv)
    if build.needs_build():
        build.build()
    g, prm = make(args)
    j = solver.JoeGpu(g, prm, precision=1 if args.precision == "mixed" else 0)
    j.set_state(*case.perturbed_state(g.x_cv, prm, 0.0))
    t0 = time.perf_counter()
    res = j.runBackwardEuler(args.steps)
    dt = time.perf_counter() - t0
    for k in range(0, args.steps, max(1, args.steps // 10)):
        print("RESID: %6d %12.4e %12.4e %12.4e %12.4e %12.4e" % (k + 1, *res[k]))
    print("cells %d steps %d wall %.3f s (%.3e cell-iters/s incl. host sync)" % (g.ncv, args.steps, dt,
                                                                               g.ncv * args.steps / dt))
    if not np.all(np.isfinite(res)):
        raise SystemExit("non-finite residual")


if __name__ == "__main__":
    main()
