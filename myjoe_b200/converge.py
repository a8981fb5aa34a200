"""Time to converge one case on the GPU: the Euler channel bump (64x32x4
hex, 8,192 cells, HLLC, M 0.5, second order with the limiter, CFL 1 ramped
x1.2 every 5 steps to 20, the settings the reference converges this case
with) or the laminar flat plate (256x96x2, 49,152 cells, Roe + Sutherland,
CFL ramped to 100), run to a drop of the L1 energy residual (relative to the
first step's, or to the largest so far), FP64 or mixed.  Prints one JSON
line: steps, device seconds, cell-iters/s, converged solves per hour of one
GPU.

    python -m myjoe_b200.converge --case bump [--precision mixed] [--solver SGS] [--drop 1e-10]
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import time

import numpy as np

from . import build, case, solver


def make(which, cfl_max):
    if which == "bump":
        # the settings of the reference's own converged run of this case (tests/golden/make_converged.py)
        _, g, prm = case.bump_case(64, 32, 4)
        return g, dataclasses.replace(prm, CFL=1.0, CFL_RAMP=(10, 5, 1.2, cfl_max or 20.0), EPS=0.01), \
            "Euler bump 64x32x4 (8,192 cells), HLLC"
    _, g, prm = case.plate_case(256, 96, 2)
    return g, dataclasses.replace(prm, CFL=1.0, CFL_RAMP=(10, 5, 1.2, cfl_max or 100.0)), \
        "laminar plate 256x96x2 (49,152 cells), Roe + Sutherland"


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--case", default="bump", choices=["bump", "plate"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--solver", default="SGS", choices=["SGS", "JACOBI", "LINE", "BCGSTAB", "BCGSTAB_LINELET"])
    ap.add_argument("--sweeps", type=int, default=10)
    ap.add_argument("--drop", type=float, default=1e-10)
    ap.add_argument("--max-steps", type=int, default=4000)
    ap.add_argument("--cfl-max", type=float, default=0.0, help="MAX_CFL of the ramp (0: the case's)")
    ap.add_argument("--chunk", type=int, default=50)
    ap.add_argument("--first-order", action="store_true", help="first-order reconstruction")
    ap.add_argument("--no-limiter", action="store_true", help="second order without the Barth-Jespersen limiter")
    ap.add_argument("--drop-from", choices=["first", "max"], default=None,
                    help="drop relative to the first step's energy residual (bump default) or to the largest "
                         "so far (plate default: from the uniform start the plate's first residual is only the "
                         "wall's, and the residual grows by about ten orders before it falls)")
    a = ap.parse_args(argv)
    build.build()
    g, prm, name = make(a.case, a.cfl_max)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS=a.solver, LS_MAX_ITER=a.sweeps,
                              SECOND_ORDER=not a.first_order, LIMITER=not a.no_limiter)
    j = solver.JoeGpu(g, prm, precision=1 if a.precision == "mixed" else 0)
    j.set_state(*case.perturbed_state(g.x_cv, prm, 0.0))
    j.runBackwardEuler(1)
    j.close()
    # the timed solve: a fresh handle from the uniform start
    j = solver.JoeGpu(g, prm, precision=1 if a.precision == "mixed" else 0)
    j.set_state(*case.perturbed_state(g.x_cv, prm, 0.0))
    drop_from = a.drop_from or ("first" if a.case == "bump" else "max")
    steps, ran, rref, t, drop = 0, 0, None, 0.0, 1.0
    hist = []   # the drop every 1000 steps
    while steps < a.max_steps:
        t0 = time.perf_counter()
        r = j.runBackwardEuler(a.chunk)
        t += time.perf_counter() - t0
        ran += a.chunk
        e = r[:, 4]
        if drop_from == "first":
            rref = e[0] if rref is None else rref
            d = e / rref
        else:
            run_max = np.maximum.accumulate(np.concatenate([[rref or 0.0], e]))[1:]
            rref = run_max[-1]
            d = e / run_max
        hit = np.nonzero(d <= a.drop)[0]
        if hit.size:
            steps += int(hit[0]) + 1
            drop = float(d[hit[0]])
            break
        steps += a.chunk
        drop = float(d[-1])
        if steps % 1000 == 0:
            hist.append(drop)
        if not np.isfinite(drop):
            break
    t *= steps / max(ran, 1)  # the steps after the drop inside the last chunk do not count
    order = "first order" if a.first_order else "second order" + (" no limiter" if a.no_limiter else "")
    out = {"workload": name, "cells": g.ncv, "precision": a.precision, "solver": "%s x%d" % (a.solver, a.sweeps),
           "order": order,
           "cfl_ramp": list(prm.CFL_RAMP),
           "drop_target": a.drop, "drop_from": drop_from, "drop": drop, "converged": bool(drop <= a.drop), "steps": steps,
           "seconds": t, "cell_iters_per_s": g.ncv * steps / t, "solves_per_hour": 3600.0 / t,
           "drop_every_1000_steps": hist}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
