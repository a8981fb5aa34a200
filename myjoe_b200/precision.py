"""Precision form on a shuffled mixed prism/hex mesh: one Spalart-Allmaras
case solved twice on the GPU, with FP64 Jacobian blocks and relaxation (the
plain method) and with FP32 blocks and relaxation inside the FP64 residual
and update (the mixed form), each to the residual drop or the step limit.
Reports the steps, time and throughput of each, and the relative L2 error of
the mixed form's final fields against the FP64 ones.

The mesh: the channel bump of ``case.sa_bump_case`` (M 0.7, Re 3e6 on the
bump chord, far-field inlet/outlet/top, viscous WALL below) meshed by
``meshgen.channel_bump_mixed`` (prism rows on the wall, hexahedra above),
cells and faces shuffled from the seed, solved through a handle that
renumbers them itself (reverse Cuthill-McKee).  The shuffled order without
renumbering is timed over a few hundred steps beside it.  The linear solve
is the LINE relaxation by default (block-tridiagonal solves along the
wall-normal lines, which the stretched wall rows need), 10 sweeps per step.

    python -m myjoe_b200.precision [--nx 512 --ny 400 --nz 8 --n-prism 88] [--first-order] [--out f.json]
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import time

import numpy as np

from . import build, case, solver


def rel_l2(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def solve(g, prm, precision, max_steps, drop, chunk, renumber=True):
    j = solver.JoeGpu(g, prm, precision=precision, renumber=renumber)
    st = case.perturbed_state(g.x_cv, prm, 0.0)
    j.set_state(*st)
    j.set_scalars(np.full(g.ncv, prm.NUSA_INITIAL))
    hist, r0, steps, t_solve = [], None, 0, 0.0
    while steps < max_steps:
        n = min(chunk, max_steps - steps)
        t = time.perf_counter()
        r = j.runBackwardEuler(n)
        t_solve += time.perf_counter() - t
        if r0 is None:
            r0 = r[0].copy()
        steps += n
        rel = r[-1] / r0
        hist.append([steps] + [float(x) for x in rel])
        if not np.all(np.isfinite(rel)) or rel[4] <= drop:
            break
    fields = dict(zip(("rho", "rhou", "rhoE"), j.get_state()))
    fields["nuSA"] = j.get_scalars()
    out = {"precision": "mixed" if precision else "fp64", "steps": steps, "seconds": t_solve,
           "ms_per_step": 1e3 * t_solve / steps, "cell_iters_per_s": g.ncv * steps / t_solve,
           "final_drop": hist[-1][1:], "converged": bool(hist[-1][5] <= drop), "history": hist,
           "device_bytes": j.device_bytes()}
    j.close()
    return out, fields


def time_order(g, prm, renumber, steps=200):
    j = solver.JoeGpu(g, prm, precision=1, renumber=renumber)
    j.set_state(*case.perturbed_state(g.x_cv, prm, 0.0))
    j.set_scalars(np.full(g.ncv, prm.NUSA_INITIAL))
    j.runBackwardEuler(20)
    j.set_profiling(True)
    t = time.perf_counter()
    j.runBackwardEuler(steps)
    dt = time.perf_counter() - t
    prof = j.profile()
    j.close()
    return {"renumber": renumber, "ms_per_step": 1e3 * dt / steps, **prof}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--nx", type=int, default=512)
    ap.add_argument("--ny", type=int, default=400)
    ap.add_argument("--nz", type=int, default=8)
    ap.add_argument("--n-prism", type=int, default=88)
    ap.add_argument("--stretch", type=float, default=1.02)
    ap.add_argument("--bump-h", type=float, default=0.05)
    ap.add_argument("--mach", type=float, default=0.7)
    ap.add_argument("--re", type=float, default=3.0e6)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--first-order", action="store_true")
    ap.add_argument("--solver", default="LINE", choices=["LINE", "SGS", "JACOBI"])
    ap.add_argument("--sweeps", type=int, default=10)
    ap.add_argument("--cfl-max", type=float, default=50.0)
    ap.add_argument("--max-steps", type=int, default=6000)
    ap.add_argument("--drop", type=float, default=1e-8)
    ap.add_argument("--chunk", type=int, default=250)
    ap.add_argument("--skip-order-timing", action="store_true")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    build.build()
    t = time.perf_counter()
    raw, g, prm = case.sa_bump_case(a.nx, a.ny, a.nz, mach=a.mach, re=a.re, bump_h=a.bump_h, seed=a.seed,
                                    stretch=a.stretch, n_prism=a.n_prism, alternate=True, shuffle=True)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS=a.solver, LS_MAX_ITER=a.sweeps, CFL=1.0,
                              CFL_RAMP=(10, 5, 1.2, a.cfl_max), SECOND_ORDER=not a.first_order)
    t_mesh = time.perf_counter() - t
    nprism = 2 * a.nx * a.nz * a.n_prism
    res = {"workload": "SA bump, shuffled mixed prism/hex mesh", "ncv": g.ncv, "prisms": nprism,
           "hexahedra": g.ncv - nprism, "nfa": g.nfa, "mach": a.mach, "re": a.re, "bump_h": a.bump_h,
           "second_order": not a.first_order, "solver": a.solver, "sweeps": a.sweeps, "cfl_max": a.cfl_max,
           "drop": a.drop,
           "mesh_seconds": t_mesh}
    if not a.skip_order_timing:
        res["order_timing"] = [time_order(g, prm, False), time_order(g, prm, True)]
    r64, f64 = solve(g, prm, 0, a.max_steps, a.drop, a.chunk)
    r32, f32 = solve(g, prm, 1, a.max_steps, a.drop, a.chunk)
    res["fp64"], res["mixed"] = r64, r32
    res["mixed_vs_fp64_rel_l2"] = {k: rel_l2(f32[k], f64[k]) for k in f64}
    line = json.dumps(res)
    print(line)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
