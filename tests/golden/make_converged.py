"""Converged-field goldens: the reference solver itself (oracle/_ref/ref_harness)
run to steady state.

* converged_bump_64x32x4.npz: the 64x32x4 inviscid channel-with-bump case (8,192
  cells; HLLC, second order LSQ + Barth-Jespersen EPS 0.01, backward Euler,
  BiCGSTAB, CFL ramp 1 -> 20), stopped at a 1e-10 drop of the L1 energy
  residual or 2,000 iterations.
* converged_plate_64x32x2.npz: the laminar flat plate of the plate benchmark at
  64x32x2 (4,096 cells, geometric wall-normal stretching, Re_L 1e5, Mach 0.3,
  Roe, Sutherland viscosity, Pr 0.72; BiCGSTAB with the reference's default
  thresholds, CFL ramp 1 -> 200), PLATE_STEPS iterations.  From the uniform
  start the L1 energy residual is 0 at the first step (so the reference's own
  absolute rule RESID_ENERG_TH would stop it there), grows to about 3.4 and
  falls to a round-off floor near 1.4e-9; after PLATE_STEPS it is about
  1.7e-9, 5e-10 of its peak.

Each stores the reference's cell centroids, the converged conserved state and
the residual history.

The ramp stops at CFL 20: with its default linear-solver thresholds
(BiCGSTAB, 30 iterations, 1e-2 relative) and under-relaxation 0.3 the
reference does not converge on this case at CFL 100 (a ramp of x1.2 every 5
steps diverges at step 154; x1.1 every 10 steps stalls at a 5e-3 drop).

    python tests/golden/make_converged.py [bump] [plate]   # minutes on one core each
"""
from __future__ import annotations

import dataclasses
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from myjoe_b200 import case, meshgen  # noqa: E402
from oracle import refrun  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
DROP = 1.0e-10


def bump_config():
    raw, g, prm = case.bump_case(64, 32, 4)
    prm = dataclasses.replace(prm, CFL=1.0, CFL_RAMP=(10, 5, 1.2, 20.0), EPS=0.01)
    return raw, g, prm


PLATE_STEPS = 4000


def plate_config():
    raw, g, prm = case.plate_case(64, 32, 2)
    prm = dataclasses.replace(prm, CFL=1.0, CFL_RAMP=(10, 5, 1.2, 200.0))
    return raw, g, prm


def make_plate():
    raw, g, prm = plate_config()
    write = lambda p: meshgen.write_msh(p, raw)
    run = dataclasses.replace(prm, NSTEPS=PLATE_STEPS)
    r = refrun.run(write, run.joe_in("mesh.msh"), "run", timeout=7200)
    np.savez_compressed(os.path.join(HERE, "converged_plate_64x32x2.npz"), x_cv=r["x_cv"].reshape(-1, 3),
                        rho=r["final_rho"], rhou=r["final_rhou"].reshape(-1, 3), rhoE=r["final_rhoE"],
                        resid=r["resid"], steps=np.array(r["steps"]), seconds=np.array(r["seconds"]))
    print("plate steps", r["steps"], "seconds", r["seconds"], "final energy residual", r["resid"][-1][4])


def main():
    which = sys.argv[1:] or ["bump"]
    if "plate" in which:
        make_plate()
    if "bump" not in which:
        return
    raw, g, prm = bump_config()
    write = lambda p: meshgen.write_msh(p, raw)
    first = refrun.run(write, dataclasses.replace(prm, NSTEPS=1).joe_in("mesh.msh"), "run")
    r0 = float(first["resid"][0][4])
    run = dataclasses.replace(prm, NSTEPS=2000)
    r = refrun.run(write, run.joe_in("mesh.msh", "RESID_ENERG_TH = %.17g" % (DROP * r0)), "run", timeout=3600)
    np.savez_compressed(os.path.join(HERE, "converged_bump_64x32x4.npz"), x_cv=r["x_cv"].reshape(-1, 3),
                        rho=r["final_rho"], rhou=r["final_rhou"].reshape(-1, 3), rhoE=r["final_rhoE"],
                        resid=r["resid"], steps=np.array(r["steps"]), seconds=np.array(r["seconds"]))
    print("steps", r["steps"], "seconds", r["seconds"], "final/initial energy residual",
          r["resid"][-1][4] / r0)


if __name__ == "__main__":
    main()
