"""Restart-file fixtures: files written by the reference solver itself
(oracle/_ref/ref_harness, built from the reference's own sources), and the
reference's own continuation from one of them.

* restart_bump_step3.out: the 8x4x2 jittered channel bump (HLLC, second order,
  CFL ramp x1.5 per step to 5) after 3 runBackwardEuler steps from the
  perturbed uniform state: the restart.out runBackwardEuler leaves
  (JoeWithModels.cpp:1179, Ugp::writeRestart).
* restart_bump.npz: the reference's cell centroids and state after those 3
  steps, and after 3 more steps that the reference ran from the restart file
  (RESTART = restart.in, NSTEPS = 6): its centroids (in its order after
  reading the restart), state and residuals, and the case parameters.
* restart_sa_step2.out: the 8x4x2 Spalart-Allmaras bump (segregated SA run)
  after 2 steps; it holds nuSA and the SA model's records.

    python tests/golden/make_restart.py    # needs the reference + g++ (seconds)
"""
from __future__ import annotations

import dataclasses
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from myjoe_b200 import case, meshgen  # noqa: E402
from oracle import refrun  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
PERTURB = 0.05


def bump_case():
    raw, _, prm = case.bump_case(8, 4, 2, jitter=0.15, seed=7)
    return raw, dataclasses.replace(prm, CFL_RAMP=(1, 1, 1.5, 5.0))


def sa_case():
    raw, _, prm = case.sa_bump_case(8, 4, 2, stretch=1.3)
    return raw, prm


def main():
    sys.path.insert(0, HERE)
    from make_golden import params_json
    raw, prm = bump_case()
    write = lambda p: meshgen.write_msh(p, raw)  # noqa: E731
    first = refrun.run(write, dataclasses.replace(prm, NSTEPS=3).joe_in("mesh.msh", "HARNESS_PERTURB = %g" % PERTURB),
                       "run", collect=("restart.out",))
    blob = first["files"]["restart.out"]
    with open(os.path.join(HERE, "restart_bump_step3.out"), "wb") as f:
        f.write(blob)
    cont = refrun.run(None, dataclasses.replace(prm, NSTEPS=6).joe_in("restart.in"), "run",
                      files={"restart.in": blob})
    np.savez_compressed(os.path.join(HERE, "restart_bump.npz"),
                        x_cv3=first["x_cv"], rho3=first["final_rho"], rhou3=first["final_rhou"],
                        rhoE3=first["final_rhoE"], x_cv6=cont["x_cv"], rho6=cont["final_rho"],
                        rhou6=cont["final_rhou"], rhoE6=cont["final_rhoE"], resid6=cont["resid"],
                        steps6=np.array(cont["steps"]), params=np.array(params_json(prm)))
    print("bump: restart", len(blob), "bytes; continued to step", cont["steps"])
    raw, prm = sa_case()
    sa = refrun.run(lambda p: meshgen.write_msh(p, raw),
                    dataclasses.replace(prm, NSTEPS=2).joe_in("mesh.msh", "HARNESS_PERTURB = %g" % PERTURB), "run",
                    run_kind=1, collect=("restart.out",))
    with open(os.path.join(HERE, "restart_sa_step2.out"), "wb") as f:
        f.write(sa["files"]["restart.out"])
    with open(os.path.join(HERE, "restart_sa.json"), "w") as f:
        f.write(json.dumps({"params": params_json(prm)}))
    print("sa: restart", len(sa["files"]["restart.out"]), "bytes")


if __name__ == "__main__":
    main()
