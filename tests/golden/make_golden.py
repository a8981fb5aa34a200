"""Generates the golden fixtures in this directory by running the reference
solver itself (oracle/_ref/ref_harness, compiled from the reference's own
sources by oracle/Makefile) on small seeded meshes.

Each fixture holds the reference's mesh arrays (its own cell/face order), the
initial state, the case parameters, and the reference's outputs: primitive
and boundary-face states, local time step, gradients, RHS, the implicit
matrix A, one linear solve, and the state + L1 residuals after a few
runBackwardEuler steps.

    python tests/golden/make_golden.py [segregated] [sa] [sst] [--only=NAME_PART]   # needs the reference + g++
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
from myjoe_b200.case import BC  # noqa: E402
from oracle import refrun  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
PERTURB = 0.05
NSTEPS = 3


def cases():
    raw, _, prm = case.bump_case(8, 4, 2, jitter=0.15, seed=7)
    visc = dataclasses.replace(prm, MU_MODE="SUTHERLAND", MU_REF=1.716e-5 * 2000.0, SPACE_INTEGRATION="ROE")
    u = prm.U_INITIAL
    bc_mix = dict(prm.bcs)
    bc_mix["inlet"] = BC("CBC_SUBSONIC_INLET", (1.0, 0.0, 0.0, 300.0 * 1.05, 1.0e5 * 1.05 ** 3.5))
    bc_mix["upper"] = BC("FARFIELD", u + (1.0e5, prm.RHO_REF, 1.4))
    bc_mix["outlet"] = BC("NEUMANN")
    bc_iso = dict(visc.bcs)
    bc_iso["lower"] = BC("WALL", (350.0,))
    rawp, _, prmp = case.plate_case(12, 8, 2)
    # prism rows on the wall (triangulated wall surface extruded wall-normal), hexahedra above
    rawm = meshgen.channel_bump_mixed(12, 6, 2, n_prism=2, stretch=1.2, jitter=0.1, seed=4)
    yield "bump_hllc", raw, prm
    yield "bump_roe", raw, dataclasses.replace(prm, SPACE_INTEGRATION="ROE")
    yield "bump_ausm_first_order", raw, dataclasses.replace(prm, SPACE_INTEGRATION="AUSM", SECOND_ORDER=False)
    yield "bump_hllc_symm_analytical_lusgs", raw, dataclasses.replace(prm, SYMM_BC="ANALYTICAL",
                                                                     LINEAR_SOLVER_NS="LUSGS")
    yield "bump_hllc_symm_new_sumdt", raw, dataclasses.replace(prm, SYMM_BC="NEW_NUMERIC", TIME_STEP="SUM_BASED",
                                                               CFL_RAMP=(1, 1, 1.5, 5.0))
    yield "bump_bc_mix", raw, dataclasses.replace(prm, bcs=bc_mix)
    yield "bump_roe_laminar_isothermal", raw, dataclasses.replace(visc, bcs=bc_iso)
    yield "bump_hllc_laminar_powerlaw_novisclim", raw, dataclasses.replace(visc, MU_MODE="POWERLAW",
                                                                          SPACE_INTEGRATION="HLLC",
                                                                          VISC_LIMITER=False)
    yield "plate_roe", rawp, prmp
    # gravity (sourceHook, GX/GY/GZ), large enough to stand out of the face fluxes
    yield "bump_hllc_gravity", raw, dataclasses.replace(prm, GX=300.0, GY=-5000.0, GZ=40.0)
    yield "plate_roe_gravity", rawp, dataclasses.replace(prmp, GX=0.0, GY=-5000.0, GZ=0.0)
    # Haenel & Schwane (SPACE_INTEGRATION = HAENEL): second order, laminar, first order with NEW_NUMERIC symmetry
    # Green-Gauss gradients (GRAD_RECONSTRUCTION SCHEME=GREENGAUSS, the reference's default scheme)
    yield "bump_hllc_greengauss", raw, dataclasses.replace(prm, GRAD_SCHEME="GREENGAUSS")
    yield "plate_roe_greengauss", rawp, dataclasses.replace(prmp, GRAD_SCHEME="GREENGAUSS")
    yield "bump_roe_laminar_greengauss_novisclim", raw, dataclasses.replace(visc, bcs=bc_iso, GRAD_SCHEME="GREENGAUSS",
                                                                          VISC_LIMITER=False)
    # SDWLS gradients (GRAD_RECONSTRUCTION SCHEME=SDWLS): inviscid second order, laminar plate, isothermal wall
    yield "bump_hllc_sdwls", raw, dataclasses.replace(prm, GRAD_SCHEME="SDWLS")
    yield "plate_roe_sdwls", rawp, dataclasses.replace(prmp, GRAD_SCHEME="SDWLS")
    yield "bump_roe_laminar_sdwls_isothermal", raw, dataclasses.replace(visc, bcs=bc_iso, GRAD_SCHEME="SDWLS")
    # AUSMDV family: sonic faces from a sonic inflow, the HAENEL shock fix on faces between flagged
    # cells (CELL_FLAG_HEX), ALPHA_LR with CELL_FLAG_TET, the entropy fix on an expansion; AUSMD and AUSMV
    rawt, _, prmt = case.bump_case(8, 4, 2, jitter=0.15, seed=7, mach=1.0)
    rawt5, _, prmt5 = case.bump_case(8, 4, 2, jitter=0.15, seed=7, mach=1.05)
    yield "bump_ausmdv_m1", rawt, dataclasses.replace(prmt, SPACE_INTEGRATION="AUSMDV")
    yield "bump_ausmdv_alpha_tet_m105", rawt5, dataclasses.replace(prmt5, SPACE_INTEGRATION="AUSMDV",
                                                                   SHOCK_FIX_TYPE="ALPHA_LR",
                                                                   SHOCK_FIX_FLAG="CELL_FLAG_TET")
    yield "bump_ausmv_m105", rawt5, dataclasses.replace(prmt5, SPACE_INTEGRATION="AUSMV", SHOCK_FIX_TYPE="NONE")
    yield "bump_ausmd_first_order", raw, dataclasses.replace(prm, SPACE_INTEGRATION="AUSMD", SECOND_ORDER=False,
                                                             ENTROPY_FIX="NONE", SHOCK_FIX_TYPE="NONE")
    # JST: first and second order, and the laminar plate
    yield "bump_jst_first_order", raw, dataclasses.replace(prm, SPACE_INTEGRATION="JST", SECOND_ORDER=False)
    yield "bump_jst", raw, dataclasses.replace(prm, SPACE_INTEGRATION="JST")
    yield "plate_jst", rawp, dataclasses.replace(prmp, SPACE_INTEGRATION="JST")
    yield "bump_haenel", raw, dataclasses.replace(prm, SPACE_INTEGRATION="HAENEL")
    yield "bump_haenel_laminar_isothermal", raw, dataclasses.replace(visc, SPACE_INTEGRATION="HAENEL", bcs=bc_iso)
    yield "bump_haenel_first_order_symm_new", raw, dataclasses.replace(prm, SPACE_INTEGRATION="HAENEL",
                                                                      SECOND_ORDER=False, SYMM_BC="NEW_NUMERIC")
    yield "mixed_bump_hllc", rawm, prm
    yield "mixed_bump_roe_laminar_isothermal", rawm, dataclasses.replace(visc, bcs=bc_iso)
    # BCGSTAB_LINELET: lines from the wall through the stretched rows (and through prisms into hexahedra)
    rawl, _, prml = case.plate_case(24, 16, 2)
    yield "plate_roe_linelet", rawl, dataclasses.replace(prml, LINEAR_SOLVER_NS="BCGSTAB_LINELET", LS_MAX_ITER=10)
    yield "mixed_bump_roe_laminar_linelet", rawm, dataclasses.replace(visc, bcs=bc_iso,
                                                                      LINEAR_SOLVER_NS="BCGSTAB_LINELET")


def sa_cases():
    """Coupled Spalart-Allmaras cases (runBackwardEulerCoupled's calcRhsCoupled)."""
    raw, _, prm = case.sa_bump_case(16, 8, 2, stretch=1.2, jitter=0.1, seed=3)
    rawc, _, prmc = case.sa_bump_case(16, 8, 2, stretch=1.15, jitter=0.1, seed=5, inlet="CBC", mach=0.5)
    bc_n = dict(prmc.bcs)
    bc_n["outlet"] = BC("NEUMANN")
    yield "sa_bump_farfield", raw, prm
    yield "sa_bump_cbc_symm_original", rawc, dataclasses.replace(prmc, SYMM_BC="ORIGINAL_NUMERIC")
    rawm, _, prmm = case.sa_bump_case(12, 8, 2, stretch=1.2, jitter=0.1, seed=6, n_prism=3, alternate=True)
    yield "sa_mixed_bump_farfield", rawm, prmm
    yield "sa_bump_neumann_first_order_new_numeric", rawc, dataclasses.replace(
        prmc, bcs=bc_n, SECOND_ORDER=False, SYMM_BC="NEW_NUMERIC")
    # the coupled AUSMDV family and HAENEL (calcFluxCoupled's other flux choices): sonic inflows for the
    # shock sensor (the HAENEL shock fix with CELL_FLAG_HEX, ALPHA_LR with CELL_FLAG_TET), the entropy
    # fix, every boundary branch; HAENEL is not combined with NEW_NUMERIC symmetry, whose matrices the
    # reference leaves unset (it compares the name "Haenel" there)
    rawt, _, prmt = case.sa_bump_case(16, 8, 2, stretch=1.2, jitter=0.1, seed=7, mach=1.0)
    rawt5, _, prmt5 = case.sa_bump_case(16, 8, 2, stretch=1.15, jitter=0.1, seed=8, inlet="CBC", mach=1.05)
    yield "sa_bump_ausmdv_m1", rawt, dataclasses.replace(prmt, SPACE_INTEGRATION="AUSMDV")
    yield "sa_bump_ausmv_alpha_tet_m105_symm_original", rawt5, dataclasses.replace(
        prmt5, SPACE_INTEGRATION="AUSMV", SHOCK_FIX_TYPE="ALPHA_LR", SHOCK_FIX_FLAG="CELL_FLAG_TET",
        SYMM_BC="ORIGINAL_NUMERIC")
    yield "sa_bump_ausmd_neumann_first_order_new_numeric", rawc, dataclasses.replace(
        prmc, bcs=bc_n, SECOND_ORDER=False, SYMM_BC="NEW_NUMERIC", SPACE_INTEGRATION="AUSMD",
        SHOCK_FIX_TYPE="NONE", ENTROPY_FIX="NONE")
    yield "sa_bump_haenel_farfield", raw, dataclasses.replace(prm, SPACE_INTEGRATION="HAENEL")
    # gravity (sourceHookCoupled, GX/GY/GZ)
    yield "sa_bump_gravity", raw, dataclasses.replace(prm, GX=300.0, GY=-5000.0, GZ=40.0)
    yield "sa_mixed_bump_haenel_symm_original", rawm, dataclasses.replace(prmm, SPACE_INTEGRATION="HAENEL",
                                                                          SYMM_BC="ORIGINAL_NUMERIC")


def sst_cases():
    """Coupled Menter SST cases (runBackwardEulerCoupled's calcRhsCoupled, 7x7 blocks)."""
    raw, _, prm = case.sst_bump_case(16, 8, 2, stretch=1.2, jitter=0.1, seed=3)
    rawc, _, prmc = case.sst_bump_case(16, 8, 2, stretch=1.15, jitter=0.1, seed=5, inlet="CBC", mach=0.5)
    bc_n = dict(prmc.bcs)
    bc_n["outlet"] = BC("NEUMANN")
    yield "sst_bump_farfield", raw, prm
    yield "sst_bump_cbc_symm_original", rawc, dataclasses.replace(prmc, SYMM_BC="ORIGINAL_NUMERIC")
    rawm, _, prmm = case.sst_bump_case(12, 8, 2, stretch=1.2, jitter=0.1, seed=6, n_prism=3, alternate=True)
    yield "sst_mixed_bump_farfield", rawm, prmm
    yield "sst_bump_neumann_first_order_new_numeric", rawc, dataclasses.replace(
        prmc, bcs=bc_n, SECOND_ORDER=False, SYMM_BC="NEW_NUMERIC")
    # the coupled AUSMDV and HAENEL with k in the total enthalpy
    rawt, _, prmt = case.sst_bump_case(16, 8, 2, stretch=1.2, jitter=0.1, seed=7, mach=1.0)
    yield "sst_bump_ausmdv_m1", rawt, dataclasses.replace(prmt, SPACE_INTEGRATION="AUSMDV")
    yield "sst_bump_haenel_neumann_first_order", rawc, dataclasses.replace(
        prmc, bcs=bc_n, SECOND_ORDER=False, SYMM_BC="ORIGINAL_NUMERIC", SPACE_INTEGRATION="HAENEL")


def params_json(prm) -> str:
    d = dataclasses.asdict(prm)
    d["bcs"] = {k: [v.kind, list(v.values)] for k, v in prm.bcs.items()}
    return json.dumps(d)


def params_from_json(s: str):
    d = json.loads(s)
    bcs = {k: BC(v[0], tuple(v[1])) for k, v in d.pop("bcs").items()}
    for k in ("CFL_RAMP", "U_INITIAL"):
        d[k] = tuple(d[k])
    return case.JoeParams(bcs=bcs, **d)


def main(which=("segregated", "sa"), only=""):
    """``only``: regenerate just the fixtures whose name contains it."""
    for name, raw, prm in (cases() if "segregated" in which else ()):
        if only not in name:
            continue
        extra = "HARNESS_PERTURB = %g" % PERTURB
        d = refrun.run(lambda p: meshgen.write_msh(p, raw), prm.joe_in("mesh.msh", extra), "dump")
        prm_run = dataclasses.replace(prm, NSTEPS=NSTEPS)
        r = refrun.run(lambda p: meshgen.write_msh(p, raw), prm_run.joe_in("mesh.msh", extra), "run")
        keep = ["cvofa", "faocv_i", "faocv_v", "nbocv_i", "nbocv_v", "x_cv", "x_fa", "fa_normal", "cv_volume",
                "nbocv_lsg_coeff", "boundary_fa_lsg_coeff", "init_rho", "init_rhou", "init_rhoE",
                "press", "temp", "enthalpy", "sos", "vel", "rho_bfa", "T_bfa", "vel_bfa", "p_bfa", "h_bfa",
                "mul_fa", "lamOcp_fa", "local_dt", "grad_u", "grad_rho", "grad_p", "grad_enthalpy",
                "rhs_rho", "rhs_rhou", "rhs_rhoE", "A", "rhs_sys", "dq", "line_off", "line_cv"]
        out = {k: d[k] for k in keep if k in d}
        out["final_rho"], out["final_rhou"], out["final_rhoE"] = r["final_rho"], r["final_rhou"], r["final_rhoE"]
        out["resid"] = r["resid"]
        out["meta"] = np.array(json.dumps(d["meta"]))
        out["params"] = np.array(params_json(prm))
        out["nsteps"] = np.array(NSTEPS)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print("wrote", name, d["meta"]["ncv"], "cells")
    turb = [(n, r, p, 1) for n, r, p in (sa_cases() if "sa" in which else ())]
    turb += [(n, r, p, 2) for n, r, p in (sst_cases() if "sst" in which else ())]
    for name, raw, prm, run_kind in turb:
        if only not in name:
            continue
        extra = "HARNESS_PERTURB = %g" % PERTURB
        d = refrun.run(lambda p: meshgen.write_msh(p, raw), prm.joe_in("mesh.msh", extra), "coupled",
                       run_kind=run_kind)
        keep = ["cvofa", "faocv_i", "faocv_v", "nbocv_i", "nbocv_v", "x_cv", "x_fa", "fa_normal", "cv_volume",
                "nbocv_lsg_coeff", "boundary_fa_lsg_coeff", "init_rho", "init_rhou", "init_rhoE", "init_scal0",
                "init_scal1", "mul_fa", "lamOcp_fa", "mut_fa", "scal0_bfa", "scal1_bfa", "wallDist", "strMag",
                "vortMag", "diverg", "crossDiff", "blendFuncF1", "blendFuncF2", "local_dt", "grad_u",
                "scal0_grad", "scal0_diff", "scal1_grad", "scal1_diff", "rhs_coupled", "A_coupled"]
        out = {k: d[k] for k in keep if k in d}
        out["meta"] = np.array(json.dumps(d["meta"]))
        out["params"] = np.array(params_json(prm))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print("wrote", name, d["meta"]["ncv"], "cells")


def load(path):
    z = np.load(path)
    d = {k: z[k] for k in z.files}
    d["meta"] = json.loads(str(d["meta"]))
    d["meta"]["zones"] = [tuple(zz) for zz in d["meta"]["zones"]]
    d["params"] = params_from_json(str(d["params"]))
    return d


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--only=")]
    only = [a[len("--only="):] for a in sys.argv[1:] if a.startswith("--only=")]
    main(tuple(args) or ("segregated", "sa", "sst"), only[0] if only else "")
