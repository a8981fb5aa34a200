"""GPU parity of the coupled turbulence-model path: Spalart-Allmaras (6x6
blocks) and Menter SST (7x7 blocks).

Against the reference's own calcRhsCoupled (golden fixtures made by the
reference solver, tests/golden/make_golden.py ``sa``/``sst``): wall
distance, strain/vorticity magnitudes (SST: divergence, cross-diffusion,
blending functions), turbulent viscosity, scalar boundary values (SST's omega
wall hook included), gradients and diffusivities of the scalars, the residual
and the block Jacobian.  Against the oracle (pinned bit-exact to the same
fixtures): backward-Euler steps and converged fields, FP64 and mixed
precision.

Tolerances: model arrays and residual components 1e-11 normwise (max error /
max magnitude of the array; the GPU's pow/tanh may differ from glibc's by an
ulp); Jacobian 1e-11 normwise per block entry; steps 1e-10 normwise;
converged fields 1e-8 relative L2 in both precisions (FP64 and mixed).
"""
import dataclasses
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)
GOLDEN = sorted(glob.glob(os.path.join(HERE, "golden", "sa_*.npz")) + glob.glob(os.path.join(HERE, "golden", "sst_*.npz")))


def nrel(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def rel_l2(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def golden(request):
    from tests.golden.make_golden import load
    return load(request.param)


def _scalars(g):
    return np.stack([g["init_scal%d" % s] for s in range(g["params"].nscal)], 1)


def _gpu(g, precision=0, lin="SGS", **kw):
    from myjoe_b200 import build, solver
    build.build()
    prm = dataclasses.replace(g["params"], LINEAR_SOLVER_NS=lin, LS_MAX_ITER=10, **kw)
    j = solver.JoeGpu(dict(g), prm, precision=precision)
    j.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    j.set_scalars(_scalars(g))
    return j, prm


def test_model_arrays_match_reference(golden):
    j, prm = _gpu(golden)
    ns = prm.nscal
    assert nrel(j.turb_array("wallDist"), golden["wallDist"]) <= 1e-13
    names = ["strMag", "vortMag"] + (["diverg", "crossDiff", "blendFuncF1", "blendFuncF2"] if ns == 2 else [])
    for k in names:
        assert nrel(j.turb_array(k), golden[k]) <= 1e-11, k
    assert nrel(j.turb_array("mut_fa"), golden["mut_fa"]) <= 1e-11
    pb, gp, df = j.turb_array("phi_bfa"), j.turb_array("grad_phi"), j.turb_array("diff")
    for s in range(ns):
        assert nrel(pb[s], golden["scal%d_bfa" % s]) <= 1e-12, s
        assert nrel(gp[s], golden["scal%d_grad" % s].reshape(-1, 3)) <= 1e-11, s
        assert nrel(df[s], golden["scal%d_diff" % s]) <= 1e-11, s


def test_rhs_and_matrix_match_reference(golden):
    j, prm = _gpu(golden)
    B = 5 + prm.nscal
    rhs, A = j.calcRhsCoupled(True)
    ref_r = golden["rhs_coupled"].reshape(-1, B)
    ref_A = golden["A_coupled"].reshape(-1, B, B)
    for i in range(B):
        assert nrel(rhs[:, i], ref_r[:, i]) <= 1e-11, i
    for r in range(B):
        for c in range(B):
            if np.abs(ref_A[:, r, c]).max() == 0.0:
                assert np.abs(A[:, r, c]).max() == 0.0, (r, c)
            else:
                assert nrel(A[:, r, c], ref_A[:, r, c]) <= 1e-11, (r, c)


# HLLC on both models; the coupled AUSMDV (sonic, both fixes) and HAENEL
STEP_CASES = ["sa_bump_cbc_symm_original", "sst_bump_cbc_symm_original", "sa_bump_ausmdv_m1",
              "sst_bump_haenel_neumann_first_order"]


@pytest.mark.parametrize("name", STEP_CASES)
@pytest.mark.parametrize("lin", ["SGS", "JACOBI"])
def test_steps_match_oracle(name, lin):
    from oracle.oracle import OracleSA
    from tests.golden.make_golden import load
    g = load(os.path.join(HERE, "golden", name + ".npz"))
    j, prm = _gpu(g, lin=lin, CFL=5.0)
    o = OracleSA(dict(g), prm)
    o.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    o.set_scalar(_scalars(g))
    o.calc_state()
    rg = j.runBackwardEuler(3)
    ro = o.step(3)
    assert rg.shape == (3, 5 + prm.nscal)
    assert nrel(rg[-1], ro) <= 1e-10
    for a, b in zip(j.get_state(), o.get_state()):
        assert nrel(a, b) <= 1e-10
    sg, so = np.asarray(j.get_scalars()).reshape(j.ncv, -1), np.asarray(o.get_scalar()).reshape(j.ncv, -1)
    for s in range(prm.nscal):
        assert nrel(sg[:, s], so[:, s]) <= 1e-10, s


@pytest.mark.parametrize("model", ["sa", "sst"])
@pytest.mark.parametrize("precision", [0, 1])
def test_converged_fields_match_oracle(model, precision):
    from myjoe_b200 import build, case, solver
    from oracle.oracle import OracleSA
    build.build()
    make = case.sa_bump_case if model == "sa" else case.sst_bump_case
    raw, g, prm = make(24, 12, 2, stretch=1.15, seed=1, mach=0.5, re=1.0e5)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=10, CFL=1.0, CFL_RAMP=(10, 5, 1.2, 20.0))
    st = case.perturbed_state(g.x_cv, prm, 0.0)
    phi0 = (np.full((g.ncv, 1), prm.NUSA_INITIAL) if model == "sa"
            else np.tile([prm.KINE_INITIAL, prm.OMEGA_INITIAL], (g.ncv, 1)))
    o = OracleSA(g, prm)
    o.set_state(*st)
    o.set_scalar(phi0)
    o.calc_state()
    ro = o.step(1200)
    j = solver.JoeGpu(g, prm, precision=precision)
    j.set_state(*st)
    j.set_scalars(phi0)
    rg = j.runBackwardEuler(1200)
    assert rg[-1, 4] / rg[0, 4] < 1e-9 and ro[4] / rg[0, 4] < 1e-9   # both converged
    for a, b in zip(j.get_state(), o.get_state()):
        assert rel_l2(a, b) <= 1e-8
    sg, so = np.asarray(j.get_scalars()).reshape(g.ncv, -1), np.asarray(o.get_scalar()).reshape(g.ncv, -1)
    for s in range(prm.nscal):
        assert rel_l2(sg[:, s], so[:, s]) <= 1e-8, s
