"""GPU parity of the coupled Spalart-Allmaras path (6x6 blocks).

Against the reference's own calcRhsCoupled (golden fixtures made by the
reference solver, tests/golden/make_golden.py ``sa``): wall distance,
strain/vorticity magnitudes, turbulent viscosity, scalar boundary values,
gradient and diffusivity of nuSA, the 6-component residual and the 6x6 block
Jacobian.  Against the oracle (pinned bit-exact to the same fixtures):
backward-Euler steps and converged fields, FP64 and mixed precision.

Tolerances: model arrays and residual components 1e-11 normwise (max error /
max magnitude of the array; the GPU's pow() may differ from glibc's by an
ulp); Jacobian 1e-11 normwise per block entry; steps 1e-10 normwise;
converged fields 1e-8 relative L2, the north-star bar for both precisions.
"""
import dataclasses
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "sa_*.npz")))


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


def _gpu(g, precision=0, lin="SGS"):
    from myjoe_b200 import build, solver
    build.build()
    prm = dataclasses.replace(g["params"], LINEAR_SOLVER_NS=lin, LS_MAX_ITER=10)
    j = solver.JoeGpu(dict(g), prm, precision=precision)
    j.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    j.set_scalars(g["init_scal0"])
    return j


def test_sa_model_arrays_match_reference(golden):
    j = _gpu(golden)
    t = j.turb()
    assert nrel(t["wallDist"], golden["wallDist"]) <= 1e-13
    assert nrel(t["strMag"], golden["strMag"]) <= 1e-11
    assert nrel(t["vortMag"], golden["vortMag"]) <= 1e-11
    assert nrel(t["mut_fa"], golden["mut_fa"]) <= 1e-11
    assert np.array_equal(t["phi_bfa"], golden["scal0_bfa"])
    assert nrel(t["grad_phi"], golden["scal0_grad"]) <= 1e-11
    assert nrel(t["diff"], golden["scal0_diff"]) <= 1e-11


def test_sa_rhs_and_matrix_match_reference(golden):
    j = _gpu(golden)
    rhs, A = j.calcRhsCoupled(True)
    ref_r = golden["rhs_coupled"].reshape(-1, 6)
    ref_A = golden["A_coupled"].reshape(-1, 6, 6)
    for i in range(6):
        assert nrel(rhs[:, i], ref_r[:, i]) <= 1e-11, i
    for r in range(6):
        for c in range(6):
            if np.abs(ref_A[:, r, c]).max() == 0.0:
                assert np.abs(A[:, r, c]).max() == 0.0
            else:
                assert nrel(A[:, r, c], ref_A[:, r, c]) <= 1e-11, (r, c)


@pytest.mark.parametrize("lin", ["SGS", "JACOBI"])
def test_sa_steps_match_oracle(lin):
    from myjoe_b200 import build, solver
    from oracle.oracle import OracleSA
    from tests.golden.make_golden import load
    build.build()
    g = load(GOLDEN[0])
    prm = dataclasses.replace(g["params"], LINEAR_SOLVER_NS=lin, LS_MAX_ITER=10, CFL=5.0)
    o = OracleSA(dict(g), prm)
    o.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    o.set_scalar(g["init_scal0"])
    o.calc_state()
    j2 = solver.JoeGpu(dict(g), prm)
    j2.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    j2.set_scalars(g["init_scal0"])
    rg = j2.runBackwardEuler(3)
    ro = o.step(3)
    assert rg.shape == (3, 6)
    assert nrel(rg[-1], ro) <= 1e-10
    for a, b in zip(j2.get_state(), o.get_state()):
        assert nrel(a, b) <= 1e-10
    assert nrel(j2.get_scalars(), o.get_scalar()) <= 1e-10


@pytest.mark.parametrize("precision", [0, 1])
def test_sa_converged_fields_match_oracle(precision):
    from myjoe_b200 import build, case, solver
    from oracle.oracle import OracleSA
    build.build()
    raw, g, prm = case.sa_bump_case(24, 12, 2, stretch=1.15, seed=1, mach=0.5, re=1.0e5)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=10, CFL=1.0, CFL_RAMP=(10, 5, 1.2, 20.0))
    st = case.perturbed_state(g.x_cv, prm, 0.0)
    nu0 = np.full(g.ncv, prm.NUSA_INITIAL)
    o = OracleSA(g, prm)
    o.set_state(*st)
    o.set_scalar(nu0)
    o.calc_state()
    ro = o.step(1200)
    j = solver.JoeGpu(g, prm, precision=precision)
    j.set_state(*st)
    j.set_scalars(nu0)
    rg = j.runBackwardEuler(1200)
    assert rg[-1, 4] / rg[0, 4] < 1e-9 and ro[4] / rg[0, 4] < 1e-9   # both converged
    for a, b in zip(j.get_state(), o.get_state()):
        assert rel_l2(a, b) <= 1e-8
    assert rel_l2(j.get_scalars(), o.get_scalar()) <= 1e-8
