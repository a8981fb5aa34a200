"""LINE relaxation (JG_LS_LINE) on the GPU against the oracle's jo_line_relax.

Block line-Jacobi: the block-tridiagonal system of every line of the
reference's initializeLinelet solved exactly, block Jacobi on the other
cells.  Checked on the 5x5 path (one solve on the reference's own system,
backward-Euler steps) and on the coupled SA/SST paths (steps), FP64 against
the oracle at 1e-12 (one solve) / 1e-10 (steps) relative, and converged
fields of the FP64 and mixed forms at 1e-8 relative L2.
"""
import dataclasses
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)


def nrel(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    return float(np.abs(a - b).max() / np.abs(b).max())


def rel_l2(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _fixture(name):
    from tests.golden.make_golden import load
    return load(os.path.join(HERE, "golden", name + ".npz"))


@pytest.mark.parametrize("name", ["plate_roe_linelet", "mixed_bump_roe_laminar_linelet"])
def test_line_solve_matches_oracle(name):
    from myjoe_b200 import build, solver
    from oracle.oracle import Oracle
    build.build()
    g = _fixture(name)
    prm = dataclasses.replace(g["params"], LINEAR_SOLVER_NS="LINE")
    A = g["A"].copy()
    vol_dt = g["cv_volume"] / g["local_dt"]
    for i in range(5):
        A[g["nbocv_i"][:-1], i, i] += vol_dt
    rhs = g["rhs_sys"].reshape(-1, 5)
    o = Oracle(dict(g), prm)
    for sweeps in (1, 7):
        dq_o, _ = o.solve(A, rhs, 0, 0, sweeps, 5)
        j = solver.JoeGpu(dict(g), prm)
        dq_g, it = j.solveCoupledLinSysNS(A, rhs, 0, 0, sweeps)
        assert it == sweeps
        assert nrel(dq_g, dq_o) <= 1e-12


def test_line_steps_match_oracle_5x5():
    from myjoe_b200 import build, solver
    from oracle.oracle import Oracle
    build.build()
    g = _fixture("plate_roe_linelet")
    prm = dataclasses.replace(g["params"], LINEAR_SOLVER_NS="LINE", LS_MAX_ITER=6, CFL=5.0)
    o = Oracle(dict(g), prm)
    o.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    o.calc_state()
    j = solver.JoeGpu(dict(g), prm)
    j.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    ro = np.array([o.step(1) for _ in range(10)])
    rg = j.runBackwardEuler(10)
    assert nrel(rg, ro) <= 1e-10
    for a, b in zip(j.get_state(), o.get_state()):
        assert nrel(a, b) <= 1e-10


@pytest.mark.parametrize("name", ["sa_bump_farfield", "sst_mixed_bump_farfield"])
def test_line_steps_match_oracle_coupled(name):
    from myjoe_b200 import build, solver
    from oracle.oracle import OracleSA
    build.build()
    g = _fixture(name)
    prm = dataclasses.replace(g["params"], LINEAR_SOLVER_NS="LINE", LS_MAX_ITER=6, CFL=5.0)
    phi = np.stack([g["init_scal%d" % s] for s in range(prm.nscal)], 1)
    o = OracleSA(dict(g), prm)
    o.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    o.set_scalar(phi)
    o.calc_state()
    j = solver.JoeGpu(dict(g), prm)
    j.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    j.set_scalars(phi)
    ro = o.step(4)
    rg = j.runBackwardEuler(4)
    assert nrel(rg[-1], ro) <= 1e-10
    for a, b in zip(j.get_state(), o.get_state()):
        assert nrel(a, b) <= 1e-10
    assert nrel(j.get_scalars(), o.get_scalar()) <= 1e-10


@pytest.mark.parametrize("precision", [0, 1])
def test_line_converged_sa_field_matches_oracle(precision):
    from myjoe_b200 import build, case, solver
    from oracle.oracle import OracleSA
    build.build()
    raw, g, prm = case.sa_bump_case(24, 16, 2, stretch=1.25, seed=1, mach=0.5, re=1.0e5, n_prism=4,
                                    alternate=True, shuffle=True)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="LINE", LS_MAX_ITER=6, CFL=1.0, CFL_RAMP=(10, 5, 1.2, 50.0))
    st = case.perturbed_state(g.x_cv, prm, 0.0)
    phi0 = np.full(g.ncv, prm.NUSA_INITIAL)
    o = OracleSA(g, prm)
    o.set_state(*st)
    o.set_scalar(phi0)
    o.calc_state()
    ro = o.step(1500)
    j = solver.JoeGpu(g, prm, precision=precision, renumber=True)
    j.set_state(*st)
    j.set_scalars(phi0)
    rg = j.runBackwardEuler(1500)
    assert rg[-1, 4] / rg[0, 4] < 1e-9 and ro[4] / rg[0, 4] < 1e-9
    for a, b in zip(j.get_state(), o.get_state()):
        assert rel_l2(a, b) <= 1e-8
    assert rel_l2(j.get_scalars(), o.get_scalar()) <= 1e-8
