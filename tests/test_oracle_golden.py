"""Pins the C oracle (oracle/joe_oracle.c) against golden fixtures produced
by the reference solver itself (tests/golden/make_golden.py).  The oracle is
a bit-exact restatement: every array must match exactly, except the L1
residual history, which the reference prints with 5 significant digits."""
import glob
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from myjoe_b200.case import SOLVER_KINDS
from tests.golden.make_golden import load

GOLDEN = sorted(p for p in glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz"))
                if not os.path.basename(p).startswith(("converged_", "sa_", "sst_", "restart_")))


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def golden(request):
    return load(request.param)


def _oracle(g):
    d = dict(g)
    o = Oracle(d, g["params"])
    o.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    o.calc_state()
    return o


def test_state_and_boundary(golden):
    o = _oracle(golden)
    for k in ["press", "temp", "enthalpy", "sos", "rho_bfa", "T_bfa", "p_bfa", "h_bfa", "vel_bfa"]:
        np.testing.assert_array_equal(o.array(k).ravel(), golden[k].ravel(), err_msg=k)
    if golden["params"].MU_REF > 0:
        for k in ["mul_fa", "lamOcp_fa"]:
            np.testing.assert_array_equal(o.array(k).ravel(), golden[k].ravel(), err_msg=k)


def test_dt_gradients_rhs_matrix(golden):
    o = _oracle(golden)
    o.calc_dt()
    np.testing.assert_array_equal(o.array("local_dt"), golden["local_dt"])
    rr, ru, rE, A = o.calc_rhs(True)
    np.testing.assert_array_equal(rr, golden["rhs_rho"])
    np.testing.assert_array_equal(ru.ravel(), golden["rhs_rhou"].ravel())
    np.testing.assert_array_equal(rE, golden["rhs_rhoE"])
    np.testing.assert_array_equal(A.ravel(), golden["A"].ravel())
    np.testing.assert_array_equal(o.array("grad_u").ravel(), golden["grad_u"].ravel())
    if golden["params"].SECOND_ORDER:
        np.testing.assert_array_equal(o.array("grad_rho").ravel(), golden["grad_rho"].ravel())
        np.testing.assert_array_equal(o.array("grad_p").ravel(), golden["grad_p"].ravel())


def test_linear_solve(golden):
    o = _oracle(golden)
    o.calc_dt()
    _, _, _, A = o.calc_rhs(True)
    g = golden
    p = g["params"]
    vol_dt = g["cv_volume"] / g["local_dt"]
    nb_i = g["nbocv_i"]
    for i in range(5):
        A[nb_i[:-1], i, i] += vol_dt
    dq, _ = o.solve(A, g["rhs_sys"].reshape(-1, 5), p.LS_ABS_RESID, p.LS_REL_RESID, p.LS_MAX_ITER,
                    SOLVER_KINDS[p.LINEAR_SOLVER_NS])
    np.testing.assert_array_equal(dq.ravel(), g["dq"].ravel())


def test_backward_euler_steps(golden):
    o = _oracle(golden)
    res = np.array([o.step(1) for _ in range(int(golden["nsteps"]))])
    rho, rhou, rhoE = o.get_state()
    np.testing.assert_array_equal(rho, golden["final_rho"])
    np.testing.assert_array_equal(rhou.ravel(), golden["final_rhou"].ravel())
    np.testing.assert_array_equal(rhoE, golden["final_rhoE"])
    np.testing.assert_allclose(res, golden["resid"], rtol=6e-5, atol=0)


def test_linelets(golden):
    """initializeLinelet's lines (fixtures solved with BCGSTAB_LINELET)."""
    if "line_off" not in golden:
        pytest.skip("not a BCGSTAB_LINELET fixture")
    off, cv = _oracle(golden).linelets()
    np.testing.assert_array_equal(off, golden["line_off"])
    np.testing.assert_array_equal(cv, golden["line_cv"])
    assert (np.diff(off) >= 2).any()
