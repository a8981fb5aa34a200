"""Pins the oracle's coupled Spalart-Allmaras path (oracle/joe_oracle.c,
jo_calc_rhs_coupled and its helpers) against golden fixtures produced by the
reference solver's own calcRhsCoupled with RansTurbSA (tests/golden/
make_golden.py, ``sa`` cases).  Every array must match bit for bit: wall
distance, strain and vorticity magnitudes, turbulent viscosity, scalar
boundary values, time step, gradients, scalar diffusivity, the 6-component
residual and the 6x6 block Jacobian."""
import glob
import os

import numpy as np
import pytest

from oracle.oracle import OracleSA
from tests.golden.make_golden import load

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "sa_*.npz")))


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def golden(request):
    return load(request.param)


def _oracle(g):
    o = OracleSA(dict(g), g["params"])
    o.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    o.set_scalar(g["init_scal0"])
    o.calc_state()
    return o


def test_turbulence_arrays(golden):
    o = _oracle(golden)
    for k, ref in (("wallDist", "wallDist"), ("strMag", "strMag"), ("vortMag", "vortMag"), ("phi_bfa", "scal0_bfa")):
        np.testing.assert_array_equal(o.sa_array(k), golden[ref], err_msg=k)
    for k in ("mut_fa", "mul_fa", "lamOcp_fa"):
        np.testing.assert_array_equal(o.array(k), golden[k], err_msg=k)


def test_coupled_rhs_and_matrix(golden):
    o = _oracle(golden)
    o.calc_dt(golden["params"].CFL)
    np.testing.assert_array_equal(o.array("local_dt"), golden["local_dt"])
    rhs, A = o.calc_rhs(True)
    np.testing.assert_array_equal(o.array("grad_u").ravel(), golden["grad_u"].ravel())
    np.testing.assert_array_equal(o.sa_array("grad_phi").ravel(), golden["scal0_grad"].ravel())
    if golden["params"].MU_REF > 0.0:
        np.testing.assert_array_equal(o.sa_array("diff"), golden["scal0_diff"])
    np.testing.assert_array_equal(rhs.ravel(), golden["rhs_coupled"])
    np.testing.assert_array_equal(A.ravel(), golden["A_coupled"])
    assert np.abs(A[:, 5, :]).max() > 0.0 and np.abs(rhs[:, 5]).max() > 0.0   # the scalar row is populated


def test_coupled_step_is_finite_and_clipped():
    g = load(GOLDEN[0])
    o = _oracle(g)
    r = o.step(3)
    assert np.all(np.isfinite(r))
    phi = o.get_scalar()
    assert phi.min() >= 1.0e-10 and phi.max() <= 1.0
