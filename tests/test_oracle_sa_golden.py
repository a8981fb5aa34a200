"""Pins the oracle's coupled turbulence-model path (oracle/joe_oracle.c,
jo_calc_rhs_coupled and its helpers) against golden fixtures produced by the
reference solver's own calcRhsCoupled with RansTurbSA (``sa_*``, 6x6 blocks)
and RansTurbKOmSST (``sst_*``, 7x7 blocks) (tests/golden/make_golden.py).
Every array must match bit for bit: wall distance, strain/vorticity (and for
SST divergence, cross-diffusion, blending functions F1/F2), turbulent
viscosity, scalar boundary values (including SST's omega wall hook), time
step, gradients and diffusivities of the scalars, the residual and the block
Jacobian."""
import glob
import os

import numpy as np
import pytest

from oracle.oracle import OracleSA
from tests.golden.make_golden import load

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "sa_*.npz")) +
                glob.glob(os.path.join(os.path.dirname(__file__), "golden", "sst_*.npz")))


@pytest.fixture(params=GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def golden(request):
    return load(request.param)


def _scalars(g):
    ns = g["params"].nscal
    return np.stack([g["init_scal%d" % s] for s in range(ns)], 1)


def _oracle(g):
    o = OracleSA(dict(g), g["params"])
    o.set_state(g["init_rho"], g["init_rhou"].reshape(-1, 3), g["init_rhoE"])
    o.set_scalar(_scalars(g))
    o.calc_state()
    return o


def test_turbulence_arrays(golden):
    o = _oracle(golden)
    names = ["wallDist", "strMag", "vortMag"]
    if golden["params"].TURB_MODEL == "SST":
        names += ["diverg", "crossDiff", "blendFuncF1", "blendFuncF2"]
    for k in names:
        np.testing.assert_array_equal(o.sa_array(k), golden[k], err_msg=k)
    for s in range(golden["params"].nscal):
        np.testing.assert_array_equal(o.sa_array("phi_bfa" if s == 0 else "phi1_bfa"), golden["scal%d_bfa" % s])
    for k in ("mut_fa", "mul_fa", "lamOcp_fa"):
        np.testing.assert_array_equal(o.array(k), golden[k], err_msg=k)


def test_coupled_rhs_and_matrix(golden):
    o = _oracle(golden)
    B = 5 + golden["params"].nscal
    o.calc_dt(golden["params"].CFL)
    np.testing.assert_array_equal(o.array("local_dt"), golden["local_dt"])
    rhs, A = o.calc_rhs(True)
    np.testing.assert_array_equal(o.array("grad_u").ravel(), golden["grad_u"].ravel())
    for s in range(golden["params"].nscal):
        sfx = "" if s == 0 else "1"
        np.testing.assert_array_equal(o.sa_array("grad_phi" + sfx).ravel(), golden["scal%d_grad" % s].ravel())
        if golden["params"].MU_REF > 0.0:
            np.testing.assert_array_equal(o.sa_array("diff" + sfx), golden["scal%d_diff" % s])
    np.testing.assert_array_equal(rhs.ravel(), golden["rhs_coupled"])
    np.testing.assert_array_equal(A.ravel(), golden["A_coupled"])
    assert A.shape[1:] == (B, B)
    for s in range(5, B):   # the scalar rows are populated
        assert np.abs(A[:, s, :]).max() > 0.0 and np.abs(rhs[:, s]).max() > 0.0


@pytest.mark.parametrize("model", ["sa", "sst"])
def test_coupled_step_is_finite_and_clipped(model):
    g = load(os.path.join(os.path.dirname(__file__), "golden", model + "_bump_cbc_symm_original.npz"))
    o = _oracle(g)
    r = o.step(3)
    assert np.all(np.isfinite(r)) and r.shape == (5 + g["params"].nscal,)
    phi = np.asarray(o.get_scalar()).reshape(o.ncv, -1)
    lo = [1.0e-10] if model == "sa" else [1.0e-10, 1.0e-4]
    hi = [1.0] if model == "sa" else [1.0e10, 1.0e15]
    for s in range(phi.shape[1]):
        assert phi[:, s].min() >= lo[s] and phi[:, s].max() <= hi[s]
