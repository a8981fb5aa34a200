"""The handle's own renumbering (jg_params.renumber = JG_RENUMBER_RCM) on
shuffled mixed prism/hex meshes.

Renumbering keeps every per-cell list in the caller's order and only changes
ids, so each per-cell and per-face operation is the same arithmetic on the
same operands: calcRhs (residual and Jacobian), gradients, boundary states,
time steps, the coupled SA/SST assembly and block-Jacobi steps must come back
bit for bit equal to the handle that keeps the caller's order, in the
caller's order.  The L1 residual sums run in the internal order (1e-13
relative), BiCGSTAB's dot products too (1e-10), and multicolour Gauss-Seidel
colours in the internal order, so its converged field is compared at the
1e-8 bar of the converged-field tests.
"""
import dataclasses
import glob
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)


def _pair(g, prm, precision=0):
    from myjoe_b200 import build, solver
    build.build()
    return (solver.JoeGpu(g, prm, precision=precision, renumber=False),
            solver.JoeGpu(g, prm, precision=precision, renumber=True))


def _euler_mixed(shuffle=True, visc=False):
    from myjoe_b200 import case, geometry, meshgen
    raw = meshgen.channel_bump_mixed(40, 20, 3, n_prism=5, stretch=1.15, jitter=0.1, seed=11)
    g = geometry.build_cv_mesh(raw, seed=12, shuffle=shuffle)
    _, _, prm = case.bump_case(8, 4, 2)
    if visc:
        prm = dataclasses.replace(prm, MU_MODE="SUTHERLAND", MU_REF=1.716e-5 * 2000.0, SPACE_INTEGRATION="ROE")
    return g, dataclasses.replace(prm, LINEAR_SOLVER_NS="JACOBI", LS_MAX_ITER=6, CFL=5.0)


@pytest.mark.parametrize("visc", [False, True], ids=["euler_hllc", "laminar_roe"])
def test_renumbered_operators_are_bitwise_equal(visc):
    from myjoe_b200 import case
    g, prm = _euler_mixed(visc=visc)
    a, b = _pair(g, prm)
    st = case.perturbed_state(g.x_cv, prm, 0.05)
    for j in (a, b):
        j.set_state(*st)
    for x, y in zip(a.calcRhs(True), b.calcRhs(True)):
        np.testing.assert_array_equal(x, y)
    for k, v in a.gradients().items():
        np.testing.assert_array_equal(v, b.gradients()[k], err_msg=k)
    for k, v in a.primitives().items():
        np.testing.assert_array_equal(v, b.primitives()[k], err_msg=k)
    for k, v in a.boundary().items():
        np.testing.assert_array_equal(v, b.boundary()[k], err_msg=k)
    da, db = a.calcDt(), b.calcDt()
    assert da[0] == db[0]
    np.testing.assert_array_equal(da[1], db[1])


def test_renumbered_jacobi_steps_are_bitwise_equal():
    from myjoe_b200 import case
    g, prm = _euler_mixed()
    a, b = _pair(g, prm)
    st = case.perturbed_state(g.x_cv, prm, 0.02)
    for j in (a, b):
        j.set_state(*st)
    ra, rb = a.runBackwardEuler(25), b.runBackwardEuler(25)
    np.testing.assert_allclose(rb, ra, rtol=1e-13, atol=0.0)
    for x, y in zip(a.get_state(), b.get_state()):
        np.testing.assert_array_equal(x, y)


def test_renumbered_linear_solve():
    from myjoe_b200 import case
    g, prm = _euler_mixed()
    for solver_name, tol in (("JACOBI", 0.0), ("BCGSTAB", 1e-10)):
        p = dataclasses.replace(prm, LINEAR_SOLVER_NS=solver_name, LS_MAX_ITER=8)
        a, b = _pair(g, p)
        st = case.perturbed_state(g.x_cv, p, 0.05)
        for j in (a, b):
            j.set_state(*st)
        rr, ru, rE, A = a.calcRhs(True)
        rhs = np.concatenate([rr[:, None], ru, rE[:, None]], 1)
        A = A.copy()
        A[g.nbocv_i[:-1]] += np.eye(5) * (g.cv_volume / 1e-6)[:, None, None]
        xa, _ = a.solveCoupledLinSysNS(A, rhs, 1e-14, 1e-12, 8)
        xb, _ = b.solveCoupledLinSysNS(A, rhs, 1e-14, 1e-12, 8)
        if tol == 0.0:
            np.testing.assert_array_equal(xa, xb)
        else:
            assert np.abs(xa - xb).max() <= tol * np.abs(xa).max()


@pytest.mark.parametrize("model", ["sa", "sst"])
def test_renumbered_coupled_path_is_bitwise_equal(model):
    from myjoe_b200 import case
    make = case.sa_bump_case if model == "sa" else case.sst_bump_case
    _, g, prm = make(32, 16, 2, stretch=1.2, jitter=0.1, seed=7, n_prism=4, shuffle=True, mach=0.5, re=1e5)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="JACOBI", LS_MAX_ITER=6, CFL=2.0)
    a, b = _pair(g, prm)
    st = case.perturbed_state(g.x_cv, prm, 0.03)
    values = [prm.NUSA_INITIAL] if model == "sa" else [prm.KINE_INITIAL, prm.OMEGA_INITIAL]
    phi0 = np.stack([case.perturbed_scalar(g.x_cv, v, 0.1) for v in values], 1)
    for j in (a, b):
        j.set_state(*st)
        j.set_scalars(phi0)
    for k in ("wallDist", "strMag", "vortMag", "mut_fa", "phi_bfa", "grad_phi", "diff"):
        np.testing.assert_array_equal(a.turb_array(k), b.turb_array(k), err_msg=k)
    for x, y in zip(a.calcRhsCoupled(True), b.calcRhsCoupled(True)):
        np.testing.assert_array_equal(x, y)
    a.runBackwardEuler(10)
    b.runBackwardEuler(10)
    for x, y in zip(a.get_state(), b.get_state()):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a.get_scalars(), b.get_scalars())


def test_renumbered_golden_mixed_mesh_matches_reference():
    """The reference's own residual and Jacobian on a mixed prism/hex mesh,
    through a renumbering handle."""
    from myjoe_b200 import build, solver
    from tests.golden.make_golden import load
    build.build()
    for path in sorted(glob.glob(os.path.join(HERE, "golden", "mixed_*.npz"))):
        gd = load(path)
        prm = gd["params"]
        j = solver.JoeGpu(dict(gd), prm, renumber=True)
        j.set_state(gd["init_rho"], gd["init_rhou"].reshape(-1, 3), gd["init_rhoE"])
        j.calcDt(prm.CFL)
        rr, ru, rE, A = j.calcRhs(True)
        for x, ref in ((rr, gd["rhs_rho"]), (ru.ravel(), gd["rhs_rhou"].ravel()), (rE, gd["rhs_rhoE"])):
            assert np.abs(x - ref).max() <= 1e-12 * np.abs(ref).max()
        ref_A = gd["A"].reshape(A.shape)
        assert np.abs(A - ref_A).max() <= 1e-12 * np.abs(ref_A).max()


def test_renumbered_sgs_converges_to_the_same_field():
    from myjoe_b200 import case
    g, prm = _euler_mixed()
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=6, CFL=2.0, CFL_RAMP=(10, 5, 1.2, 20.0))
    a, b = _pair(g, prm)
    st = case.perturbed_state(g.x_cv, prm, 0.0)
    for j in (a, b):
        j.set_state(*st)
    ra, rb = a.runBackwardEuler(3200), b.runBackwardEuler(3200)
    assert ra[-1, 4] / ra[0, 4] < 1e-9 and rb[-1, 4] / rb[0, 4] < 1e-9
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.linalg.norm(x - y) <= 1e-8 * np.linalg.norm(x)


def test_color_grouped_order_gives_the_rcm_sgs_bits():
    """JG_RENUMBER_RCM_COLOR keeps the RCM order's colour classes, so multicolour
    Gauss-Seidel steps give the RCM handle's states bit for bit (only the L1
    residual sums run in another order); each colour pass now launches over the
    slices of that colour only."""
    from myjoe_b200 import case, solver
    g, prm = _euler_mixed()
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=6, CFL=2.0, CFL_RAMP=(10, 5, 1.2, 20.0))
    for precision in (0, 1):
        a = solver.JoeGpu(g, prm, precision=precision, renumber=solver.RENUMBER_RCM)
        b = solver.JoeGpu(g, prm, precision=precision, renumber=solver.RENUMBER_RCM_COLOR)
        st = case.perturbed_state(g.x_cv, prm, 0.02)
        for j in (a, b):
            j.set_state(*st)
        ra, rb = a.runBackwardEuler(30), b.runBackwardEuler(30)
        np.testing.assert_allclose(rb, ra, rtol=1e-13, atol=0.0)
        for x, y in zip(a.get_state(), b.get_state()):
            np.testing.assert_array_equal(x, y)
        a.close()
        b.close()


@pytest.mark.parametrize("turb", ["NONE", "SA"])
def test_line_grouped_order_gives_the_rcm_line_relaxation_bits(turb):
    """JG_RENUMBER_RCM_LINES makes each LINE relaxation line consecutive; the lines and
    every per-cell operation are those of the RCM handle, so LINE steps (5x5 laminar and
    6x6 coupled SA, FP64 and mixed) give its states bit for bit."""
    from myjoe_b200 import case, solver
    _, g, prm = case.sa_bump_case(48, 40, 2, stretch=1.1, n_prism=8, bump_h=0.05, alternate=True,
                                  shuffle=True, seed=3)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="LINE", LS_MAX_ITER=5, CFL=5.0, CFL_RAMP=(5, 5, 1.2, 50.0))
    if turb == "NONE":
        prm = dataclasses.replace(prm, TURB_MODEL="NONE", scalar_bcs={})
    st = case.perturbed_state(g.x_cv, prm, 0.0)
    for precision in (0, 1):
        hs = [solver.JoeGpu(g, prm, precision=precision, renumber=m)
              for m in (solver.RENUMBER_RCM, solver.RENUMBER_RCM_LINES)]
        for j in hs:
            j.set_state(*st)
            if turb == "SA":
                j.set_scalars(np.full(g.ncv, prm.NUSA_INITIAL))
        ra, rb = (j.runBackwardEuler(12) for j in hs)
        np.testing.assert_allclose(rb, ra, rtol=1e-13, atol=0.0)
        for x, y in zip(hs[0].get_state(), hs[1].get_state()):
            np.testing.assert_array_equal(x, y)
        for j in hs:
            j.close()
