"""The driver-level entry points: jg_run_to (runBackwardEuler until the
energy-residual drop, as doneSolver stops it), jg_set_params (run-time
settings of a live handle), jg_calc_grad (the gradient pass on its own) and
jg_step_host (a host-resident state stepped in place).
Each is checked against the plain calls it must agree with, bit for bit."""
import dataclasses

import numpy as np
import pytest

from myjoe_b200 import case, solver

pytestmark = pytest.mark.gpu


def _bump(**kw):
    _, g, prm = case.bump_case(24, 12, 2, jitter=0.1, seed=4)
    return g, dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=10, CFL=1.0,
                                  CFL_RAMP=(10, 5, 1.2, 20.0), **kw)


def _fresh(g, prm):
    j = solver.JoeGpu(g, prm)
    j.set_state(*case.perturbed_state(g.x_cv, prm, 0.0))
    return j


@pytest.mark.parametrize("check_every", [1, 25])
def test_run_to_stops_where_the_drop_is_met(check_every):
    g, prm = _bump()
    a = _fresh(g, prm)
    n, d = a.run_to(1e-6, 4000, check_every)
    b = _fresh(g, prm)
    r = b.runBackwardEuler(n)
    drops = r[:, 4] / r[0, 4]
    assert d == drops[-1]
    first = int(np.nonzero(drops <= 1e-6)[0][0]) + 1
    if check_every == 1:
        assert n == first
    else:
        assert first <= n < first + check_every and n % check_every == 0
    for x, y in zip(a.get_state(), b.get_state()):
        np.testing.assert_array_equal(x, y)
    a.close()
    b.close()


def test_run_to_absolute_threshold_is_strict():
    """resid_drop < 0: the reference's doneSolver rule, the absolute energy
    residual strictly below the threshold (RESID_ENERG_TH)."""
    g, prm = _bump()
    b = _fresh(g, prm)
    r = b.runBackwardEuler(400)
    th = float(r[250, 4])           # a residual the run reaches exactly
    first = int(np.nonzero(r[:, 4] < th)[0][0]) + 1
    a = _fresh(g, prm)
    n, _ = a.run_to(-th, 400, 1)
    assert n == first and n != 251   # step 251's residual equals the threshold: not below it
    b.close()
    a.close()


def test_run_to_max_steps():
    g, prm = _bump()
    j = _fresh(g, prm)
    n, d = j.run_to(0.0, 30, 7)
    assert n == 30 and 0.0 < d
    assert j.cfl_step()[1] == 30
    j.close()


def test_set_params_equals_a_handle_made_with_them():
    g, prm = _bump()
    new = dataclasses.replace(prm, CFL=2.0, CFL_RAMP=(5, 3, 1.3, 40.0), UNDER_RELAXATION=0.5, LS_MAX_ITER=6,
                              EPS=0.02)
    a = _fresh(g, prm)
    a.runBackwardEuler(3)   # a captured step with the old settings, then the new ones
    a.set_params(new)
    a.set_cfl_step(new.CFL, 0)
    a.set_state(*case.perturbed_state(g.x_cv, prm, 0.0))
    ra = a.runBackwardEuler(20)
    b = _fresh(g, new)
    rb = b.runBackwardEuler(20)
    np.testing.assert_array_equal(ra, rb)
    for x, y in zip(a.get_state(), b.get_state()):
        np.testing.assert_array_equal(x, y)
    with pytest.raises(solver.JoeGpuError) as e:
        a.set_params(dataclasses.replace(new, SPACE_INTEGRATION="ROE"))
    assert e.value.code == -1
    a.close()
    b.close()


def test_calc_grad_equals_the_gradients_of_calc_rhs():
    g, prm = _bump()
    prm = dataclasses.replace(prm, MU_MODE="SUTHERLAND", MU_REF=1.716e-5 * 2000.0)
    j = solver.JoeGpu(g, prm)
    j.set_state(*case.perturbed_state(g.x_cv, prm, 0.05))
    got = j.calcGrad()
    j.calcDt()
    j.calcRhs()
    ref = j.gradients()
    for k in ("grad_u", "grad_rho", "grad_p", "grad_enthalpy"):
        np.testing.assert_array_equal(got[k], ref[k])
    j.close()


@pytest.mark.parametrize("renumber,pinned", [(0, False), (2, False), (0, True), (2, True)])
def test_step_host_is_set_step_get(renumber, pinned):
    """jg_step_host (a host-resident state stepped in place, one synchronisation) gives, bit for
    bit, what jg_set_state + jg_step + jg_get_state give, step after step, in the caller's order,
    from pageable and from page-locked arrays."""
    import torch
    g, prm = _bump()
    st = case.perturbed_state(g.x_cv, prm, 0.0)
    a = solver.JoeGpu(g, prm, renumber=renumber)
    b = solver.JoeGpu(g, prm, renumber=renumber)
    a.set_state(*st)
    b.set_state(*st)
    if pinned:
        rho, rhou, rhoE = (torch.empty(np.shape(x), dtype=torch.float64, pin_memory=True).numpy() for x in st)
        for x, y in zip((rho, rhou, rhoE), st):
            x[...] = y
    else:
        rho, rhou, rhoE = (np.array(x, dtype=np.float64, order="C") for x in st)
    ns = 1 if pinned else 3   # one step on page-locked arrays: the call's own captured graph
    ra = np.zeros((ns, 5))
    for k in range(4):
        a.step_host(rho, rhou, rhoE, ns, ra)
        b.set_state(*b.get_state())
        rb = b.runBackwardEuler(ns)
        np.testing.assert_array_equal(ra, rb)
        for x, y in zip((rho, rhou, rhoE), b.get_state()):
            np.testing.assert_array_equal(x, y)
    a.close()
    b.close()


def test_step_host_reports_a_nonphysical_state():
    g, prm = _bump()
    st = [np.array(x, dtype=np.float64, order="C") for x in case.perturbed_state(g.x_cv, prm, 0.0)]
    j = solver.JoeGpu(g, prm)
    j.set_state(*st)
    st[2][7] = -abs(st[2][7])     # negative energy, so negative pressure, in one cell
    with pytest.raises(solver.JoeGpuError) as e:
        j.step_host(st[0], st[1], st[2], 1)
    assert e.value.code == -4   # JG_ERR_STATE
    j.close()
