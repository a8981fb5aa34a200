"""Lagged Jacobian (jg_params.jac_lag): the flux Jacobian blocks of each case
are formed every jac_lag-th step; the steps between add their own vol/dt to
the kept diagonal and invert it.

* jac_lag = 1 is the plain iteration, bit for bit;
* a lagged run's first step equals the plain run's first step (the blocks
  are fresh), and the first step after a new state is fresh again;
* a batch of lagged cases gives each case the bits it gets alone;
* the converged field does not depend on the lag (tests/test_gpu_converged.py
  runs the reference's converged bump with jac_lag = 5).
"""
import dataclasses

import numpy as np
import pytest

from myjoe_b200 import case, solver

pytestmark = pytest.mark.gpu


def _bump(seed=4, nx=24, ny=12):
    _, g, prm = case.bump_case(nx, ny, 2, jitter=0.1, seed=seed)
    return g, dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=8, CFL=2.0, CFL_RAMP=(3, 2, 1.3, 30.0))


def _run(g, prm, lag, nsteps, precision=0):
    j = solver.JoeGpu(g, prm, precision=precision, jac_lag=lag)
    j.set_state(*case.perturbed_state(g.x_cv, prm, 0.02))
    r = j.runBackwardEuler(nsteps)
    st = j.get_state()
    j.close()
    return st, r


@pytest.mark.parametrize("precision", [0, 1])
def test_lag_one_is_the_plain_iteration(precision):
    g, prm = _bump()
    a = _run(g, prm, 0, 12, precision)
    b = _run(g, prm, 1, 12, precision)
    for x, y in zip(a[0], b[0]):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a[1], b[1])


@pytest.mark.parametrize("precision", [0, 1])
def test_lagged_steps(precision):
    g, prm = _bump()
    plain1 = _run(g, prm, 1, 1, precision)
    lag1 = _run(g, prm, 4, 1, precision)
    for x, y in zip(plain1[0], lag1[0]):
        np.testing.assert_array_equal(x, y)     # step 1: fresh blocks, the same bits
    plain = _run(g, prm, 1, 12, precision)
    lag = _run(g, prm, 4, 12, precision)
    assert np.all(np.isfinite(lag[1]))
    assert not np.array_equal(plain[0][0], lag[0][0])   # the lag does change the iterates
    # a new state starts with fresh blocks again
    j = solver.JoeGpu(g, prm, precision=precision, jac_lag=4)
    st0 = case.perturbed_state(g.x_cv, prm, 0.02)
    j.set_state(*st0)
    j.runBackwardEuler(6)
    j.set_state(*st0)
    j.set_cfl_step(prm.CFL, 0)
    j.runBackwardEuler(1)
    for x, y in zip(j.get_state(), plain1[0]):
        np.testing.assert_array_equal(x, y)
    j.close()


def test_lagged_batch_is_bitwise_equal_to_alone():
    cs = [_bump(seed=k, nx=nx, ny=ny) for k, (nx, ny) in enumerate([(24, 12), (40, 16), (16, 8)])]
    alone = [_run(g, prm, 3, 10, 1) for g, prm in cs]
    b = solver.JoeGpuBatch(cs, precision=1, jac_lag=3)
    for k, (g, prm) in enumerate(cs):
        b.set_case_state(k, *case.perturbed_state(g.x_cv, prm, 0.02))
    rb = b.runBackwardEulerCases(10)
    for k in range(len(cs)):
        for x, y in zip(b.get_case_state(k), alone[k][0]):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(rb[:, k, :], alone[k][1])
    b.close()


def test_lag_refused_where_it_does_not_apply():
    g, prm = _bump()
    with pytest.raises(solver.JoeGpuError):
        solver.JoeGpu(g, dataclasses.replace(prm, LINEAR_SOLVER_NS="BCGSTAB"), jac_lag=3)
