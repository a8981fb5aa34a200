"""Batching form: independent cases of different sizes and inflow
conditions advanced in one batch must give, per case, bit-identical states
and residual histories to the same case run alone (no cross-case reduction,
no cross-case data)."""
import dataclasses

import numpy as np
import pytest

from myjoe_b200 import case, solver

pytestmark = pytest.mark.gpu


def cases():
    out = []
    for k, (nx, ny, mach, aoa, bump) in enumerate([(24, 12, 0.5, 0.0, 0.1), (40, 16, 0.6, 2.0, 0.07),
                                                   (16, 8, 0.4, -3.0, 0.12)]):
        _, g, prm = case.bump_case(nx, ny, 2, mach=mach, aoa_deg=aoa, bump_h=bump, jitter=0.1, seed=k)
        prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=6, CFL=2.0, CFL_RAMP=(3, 2, 1.3, 30.0))
        out.append((g, prm))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_is_bitwise_equal_to_alone(precision):
    cs = cases()
    nsteps = 12
    alone = []
    for g, prm in cs:
        j = solver.JoeGpu(g, prm, precision=precision)
        j.set_state(*case.perturbed_state(g.x_cv, prm, 0.02))
        r = j.runBackwardEuler(nsteps)
        alone.append((j.get_state(), r))
        j.close()
    b = solver.JoeGpuBatch(cs, precision=precision)
    for k, (g, prm) in enumerate(cs):
        b.set_case_state(k, *case.perturbed_state(g.x_cv, prm, 0.02))
    rb = b.runBackwardEulerCases(nsteps)
    for k in range(len(cs)):
        st = b.get_case_state(k)
        for a, c in zip(st, alone[k][0]):
            np.testing.assert_array_equal(a, c)
        np.testing.assert_array_equal(rb[:, k, :], alone[k][1])
    b.close()


def test_diverging_case_is_retired_without_disturbing_the_batch():
    """A case started from a non-physical state (negative pressure injected on
    the host into its initial state) is flagged and frozen; the other cases'
    states stay bit-identical to their runs alone."""
    cs = cases()
    nsteps = 6
    alone = []
    for g, prm in cs[1:]:
        j = solver.JoeGpu(g, prm)
        j.set_state(*case.perturbed_state(g.x_cv, prm, 0.02))
        j.runBackwardEuler(nsteps)
        alone.append(j.get_state())
        j.close()
    b = solver.JoeGpuBatch(cs)
    for k, (g, prm) in enumerate(cs):
        rho, rhou, rhoE = case.perturbed_state(g.x_cv, prm, 0.02)
        if k == 0:
            rhoE = rhoE.copy()
            rhoE[len(rhoE) // 2] = -abs(rhoE[len(rhoE) // 2])  # the fault: negative energy in one cell
        b.set_case_state(k, rho, rhou, rhoE)
    with pytest.raises(solver.JoeGpuError):
        b.runBackwardEulerCases(1)         # the preamble reports the bad input state
    b.set_active(0, False)
    b.status()
    r = b.runBackwardEulerCases(nsteps)
    for k in range(1, len(cs)):
        for a, c in zip(b.get_case_state(k), alone[k - 1]):
            np.testing.assert_array_equal(a, c)
    assert np.all(np.isfinite(r[:, 1:, :]))
    b.close()
