"""Batching form: independent cases of different sizes and inflow
conditions advanced in one batch must give, per case, bit-identical states
and residual histories to the same case run alone (no cross-case reduction,
no cross-case data)."""
import dataclasses

import numpy as np
import pytest

from myjoe_b200 import case, solver

pytestmark = pytest.mark.gpu


def cases(flux="HLLC", machs=(0.5, 0.6, 0.4)):
    out = []
    for k, (nx, ny, aoa, bump) in enumerate([(24, 12, 0.0, 0.1), (40, 16, 2.0, 0.07), (16, 8, -3.0, 0.12)]):
        _, g, prm = case.bump_case(nx, ny, 2, mach=machs[k], aoa_deg=aoa, bump_h=bump, jitter=0.1, seed=k)
        prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=6, CFL=2.0, CFL_RAMP=(3, 2, 1.3, 30.0),
                                  SPACE_INTEGRATION=flux)
        out.append((g, prm))
    return out


# AUSMDV on sonic inflows (the shock sensor's flags and the Haenel shock fix per case) and JST
# (its per-cell sensors) keep every per-cell quantity inside its case as well
@pytest.mark.parametrize("flux,machs", [("HLLC", (0.5, 0.6, 0.4)), ("AUSMDV", (1.0, 0.95, 1.05)),
                                        ("JST", (0.5, 0.6, 0.4))])
@pytest.mark.parametrize("precision", [0, 1])
def test_batch_is_bitwise_equal_to_alone(precision, flux, machs):
    cs = cases(flux, machs)
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


def turb_cases(model, solver_name="SGS"):
    make = case.sa_bump_case if model == "sa" else case.sst_bump_case
    out = []
    for k, (nx, ny, npr, mach, bump) in enumerate([(24, 12, 0, 0.5, 0.08), (32, 16, 4, 0.6, 0.05),
                                                   (16, 10, 0, 0.4, 0.1)]):
        # one fluid for the whole batch: Re grows with the Mach number at a fixed viscosity
        _, g, prm = make(nx, ny, 2, mach=mach, mu_ref=2.0e-3, bump_h=bump, stretch=1.15, jitter=0.05, seed=k,
                         n_prism=npr, alternate=True)
        prm = dataclasses.replace(prm, LINEAR_SOLVER_NS=solver_name, LS_MAX_ITER=6, CFL=1.0,
                                  CFL_RAMP=(3, 2, 1.2, 10.0))
        out.append((g, prm))
    return out


def _phi0(g, prm):
    vals = [prm.NUSA_INITIAL] if prm.TURB_MODEL == "SA" else [prm.KINE_INITIAL, prm.OMEGA_INITIAL]
    return np.stack([case.perturbed_scalar(g.x_cv, v, 0.05) for v in vals], 1)


@pytest.mark.parametrize("model,solver_name", [("sa", "SGS"), ("sst", "SGS"), ("sa", "LINE"), ("sst", "LINE")])
@pytest.mark.parametrize("precision", [0, 1])
def test_turbulence_batch_is_bitwise_equal_to_alone(model, solver_name, precision):
    """SA (6x6) and SST (7x7) cases of different sizes, hex and mixed
    prism/hex meshes, in one batch, relaxed by SGS or LINE (every case grows
    its own lines from its own walls): per case the state, the transported
    scalars and the residual history are those of the case run alone (each
    case's wall distance is taken to its own walls)."""
    cs = turb_cases(model, solver_name)
    nsteps = 10
    alone = []
    for g, prm in cs:
        j = solver.JoeGpu(g, prm, precision=precision)
        j.set_state(*case.perturbed_state(g.x_cv, prm, 0.02))
        j.set_scalars(_phi0(g, prm))
        wd = j.turb_array("wallDist")
        r = j.runBackwardEuler(nsteps)
        alone.append((j.get_state(), j.get_scalars(), r, wd))
        j.close()
    b = solver.JoeGpuBatch(cs, precision=precision)
    for k, (g, prm) in enumerate(cs):
        b.set_case_state(k, *case.perturbed_state(g.x_cv, prm, 0.02))
        b.set_case_scalars(k, _phi0(g, prm))
    wd = b.turb_array("wallDist")
    off = np.concatenate([[0], np.cumsum(b.sizes)])
    for k in range(len(cs)):
        np.testing.assert_array_equal(wd[off[k]:off[k + 1]], alone[k][3])
    rb = b.runBackwardEulerCases(nsteps)
    assert rb.shape == (nsteps, len(cs), 5 + cs[0][1].nscal)
    for k in range(len(cs)):
        for a, c in zip(b.get_case_state(k), alone[k][0]):
            np.testing.assert_array_equal(a, c)
        np.testing.assert_array_equal(b.get_case_scalars(k), alone[k][1])
        np.testing.assert_array_equal(rb[:, k, :], alone[k][2])
    # a frozen case keeps its state while the others advance
    b.set_active(1, False)
    frozen = b.get_case_state(1)
    b.runBackwardEulerCases(3)
    for a, c in zip(b.get_case_state(1), frozen):
        np.testing.assert_array_equal(a, c)
    b.close()


def test_batch_refuses_cases_with_different_fluids():
    cs = turb_cases("sa")
    g, prm = cs[1]
    cs[1] = (g, dataclasses.replace(prm, MU_REF=2.0 * prm.MU_REF))
    with pytest.raises(ValueError):
        solver.JoeGpuBatch(cs)


def test_batch_refuses_a_coupling_time_step_mode_after_creation():
    """jg_set_params on a batch handle refuses CFL_MIN (one minimum over the
    cells of every case would couple them), as jg_batch_create does; the
    handle keeps stepping with its old settings."""
    import ctypes as C
    from myjoe_b200.abi import jg_params
    cs = cases()
    b = solver.JoeGpuBatch(cs)
    for k, (g, prm) in enumerate(cs):
        b.set_case_state(k, *case.perturbed_state(g.x_cv, prm, 0.02))
    q = jg_params()
    C.memmove(C.byref(q), C.byref(b.jp), C.sizeof(jg_params))
    q.time_step_mode = 1  # JG_TS_CFL_MIN
    assert solver.lib().jg_set_params(b.h, C.byref(q)) == -1  # JG_ERR_ARG
    r = b.runBackwardEulerCases(2)
    assert np.all(np.isfinite(r))
    b.close()


@pytest.mark.parametrize("method", [1, 2])
def test_renumbered_batch_is_bitwise_equal_to_renumbered_alone(method):
    """A batch renumbers each case on its own (RCM, or RCM grouped by colour):
    each case's state and residual history equal the same case renumbered on
    its own handle, and states come back in the caller's cell order."""
    cs = cases()
    nsteps = 10
    alone = []
    for g, prm in cs:
        j = solver.JoeGpu(g, prm, precision=1, renumber=method)
        j.set_state(*case.perturbed_state(g.x_cv, prm, 0.02))
        r = j.runBackwardEuler(nsteps)
        alone.append((j.get_state(), r))
        j.close()
    b = solver.JoeGpuBatch(cs, precision=1, renumber=method)
    for k, (g, prm) in enumerate(cs):
        b.set_case_state(k, *case.perturbed_state(g.x_cv, prm, 0.02))
    rb = b.runBackwardEulerCases(nsteps)
    for k in range(len(cs)):
        for x, y in zip(b.get_case_state(k), alone[k][0]):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(rb[:, k, :], alone[k][1])
    b.close()


def test_renumbered_turbulence_batch_scalars_in_caller_order():
    """SST cases renumbered inside a batch: scalars go in and come out in each
    case's own cell order, and equal the same case renumbered alone."""
    cs = turb_cases("sst")
    nsteps = 6
    alone = []
    for g, prm in cs:
        j = solver.JoeGpu(g, prm, renumber=1)
        j.set_state(*case.perturbed_state(g.x_cv, prm, 0.02))
        j.set_scalars(_phi0(g, prm))
        j.runBackwardEuler(nsteps)
        alone.append((j.get_state(), np.asarray(j.get_scalars()).reshape(g.ncv, -1)))
        j.close()
    b = solver.JoeGpuBatch(cs, renumber=1)
    for k, (g, prm) in enumerate(cs):
        b.set_case_state(k, *case.perturbed_state(g.x_cv, prm, 0.02))
        b.set_case_scalars(k, _phi0(g, prm))
    b.runBackwardEulerCases(nsteps)
    for k in range(len(cs)):
        for x, y in zip(b.get_case_state(k), alone[k][0]):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(np.asarray(b.get_case_scalars(k)).reshape(alone[k][1].shape), alone[k][1])
    b.close()


def test_line_grouped_batch_is_bitwise_equal_to_alone():
    """SA cases relaxed by LINE in a batch renumbered case by case with
    JG_RENUMBER_RCM_LINES (each case's lines from its own walls, consecutive in
    its own order): per case the state, the scalars and the residual history
    equal the case alone with the same order and alone with plain RCM."""
    cs = turb_cases("sa", "LINE")
    nsteps = 8
    runs = {}
    for method in (solver.RENUMBER_RCM, solver.RENUMBER_RCM_LINES):
        out = []
        for g, prm in cs:
            j = solver.JoeGpu(g, prm, precision=1, renumber=method)
            j.set_state(*case.perturbed_state(g.x_cv, prm, 0.02))
            j.set_scalars(_phi0(g, prm))
            r = j.runBackwardEuler(nsteps)
            out.append((j.get_state(), j.get_scalars(), r))
            j.close()
        runs[method] = out
    b = solver.JoeGpuBatch(cs, precision=1, renumber=solver.RENUMBER_RCM_LINES)
    for k, (g, prm) in enumerate(cs):
        b.set_case_state(k, *case.perturbed_state(g.x_cv, prm, 0.02))
        b.set_case_scalars(k, _phi0(g, prm))
    rb = b.runBackwardEulerCases(nsteps)
    for k in range(len(cs)):
        for ref in (runs[solver.RENUMBER_RCM_LINES][k], runs[solver.RENUMBER_RCM][k]):
            for x, y in zip(b.get_case_state(k), ref[0]):
                np.testing.assert_array_equal(x, y)
            np.testing.assert_array_equal(b.get_case_scalars(k), ref[1])
        np.testing.assert_array_equal(rb[:, k, :], runs[solver.RENUMBER_RCM_LINES][k][2])
        np.testing.assert_allclose(rb[:, k, :], runs[solver.RENUMBER_RCM][k][2], rtol=1e-13, atol=0.0)
    b.close()
