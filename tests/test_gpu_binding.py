"""The drop-in binding compiled and run: include/joe_gpu.hpp's JoeGpu (a
JoeWithModels subclass whose loop runs on the GPU through the C ABI) built
into the reference's own case harness (oracle/Makefile target ``binding``:
the reference's objects + libjoe_b200.so) runs the reference's case path --
Joe.in, the .msh reader, geometry, LSQ coefficients, initial condition,
doneSolver, showResidue -- and must end where the reference's own
runBackwardEuler ends (JoeWithModels.cpp:881-1198): the 64x32x4 inviscid bump,
HLLC, second order, BiCGSTAB with the reference's thresholds, from a perturbed
state.  States after the run within 1e-10 relative, residual histories to the
5 digits the reference prints."""
import dataclasses
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nsteps", [25])
def test_binding_runs_the_reference_case_path(nsteps):
    from myjoe_b200 import build, case, meshgen
    from oracle import refrun
    build.build()
    if not os.path.exists(refrun.BINDING):
        pytest.fail("binding not built: make -C oracle binding REF=<the reference src directory>")
    raw, g, prm = case.bump_case(64, 32, 4)
    prm = dataclasses.replace(prm, CFL=1.0, CFL_RAMP=(5, 5, 1.2, 20.0), NSTEPS=nsteps)
    joe_in = prm.joe_in("mesh.msh", "HARNESS_PERTURB = 0.02")
    write = lambda p: meshgen.write_msh(p, raw)
    ref = refrun.run(write, joe_in, "run")
    gpu = refrun.run(write, joe_in, "gpu", harness=refrun.BINDING)
    assert ref["steps"] == gpu["steps"] == nsteps
    for k in ("final_rho", "final_rhoE"):
        a, b = gpu[k], ref[k]
        assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max(), k
    a, b = gpu["final_rhou"], ref["final_rhou"]
    assert np.abs(a - b).max() <= 1e-10 * np.abs(b).max()
    assert gpu["resid"].shape == ref["resid"].shape == (nsteps, 5)   # CHECK_INTERVAL = 1: every step
    np.testing.assert_allclose(gpu["resid"], ref["resid"], rtol=6e-5)
