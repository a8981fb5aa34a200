"""Restart files and the GPU handle: a case resumed on the GPU from a restart
the reference wrote continues as the reference itself continues from it, and
the handle's state written to a restart reads back bit for bit.

Fixtures (tests/golden/make_restart.py): restart_bump_step3.out, the
reference's restart after 3 steps of the 8x4x2 bump; restart_bump.npz, the
reference's state after 3 more steps run from that file; restart_sa_step2.out,
an SA case with nuSA and the reference's wall distance.

Tolerance: states after backward-Euler steps 1e-10 relative (the GPU sums
faces in its own order and contracts to fused multiply-adds); the wall
distance 1e-12 relative.
"""
import dataclasses
import json
import os

import numpy as np
import pytest
from scipy.spatial import cKDTree

from myjoe_b200 import case, restart, solver
from tests.golden.make_golden import params_from_json

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from myjoe_b200 import build
    build.build()
    if solver.device_count() == 0:
        pytest.fail("no CUDA device visible to libjoe_b200.so")


def rel(a, b):
    a, b = np.asarray(a).reshape(len(b), -1), np.asarray(b).reshape(len(b), -1)
    s = np.abs(b).max(axis=0)
    s[s == 0] = 1.0
    return float((np.abs(a - b).max(axis=0) / s).max())


def test_gpu_resumes_the_reference_restart(tmp_path):
    ref = np.load(os.path.join(GOLD, "restart_bump.npz"))
    prm = params_from_json(str(ref["params"]))
    g, r = restart.read_restart(os.path.join(GOLD, "restart_bump_step3.out"))
    j = solver.JoeGpu(g, prm)
    r.load_state(j)
    assert j.cfl_step() == (prm.CFL, 3)
    rho, rhou, rhoE = j.get_state()
    assert np.array_equal(rho, ref["rho3"]) and np.array_equal(rhou, ref["rhou3"])
    j.runBackwardEuler(3)
    assert j.cfl_step()[1] == 6
    _, m = cKDTree(g.x_cv).query(ref["x_cv6"])
    rho, rhou, rhoE = j.get_state()
    assert rel(rho[m], ref["rho6"]) < 1e-10
    assert rel(rhou[m], ref["rhou6"]) < 1e-10
    assert rel(rhoE[m], ref["rhoE6"]) < 1e-10
    # the GPU state written into the reference's file and read back
    r.save_state(j)
    p = str(tmp_path / "gpu.out")
    r.write(p)
    back = restart.Restart.read(p)
    assert back.get("STEP")[1] == 6
    assert np.array_equal(back.get("RHO")[1], rho)
    assert np.array_equal(back.get("RHOU")[1], rhou)
    assert np.array_equal(back.get("RHOE")[1], rhoE)
    assert back.record_names() == r.record_names()
    j.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_state_through_a_library_file(precision, tmp_path):
    """A handle's state written with the handle's own mesh, read into a fresh
    handle on the mesh rebuilt from the file: identical state and step, and,
    once both ramps stand at the same CFL, identical steps after it."""
    ref = np.load(os.path.join(GOLD, "restart_bump.npz"))
    prm = params_from_json(str(ref["params"]))
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=10)
    g, r = restart.read_restart(os.path.join(GOLD, "restart_bump_step3.out"))
    a = solver.JoeGpu(g, prm, precision=precision)
    r.load_state(a)
    a.runBackwardEuler(2)
    p = str(tmp_path / "a.out")
    restart.write_restart(p, g, a)
    g2, r2 = restart.read_restart(p)
    b = solver.JoeGpu(g2, prm, precision=precision)
    r2.load_state(b)
    # a restart resumes at STEP with the CFL back at its start value (JoeWithModels.cpp:975-978)
    assert b.cfl_step() == (prm.CFL, 5)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(x, y)
    a.set_cfl_step(prm.CFL, 5)
    a.runBackwardEuler(2)
    b.runBackwardEuler(2)
    for x, y in zip(a.get_state(), b.get_state()):
        assert rel(x, y) < 1e-13
    a.close()
    b.close()


def test_gpu_sa_restart_scalars_and_wall_distance(tmp_path):
    prm = params_from_json(json.load(open(os.path.join(GOLD, "restart_sa.json")))["params"])
    # the coupled SA path relaxes point-wise (the reference's coupled solve is PETSc)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=10)
    g, r = restart.read_restart(os.path.join(GOLD, "restart_sa_step2.out"))
    j = solver.JoeGpu(g, prm)
    r.load_state(j)
    assert np.array_equal(j.get_scalars(), r.get("nuSA")[1])
    # the reference's calcWallDistance, stored in its restart, against the GPU's
    wd = r.get("wallDist")[1]
    assert rel(j.turb_array("wallDist"), wd) < 1e-12
    j.runBackwardEuler(2)
    r.save_state(j)
    p = str(tmp_path / "sa.out")
    r.write(p)
    back = restart.Restart.read(p)
    assert np.array_equal(back.get("nuSA")[1], j.get_scalars())
    assert back.get("STEP")[1] == 4
    j.close()


def test_load_state_rejects_a_mismatched_file():
    ref = np.load(os.path.join(GOLD, "restart_bump.npz"))
    prm = params_from_json(str(ref["params"]))
    g, _ = restart.read_restart(os.path.join(GOLD, "restart_bump_step3.out"))
    j = solver.JoeGpu(g, prm)
    blank = restart.Restart.from_cv_mesh(g)
    with pytest.raises(solver.JoeGpuError) as e:
        blank.load_state(j)                # no RHO / RHOU / RHOE records
    assert e.value.code == -1
    _, small, _ = case.bump_case(6, 4, 2)
    other = restart.Restart.from_cv_mesh(small)
    for name, kind, shape in (("RHO", restart.CV_D1, (small.ncv,)), ("RHOE", restart.CV_D1, (small.ncv,)),
                              ("RHOU", restart.CV_D3, (small.ncv, 3))):
        other.put(name, kind, np.ones(shape))
    with pytest.raises(solver.JoeGpuError) as e:
        other.load_state(j)                # another mesh
    assert e.value.code == -1
    j.close()
