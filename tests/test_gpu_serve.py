"""Serving form (jg_serve_*): results are the same alone and in the mix.

Cases of different sizes and inflow conditions go through one server that
keeps them all resident at once, through one that admits a single case at a
time, and through one whose device-memory budget admits only what fits.  Each
case runs on its own handle and stream and retires at the same step in every
run, so its final state must be bitwise identical across the three.  A case
with a non-physical initial state sits in the mix: it must be restarted up to
the limit, retired as failed, and leave the other cases' results untouched.
The exact device-footprint estimate used for admission is checked against the
bytes a handle really allocates.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPECS = [  # (nx, ny, mach, aoa, bump)
    (24, 12, 0.40, 1.0, 0.06),
    (40, 20, 0.50, -2.0, 0.08),
    (32, 16, 0.35, 3.0, 0.05),
    (20, 10, 0.45, 0.0, 0.07),
]
DROP = 1e-6


def _cases():
    from myjoe_b200 import case
    out = []
    for k, (nx, ny, mach, aoa, bump) in enumerate(SPECS):
        _, g, prm = case.bump_case(nx, ny, 2, mach=mach, aoa_deg=aoa, bump_h=bump, seed=k, inlet="FARFIELD")
        prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=10, CFL=1.0, CFL_RAMP=(10, 5, 1.2, 20.0))
        out.append((g, prm, case.perturbed_state(g.x_cv, prm, 0.0)))
    return out


def _serve(cases, bad, precision, **kw):
    from myjoe_b200 import solver
    srv = solver.JoeServer(steps_per_poll=25, resid_drop=DROP, max_steps=3000, max_restarts=1,
                           restart_cfl_factor=0.5, **kw)
    ids = [srv.submit(g, prm, st, precision=precision) for g, prm, st in cases]
    g, prm, st = bad
    bad_id = srv.submit(g, prm, st, precision=precision)
    res = {}
    peak_resident, peak_shared_bytes = 0, 0.0
    while len(res) < len(ids) + 1:
        for r in srv.poll(max_wait=0.01):
            res[r["id"]] = (r, srv.fetch(r["id"]))
        st = srv.stats()
        peak_resident = max(peak_resident, st["resident"])
        if st["resident"] > 1:
            peak_shared_bytes = max(peak_shared_bytes, st["bytes_resident"])
    srv.close()
    return [res[i] for i in ids], res[bad_id], (peak_resident, peak_shared_bytes)


@pytest.mark.parametrize("precision", [0, 1])
def test_serve_same_alone_and_in_mix(precision):
    from myjoe_b200 import build, solver
    build.build()
    assert solver.device_count() > 0
    cases = _cases()
    g, prm, (rho, rhou, rhoE) = cases[0]
    rhoE_bad = rhoE.copy()
    rhoE_bad[5] = -abs(rhoE_bad[5])  # negative pressure in one cell: non-physical from the start
    bad = (g, prm, (rho, rhou, rhoE_bad))

    fp = [solver.case_footprint(c[0], c[1], precision) for c in cases]
    budget = 1.05 * max(fp)
    mix, bad_mix, (peak_mix, _) = _serve(cases, bad, precision, max_resident=8)
    alone, bad_alone, (peak_alone, _) = _serve(cases, bad, precision, max_resident=1)
    tight, _, (_, tight_bytes) = _serve(cases, bad, precision, max_resident=8, hbm_budget=budget)
    assert peak_alone == 1 and peak_mix > 1
    assert tight_bytes <= budget   # cases share the device only within the memory budget

    for (rm, sm), (ra, sa), (rt, stt) in zip(mix, alone, tight):
        assert rm["status"] == 0, rm          # converged
        assert rm["drop"] <= DROP and rm["restarts"] == 0
        for r in (ra, rt):
            assert (r["status"], r["steps"], r["conv_step"]) == (rm["status"], rm["steps"], rm["conv_step"])
        for x, y, z in zip(sm, sa, stt):
            assert np.array_equal(x, y) and np.array_equal(x, z)   # bitwise
    for b in (bad_mix, bad_alone):
        r, _ = b
        assert r["status"] == 2 and r["restarts"] == 1


@pytest.mark.parametrize("precision", [0, 1])
def test_footprint_is_exact(precision):
    from myjoe_b200 import case, solver
    _, g, prm = case.bump_case(24, 12, 2, seed=3)
    _, gp, pp = case.plate_case(32, 16, 2)
    for mesh, p in ((g, prm), (gp, pp)):
        p = dataclasses.replace(p, LINEAR_SOLVER_NS="SGS")
        est = solver.case_footprint(mesh, p, precision)
        j = solver.JoeGpu(mesh, p, precision=precision)
        j.set_state(*case.perturbed_state(mesh.x_cv, p, 0.0))
        assert j.device_bytes() == est
        j.close()


def test_case_above_the_budget_is_reported_failed():
    """A case whose footprint exceeds the whole memory budget can never be
    admitted: poll reports it as failed, with its initial state, and the
    cases that fit are served as usual."""
    from myjoe_b200 import solver
    cases = _cases()
    fp = [solver.case_footprint(c[0], c[1], 0) for c in cases]
    small = int(np.argmin(fp))
    big = int(np.argmax(fp))
    assert fp[big] > 1.2 * fp[small]
    srv = solver.JoeServer(steps_per_poll=25, resid_drop=DROP, max_steps=3000, max_restarts=0,
                           hbm_budget=1.1 * fp[small])
    g, prm, st = cases[big]
    id_big = srv.submit(g, prm, st)
    g, prm, st = cases[small]
    id_small = srv.submit(g, prm, st)
    res = {}
    while len(res) < 2:
        for r in srv.poll(max_wait=0.01):
            res[r["id"]] = (r, srv.fetch(r["id"]))
    srv.close()
    r, state = res[id_big]
    assert r["status"] == 2 and r["steps"] == 0
    for a, b in zip(state, cases[big][2]):
        np.testing.assert_array_equal(np.asarray(a).reshape(np.shape(b)), b)
    assert res[id_small][0]["status"] == 0
