"""Operator parity at the precision form's scale.

calcRhsCoupled (JoeWithModels.cpp:4597-4611: the SA residual and the 6x6 block
Jacobian) on a shuffled mixed prism/hex mesh of about a million cells -- the
precision form's workload at half its 2M cells -- through a handle that
renumbers the shuffled mesh itself, against the oracle (pinned bit-exact to the
reference's own calcRhsCoupled on the small fixtures).  One call, no steps:
each residual component and each Jacobian entry within 1e-11 of its largest
magnitude over the mesh -- the bar of the small coupled fixtures against the
reference itself (tests/test_gpu_sa.py).
"""
import dataclasses
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_calc_rhs_coupled_million_cell_shuffled_mixed_mesh():
    from myjoe_b200 import build, case, solver
    from oracle.oracle import OracleSA
    build.build()
    t = time.time()
    # 512 x 8 columns of 210 + 44 cell rows: 44 wall-normal rows of prisms (two per quad), hexes above
    _, g, prm = case.sa_bump_case(512, 210, 8, mach=0.7, re=3.0e6, bump_h=0.05, stretch=1.02, n_prism=44,
                                  shuffle=True, seed=3)
    assert g.ncv >= 1_000_000
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="SGS", LS_MAX_ITER=10)
    st = case.perturbed_state(g.x_cv, prm, 0.03)
    phi = case.perturbed_scalar(g.x_cv, prm.NUSA_INITIAL, 0.1)
    j = solver.JoeGpu(g, prm, renumber=True)
    j.set_state(*st)
    j.set_scalars(phi[:, None])
    rhs_g, A_g = j.calcRhsCoupled(True)
    j.close()
    o = OracleSA(g, prm)
    o.set_state(*st)
    o.set_scalar(phi)
    o.calc_state()
    rhs_o, A_o = o.calc_rhs(True)
    B = 6
    for i in range(B):
        ref = rhs_o[:, i]
        assert np.abs(rhs_g[:, i] - ref).max() <= 1e-11 * np.abs(ref).max(), i
    for r in range(B):
        for c in range(B):
            ref = A_o[:, r, c]
            m = np.abs(ref).max()
            if m == 0.0:
                assert np.abs(A_g[:, r, c]).max() == 0.0, (r, c)
            else:
                assert np.abs(A_g[:, r, c] - ref).max() <= 1e-11 * m, (r, c)
    print("cells %d, %.1f s" % (g.ncv, time.time() - t))
