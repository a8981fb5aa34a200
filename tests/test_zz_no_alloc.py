"""The allocation-free relaxation entry point (jg_relax_csr_noalloc).

It exists for host programs that cannot call cudaMalloc at solve time (their
device memory belongs to another allocator, or a mid-run allocation's
synchronisation or out-of-memory failure is not acceptable), so it works on
device buffers the caller already owns plus a fixed scratch array inside the
library.  This test gives it caller-owned device buffers (allocated here with
torch, as such a host would have them) and checks its result against the
regular entry point, jg_solve_lin_sys with block Jacobi, on the same system --
twice in a row with different data and sweep counts, so that a second call
reading stale scratch contents would be caught.  Same 1e-12 normwise tolerance
as the other relaxation parity tests.  The file sorts last so that a run
stopping at the first failure has run every other test before it.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def nrel(a, b):
    a, b = np.asarray(a).reshape(len(b), -1), np.asarray(b).reshape(len(b), -1)
    scale = np.abs(b).max(axis=0)
    scale[scale == 0] = 1.0
    return float((np.abs(a - b).max(axis=0) / scale).max())


def test_noalloc_relaxation_matches_regular_entry_point():
    import torch

    from myjoe_b200 import build, case, solver
    build.build()
    L = solver.lib()
    L.jg_relax_csr_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int, C.c_void_p]
    L.jg_relax_csr_noalloc.restype = C.c_int
    assert solver.device_count() > 0

    _, g, prm = case.bump_case(24, 12, 2, jitter=0.1, seed=4)
    prm = dataclasses.replace(prm, LINEAR_SOLVER_NS="JACOBI")
    j = solver.JoeGpu(g, prm)
    j.set_state(*case.perturbed_state(g.x_cv, prm, 0.03))
    _, local_dt = j.calcDt()
    rr, ru, rE, A = j.calcRhs(True)
    for i in range(5):
        A[g.nbocv_i[:-1], i, i] += g.cv_volume / local_dt
    rhs = np.column_stack([rr, ru, rE]) * prm.UNDER_RELAXATION

    dev = torch.device("cuda", torch.cuda.current_device())
    d_i = torch.from_numpy(np.ascontiguousarray(g.nbocv_i, np.int32)).to(dev)
    d_v = torch.from_numpy(np.ascontiguousarray(g.nbocv_v, np.int32)).to(dev)
    d_A = torch.from_numpy(np.ascontiguousarray(A)).to(dev)
    stream = torch.cuda.current_stream()

    for sweeps, scale in ((7, 1.0), (4, -0.5)):
        b = np.ascontiguousarray(rhs * scale)
        d_b = torch.from_numpy(b).to(dev)
        d_dq = torch.full((g.ncv, 5), float("nan"), dtype=torch.float64, device=dev)
        rc = L.jg_relax_csr_noalloc(g.ncv, d_i.data_ptr(), d_v.data_ptr(), d_A.data_ptr(), d_b.data_ptr(),
                                    d_dq.data_ptr(), sweeps, stream.cuda_stream)
        assert rc == 0, L.jg_last_error().decode()
        torch.cuda.synchronize()
        dq_new = d_dq.cpu().numpy()
        dq_ref, _ = j.solveCoupledLinSysNS(A, b, 0.0, 0.0, sweeps)
        assert np.all(np.isfinite(dq_new))
        assert nrel(dq_new, dq_ref) <= TOL

    # sizes beyond the fixed scratch are refused before any device work
    too_many = 65536 + 1
    rc = L.jg_relax_csr_noalloc(too_many, d_i.data_ptr(), d_v.data_ptr(), d_A.data_ptr(), d_b.data_ptr(),
                                d_dq.data_ptr(), 1, stream.cuda_stream)
    assert rc == -1
    assert b"exceed the limit" in L.jg_last_error()
