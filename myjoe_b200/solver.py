"""Python host mirror of the reference's operator surface over libjoe_b200.so.

``JoeGpu`` keeps the names of the reference's ``UgpWithCvCompFlow`` /
``JoeWithModels`` operators (calcStateVariables, calcDt, calcRhs,
solveCoupledLinSysNS, runBackwardEuler) and forwards each to the C ABI in
include/joe_b200.h.  The library must be the CUDA build: loading fails loudly
when it is missing; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
import types

import numpy as np

from .abi import MeshArrays, dptr, jg_mesh, jg_params, jg_serve_config, jg_serve_result, make_params
from .case import JoeParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libjoe_b200.so")
_lib = None

FLUX_SPLIT = 32        # JG_FLUX_SPLIT: face-loop shapes split into a residual and a Jacobian kernel
FLUX_CL1_3BLK = 17     # JG_FLUX_CL1_3BLK
RENUMBER_RCM, RENUMBER_RCM_COLOR, RENUMBER_RCM_LINES = 1, 2, 3   # jg_params.renumber
JG_ERR = {-1: "bad argument", -2: "CUDA error", -3: "out of device memory", -4: "non-physical state",
          -5: "no CUDA device", -6: "file error"}


class JoeGpuError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (JG_ERR.get(code, "error"), code, msg))
        self.code = code


def lib():
    """Load libjoe_b200.so (built by myjoe_b200.build); raise if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError("libjoe_b200.so is not built (python -m myjoe_b200.build): %s" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        I = C.c_int
        L.jg_last_error.restype = C.c_char_p
        L.jg_version.restype = I
        L.jg_device_count.argtypes = [C.POINTER(I)]
        L.jg_create.argtypes = [C.POINTER(jg_mesh), C.POINTER(jg_params), C.POINTER(P)]
        L.jg_renumber_cells.argtypes = [C.POINTER(jg_mesh), I, C.POINTER(I)]
        L.jg_set_launch_config.argtypes = [P, I, I]
        L.jg_get_launch_config.argtypes = [P, C.POINTER(I), C.POINTER(I)]
        L.jg_autotune.argtypes = [P, I, C.POINTER(I), C.POINTER(I), C.POINTER(C.c_float)]
        L.jg_destroy.argtypes = [P]
        L.jg_get_stream.argtypes = [P, C.POINTER(P)]
        L.jg_set_state.argtypes = [P, D, D, D]
        L.jg_get_state.argtypes = [P, D, D, D]
        L.jg_step_host.argtypes = [P, D, D, D, I, D]
        L.jg_calc_state.argtypes = [P]
        L.jg_get_primitives.argtypes = [P, D, D, D, D, D]
        L.jg_get_bfa.argtypes = [P, D, D, D, D, D, D, D]
        L.jg_calc_dt.argtypes = [P, C.c_double, D, D]
        L.jg_calc_rhs.argtypes = [P, D, D, D, D, I]
        L.jg_get_gradients.argtypes = [P, D, D, D, D]
        L.jg_solve_lin_sys.argtypes = [P, D, D, D, C.c_double, C.c_double, I, C.POINTER(I)]
        L.jg_step.argtypes = [P, I, D]
        L.jg_step_async.argtypes = [P, I]
        L.jg_get_cfl_step.argtypes = [P, D, C.POINTER(I)]
        L.jg_set_cfl_step.argtypes = [P, C.c_double, I]
        L.jg_run_to.argtypes = [P, C.c_double, I, I, C.POINTER(I), D]
        L.jg_set_params.argtypes = [P, C.POINTER(jg_params)]
        L.jg_calc_grad.argtypes = [P, D, D, D, D]
        L.jg_euler_flux_faces.argtypes = [I, I, D, D, D, D, D, D, D]
        L.jg_batch_create.argtypes = [I, C.POINTER(jg_mesh), C.POINTER(jg_params), C.POINTER(P)]
        L.jg_batch_info.argtypes = [P, C.POINTER(I), C.POINTER(I)]
        L.jg_batch_set_state.argtypes = [P, I, D, D, D]
        L.jg_batch_set_scalars.argtypes = [P, I, D]
        L.jg_batch_get_scalars.argtypes = [P, I, D]
        L.jg_batch_get_state.argtypes = [P, I, D, D, D]
        L.jg_batch_step.argtypes = [P, I, D]
        L.jg_batch_status.argtypes = [P, C.POINTER(I)]
        L.jg_batch_set_active.argtypes = [P, I, I]
        L.jg_set_profiling.argtypes = [P, I]
        L.jg_get_profile.argtypes = [P, D]
        L.jg_step_kernel_count.argtypes = [P, C.POINTER(I)]
        L.jg_set_scalars.argtypes = [P, D]
        L.jg_get_scalars.argtypes = [P, D]
        L.jg_calc_rhs_coupled.argtypes = [P, D, D, I]
        L.jg_get_turb.argtypes = [P, D, D, D, D, D, D, D]
        L.jg_get_turb_array.argtypes = [P, C.c_char_p, D]
        L.jg_case_footprint.argtypes = [C.POINTER(jg_mesh), C.POINTER(jg_params), D]
        L.jg_case_device_bytes.argtypes = [P, D]
        L.jg_serve_create.argtypes = [C.POINTER(jg_serve_config), C.POINTER(P)]
        L.jg_serve_now.argtypes = [P, D]
        L.jg_serve_submit.argtypes = [P, C.POINTER(jg_mesh), C.POINTER(jg_params), D, D, D, C.c_double,
                                      C.POINTER(C.c_longlong)]
        L.jg_serve_poll.argtypes = [P, C.c_double, C.POINTER(jg_serve_result), I, C.POINTER(I)]
        L.jg_serve_fetch.argtypes = [P, C.c_longlong, D, D, D]
        L.jg_serve_stats.argtypes = [P, C.POINTER(I), C.POINTER(I), C.POINTER(I), D]
        L.jg_serve_destroy.argtypes = [P]
        _lib = L
    return _lib


def _ck(rc):
    if rc != 0:
        raise JoeGpuError(rc, lib().jg_last_error().decode())


def _p(a):
    return None if a is None else dptr(a)


def device_count() -> int:
    n = C.c_int(0)
    lib().jg_device_count(C.byref(n))
    return n.value


class JoeGpu:
    """One case on the GPU.  ``mesh_src`` is a ``geometry.CvMesh`` or a dict of
    reference-layout arrays; ``params`` a ``case.JoeParams``."""

    def __init__(self, mesh_src, params: JoeParams, precision: int = 0, renumber: bool = False, jac_lag: int = 1):
        self.params = params
        self.ma = MeshArrays(mesh_src, params)
        self.jp = make_params(params, precision, renumber, jac_lag)
        self.ncv = self.ma.ncv
        h = C.c_void_p()
        _ck(lib().jg_create(C.byref(self.ma.mesh), C.byref(self.jp), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().jg_destroy(self.h)
            self.h = None

    __del__ = close

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        _ck(lib().jg_get_stream(self.h, C.byref(s)))
        return s.value or 0

    # -- state ---------------------------------------------------------------
    def set_state(self, rho, rhou, rhoE):
        rho, rhou, rhoE = (np.ascontiguousarray(a, np.float64) for a in (rho, rhou, rhoE))
        _ck(lib().jg_set_state(self.h, dptr(rho), dptr(rhou), dptr(rhoE)))

    def get_state(self):
        n = self.ncv
        rho, rhou, rhoE = np.empty(n), np.empty((n, 3)), np.empty(n)
        _ck(lib().jg_get_state(self.h, dptr(rho), dptr(rhou), dptr(rhoE)))
        return rho, rhou, rhoE

    def calcStateVariables(self):
        """calcStateVariables + calcMaterialProperties + setBC."""
        _ck(lib().jg_calc_state(self.h))

    def primitives(self):
        n = self.ncv
        vel, p, T, h, c = np.empty((n, 3)), np.empty(n), np.empty(n), np.empty(n), np.empty(n)
        _ck(lib().jg_get_primitives(self.h, dptr(vel), dptr(p), dptr(T), dptr(h), dptr(c)))
        return {"vel": vel, "press": p, "temp": T, "enthalpy": h, "sos": c}

    def boundary(self):
        nb, nf = self.ma.nfa_b, self.ma.nfa
        out = {"rho_bfa": np.empty(nb), "vel_bfa": np.empty((nb, 3)), "p_bfa": np.empty(nb), "T_bfa": np.empty(nb),
               "h_bfa": np.empty(nb), "mul_fa": np.empty(nf), "lamOcp_fa": np.empty(nf)}
        _ck(lib().jg_get_bfa(self.h, *(dptr(out[k]) for k in ("rho_bfa", "vel_bfa", "p_bfa", "T_bfa", "h_bfa",
                                                              "mul_fa", "lamOcp_fa"))))
        return out

    # -- operators -----------------------------------------------------------
    def calcDt(self, cfl=None):
        dtmin = C.c_double(0.0)
        local = np.empty(self.ncv)
        _ck(lib().jg_calc_dt(self.h, self.params.CFL if cfl is None else cfl, C.byref(dtmin), dptr(local)))
        return dtmin.value, local

    def calcRhs(self, flagImplicit=True):
        n = self.ncv
        rr, ru, rE = np.empty(n), np.empty((n, 3)), np.empty(n)
        A = np.empty((self.ma.nbocv_s, 5, 5)) if flagImplicit else None
        _ck(lib().jg_calc_rhs(self.h, dptr(rr), dptr(ru), dptr(rE), _p(A), int(flagImplicit)))
        return rr, ru, rE, A

    def gradients(self):
        n = self.ncv
        gu, gr, gp, gh = np.empty((n, 3, 3)), np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        _ck(lib().jg_get_gradients(self.h, dptr(gu), dptr(gr), dptr(gp), dptr(gh)))
        return {"grad_u": gu, "grad_rho": gr, "grad_p": gp, "grad_enthalpy": gh}

    def solveCoupledLinSysNS(self, A, rhs, zeroAbs, zeroRel, maxIter, dq0=None):
        dq = np.zeros((self.ncv, 5)) if dq0 is None else np.array(dq0, np.float64, order="C")
        A = np.ascontiguousarray(A, np.float64)
        rhs = np.ascontiguousarray(rhs, np.float64)
        it = C.c_int(0)
        _ck(lib().jg_solve_lin_sys(self.h, dptr(dq), dptr(A), dptr(rhs), zeroAbs, zeroRel, int(maxIter),
                                   C.byref(it)))
        return dq, it.value

    # -- coupled path (turbulence model) -------------------------------------
    @property
    def nvar(self) -> int:
        return 5 + self.params.nscal

    def set_scalars(self, phi):
        """phi[ncv] (SA: nuSA) or phi[ncv][2] (SST: kine, omega)."""
        phi = np.ascontiguousarray(np.asarray(phi, np.float64).reshape(self.ncv, self.params.nscal))
        _ck(lib().jg_set_scalars(self.h, dptr(phi)))

    def get_scalars(self):
        ns = self.params.nscal
        phi = np.empty((self.ncv, ns))
        _ck(lib().jg_get_scalars(self.h, dptr(phi)))
        return phi[:, 0] if ns == 1 else phi

    def turb_array(self, name):
        """one model array by its reference name (jg_get_turb_array); per-scalar arrays come
        back as [nscal][...]."""
        n, nf, nb, ns = self.ncv, self.ma.nfa, self.ma.nfa_b, self.params.nscal
        shape = {"mut_fa": (nf,), "phi_bfa": (ns, nb), "grad_phi": (ns, n, 3), "diff": (ns, nf)}.get(name, (n,))
        out = np.empty(shape)
        _ck(lib().jg_get_turb_array(self.h, name.encode(), dptr(out)))
        return out

    def calcRhsCoupled(self, flagImplicit=True):
        """rhs[ncv][6], A[nbocv_s][6][6] (None without flagImplicit)."""
        B = self.nvar
        rhs = np.zeros((self.ncv, B))
        A = np.zeros((self.ma.nbocv_s, B, B)) if flagImplicit else None
        _ck(lib().jg_calc_rhs_coupled(self.h, dptr(rhs), _p(A), int(flagImplicit)))
        return rhs, A

    def turb(self):
        """wallDist, mut_fa, strMag, vortMag, phi_bfa, grad_phi, diff of the current state."""
        n, nf, nb = self.ncv, self.ma.nfa, self.ma.nfa_b
        out = {"wallDist": np.empty(n), "mut_fa": np.empty(nf), "strMag": np.empty(n), "vortMag": np.empty(n),
               "phi_bfa": np.empty(nb), "grad_phi": np.empty((n, 3)), "diff": np.empty(nf)}
        _ck(lib().jg_get_turb(self.h, *(dptr(out[k]) for k in ("wallDist", "mut_fa", "strMag", "vortMag",
                                                                  "phi_bfa", "grad_phi", "diff"))))
        return out

    def runBackwardEuler(self, nsteps):
        """``nsteps`` iterations of the backward-Euler loop; returns the L1
        residual history [nsteps][5] ([nsteps][6] on the coupled SA path)."""
        r = np.zeros((max(nsteps, 1), self.nvar))
        _ck(lib().jg_step(self.h, int(nsteps), dptr(r)))
        return r[:nsteps]

    def step_async(self, nsteps):
        _ck(lib().jg_step_async(self.h, int(nsteps)))

    def step_host(self, rho, rhou, rhoE, nsteps, resid=None):
        """``nsteps`` steps of a host-resident state, in place (jg_step_host): the arrays (C-contiguous
        float64, ``rhou`` [ncv][3]) go up, the steps run, the new state comes back into them, with one
        synchronisation.  ``resid`` ([nsteps][nvar] float64) receives the residual history."""
        for a in (rho, rhou, rhoE):
            if a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("step_host updates C-contiguous float64 arrays in place")
        _ck(lib().jg_step_host(self.h, dptr(rho), dptr(rhou), dptr(rhoE), int(nsteps),
                               dptr(resid) if resid is not None else None))

    def set_profiling(self, on=True):
        _ck(lib().jg_set_profiling(self.h, int(on)))

    def profile(self):
        ms = np.zeros(2)
        _ck(lib().jg_get_profile(self.h, dptr(ms)))
        return {"face_loop_ms": float(ms[0]), "linear_solve_ms": float(ms[1])}

    def step_kernel_count(self):
        n = C.c_int(0)
        _ck(lib().jg_step_kernel_count(self.h, C.byref(n)))
        return n.value

    def device_bytes(self) -> float:
        b = C.c_double()
        _ck(lib().jg_case_device_bytes(self.h, C.byref(b)))
        return b.value

    def autotune(self, trials=5):
        """time the launch shapes on this handle and keep the fastest: returns
        (lanes per cell of the face loop, sweep kernel, {shape: ms per launch})"""
        cl, rv = C.c_int(0), C.c_int(0)
        ms = (C.c_float * 10)()
        _ck(lib().jg_autotune(self.h, int(trials), C.byref(cl), C.byref(rv), ms))
        times = {"flux_cl1": ms[0], "flux_cl2": ms[1], "flux_cl4": ms[2], "sweep0": ms[3], "sweep1": ms[4],
                 "flux_cl17": ms[5]}
        for k, fl in enumerate((1, 2, 4, 8)):
            times["flux_cl%d" % (FLUX_SPLIT + fl)] = ms[6 + k]
        return cl.value, rv.value, times

    def set_launch_config(self, flux_cl, relax_variant):
        _ck(lib().jg_set_launch_config(self.h, int(flux_cl), int(relax_variant)))

    def launch_config(self):
        cl, rv = C.c_int(0), C.c_int(0)
        _ck(lib().jg_get_launch_config(self.h, C.byref(cl), C.byref(rv)))
        return cl.value, rv.value

    def cfl_step(self):
        cfl = C.c_double(0.0)
        step = C.c_int(0)
        _ck(lib().jg_get_cfl_step(self.h, C.byref(cfl), C.byref(step)))
        return cfl.value, step.value

    def run_to(self, resid_drop, max_steps, check_every=1):
        """runBackwardEuler until the energy residual drops to resid_drop x the first
        step's (resid_drop >= 0), or falls strictly below -resid_drop (resid_drop < 0:
        the reference's RESID_ENERG_TH rule), or max_steps (jg_run_to): returns
        (steps run, last relative drop)"""
        n, d = C.c_int(0), C.c_double(0.0)
        _ck(lib().jg_run_to(self.h, float(resid_drop), int(max_steps), int(check_every), C.byref(n), C.byref(d)))
        return n.value, d.value

    def set_params(self, params: JoeParams):
        """new run-time settings (CFL, ramp, under-relaxation, solver thresholds, EPS) for this handle"""
        jp = make_params(params, self.jp.precision, bool(self.jp.renumber), self.jp.jac_lag)
        _ck(lib().jg_set_params(self.h, C.byref(jp)))
        self.jp = jp
        self.params = params

    def calcGrad(self):
        """calcCvVectorGrad / calcCvScalarGrad of the current state on their own
        (jg_calc_grad), keyed as ``gradients()``"""
        n = self.ncv
        gu, gr, gp, gh = np.empty((n, 3, 3)), np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        _ck(lib().jg_calc_grad(self.h, dptr(gu), dptr(gr), dptr(gp), dptr(gh)))
        return {"grad_u": gu, "grad_rho": gr, "grad_p": gp, "grad_enthalpy": gh}

    def set_cfl_step(self, cfl, step):
        """the CFL and step count the next step's ramp starts from (jg_set_cfl_step)"""
        _ck(lib().jg_set_cfl_step(self.h, float(cfl), int(step)))


def euler_flux_faces(kind, L, R, area, nvec, matrices=True):
    n = L.shape[0]
    L, R, area, nvec = (np.ascontiguousarray(a, np.float64) for a in (L, R, area, nvec))
    F = np.zeros((n, 5))
    AL = np.zeros((n, 5, 5)) if matrices else None
    AR = np.zeros((n, 5, 5)) if matrices else None
    _ck(lib().jg_euler_flux_faces(kind, n, dptr(L), dptr(R), dptr(area), dptr(nvec), dptr(F), _p(AL), _p(AR)))
    return F, AL, AR


def visc_flux_faces(S0, S1, gu0, gu1, gh0, gh1, mul, lamOcp, u_fa, area, nvec, svec, smag, matrices=True):
    """addViscFlux per face on the GPU (jg_visc_flux_faces): (F[n,4], A0[n,5,5], A1[n,5,5])"""
    a = [np.ascontiguousarray(x, np.float64) for x in (S0, S1, gu0, gu1, gh0, gh1, mul, lamOcp, u_fa, area, nvec,
                                                        svec, smag)]
    n = a[0].shape[0]
    F = np.zeros((n, 4))
    A0 = np.zeros((n, 5, 5)) if matrices else None
    A1 = np.zeros((n, 5, 5)) if matrices else None
    L = lib()
    L.jg_visc_flux_faces.argtypes = [C.c_int] + [C.POINTER(C.c_double)] * 16
    _ck(L.jg_visc_flux_faces(n, *[dptr(x) for x in a], dptr(F), _p(A0), _p(A1)))
    return F, A0, A1


class JoeGpuBatch(JoeGpu):
    """Many independent cases advanced together (jg_batch_create): one launch
    per stage over all cases.  ``cases`` is a list of (mesh, JoeParams); the
    cases share one jg_params (the fluid: gamma, R, viscosity law and MU_REF,
    Pr; the solver settings: flux, linear solver, CFL ramp, turbulence model)
    and each brings its own boundary values.  Cases whose shared settings
    differ (two fluids, say) are refused."""

    def __init__(self, cases, precision: int = 0, jac_lag: int = 1, renumber: int = 0):
        self.params = cases[0][1]
        self.mas = [MeshArrays(m, p) for m, p in cases]
        self.jp = make_params(self.params, precision, renumber, jac_lag)
        for k, (_, prm) in enumerate(cases[1:], 1):
            q = make_params(prm, precision, renumber, jac_lag)
            val = lambda x: list(x) if isinstance(x, C.Array) else x  # noqa: E731 (array fields by value)
            diff = [f for f, _ in jg_params._fields_ if val(getattr(q, f)) != val(getattr(self.jp, f))]
            if diff:
                raise ValueError("case %d differs from case 0 in the batch-wide settings %s" % (k, diff))
        arr = (jg_mesh * len(cases))(*[ma.mesh for ma in self.mas])
        h = C.c_void_p()
        _ck(lib().jg_batch_create(len(cases), arr, C.byref(self.jp), C.byref(h)))
        self.h = h
        self.ncases = len(cases)
        self.sizes = [ma.ncv for ma in self.mas]
        self.ncv = sum(self.sizes)
        # the concatenated system's sizes (the single-case calls of the base class use them)
        self.ma = types.SimpleNamespace(ncv=self.ncv, nfa=sum(ma.nfa for ma in self.mas),
                                        nfa_b=sum(ma.nfa_b for ma in self.mas),
                                        nbocv_s=sum(ma.nbocv_s for ma in self.mas))

    def set_case_state(self, k, rho, rhou, rhoE):
        rho, rhou, rhoE = (np.ascontiguousarray(a, np.float64) for a in (rho, rhou, rhoE))
        _ck(lib().jg_batch_set_state(self.h, int(k), dptr(rho), dptr(rhou), dptr(rhoE)))

    def get_case_state(self, k):
        n = self.sizes[k]
        rho, rhou, rhoE = np.empty(n), np.empty((n, 3)), np.empty(n)
        _ck(lib().jg_batch_get_state(self.h, int(k), dptr(rho), dptr(rhou), dptr(rhoE)))
        return rho, rhou, rhoE

    def set_case_scalars(self, k, phi):
        """case k's transported scalars, phi[ncv_k] (SA) or phi[ncv_k][2] (SST)"""
        phi = np.ascontiguousarray(np.asarray(phi, np.float64).reshape(self.sizes[k], self.params.nscal))
        _ck(lib().jg_batch_set_scalars(self.h, int(k), dptr(phi)))

    def get_case_scalars(self, k):
        ns = self.params.nscal
        phi = np.empty((self.sizes[k], ns))
        _ck(lib().jg_batch_get_scalars(self.h, int(k), dptr(phi)))
        return phi[:, 0] if ns == 1 else phi

    def status(self):
        st = (C.c_int * self.ncases)()
        _ck(lib().jg_batch_status(self.h, st))
        return np.array(list(st))

    def set_active(self, k, active):
        _ck(lib().jg_batch_set_active(self.h, int(k), int(bool(active))))

    def runBackwardEulerCases(self, nsteps):
        """residuals [nsteps][ncases][5 + nscal]"""
        r = np.zeros((max(nsteps, 1), self.ncases, self.nvar))
        _ck(lib().jg_batch_step(self.h, int(nsteps), dptr(r)))
        return r[:nsteps]


SERVE_STATUS = {0: "converged", 1: "max_steps", 2: "failed", 3: "stalled"}


class JoeServer:
    """Serving form over the C ABI (jg_serve_*): cases are submitted with their
    mesh, parameters and initial state, admitted by device-memory footprint,
    stepped concurrently (one stream and captured step per case) and retired
    at the residual drop.  ``poll`` runs the progress engine and returns the
    retired cases as dicts; ``fetch`` returns a retired case's final state."""

    def __init__(self, max_resident=32, hbm_budget=0.0, steps_per_poll=20, resid_drop=1e-8, max_steps=20000,
                 max_restarts=2, restart_cfl_factor=0.25, stall_steps=0, admission="fifo", device=0):
        cfg = jg_serve_config(device=device, max_resident=max_resident, hbm_budget=float(hbm_budget),
                              steps_per_poll=steps_per_poll, resid_drop=resid_drop, max_steps=max_steps,
                              max_restarts=max_restarts, restart_cfl_factor=restart_cfl_factor,
                              stall_steps=stall_steps, admission={"fifo": 0, "smallest": 1}[admission])
        h = C.c_void_p()
        _ck(lib().jg_serve_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.sizes = {}

    def close(self):
        if getattr(self, "h", None):
            lib().jg_serve_destroy(self.h)
            self.h = None

    __del__ = close

    def now(self) -> float:
        t = C.c_double()
        _ck(lib().jg_serve_now(self.h, C.byref(t)))
        return t.value

    def submit(self, mesh_src, params: JoeParams, state, precision: int = 0, t_arrival: float = -1.0,
               jac_lag: int = 1, renumber: int = 0) -> int:
        ma = mesh_src if isinstance(mesh_src, MeshArrays) else MeshArrays(mesh_src, params)
        jp = make_params(params, precision, renumber, jac_lag)
        rho, rhou, rhoE = (np.ascontiguousarray(a, np.float64) for a in state)
        i = C.c_longlong()
        _ck(lib().jg_serve_submit(self.h, C.byref(ma.mesh), C.byref(jp), dptr(rho), dptr(rhou), dptr(rhoE),
                                  float(t_arrival), C.byref(i)))
        self.sizes[i.value] = ma.ncv
        return i.value

    def poll(self, max_wait=0.05, cap=64):
        out = (jg_serve_result * cap)()
        n = C.c_int()
        _ck(lib().jg_serve_poll(self.h, float(max_wait), out, cap, C.byref(n)))
        return [{f: getattr(out[k], f) for f, _ in jg_serve_result._fields_} for k in range(n.value)]

    def fetch(self, rid):
        n = self.sizes.pop(rid)
        rho, rhou, rhoE = np.empty(n), np.empty((n, 3)), np.empty(n)
        _ck(lib().jg_serve_fetch(self.h, C.c_longlong(rid), dptr(rho), dptr(rhou), dptr(rhoE)))
        return rho, rhou, rhoE

    def stats(self):
        r, q, f = C.c_int(), C.c_int(), C.c_int()
        b = C.c_double()
        _ck(lib().jg_serve_stats(self.h, C.byref(r), C.byref(q), C.byref(f), C.byref(b)))
        return {"resident": r.value, "queued": q.value, "unfetched": f.value, "bytes_resident": b.value}


def case_footprint(mesh_src, params: JoeParams, precision: int = 0, renumber: bool = False,
                   jac_lag: int = 1) -> float:
    """Device bytes jg_create + jg_set_state allocate for this case."""
    ma = mesh_src if isinstance(mesh_src, MeshArrays) else MeshArrays(mesh_src, params)
    jp = make_params(params, precision, renumber, jac_lag)
    b = C.c_double()
    _ck(lib().jg_case_footprint(C.byref(ma.mesh), C.byref(jp), C.byref(b)))
    return b.value


def renumber_cells(mesh_src, params: JoeParams, method: int = RENUMBER_RCM) -> np.ndarray:
    """The cell order a handle made with ``renumber=method`` uses: the caller's id
    of each cell (reverse Cuthill-McKee, or RCM grouped by Gauss-Seidel colour;
    host only, no GPU needed)."""
    ma = mesh_src if isinstance(mesh_src, MeshArrays) else MeshArrays(mesh_src, params)
    out = np.empty(ma.ncv, np.int32)
    _ck(lib().jg_renumber_cells(C.byref(ma.mesh), int(method), out.ctypes.data_as(C.POINTER(C.c_int))))
    return out
