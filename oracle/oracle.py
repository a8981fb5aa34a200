"""ctypes wrapper of the C oracle (oracle/_ref/libjoe_oracle.so, built from
oracle/joe_oracle.c).  Test infrastructure only: the checker for the GPU
library and the CPU "port" baseline of bench.py."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from myjoe_b200.abi import MeshArrays, dptr, jg_mesh, jg_params, make_params

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libjoe_oracle.so")
_lib = None


def build():
    subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        D = C.POINTER(C.c_double)
        L.jo_create.restype = P
        L.jo_create.argtypes = [C.POINTER(jg_mesh), C.POINTER(jg_params)]
        L.jo_destroy.argtypes = [P]
        L.jo_visc_flux_faces.argtypes = [C.c_int] + [D] * 16
        L.jo_set_state.argtypes = [P, D, D, D]
        L.jo_get_state.argtypes = [P, D, D, D]
        L.jo_calc_state.argtypes = [P]
        L.jo_calc_state.restype = C.c_int
        L.jo_calc_dt.argtypes = [P, C.c_double]
        L.jo_calc_dt.restype = C.c_double
        L.jo_calc_rhs.argtypes = [P, D, D, D, D, C.c_int]
        L.jo_solve.argtypes = [P, D, D, D, C.c_double, C.c_double, C.c_int, C.c_int]
        L.jo_solve.restype = C.c_int
        L.jo_step.argtypes = [P, C.c_int, D]
        L.jo_step.restype = C.c_int
        L.jo_array.argtypes = [P, C.c_char_p]
        L.jo_array.restype = D
        L.jo_cfl.argtypes = [P]
        L.jo_cfl.restype = C.c_double
        L.jo_euler_flux_faces.argtypes = [C.c_int, C.c_int, D, D, D, D, D, D, D]
        L.jo_set_scalars.argtypes = [P, D]
        L.jo_get_scalars.argtypes = [P, D]
        L.jo_wall_distance.argtypes = [P]
        L.jo_calc_state_coupled.argtypes = [P]
        L.jo_calc_state_coupled.restype = C.c_int
        L.jo_calc_rhs_coupled.argtypes = [P, D, D, C.c_int]
        L.jo_solve_blocks.argtypes = [P, C.c_int, D, D, D, C.c_int, C.c_int]
        L.jo_step_coupled.argtypes = [P, C.c_int, D]
        L.jo_step_coupled.restype = C.c_int
        L.jo_sa_array.argtypes = [P, C.c_char_p]
        L.jo_sa_array.restype = D
        L.jo_sa_release.argtypes = [P]
        L.jo_linelets.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.jo_line_relax.argtypes = [P, C.c_int, D, D, D, C.c_int]
        L.jo_relax_lines.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.jo_relax_lines.restype = C.c_int
        L.jo_linelets.restype = C.c_int
        _lib = L
    return _lib


_SIZES = {"flux_scale": 5, "vel": 3, "grad_u": 9, "grad_rho": 3, "grad_p": 3, "grad_enthalpy": 3, "vel_bfa": 3, "rhou": 3}
_BFA = {"rho_bfa", "T_bfa", "vel_bfa", "p_bfa", "h_bfa", "gam_bfa", "RoM_bfa"}
_FA = {"mul_fa", "lamOcp_fa", "mut_fa"}


class Oracle:
    def __init__(self, mesh_src, params, precision=0):
        self.params = params
        self.ma = MeshArrays(mesh_src, params)
        self.jp = make_params(params, precision)
        self.h = lib().jo_create(C.byref(self.ma.mesh), C.byref(self.jp))
        self.ncv = self.ma.ncv

    def __del__(self):
        if getattr(self, "h", None):
            lib().jo_sa_release(self.h)
            lib().jo_destroy(self.h)
            self.h = None

    def set_state(self, rho, rhou, rhoE):
        rho, rhou, rhoE = (np.ascontiguousarray(a, np.float64) for a in (rho, rhou, rhoE))
        lib().jo_set_state(self.h, dptr(rho), dptr(rhou), dptr(rhoE))

    def get_state(self):
        n = self.ncv
        rho, rhou, rhoE = np.empty(n), np.empty((n, 3)), np.empty(n)
        lib().jo_get_state(self.h, dptr(rho), dptr(rhou), dptr(rhoE))
        return rho, rhou, rhoE

    def calc_state(self):
        if lib().jo_calc_state(self.h) != 0:
            raise ValueError("unsupported boundary condition")

    def array(self, name):
        if name in _BFA:
            n = self.ma.nfa_b
        elif name in _FA:
            n = self.ma.nfa
        else:
            n = self.ncv
        k = _SIZES.get(name, 1)
        ptr = lib().jo_array(self.h, name.encode())
        a = np.ctypeslib.as_array(ptr, shape=(n * k,)).copy()
        return a.reshape(n, k) if k > 1 else a

    def calc_dt(self, cfl=None):
        return lib().jo_calc_dt(self.h, self.params.CFL if cfl is None else cfl)

    def calc_rhs(self, implicit=True):
        n = self.ncv
        rr, ru, rE = np.zeros(n), np.zeros((n, 3)), np.zeros(n)
        A = np.zeros((self.ma.nbocv_s, 5, 5)) if implicit else None
        lib().jo_calc_rhs(self.h, dptr(rr), dptr(ru), dptr(rE), dptr(A) if implicit else None, int(implicit))
        return rr, ru, rE, A

    def solve(self, A, rhs, zero_abs, zero_rel, max_iter, solver=0, dq0=None):
        dq = np.zeros((self.ncv, 5)) if dq0 is None else np.ascontiguousarray(dq0, np.float64).copy()
        A = np.ascontiguousarray(A, np.float64)
        rhs = np.ascontiguousarray(rhs, np.float64)
        it = lib().jo_solve(self.h, dptr(dq), dptr(A), dptr(rhs), zero_abs, zero_rel, max_iter, solver)
        return dq, it

    def linelets(self):
        """initializeLinelet's lines: (off[nlines+1], cells)"""
        n = lib().jo_linelets(self.h, None, None)
        off = np.zeros(n + 1, np.int32)
        lib().jo_linelets(self.h, off.ctypes.data_as(C.POINTER(C.c_int)), None)
        cv = np.zeros(max(int(off[-1]), 1), np.int32)
        lib().jo_linelets(self.h, off.ctypes.data_as(C.POINTER(C.c_int)), cv.ctypes.data_as(C.POINTER(C.c_int)))
        return off, cv[:off[-1]]

    def relax_lines(self):
        """the LINE relaxation's lines: (off[nlines+1], cells)"""
        n = lib().jo_relax_lines(self.h, None, None)
        off = np.zeros(n + 1, np.int32)
        lib().jo_relax_lines(self.h, off.ctypes.data_as(C.POINTER(C.c_int)), None)
        cv = np.zeros(max(int(off[-1]), 1), np.int32)
        lib().jo_relax_lines(self.h, off.ctypes.data_as(C.POINTER(C.c_int)), cv.ctypes.data_as(C.POINTER(C.c_int)))
        return off, cv[:off[-1]]

    def step(self, nsteps=1):
        r = np.zeros(5)
        err = lib().jo_step(self.h, nsteps, dptr(r))
        if err:
            raise ValueError("oracle step failed")
        return r


class OracleSA(Oracle):
    """The coupled path with a turbulence model: SA (6x6 blocks, nuSA) or SST
    (7x7, kine and omega).  ``set_scalar`` takes phi[ncv] (SA) or phi[ncv][2]."""

    def __init__(self, mesh_src, params, precision=0):
        super().__init__(mesh_src, params, precision)
        self.ns = params.nscal
        self.B = 5 + self.ns
        lib().jo_wall_distance(self.h)

    def set_scalar(self, phi):
        phi = np.ascontiguousarray(np.asarray(phi, np.float64).reshape(self.ncv, self.ns))
        lib().jo_set_scalars(self.h, dptr(phi))

    def get_scalar(self):
        phi = np.empty((self.ncv, self.ns))
        lib().jo_get_scalars(self.h, dptr(phi))
        return phi[:, 0] if self.ns == 1 else phi

    def calc_state(self):
        if lib().jo_calc_state_coupled(self.h) != 0:
            raise ValueError("unsupported boundary condition")

    def sa_array(self, name):
        n = {"phi_bfa": self.ma.nfa_b, "diff": self.ma.nfa, "phi1_bfa": self.ma.nfa_b, "diff1": self.ma.nfa}.get(
            name, self.ncv)
        k = 3 if name in ("grad_phi", "grad_phi1") else 1
        ptr = lib().jo_sa_array(self.h, name.encode())
        a = np.ctypeslib.as_array(ptr, shape=(n * k,)).copy()
        return a.reshape(n, k) if k > 1 else a

    def calc_rhs(self, implicit=True):
        n, B = self.ncv, self.B
        rhs = np.zeros((n, B))
        A = np.zeros((self.ma.nbocv_s, B, B))
        lib().jo_calc_rhs_coupled(self.h, dptr(rhs), dptr(A), int(implicit))
        return rhs, A

    def solve_blocks(self, A, rhs, sweeps, sgs=True, line=False):
        x = np.zeros((self.ncv, self.B))
        A = np.ascontiguousarray(A, np.float64)
        rhs = np.ascontiguousarray(rhs, np.float64)
        if line:
            lib().jo_line_relax(self.h, self.B, dptr(x), dptr(A), dptr(rhs), int(sweeps))
        else:
            lib().jo_solve_blocks(self.h, self.B, dptr(x), dptr(A), dptr(rhs), int(sweeps), int(sgs))
        return x

    def step(self, nsteps=1):
        r = np.zeros(self.B)
        if lib().jo_step_coupled(self.h, nsteps, dptr(r)):
            raise ValueError("oracle step failed")
        return r


def visc_flux_faces(S0, S1, gu0, gu1, gh0, gh1, mul, lamOcp, u_fa, area, nvec, svec, smag, matrices=True):
    """addViscFlux per face (jo_visc_flux_faces): (F[n,4], A0[n,5,5], A1[n,5,5])"""
    a = [np.ascontiguousarray(x, np.float64) for x in (S0, S1, gu0, gu1, gh0, gh1, mul, lamOcp, u_fa, area, nvec,
                                                        svec, smag)]
    n = a[0].shape[0]
    F = np.zeros((n, 4))
    A0 = np.zeros((n, 5, 5)) if matrices else None
    A1 = np.zeros((n, 5, 5)) if matrices else None
    lib().jo_visc_flux_faces(n, *[dptr(x) for x in a], dptr(F), dptr(A0) if matrices else None,
                             dptr(A1) if matrices else None)
    return F, A0, A1


def euler_flux_faces(kind, L, R, area, nvec, matrices=True):
    n = L.shape[0]
    L, R, area, nvec = (np.ascontiguousarray(a, np.float64) for a in (L, R, area, nvec))
    F = np.zeros((n, 5))
    AL = np.zeros((n, 5, 5)) if matrices else None
    AR = np.zeros((n, 5, 5)) if matrices else None
    lib().jo_euler_flux_faces(kind, n, dptr(L), dptr(R), dptr(area), dptr(nvec), dptr(F),
                              dptr(AL) if matrices else None, dptr(AR) if matrices else None)
    return F, AL, AR
