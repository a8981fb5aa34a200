"""ctypes mirror of the structs in include/joe_b200.h and converters from
the Python-side case description (``case.JoeParams`` + a control-volume
mesh in the reference's layout)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from .case import (AUSM_TYPES, BC_KINDS, FLUX_KINDS, SHOCK_FIX_KINDS, SHOCK_FLAG_KINDS, SOLVER_KINDS, SYMM_BC_KINDS,
                   JoeParams)


class jg_zone(C.Structure):
    _fields_ = [("ifa_f", C.c_int), ("ifa_l", C.c_int), ("kind", C.c_int), ("scal_bc", C.c_int),
                ("v", C.c_double * 8)]


class jg_mesh(C.Structure):
    _fields_ = [("ncv", C.c_int), ("nfa", C.c_int), ("nfa_b", C.c_int), ("nbocv_s", C.c_int),
                ("nzones", C.c_int),
                ("cvofa", C.POINTER(C.c_int)),
                ("faocv_i", C.POINTER(C.c_int)), ("faocv_v", C.POINTER(C.c_int)),
                ("nbocv_i", C.POINTER(C.c_int)), ("nbocv_v", C.POINTER(C.c_int)),
                ("x_cv", C.POINTER(C.c_double)), ("x_fa", C.POINTER(C.c_double)),
                ("fa_normal", C.POINTER(C.c_double)), ("cv_volume", C.POINTER(C.c_double)),
                ("nbocv_lsg_coeff", C.POINTER(C.c_double)),
                ("boundary_fa_lsg_coeff", C.POINTER(C.c_double)),
                ("zones", C.POINTER(jg_zone))]


class jg_params(C.Structure):
    _fields_ = [("gamma", C.c_double), ("R_gas", C.c_double), ("Pr", C.c_double), ("PrTurb", C.c_double),
                ("mu_mode", C.c_int), ("flux", C.c_int),
                ("mu_ref", C.c_double), ("mu_power_law", C.c_double), ("SL_Tref", C.c_double),
                ("SL_Sref", C.c_double), ("T_ref", C.c_double),
                ("second_order", C.c_int), ("limiter", C.c_int), ("eps", C.c_double),
                ("visc_limiter", C.c_int), ("symm_bc", C.c_int),
                ("time_step_mode", C.c_int), ("time_step", C.c_int),
                ("cfl", C.c_double), ("dt", C.c_double),
                ("cfl_after", C.c_int), ("cfl_interval", C.c_int),
                ("cfl_factor", C.c_double), ("cfl_max", C.c_double),
                ("under_relax", C.c_double),
                ("lin_solver", C.c_int), ("ls_max_iter", C.c_int),
                ("ls_abs", C.c_double), ("ls_rel", C.c_double),
                ("precision", C.c_int), ("nscal", C.c_int), ("turb_model", C.c_int), ("renumber", C.c_int),
                ("grad_scheme", C.c_int),
                ("ausm_type", C.c_int), ("shock_fix", C.c_int), ("shock_flag", C.c_int), ("entropy_fix", C.c_int),
                ("jac_lag", C.c_int), ("gravity", C.c_double * 3)]


class jg_serve_config(C.Structure):
    _fields_ = [("device", C.c_int), ("max_resident", C.c_int), ("hbm_budget", C.c_double),
                ("steps_per_poll", C.c_int), ("resid_drop", C.c_double), ("max_steps", C.c_int),
                ("max_restarts", C.c_int), ("restart_cfl_factor", C.c_double), ("stall_steps", C.c_int),
                ("admission", C.c_int)]


class jg_serve_result(C.Structure):
    _fields_ = [("id", C.c_longlong), ("status", C.c_int), ("steps", C.c_int), ("steps_total", C.c_int),
                ("restarts", C.c_int), ("ncv", C.c_int), ("conv_step", C.c_int), ("drop", C.c_double),
                ("t_arrival", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("bytes", C.c_double)]


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int))


def make_params(p: JoeParams, precision: int = 0, renumber: bool = False, jac_lag: int = 1) -> jg_params:
    """jac_lag: form the flux Jacobian blocks every jac_lag-th step (1: every step, as the reference)"""
    q = jg_params()
    q.jac_lag = int(jac_lag)
    for i, g in enumerate((p.GX, p.GY, p.GZ)):
        q.gravity[i] = g
    q.gamma = p.GAMMA
    q.R_gas = p.R_gas
    q.Pr = p.PR
    q.PrTurb = p.PRTURB
    q.mu_mode = 1 if p.MU_MODE == "SUTHERLAND" else 0
    q.flux = FLUX_KINDS[p.SPACE_INTEGRATION]
    if q.flux == 4:
        q.ausm_type = AUSM_TYPES[p.SPACE_INTEGRATION]
        q.shock_fix = SHOCK_FIX_KINDS[p.SHOCK_FIX_TYPE]
        q.shock_flag = SHOCK_FLAG_KINDS[p.SHOCK_FIX_FLAG]
        q.entropy_fix = int(p.ENTROPY_FIX == "EXPANSION_FAN")
    q.mu_ref = p.MU_REF
    q.mu_power_law = p.MU_POWER_LAW
    q.SL_Tref = p.SL_TREF
    q.SL_Sref = p.SL_SREF
    q.T_ref = p.T_REF
    q.second_order = int(p.SECOND_ORDER)
    q.limiter = int(p.LIMITER)
    q.eps = p.EPS
    q.visc_limiter = int(p.VISC_LIMITER)
    q.symm_bc = SYMM_BC_KINDS[p.SYMM_BC]
    q.time_step_mode = 0
    q.time_step = 0 if p.TIME_STEP == "MAX_BASED" else 1
    q.cfl = p.CFL
    q.dt = 0.0
    q.cfl_after, q.cfl_interval, q.cfl_factor, q.cfl_max = p.CFL_RAMP
    q.under_relax = p.UNDER_RELAXATION
    q.lin_solver = SOLVER_KINDS[p.LINEAR_SOLVER_NS]
    q.ls_max_iter = p.LS_MAX_ITER
    q.ls_abs = p.LS_ABS_RESID
    q.ls_rel = p.LS_REL_RESID
    q.precision = precision
    q.nscal = p.nscal
    q.turb_model = {"SA": 1, "SST": 2}.get(p.TURB_MODEL, 0)
    q.renumber = int(renumber)   # False/True: none/RCM; 2: RCM grouped by Gauss-Seidel colour; 3: RCM, LINE lines consecutive
    q.grad_scheme = {"LEASTSQUARES": 0, "GREENGAUSS": 1, "SDWLS": 2}[p.GRAD_SCHEME]
    if q.grad_scheme == 2:
        q.limiter = 0   # SDWLS applies no limiter (limiterNavierS = 0, UgpWithCvCompFlow.h:275-280)
    return q


class MeshArrays:
    """Contiguous arrays (reference layout) + the jg_mesh struct over them.
    ``src`` is a ``geometry.CvMesh`` or a dict of reference dumps."""

    def __init__(self, src, params: JoeParams):
        g = (lambda k: getattr(src, k)) if not isinstance(src, dict) else (lambda k: src[k])
        self.ncv = int(g("ncv")) if not isinstance(src, dict) else int(src["meta"]["ncv"])
        ii = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        dd = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        self.cvofa = ii(g("cvofa")).reshape(-1, 2)
        self.nfa = self.cvofa.shape[0]
        self.faocv_i, self.faocv_v = ii(g("faocv_i")), ii(g("faocv_v"))
        self.nbocv_i, self.nbocv_v = ii(g("nbocv_i")), ii(g("nbocv_v"))
        self.x_cv = dd(g("x_cv")).reshape(-1, 3)
        self.x_fa = dd(g("x_fa")).reshape(-1, 3)
        self.fa_normal = dd(g("fa_normal")).reshape(-1, 3)
        self.cv_volume = dd(g("cv_volume"))
        self.nbocv_lsg_coeff = dd(g("nbocv_lsg_coeff")).reshape(-1, 3)
        self.boundary_fa_lsg_coeff = dd(g("boundary_fa_lsg_coeff")).reshape(-1, 3)
        zones = src["meta"]["zones"] if isinstance(src, dict) else src.zones
        self.nfa_b = int(src["meta"]["nfa_b"]) if isinstance(src, dict) else int(src.nfa_b)
        self.zone_names = [z[0] for z in zones]
        zarr = (jg_zone * max(1, len(zones)))()
        for i, (name, f0, f1) in enumerate(zones):
            bc = params.bcs[name]
            zarr[i].ifa_f, zarr[i].ifa_l = f0, f1
            zarr[i].kind = BC_KINDS[bc.kind]
            vals = list(bc.values) + [0.0] * (8 - len(bc.values))
            bits = 0
            for sc, (kind, v) in enumerate(params.zone_scalar_bcs(name)):
                if kind == "dirichlet":
                    bits |= 1 << sc
                    vals[6 + sc] = v
                elif kind == "hook":
                    bits |= 1 << (4 + sc)
            zarr[i].scal_bc = bits
            for k in range(8):
                zarr[i].v[k] = vals[k]
        self.zarr = zarr
        m = jg_mesh()
        m.ncv, m.nfa, m.nfa_b, m.nbocv_s, m.nzones = (self.ncv, self.nfa, self.nfa_b,
                                                       self.nbocv_v.shape[0], len(zones))
        m.cvofa = iptr(self.cvofa)
        m.faocv_i, m.faocv_v = iptr(self.faocv_i), iptr(self.faocv_v)
        m.nbocv_i, m.nbocv_v = iptr(self.nbocv_i), iptr(self.nbocv_v)
        m.x_cv, m.x_fa, m.fa_normal = dptr(self.x_cv), dptr(self.x_fa), dptr(self.fa_normal)
        m.cv_volume = dptr(self.cv_volume)
        m.nbocv_lsg_coeff = dptr(self.nbocv_lsg_coeff)
        m.boundary_fa_lsg_coeff = dptr(self.boundary_fa_lsg_coeff)
        m.zones = C.cast(zarr, C.POINTER(jg_zone))
        self.mesh = m

    @property
    def nbocv_s(self) -> int:
        return int(self.nbocv_v.shape[0])
