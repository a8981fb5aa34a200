"""Case description for the implicit finite-volume path: the reference's
input-file keys on the hot path (``src/joe/UgpWithCvCompFlow.h:57-502``,
``src/joe/JoeWithModels.cpp:881-924``) as a dataclass, the boundary-condition
table, and the seeded synthetic workloads.

``JoeParams.joe_in()`` renders the same settings as a reference ``Joe.in`` so
that the reference solver and this library run identical cases.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, Tuple

import numpy as np

from . import geometry, meshgen

# boundary kinds (values shared with include/joe_b200.h JG_BC_*)
BC_KINDS = {
    "SYMMETRY": 1, "WALL": 2, "CBC": 3, "CBC_SUBSONIC_INLET": 4,
    "CBC_SUBSONIC_OUTLET": 5, "NEUMANN": 6, "FARFIELD": 7, "NOTHING": 8,
}
FLUX_KINDS = {"HLLC": 0, "ROE": 1, "AUSM": 2, "HAENEL": 3, "AUSMDV": 4, "AUSMV": 4, "AUSMD": 4, "JST": 5}
AUSM_TYPES = {"AUSMDV": 0, "AUSMV": 1, "AUSMD": 2}
SHOCK_FIX_KINDS = {"NONE": 0, "HAENEL": 1, "ALPHA_LR": 2}
SHOCK_FLAG_KINDS = {"CELL_FLAG_HEX": 0, "CELL_FLAG_TET": 1}
SYMM_BC_KINDS = {"ORIGINAL_NUMERIC": 0, "NEW_NUMERIC": 1, "ANALYTICAL": 2}
SOLVER_KINDS = {"BCGSTAB": 0, "LUSGS": 1, "JACOBI": 2, "SGS": 3, "BCGSTAB_LINELET": 4, "LINE": 5}


@dataclasses.dataclass
class BC:
    kind: str
    values: Tuple[float, ...] = ()

    def joe_in(self) -> str:
        if self.kind == "WALL" and self.values and self.values[0] > 0.0:
            return "WALL TEMP %.17g" % self.values[0]
        if self.kind == "WALL":
            return "WALL"
        return " ".join([self.kind] + ["%.17g" % v for v in self.values])


@dataclasses.dataclass
class JoeParams:
    T_REF: float = 300.0
    P_REF: float = 1.0e5
    RHO_REF: float = 1.0e5 / (287.0 * 300.0)
    GAMMA: float = 1.4
    PR: float = 0.72
    PRTURB: float = 0.9
    MU_MODE: str = "POWERLAW"
    MU_REF: float = 0.0
    MU_POWER_LAW: float = 0.76
    SL_TREF: float = 273.15
    SL_SREF: float = 110.4
    SECOND_ORDER: bool = True
    SPACE_INTEGRATION: str = "HLLC"
    LIMITER: bool = True
    EPS: float = 0.01
    GRAD_SCHEME: str = "LEASTSQUARES"   # GRAD_RECONSTRUCTION SCHEME: LEASTSQUARES, GREENGAUSS or SDWLS
    # AUSMDV / AUSMV / AUSMD only (the reference's defaults)
    SHOCK_FIX_TYPE: str = "HAENEL"      # NONE, HAENEL or ALPHA_LR
    SHOCK_FIX_FLAG: str = "CELL_FLAG_HEX"   # or CELL_FLAG_TET
    ENTROPY_FIX: str = "EXPANSION_FAN"  # or NONE
    VISC_LIMITER: bool = True
    SYMM_BC: str = "ORIGINAL_NUMERIC"
    GX: float = 0.0                     # gravity of sourceHook (GX, GY, GZ)
    GY: float = 0.0
    GZ: float = 0.0
    TIME_STEP: str = "MAX_BASED"
    CFL: float = 1.0
    CFL_RAMP: Tuple[int, int, float, float] = (100, 10, 1.0, 100.0)
    NSTEPS: int = 100
    UNDER_RELAXATION: float = 0.3
    LINEAR_SOLVER_NS: str = "BCGSTAB"
    LS_MAX_ITER: int = 30
    LS_ABS_RESID: float = 1.0e-8
    LS_REL_RESID: float = 1.0e-2
    U_INITIAL: Tuple[float, float, float] = (0.0, 0.0, 0.0)
    P_INITIAL: float = 1.0e5
    RHO_INITIAL: float = 1.0e5 / (287.0 * 300.0)
    bcs: Dict[str, BC] = dataclasses.field(default_factory=dict)
    TURB_MODEL: str = "NONE"          # "SA" (coupled 6x6) or "SST" (Menter k-omega SST, coupled 7x7)
    NUSA_INITIAL: float = 0.0         # INITIAL_CONDITION_TURB for SA (nuSA)
    KINE_INITIAL: float = 0.0         # INITIAL_CONDITION_TURB for SST (kine, omega)
    OMEGA_INITIAL: float = 0.0
    # scalar boundary values per zone ("<zone>.<scalar> = v" / "= HOOK"); absent: zero flux.
    # SA: {zone: nuSA}; SST: {zone: (kine or None, omega or "HOOK" or None)}
    scalar_bcs: Dict[str, object] = dataclasses.field(default_factory=dict)

    @property
    def nscal(self) -> int:
        return {"SA": 1, "SST": 2}.get(self.TURB_MODEL, 0)

    @property
    def scalar_names(self):
        return {"SA": ["nuSA"], "SST": ["kine", "omega"]}.get(self.TURB_MODEL, [])

    def zone_scalar_bcs(self, zone):
        """[(kind, value)] per scalar for a zone: kind "dirichlet", "hook" or None."""
        v = self.scalar_bcs.get(zone)
        vals = [v] if (self.TURB_MODEL == "SA" and v is not None) else (list(v) if v is not None else [])
        out = []
        for s in range(self.nscal):
            x = vals[s] if s < len(vals) else None
            if x is None:
                out.append((None, 0.0))
            elif isinstance(x, str):
                out.append(("hook", 0.0))
            else:
                out.append(("dirichlet", float(x)))
        return out

    @property
    def R_gas(self) -> float:
        # ideal gas law as the reference sets it (UgpWithCvCompFlow.h:219)
        return self.P_REF / self.RHO_REF / self.T_REF

    def joe_in(self, restart: str, extra: str = "") -> str:
        L = [
            "RESTART = %s" % restart,
            "T_REF = %.17g" % self.T_REF, "P_REF = %.17g" % self.P_REF, "RHO_REF = %.17g" % self.RHO_REF,
            "GAMMA = %.17g" % self.GAMMA, "PR = %.17g" % self.PR, "PRTURB = %.17g" % self.PRTURB,
            "MU_MODE = %s" % self.MU_MODE, "MU_REF = %.17g" % self.MU_REF,
            "MU_POWER_LAW = %.17g" % self.MU_POWER_LAW, "SL_TREF = %.17g" % self.SL_TREF,
            "SL_SREF = %.17g" % self.SL_SREF,
            "SPACE_INTEGRATION = %s" % self.SPACE_INTEGRATION,
            "SHOCK_FIX_TYPE = %s" % self.SHOCK_FIX_TYPE, "SHOCK_FIX_FLAG = %s" % self.SHOCK_FIX_FLAG,
            "ENTROPY_FIX = %s" % self.ENTROPY_FIX,
            "GRAD_RECONSTRUCTION  SCHEME=%s  LIMITER=%s  EPS=%.17g" % (self.GRAD_SCHEME,
                "YES" if self.LIMITER else "NO", self.EPS),
            "VISC_LIMITER = %s" % ("YES" if self.VISC_LIMITER else "NO"),
            "SYMM_BC = %s" % self.SYMM_BC,
            "GX = %.17g" % self.GX, "GY = %.17g" % self.GY, "GZ = %.17g" % self.GZ,
            "TIME_STEP = %s" % self.TIME_STEP,
            "TIME_INTEGRATION = BACKWARD_EULER",
            "CFL = %.17g" % self.CFL,
            "CFL_RAMP AFTER_ITER=%d  INTERVAL_ITER=%d  FACTOR_CFL=%.17g  MAX_CFL=%.17g" % self.CFL_RAMP,
            "NSTEPS = %d" % self.NSTEPS,
            "UNDER_RELAXATION = %.17g" % self.UNDER_RELAXATION,
            "LINEAR_SOLVER_NS = %s" % self.LINEAR_SOLVER_NS,
            "LINEAR_SOLVER_NS_TRESHOLDS  MAX_ITER=%d  ABS_RESID=%.17g  REL_RESID=%.17g" % (
                self.LS_MAX_ITER, self.LS_ABS_RESID, self.LS_REL_RESID),
            "U_INITIAL = %.17g %.17g %.17g" % tuple(self.U_INITIAL),
            "P_INITIAL = %.17g" % self.P_INITIAL, "RHO_INITIAL = %.17g" % self.RHO_INITIAL,
            ("INITIAL_CONDITION_TURB = %.17g %.17g" % (self.KINE_INITIAL, self.OMEGA_INITIAL)
             if self.TURB_MODEL == "SST" else "INITIAL_CONDITION_TURB = %.17g 0.0" % self.NUSA_INITIAL),
            "CHECK_INTERVAL = 1",
            "INITIAL_FLOWFIELD_OUTPUT = NO",
        ]
        if self.SECOND_ORDER:
            L.append("SPATIAL_SECOND_ORDER")
        for name, bc in self.bcs.items():
            L.append("%s = %s" % (name, bc.joe_in()))
        for name in self.scalar_bcs:
            for (kind, v), sname in zip(self.zone_scalar_bcs(name), self.scalar_names):
                if kind == "dirichlet":
                    L.append("%s.%s = %.17g" % (name, sname, v))
                elif kind == "hook":
                    L.append("%s.%s = HOOK" % (name, sname))
        if extra:
            L.append(extra)
        return "\n".join(L) + "\n"


def perturbed_state(x_cv: np.ndarray, params: JoeParams, amp: float):
    """Uniform initial state from U/P/RHO_INITIAL, smoothly perturbed by
    ``amp`` (the identical formula is compiled into the reference harness,
    oracle/ref_harness.cpp ``perturb``)."""
    n = x_cv.shape[0]
    g = params.GAMMA
    u0 = np.asarray(params.U_INITIAL, float)
    r0 = np.full(n, params.RHO_INITIAL)
    rhou = np.tile(r0[:, None] * u0[None, :], 1)
    rhoE = params.P_INITIAL / (g - 1.0) + 0.5 * params.RHO_INITIAL * float(u0 @ u0)
    rhoE = np.full(n, rhoE)
    if amp == 0.0:
        return r0, rhou, rhoE
    x, y, z = x_cv[:, 0], x_cv[:, 1], x_cv[:, 2]
    a = amp
    f0 = 1.0 + a * np.sin(2.1 * x + 0.3) * np.cos(1.7 * y + 0.2) * (1.0 + 0.3 * np.sin(3.1 * z))
    f1 = a * np.cos(1.3 * x + 0.1) * np.sin(2.3 * y + 0.4)
    f2 = a * np.sin(1.9 * x + 0.7) * np.cos(0.9 * y + 0.5)
    f3 = 0.5 * a * np.sin(2.7 * z + 0.2) * np.cos(1.1 * x)
    f4 = 1.0 + 0.5 * a * np.cos(1.5 * x + 0.6) * np.sin(1.2 * y + 0.8)
    umag = math.sqrt(float(u0 @ u0)) + 1.0
    u = rhou / r0[:, None]
    p0 = (g - 1.0) * (rhoE - 0.5 * r0 * (u * u).sum(1))
    r = r0 * f0
    v = np.stack([u[:, 0] + umag * f1, u[:, 1] + umag * f2, u[:, 2] + umag * f3], 1)
    pp = p0 * f4
    return r, r[:, None] * v, pp / (g - 1.0) + 0.5 * r * (v * v).sum(1)


def perturbed_scalar(x_cv: np.ndarray, value: float, amp: float) -> np.ndarray:
    """Uniform transported scalar times the perturbation factor compiled into
    the reference harness (oracle/ref_harness.cpp ``scal_perturb``)."""
    x, y, z = x_cv[:, 0], x_cv[:, 1], x_cv[:, 2]
    f = 1.0 + amp * np.sin(1.3 * x + 0.4) * np.cos(0.7 * y + 0.1) * (1.0 + 0.2 * np.cos(2.3 * z))
    return value * f


# ----------------------------------------------------------------------------
# seeded workloads
# ----------------------------------------------------------------------------

def bump_case(nx=64, ny=32, nz=4, mach=0.5, p=1.0e5, T=300.0, flux="HLLC", jitter=0.0,
              seed=0, bump_h=0.1, aoa_deg=0.0, shuffle=False, inlet="CBC"):
    """Inviscid channel-with-bump (channel length 3 chords, height 1; the
    bump is bump_h sin^2 on the middle chord): WALL lower, SYMMETRY upper and
    z planes, CBC_SUBSONIC_OUTLET at p.  ``inlet="CBC"`` prescribes the inflow
    state (u, T, p), i.e. the mass flow; ``inlet="TOTAL"`` prescribes total
    pressure and temperature for the inflow Mach number and direction
    (CBC_SUBSONIC_INLET), so the mass flow follows from the pressure ratio and
    a choked throat with a shock is a valid steady state; ``inlet="FARFIELD"``
    makes inlet, outlet and top far-field boundaries (flow over a bump at an
    angle of attack)."""
    gam, R = 1.4, 287.0
    rho = p / (R * T)
    c = math.sqrt(gam * R * T)
    a = math.radians(aoa_deg)
    u = (mach * c * math.cos(a), mach * c * math.sin(a), 0.0)
    raw = meshgen.channel_bump(nx, ny, nz, bump_h=bump_h, jitter=jitter, seed=seed)
    bcs = {"outlet": BC("CBC_SUBSONIC_OUTLET", (p,)), "lower": BC("WALL"), "upper": BC("SYMMETRY"),
           "sides": BC("SYMMETRY")}
    if inlet == "TOTAL":
        f = 1.0 + 0.5 * (gam - 1.0) * mach * mach
        bcs["inlet"] = BC("CBC_SUBSONIC_INLET", (math.cos(a), math.sin(a), 0.0, T * f, p * f ** (gam / (gam - 1.0))))
    elif inlet == "FARFIELD":
        # external flow over the bump: Riemann-invariant far field on inlet, outlet and top
        ff = BC("FARFIELD", u + (p, rho, gam))
        bcs.update(inlet=ff, outlet=ff, upper=ff)
    else:
        bcs["inlet"] = BC("CBC", u + (T, p))
    prm = JoeParams(T_REF=T, P_REF=p, RHO_REF=rho, GAMMA=gam, SPACE_INTEGRATION=flux,
                    U_INITIAL=u, P_INITIAL=p, RHO_INITIAL=rho, bcs=bcs)
    return raw, geometry.build_cv_mesh(raw, seed=seed, shuffle=shuffle), prm


def plate_case(nx=256, ny=96, nz=2, mach=0.3, re_l=1.0e5, p=1.0e5, T=300.0, flux="ROE"):
    """Laminar flat plate, Sutherland viscosity, Pr 0.72: CBC inlet and top,
    CBC_SUBSONIC_OUTLET outlet, SYMMETRY ahead of the plate and on the z
    planes, adiabatic WALL on the plate.  The plate length is set so that
    Re_L = rho U L / mu(T) equals ``re_l``."""
    gam, R = 1.4, 287.0
    rho = p / (R * T)
    c = math.sqrt(gam * R * T)
    U = mach * c
    mu_ref, tref, sref = 1.716e-5, 273.15, 110.4
    mu = mu_ref * (T / tref) ** 1.5 * (tref + sref) / (T + sref)
    L = re_l * mu / (rho * U)
    raw = meshgen.flat_plate(nx, ny, nz, plate_length=L, lead=0.25 * L, re_l=re_l)
    u = (U, 0.0, 0.0)
    prm = JoeParams(T_REF=T, P_REF=p, RHO_REF=rho, GAMMA=gam, SPACE_INTEGRATION=flux,
                    MU_MODE="SUTHERLAND", MU_REF=mu_ref, SL_TREF=tref, SL_SREF=sref, PR=0.72,
                    U_INITIAL=u, P_INITIAL=p, RHO_INITIAL=rho,
                    bcs={"inlet": BC("CBC", u + (T, p)), "outlet": BC("CBC_SUBSONIC_OUTLET", (p,)),
                         "lower_sym": BC("SYMMETRY"), "plate": BC("WALL"),
                         "upper": BC("CBC", u + (T, p)), "sides": BC("SYMMETRY")})
    return raw, geometry.build_cv_mesh(raw), prm


def sa_bump_case(nx=64, ny=32, nz=2, mach=0.7, re=3.0e6, p=1.0e5, T=300.0, bump_h=0.1, jitter=0.0, seed=0,
                 stretch=1.0, inlet="FARFIELD", nu_factor=3.0, n_prism=0, shuffle=False, alternate=False,
                 aoa_deg=0.0, mu_ref=None):
    """Turbulent (SA) flow over the channel bump: viscous WALL lower (nuSA = 0),
    HLLC, Sutherland viscosity with MU_REF set so that the Reynolds number on
    the bump chord (length 1) is ``re``; inflow nuSA = ``nu_factor`` x the
    kinematic viscosity (the usual SA free-stream value), far-field inlet,
    outlet and top (or CBC inlet with ``inlet="CBC"``), SYMMETRY z planes.
    ``stretch`` > 1 clusters the rows towards the lower wall.  ``n_prism`` > 0
    meshes that many wall rows with triangular prisms (``channel_bump_mixed``);
    ``shuffle`` permutes cells and faces from ``seed``; ``aoa_deg`` tilts the
    inflow (far-field inlet).  ``mu_ref`` given fixes the fluid instead (``re``
    is then unused): cases of one batch share it."""
    gam, R = 1.4, 287.0
    rho = p / (R * T)
    c = math.sqrt(gam * R * T)
    U = mach * c
    tref, sref = 273.15, 110.4
    sutherland = (T / tref) ** 1.5 * (tref + sref) / (T + sref)
    if mu_ref is None:
        mu_ref = rho * U * 1.0 / re / sutherland
    mu = mu_ref * sutherland
    nu_inf = nu_factor * mu / rho
    a = math.radians(aoa_deg)
    u = (U * math.cos(a), U * math.sin(a), 0.0)
    if n_prism > 0:
        raw = meshgen.channel_bump_mixed(nx, ny, nz, n_prism=n_prism, bump_h=bump_h, jitter=jitter, seed=seed,
                                         stretch=stretch, alternate=alternate)
    else:
        raw = meshgen.channel_bump(nx, ny, nz, bump_h=bump_h, jitter=jitter, seed=seed, stretch=stretch)
    bcs = {"lower": BC("WALL"), "sides": BC("SYMMETRY")}
    if inlet == "CBC":
        bcs.update(inlet=BC("CBC", u + (T, p)), outlet=BC("CBC_SUBSONIC_OUTLET", (p,)), upper=BC("SYMMETRY"))
        sbc = {"inlet": nu_inf, "lower": 0.0}
    else:
        ff = BC("FARFIELD", u + (p, rho, gam))
        bcs.update(inlet=ff, outlet=ff, upper=ff)
        sbc = {"inlet": nu_inf, "outlet": nu_inf, "upper": nu_inf, "lower": 0.0}
    prm = JoeParams(T_REF=T, P_REF=p, RHO_REF=rho, GAMMA=gam, SPACE_INTEGRATION="HLLC", MU_MODE="SUTHERLAND",
                    MU_REF=mu_ref, SYMM_BC="ANALYTICAL", U_INITIAL=u, P_INITIAL=p, RHO_INITIAL=rho, bcs=bcs,
                    TURB_MODEL="SA", NUSA_INITIAL=nu_inf, scalar_bcs=sbc)
    return raw, geometry.build_cv_mesh(raw, seed=seed, shuffle=shuffle), prm


def sst_bump_case(nx=64, ny=32, nz=2, mach=0.7, re=3.0e6, p=1.0e5, T=300.0, bump_h=0.1, jitter=0.0, seed=0,
                  stretch=1.0, inlet="FARFIELD", tu=0.005, visc_ratio=0.1, n_prism=0, shuffle=False,
                  alternate=False, aoa_deg=0.0, mu_ref=None):
    """Turbulent (Menter SST) flow over the channel bump, set up like
    ``sa_bump_case``: free-stream k = 1.5 (tu U)^2 and omega from the
    free-stream eddy-viscosity ratio mu_t/mu = ``visc_ratio``; at the wall
    k = 0 and omega from the model's wall hook (60 nu / (beta_1 d^2))."""
    raw, g, prm = sa_bump_case(nx, ny, nz, mach=mach, re=re, p=p, T=T, bump_h=bump_h, jitter=jitter, seed=seed,
                               stretch=stretch, inlet=inlet, n_prism=n_prism, shuffle=shuffle, alternate=alternate,
                               aoa_deg=aoa_deg, mu_ref=mu_ref)
    U = math.hypot(prm.U_INITIAL[0], prm.U_INITIAL[1])
    rho = prm.RHO_INITIAL
    tref, sref = 273.15, 110.4
    mu = prm.MU_REF * (T / tref) ** 1.5 * (tref + sref) / (T + sref)
    k = 1.5 * (tu * U) ** 2
    om = rho * k / (visc_ratio * mu)
    sbc = {z: (k, om) for z, v in prm.scalar_bcs.items() if z != "lower"}
    sbc["lower"] = (0.0, "HOOK")
    prm = dataclasses.replace(prm, TURB_MODEL="SST", NUSA_INITIAL=0.0, KINE_INITIAL=k, OMEGA_INITIAL=om,
                              scalar_bcs=sbc)
    return raw, g, prm
