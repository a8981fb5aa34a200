/*
 * joe_b200.h -- C ABI of the B200 implicit finite-volume library (libjoe_b200.so).
 *
 * Drop-in for the implicit iteration of the Joe RANS solver (MUM suite):
 * the host keeps the reference's mesh objects (Ugp / UgpWithCv) and hands
 * their arrays, in the reference's own layouts, to these entry points.
 * Every call returns an int status (JG_OK == 0, < 0 on error; the
 * reference's `throw(-1)`), never throws across the ABI, and never reads
 * host memory after it returns.  A handle is used by one thread at a time;
 * distinct handles run concurrently on their own CUDA streams.
 *
 * Layouts (all host arrays, caller-owned, reference order):
 *   cvofa[nfa][2]            boundary faces first (cvofa[f][1] == -1), zones contiguous
 *   faocv_i[ncv+1]/faocv_v   faces of a cell, CSR
 *   nbocv_i[ncv+1]/nbocv_v   cell neighbours, CSR, diagonal first
 *   x_cv[ncv][3], cv_volume[ncv], x_fa[nfa][3], fa_normal[nfa][3] (area-weighted,
 *   pointing from cvofa[f][0] to cvofa[f][1])
 *   nbocv_lsg_coeff[nbocv_s][3], boundary_fa_lsg_coeff[nfa_b][3]
 *   rho[ncv], rhou[ncv][3], rhoE[ncv]
 *   A[nbocv_s][5][5] (block CSR over nbocv), rhs/dq[ncv][5]
 */
#ifndef JOE_B200_H
#define JOE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define JG_OK 0
#define JG_ERR_ARG (-1)       /* bad argument / unsupported option */
#define JG_ERR_CUDA (-2)      /* CUDA runtime error (message: jg_last_error) */
#define JG_ERR_NOMEM (-3)     /* device allocation failed */
#define JG_ERR_STATE (-4)     /* non-physical state (NaN, rho<=0) detected */
#define JG_ERR_NODEVICE (-5)  /* no CUDA device */
#define JG_ERR_IO (-6)        /* file cannot be opened, read or written, or is not in the expected format */

/* boundary kinds: setBC, src/joe/JoeWithModels.cpp:3857-4300 */
enum {
  JG_BC_SYMMETRY = 1,             /* v: -                                   */
  JG_BC_WALL = 2,                 /* v[0] = wall T (<= 0: adiabatic)         */
  JG_BC_CBC = 3,                  /* v[0..2] = u, v[3] = T, v[4] = p         */
  JG_BC_CBC_SUBSONIC_INLET = 4,   /* v[0..2] = flow direction, v[3] = Ttot, v[4] = ptot */
  JG_BC_CBC_SUBSONIC_OUTLET = 5,  /* v[0] = p                                */
  JG_BC_NEUMANN = 6,              /* v: -                                    */
  JG_BC_FARFIELD = 7              /* v[0..2] = u, v[3] = p, v[4] = rho, v[5] = gamma */
};
/* SPACE_INTEGRATION: HLLC, ROE, AUSM (implicit side: the HLLC matrices) and HAENEL
 * (Haenel & Schwane, calcEulerFlux_HAENEL / calcEulerFluxMatrices_HAENEL,
 * UgpWithCvCompFlow.cpp:1329-1505; also AUSMDV with SHOCK_FIX_TYPE = HAENEL) */
/* JST: Jameson-Schmidt-Turkel central flux with blended second / fourth difference dissipation
 * (calcEulerFlux_JST, UgpWithCvCompFlow.cpp:4050-4160; the pressure sensor, spectral radii and
 * undivided Laplacian of calcJSTCoeff_Const / calcJSTCoeff_Var, JoeWithModels.cpp:13380-13492,
 * recomputed every residual); implicit side: the HLLC matrices (JoeWithModels.cpp:3067-3071) */
enum { JG_FLUX_HLLC = 0, JG_FLUX_ROE = 1, JG_FLUX_AUSM = 2, JG_FLUX_HAENEL = 3, JG_FLUX_AUSMDV = 4, JG_FLUX_JST = 5 };
enum { JG_MU_POWERLAW = 0, JG_MU_SUTHERLAND = 1 };
enum { JG_SYMM_ORIGINAL_NUMERIC = 0, JG_SYMM_NEW_NUMERIC = 1, JG_SYMM_ANALYTICAL = 2 };
enum { JG_TS_CFL = 0, JG_TS_CFL_MIN = 1, JG_TS_DT = 2 };
enum { JG_DT_MAX_BASED = 0, JG_DT_SUM_BASED = 1 };
/* linear solvers: BCGSTAB and LUSGS follow the reference (UgpWithCv.cpp:2660, 3172);
 * JACOBI / SGS are block point relaxation (fixed sweep count) */
enum { JG_LS_BCGSTAB = 0, JG_LS_LUSGS = 1, JG_LS_JACOBI = 2, JG_LS_SGS = 3,
       /* BCGSTAB_LINELET: BiCGSTAB preconditioned by block-tridiagonal solves along the
        * wall-normal lines of initializeLinelet (JoeWithModels.cpp:7471-7559) and the
        * block diagonal elsewhere, solveCvVectorR5BcgstabLine (UgpWithCv.cpp:3627-3992) */
       JG_LS_BCGSTAB_LINELET = 4,
       /* LINE (no reference counterpart; the reference's coupled solve is PETSc): ls_max_iter
        * block line-Jacobi sweeps from zero: the block-tridiagonal system of every line solved
        * exactly (block Thomas), the block diagonal on the other cells, the couplings across
        * lines lagged.  The lines follow initializeLinelet's rule from the faces of every
        * WALL zone, except that where several neighbours pass a line goes on to the strongest
        * coupling if it is 1.1 times the next (so it crosses prism/hexahedron interfaces).
        * 5x5 and coupled paths, FP64 or mixed, single cases and batches. */
       JG_LS_LINE = 5 };
enum { JG_PREC_FP64 = 0, JG_PREC_MIXED = 1 };

typedef struct jg_zone {
  int ifa_f, ifa_l;   /* inclusive boundary-face range */
  int kind;           /* JG_BC_* */
  int scal_bc;        /* bit s set: transported scalar s is Dirichlet here with value v[6+s]
                         (Joe.in key "<zone>.<scalar> = value", Scalars.cpp:289-360);
                         bit 4+s: the model's HOOK boundary ("<zone>.<scalar> = HOOK");
                         neither: zero flux (phi_bfa = phi of the cell) */
  double v[8];        /* parameters, see JG_BC_* (v[6], v[7]: scalar Dirichlet values) */
} jg_zone;

typedef struct jg_mesh {
  int ncv, nfa, nfa_b, nbocv_s, nzones;
  const int *cvofa;
  const int *faocv_i, *faocv_v;
  const int *nbocv_i, *nbocv_v;
  const double *x_cv, *x_fa, *fa_normal, *cv_volume;
  const double *nbocv_lsg_coeff, *boundary_fa_lsg_coeff;
  const jg_zone *zones;
} jg_mesh;

/* Input-file keys of the hot path (UgpWithCvCompFlow.h:57-502, JoeWithModels.cpp:881-924). */
typedef struct jg_params {
  double gamma;        /* GAMMA */
  double R_gas;        /* P_REF / RHO_REF / T_REF */
  double Pr, PrTurb;   /* PR, PRTURB */
  int mu_mode;         /* MU_MODE: JG_MU_* (used when mu_ref > 0) */
  int flux;            /* SPACE_INTEGRATION: JG_FLUX_* */
  double mu_ref, mu_power_law, SL_Tref, SL_Sref, T_ref;
  int second_order;    /* SPATIAL_SECOND_ORDER */
  int limiter;         /* GRAD_RECONSTRUCTION LIMITER=YES */
  double eps;          /* GRAD_RECONSTRUCTION EPS */
  int visc_limiter;    /* VISC_LIMITER */
  int symm_bc;         /* SYMM_BC: JG_SYMM_* */
  int time_step_mode;  /* JG_TS_* */
  int time_step;       /* TIME_STEP: JG_DT_* */
  double cfl, dt;      /* CFL (or CFL_MIN) and DT */
  int cfl_after, cfl_interval;   /* CFL_RAMP AFTER_ITER, INTERVAL_ITER */
  double cfl_factor, cfl_max;    /* CFL_RAMP FACTOR_CFL, MAX_CFL */
  double under_relax;  /* UNDER_RELAXATION */
  int lin_solver;      /* LINEAR_SOLVER_NS: JG_LS_* */
  int ls_max_iter;     /* LINEAR_SOLVER_NS_TRESHOLDS MAX_ITER (BCGSTAB) or sweeps (JACOBI/SGS) */
  double ls_abs, ls_rel;
  int precision;       /* JG_PREC_* */
  int nscal;           /* transported scalars: 0 (laminar / inviscid), 1 (SA), 2 (SST) */
  int turb_model;      /* JG_TURB_*: with a model the case runs runBackwardEulerCoupled's
                          (5+nscal)^2 block system (JoeWithModels.cpp:4326-4611) */
  int renumber;        /* JG_RENUMBER_*: the handle's own cell/face order (a batch renumbers each case on its own) */
  int grad_scheme;     /* GRAD_RECONSTRUCTION SCHEME: JG_GRAD_* (the flow gradients of calcEulerFlux) */
  /* AUSMDV family (flux = JG_FLUX_AUSMDV; UgpWithCvCompFlow.h:198-234): */
  int ausm_type;       /* SPACE_INTEGRATION AUSMDV / AUSMV / AUSMD: JG_AUSM_* */
  int shock_fix;       /* SHOCK_FIX_TYPE: JG_SHOCK_FIX_* */
  int shock_flag;      /* SHOCK_FIX_FLAG: JG_SHOCK_FLAG_* */
  int entropy_fix;     /* ENTROPY_FIX EXPANSION_FAN: 1, NONE: 0 */
  /* Lagged Jacobian (no reference counterpart; the reference forms the blocks every
   * step): 0 or 1 forms the flux Jacobian blocks every step; k > 1 forms them every
   * k-th step of each case (and at its first step after a new state), adding each
   * step's own vol/dt to the kept diagonal.  The residual and the update are exact
   * every step, so the converged field does not depend on it.  Cases without a
   * turbulence model, captured linear solvers (JACOBI, SGS, LINE, LUSGS). */
  int jac_lag;
  /* GX, GY, GZ: the gravity of JoeWithModels::sourceHook / sourceHookCoupled
   * (src/joe/JoeWithModels.h:111-152), added to the momentum and energy rows of the
   * residual and to the diagonal blocks (zero: none) */
  double gravity[3];
} jg_params;
/* AUSMDV (Wada & Liou, calcEulerFlux_AUSMDV / calcEulerFluxMatrices_AUSMDV,
 * UgpWithCvCompFlow.cpp:879-1322): the AUSMD / AUSMV blend, the entropy fix for
 * single expansion waves, and the shock fix of JoeWithModels.cpp:2753-2781 and
 * 2933-2957: every step the cells beside a sonic internal face are flagged; an
 * internal face whose two cells are flagged (JG_SHOCK_FLAG_HEX; either cell:
 * JG_SHOCK_FLAG_TET), sonic faces included (the reference defines
 * SHOCKFIX_ACROSS_SHOCK), takes the Haenel & Schwane flux (JG_SHOCK_FIX_HAENEL)
 * or AUSMDV with alpha from the densities (JG_SHOCK_FIX_ALPHA_LR).
 * Boundary faces take AUSMDV without the shock fix.  Cases without a turbulence model. */
enum { JG_AUSM_DV = 0, JG_AUSM_V = 1, JG_AUSM_D = 2 };
enum { JG_SHOCK_FIX_NONE = 0, JG_SHOCK_FIX_HAENEL = 1, JG_SHOCK_FIX_ALPHA_LR = 2 };
enum { JG_SHOCK_FLAG_HEX = 0, JG_SHOCK_FLAG_TET = 1 };
/* JG_GRAD_LSQ: least squares (calcCvScalarGrad / calcCvVectorGrad, UgpWithCv.h:1009-1083);
 * JG_GRAD_GREENGAUSS: Green-Gauss with distance-weighted face values
 * (calcCvScalarGradGreenGauss / calcCvVectorGradGreenGauss, UgpWithCv.h:1091-1184, GG_WITH_DIST);
 * both followed by the same Barth-Jespersen limiter.
 * JG_GRAD_SDWLS: solution-dependent weighted least squares (calcCvScalarGradSDWLS /
 * calcCvVectorGradSDWLS, UgpWithCv.h:1418-1800): per cell and per quantity, the neighbours and
 * boundary faces weighted 1 / (|dx|^2 (|dphi| + eps ref)), ref = rho, p, h, and the speed of sound
 * for the velocity; no limiter (limiter must be 0, as the reference sets it).
 * Green-Gauss and SDWLS: cases without a turbulence model. */
enum { JG_GRAD_LSQ = 0, JG_GRAD_GREENGAUSS = 1, JG_GRAD_SDWLS = 2 };
/* Cell and face order inside a handle.  JG_RENUMBER_NONE keeps the caller's
 * order (a mesh the reference loaded is already in reverse Cuthill-McKee
 * order, Ugp::init, src/common/Ugp.cpp:3389-3399).  JG_RENUMBER_RCM renumbers
 * cells by reverse Cuthill-McKee and sorts faces by their cells inside the
 * handle; every entry point still takes and returns arrays in the caller's
 * order (cells, faces and nbocv entries), so only the speed changes.  Block
 * Jacobi steps and calcRhs give bit-identical results either way; the L1
 * residual sum and the Gauss-Seidel colouring follow the internal order. */
/* JG_RENUMBER_RCM_COLOR: the RCM order grouped by Gauss-Seidel colour, so that each colour
 * pass of the SGS relaxation reads a contiguous part of the matrix; the same colour classes,
 * so SGS gives the same bits as with JG_RENUMBER_RCM. */
/* JG_RENUMBER_RCM_LINES: the RCM order with the cells of each LINE relaxation line made
 * consecutive, in line order from the wall (each line placed where RCM meets its first cell;
 * the lines are the handle's own, built from the WALL zones by the relaxed rule of
 * JG_LS_LINE).  The line factorisation and substitutions then stream each line's blocks, and
 * the gathers of a cell's off-line neighbours read the next line's consecutive cells.  Per-cell
 * operations keep their operands and order, so results are those of JG_RENUMBER_RCM; a mesh
 * without WALL faces gets the RCM order. */
enum { JG_RENUMBER_NONE = 0, JG_RENUMBER_RCM = 1, JG_RENUMBER_RCM_COLOR = 2, JG_RENUMBER_RCM_LINES = 3 };
/* turbulence models, with the reference's default constants:
 *   JG_TURB_SA  Spalart-Allmaras (src/joe/turbModels/TurbModel_SA.h): nscal 1, nuSA (1e-10 .. 1)
 *   JG_TURB_SST Menter k-omega SST (TurbModel_KOMSST.h): nscal 2, kine (1e-10 .. 1e10) and
 *               omega (1e-4 .. 1e15); Pk limiter on, shear-stress limiter = vorticity;
 *               zone.scal_bc bit 4+s marks the model's HOOK boundary for scalar s (SST:
 *               omega on a WALL = 60 mu / (rho beta_1 d^2)) */
enum { JG_TURB_NONE = 0, JG_TURB_SA = 1, JG_TURB_SST = 2 };


typedef struct jg_case jg_case_t;   /* opaque per-case handle (device state + stream + graph) */

/* Library / errors ---------------------------------------------------------- */
int jg_version(void);
const char *jg_last_error(void);   /* message of the last failing call on this thread */
int jg_device_count(int *n);

/* Case lifetime: replaces UgpWithCvCompFlow::initializeFromRestartFile's
 * data setup (src/joe/UgpWithCvCompFlow.h:504-583) for the GPU: the mesh
 * arrays are copied to device memory owned by the handle. */
int jg_create(const jg_mesh *mesh, const jg_params *params, jg_case_t **out);
int jg_destroy(jg_case_t *h);
int jg_get_stream(jg_case_t *h, void **cuda_stream);   /* cudaStream_t of the case */

/* Conserved state in/out (rho[ncv], rhou[ncv][3], rhoE[ncv]).  jg_set_state
 * also runs the runBackwardEuler preamble (src/joe/JoeWithModels.cpp:942-957):
 * calcStateVariables + calcMaterialProperties + setBC. */
int jg_set_state(jg_case_t *h, const double *rho, const double *rhou, const double *rhoE);
int jg_get_state(jg_case_t *h, double *rho, double *rhou, double *rhoE);

/* calcStateVariables (UgpWithCvCompFlow.h:1662-1694) + calcMaterialProperties
 * (1701-1753) + setBC (JoeWithModels.cpp:3857-4300) on the current state. */
int jg_calc_state(jg_case_t *h);
/* primitive cell state (vel[ncv][3], press, temp, enthalpy, sos); any pointer may be NULL */
int jg_get_primitives(jg_case_t *h, double *vel, double *press, double *temp, double *enthalpy, double *sos);
/* boundary-face state after setBC (rho_bfa, vel_bfa[nfa_b][3], p_bfa, T_bfa, h_bfa)
 * and face viscosities mul_fa[nfa], lamOcp_fa[nfa]; any pointer may be NULL */
int jg_get_bfa(jg_case_t *h, double *rho_bfa, double *vel_bfa, double *p_bfa, double *T_bfa, double *h_bfa,
               double *mul_fa, double *lamOcp_fa);

/* UgpWithCvCompFlow::calcDt (src/joe/UgpWithCvCompFlow.cpp:5-110): local time
 * step per cell (local_dt[ncv], may be NULL) and its minimum. */
int jg_calc_dt(jg_case_t *h, double cfl, double *dt_min, double *local_dt);

/* JoeWithModels::calcRhs (src/joe/JoeWithModels.cpp:2564-2619): gradients,
 * Euler + viscous fluxes, residual; with flagImplicit and A != NULL also the
 * block Jacobian A[nbocv_s][5][5] in the reference's CSR layout. */
int jg_calc_rhs(jg_case_t *h, double *rhs_rho, double *rhs_rhou, double *rhs_rhoE, double *A, int flagImplicit);

/* Coupled path (jg_params.turb_model = JG_TURB_SA with nscal = 1, or
 * JG_TURB_SST with nscal = 2 (kine, omega); HLLC, JACOBI or SGS relaxation).  The handle computes the wall distance at creation
 * (calcWallDistance, UgpWithCvCompFlow.h:1395-1535).  Transported scalars
 * phi[ncv][nscal] (nuSA; ScalarTranspEq phi) in/out: set them after
 * jg_set_state, before the first step.  jg_calc_rhs_coupled is
 * JoeWithModels::calcRhsCoupled (JoeWithModels.cpp:4597-4611) with
 * RansTurbSA's hooks: rhs[ncv][5+nscal], A[nbocv_s][5+nscal][5+nscal] (NULL:
 * residual only).  jg_step on such a handle runs runBackwardEulerCoupled's
 * iteration (4416-4529) and reports resid[nsteps][5+nscal].  jg_get_turb
 * returns the model arrays of the current state (any pointer may be NULL):
 * wallDist[ncv], mut_fa[nfa], strMag[ncv], vortMag[ncv], phi_bfa[nfa_b],
 * grad_phi[ncv][3], diff[nfa] (scalar diffusivity). */
int jg_set_scalars(jg_case_t *h, const double *phi);
int jg_get_scalars(jg_case_t *h, double *phi);
int jg_calc_rhs_coupled(jg_case_t *h, double *rhs, double *A, int flagImplicit);
int jg_get_turb(jg_case_t *h, double *wallDist, double *mut_fa, double *strMag, double *vortMag, double *phi_bfa,
                double *grad_phi, double *diff);
/* one model array by the reference's name: "wallDist", "strMag", "vortMag",
 * "diverg", "crossDiff", "blendFuncF1", "blendFuncF2" ([ncv], the last four
 * SST only), "mut_fa" [nfa], and per scalar s, component-major: "phi_bfa"
 * [nscal][nfa_b], "grad_phi" [nscal][ncv][3], "diff" [nscal][nfa] */
int jg_get_turb_array(jg_case_t *h, const char *name, double *out);
/* gradients of the last jg_calc_rhs / step: calcCvVectorGrad / calcCvScalarGrad
 * with limiting (src/common/UgpWithCv.h:803-1083); grad_u[ncv][3][3], others [ncv][3].
 * grad_u is what the reference holds after calcRhs: the viscous gradient when
 * MU_REF > 0 (unlimited under VISC_LIMITER=NO), else the Euler one. */
int jg_get_gradients(jg_case_t *h, double *grad_u, double *grad_rho, double *grad_p, double *grad_h);
/* the same gradients of the current state computed on their own (calcRhs's
 * first pass), without the face loop; 5x5 handles, second order or viscous */
int jg_calc_grad(jg_case_t *h, double *grad_u, double *grad_rho, double *grad_p, double *grad_h);

/* UgpWithCvCompFlow::solveCoupledLinSysNS (src/joe/UgpWithCvCompFlow.h:899-950):
 * solves A dq = rhs with the solver of jg_params.lin_solver; dq is the initial
 * guess on entry (BCGSTAB) and the solution on exit.  Also exported as
 * solveLinSysNSCoupled. */
int jg_solve_lin_sys(jg_case_t *h, double *dq, const double *A, const double *rhs, double zeroAbs, double zeroRel,
                     int maxIter, int *iters);
int solveLinSysNSCoupled(jg_case_t *h, double *dq, const double *A, const double *rhs, double zeroAbs,
                         double zeroRel, int maxIter, int *iters);

/* nsteps iterations of the JoeWithModels::runBackwardEuler loop body
 * (src/joe/JoeWithModels.cpp:975-1159): CFL ramp, calcDt, calcRhs, linear
 * solve, update, state + BC.  resid[nsteps][5] (may be NULL) receives the L1
 * residual of every step.  Returns JG_ERR_STATE on a negative density or
 * pressure or a NaN residual (doneSolver, JoeWithModels.h:42-95). */
int jg_step(jg_case_t *h, int nsteps, double *resid);
/* the same steps enqueued on the case stream without synchronising */
int jg_step_async(jg_case_t *h, int nsteps);
/* A host-resident state stepped in place: jg_set_state(rho, rhou, rhoE) + jg_step(nsteps, resid)
 * + jg_get_state into the same arrays, with one synchronisation (the three calls make three); for
 * a caller that keeps the state on the host between steps, as the reference's loop does.  Pinned
 * host arrays make the copies asynchronous DMA.  A single case (not a batch handle).  Returns
 * JG_ERR_STATE if the uploaded or a stepped state is non-physical (the arrays then hold the last
 * state the device computed). */
int jg_step_host(jg_case_t *h, double *rho, double *rhou, double *rhoE, int nsteps, double *resid);
int jg_get_cfl_step(jg_case_t *h, double *cfl, int *step);
/* sets the CFL and the step count the next step's ramp starts from (the
 * reference's `cfl` and `step` members, e.g. after reading a restart) */
int jg_set_cfl_step(jg_case_t *h, double cfl, int step);
/* runBackwardEuler until a residual rule stops it, or max_steps steps.
 * resid_drop >= 0: a RELATIVE drop, the energy residual at or below
 * resid_drop x the first step's (not the reference's rule).  resid_drop < 0:
 * the reference's doneSolver rule (JoeWithModels.h:64, RESID_ENERG_TH): the
 * absolute energy residual strictly below -resid_drop.  The residual is checked
 * every check_every steps (1: step by step as the reference; more: fewer host
 * round trips, the state then up to check_every - 1 steps past the step that
 * met the rule).  steps / drop (may be NULL): steps run and the last step's
 * relative drop.  Single-case handles. */
int jg_run_to(jg_case_t *h, double resid_drop, int max_steps, int check_every, int *steps, double *drop);
/* new run-time settings for a live handle: CFL / DT and the ramp,
 * under-relaxation, linear-solver thresholds and sweeps, limiter EPS,
 * time-step mode.  Any other field must equal the handle's (JG_ERR_ARG).  The
 * CFL the ramp stands at is unchanged (jg_set_cfl_step). */
int jg_set_params(jg_case_t *h, const jg_params *params);
/* Batching form (no reference counterpart; the reference runs one case per
 * process): ncases independent cases, each with its own mesh and boundary
 * values, concatenated into one block-diagonal system so that every stage of
 * the iteration is one launch over all cases.  Each case keeps its own
 * residual reduction and never reads another case's data, so its results are
 * bit-identical alone and in any batch.  Linear solver JACOBI, SGS, LINE or
 * LUSGS (JACOBI, SGS or LINE with a turbulence model); time step CFL or DT.  All cases
 * share one model: none, SA or SST (each case's wall distance is taken to its
 * own WALL faces).  The batch handle accepts every single-case call (jg_step
 * reports the residual summed over the cases). */
int jg_batch_create(int ncases, const jg_mesh *meshes, const jg_params *params, jg_case_t **out);
int jg_batch_info(jg_case_t *h, int *ncases, int *cell_offsets /* [ncases+1], may be NULL */);
/* sets one case's state; the state/BC preamble runs at the next step (set every case first) */
int jg_batch_set_state(jg_case_t *h, int case_id, const double *rho, const double *rhou, const double *rhoE);
int jg_batch_get_state(jg_case_t *h, int case_id, double *rho, double *rhou, double *rhoE);
/* a turbulence-model batch: one case's transported scalars phi[ncv_k][nscal] in/out */
int jg_batch_set_scalars(jg_case_t *h, int case_id, const double *phi);
int jg_batch_get_scalars(jg_case_t *h, int case_id, double *phi);
/* resid[nsteps][ncases][5 + nscal]: the L1 residual of every case at every step.  A
 * case that goes non-physical does not stop the batch: see jg_batch_status. */
int jg_batch_step(jg_case_t *h, int nsteps, double *resid);
/* status[ncases]: error flags of each case since the last call (1: density or
 * pressure <= 0, 4: NaN residual); cleared by the call */
int jg_batch_status(jg_case_t *h, int *status);
/* freeze (0) or resume (1) a case: a frozen case keeps its state (retired) */
int jg_batch_set_active(jg_case_t *h, int case_id, int active);

/* Launch shapes (no reference counterpart).  The 5x5 face loop runs either
 * fused -- residual and Jacobian blocks in one kernel, flux_cl = 1, 2 or 4
 * lanes per cell with registers for two 128-thread blocks per SM, or
 * JG_FLUX_CL1_3BLK: one lane, registers capped for three blocks per SM -- or
 * split (flux_cl = JG_FLUX_SPLIT + FL, FL = 1, 2, 4 or 8; the default is
 * JG_FLUX_SPLIT + 4): a residual kernel with FL lanes per cell and a Jacobian
 * kernel (one thread per cell, the face matrices formed row by row) on two
 * streams.  Second: the kernel of the 5x5 Jacobi sweep (0: a block per 32-cell
 * slice, a thread per block row, the default; 1: a thread per cell).
 * jg_autotune times each candidate on the handle's own mesh (trials launches,
 * CUDA events) and keeps the fastest; ms[10] (may be NULL) gets the face loop
 * time per launch: fused 1, 2, 4 lanes (ms[0..2]), fused JG_FLUX_CL1_3BLK
 * (ms[5]), split FL = 1, 2, 4, 8 (ms[6..9]); and the sweep time for kernels 0,
 * 1 (ms[3..4]).  A handle with a lagged Jacobian (jac_lag > 1) runs split
 * shapes only.  The sweep kernels give bit-identical results; the face-loop
 * shapes change the order of each cell's diagonal-block and residual sums
 * (rounding-level differences).  Handles without a turbulence model; others
 * keep their single shape.  A batch handle tunes for all its cases. */
#define JG_FLUX_CL1_3BLK 17
#define JG_FLUX_SPLIT 32
int jg_set_launch_config(jg_case_t *h, int flux_cl, int relax_variant);
int jg_get_launch_config(jg_case_t *h, int *flux_cl, int *relax_variant);
int jg_autotune(jg_case_t *h, int trials, int *flux_cl, int *relax_variant, float *ms);

/* Device bytes jg_create + jg_set_state allocate for a case (exact, before
 * creating it) and the bytes a live handle holds. */
int jg_case_footprint(const jg_mesh *mesh, const jg_params *params, double *bytes);
int jg_case_device_bytes(jg_case_t *h, double *bytes);

/* The cell order jg_create uses with params.renumber = method:
 * cell_old[ncv] = the caller's id of each cell in the handle's order.  Host
 * only (no device needed).  For JG_RENUMBER_RCM: reverse Cuthill-McKee over
 * the nbocv graph, each connected component from a pseudo-peripheral cell;
 * JG_RENUMBER_RCM_COLOR and JG_RENUMBER_RCM_LINES as above. */
int jg_renumber_cells(const jg_mesh *mesh, int method, int *cell_old);

/* Serving form (no reference counterpart; the reference solves one case per
 * run): a request loop on one GPU.  Submitted cases wait in a FIFO queue and
 * are admitted while the device-memory budget and the resident-case limit
 * allow; each resident case has its own handle, stream and captured step, so
 * the cases' steps overlap on the device and every case's result is the one
 * it gets alone.  jg_serve_poll is the progress engine: it launches
 * steps_per_poll steps per resident case, reads each case's residuals without
 * blocking the others, retires a case when its L1 energy residual has fallen
 * to resid_drop x its first-step value (or after max_steps), and admits queued
 * cases into the freed memory.  A case that reaches a non-physical state is
 * restarted from its initial state with CFL_RAMP MAX_CFL (and the starting
 * CFL, if above it) multiplied by restart_cfl_factor, up to max_restarts
 * times; with stall_steps > 0 a case whose residual has stopped falling is
 * retired early as stalled.  Admission is in arrival order, or smallest
 * footprint first among the queued cases (JG_ADMIT_SMALLEST).
 * Single-threaded: call every jg_serve_* of one server from one thread. */
typedef struct jg_server jg_server_t;
typedef struct {
  int device;                /* CUDA device */
  int max_resident;          /* cases on the device at once (>= 1) */
  double hbm_budget;         /* device bytes the resident cases may hold; <= 0: 90% of the free memory.
                              * A case whose footprint is above it is retired as JG_SERVE_FAILED
                              * (with its initial state) without being started. */
  int steps_per_poll;        /* steps launched per case between residual checks (1..64) */
  double resid_drop;         /* convergence: energy residual / first-step energy residual */
  int max_steps;             /* retire unconverged after this many steps */
  int max_restarts;          /* restarts after a non-physical state */
  double restart_cfl_factor; /* CFL scaling per restart (0 < f <= 1) */
  int stall_steps;           /* > 0: retire as stalled when the best residual drop has not halved over this many steps */
  int admission;             /* JG_ADMIT_FIFO: arrival order; JG_ADMIT_SMALLEST: smallest footprint first */
} jg_serve_config;
enum { JG_ADMIT_FIFO = 0, JG_ADMIT_SMALLEST = 1 };
enum { JG_SERVE_CONVERGED = 0, JG_SERVE_MAX_STEPS = 1, JG_SERVE_FAILED = 2, JG_SERVE_STALLED = 3 };
typedef struct {
  long long id;
  int status;       /* JG_SERVE_* */
  int steps;        /* steps of the final attempt (the state returned is after these) */
  int steps_total;  /* steps over all attempts */
  int restarts;
  int ncv;
  int conv_step;    /* first step whose residual met resid_drop (-1 if none) */
  double drop;      /* energy residual / first-step energy residual at the last step */
  double t_arrival; /* server clock (seconds since jg_serve_create) */
  double t_admit;   /* first admission */
  double t_done;
  double bytes;     /* device footprint while resident */
} jg_serve_result;
int jg_serve_create(const jg_serve_config *cfg, jg_server_t **out);
/* seconds since jg_serve_create on the server's monotonic clock */
int jg_serve_now(jg_server_t *s, double *t);
/* queue a case; the server copies mesh, params and the initial state.
 * t_arrival < 0: now.  The mesh's host arrays may be freed on return. */
int jg_serve_submit(jg_server_t *s, const jg_mesh *mesh, const jg_params *params, const double *rho,
                    const double *rhou, const double *rhoE, double t_arrival, long long *id);
/* run the progress engine for up to max_wait_s seconds or until a case
 * retires; finished cases are written to out[0..*n) (at most cap) */
int jg_serve_poll(jg_server_t *s, double max_wait_s, jg_serve_result *out, int cap, int *n);
/* copy a retired case's final state and release it (each id once) */
int jg_serve_fetch(jg_server_t *s, long long id, double *rho, double *rhou, double *rhoE);
int jg_serve_stats(jg_server_t *s, int *resident, int *queued, int *finished_unfetched, double *bytes_resident);
int jg_serve_destroy(jg_server_t *s);

/* Timing hooks (no reference counterpart): with profiling on, the captured
 * step records CUDA events around the face loop and the linear solve;
 * jg_get_profile returns their device times (ms) for the last step. */
int jg_set_profiling(jg_case_t *h, int on);
int jg_get_profile(jg_case_t *h, double *ms);
/* number of kernels one captured step launches */
int jg_step_kernel_count(jg_case_t *h, int *n);

/* Block point relaxation that allocates nothing.  No counterpart in the
 * reference.  For hosts that cannot call cudaMalloc when they need the solve:
 * their device memory is owned by another allocator (a pool that claimed the
 * GPU up front, an application that budgets every byte), or an allocation's
 * device synchronisation or out-of-memory failure mid-run is not acceptable.
 * All pointers are DEVICE memory owned by the caller, in the reference's
 * layouts: nbocv_i[ncv+1], nbocv_v[nnz] (CSR, diagonal first), A[nnz][5][5],
 * rhs[ncv][5]; dq[ncv][5] receives the result of `sweeps` block Jacobi sweeps
 * from zero (the iteration of jg_solve_lin_sys with JG_LS_JACOBI, equal to it
 * to rounding: the diagonal block is applied through its LU factors, as the
 * reference's lusolv does, not through a stored inverse).  Work
 * memory is a fixed array of JG_NOALLOC_MAX_CELLS x 5 doubles (2.5 MiB) inside
 * the library, held by every GPU that loads it until the process exits;
 * ncv > JG_NOALLOC_MAX_CELLS is rejected with JG_ERR_ARG.  The first call on
 * each device looks up that array's device address (cudaGetSymbolAddress, no
 * allocation); make that first call before any stream capture.  All calls on
 * a device share the array: calls that overlap on the GPU race.  Enqueued on
 * `stream` (a cudaStream_t, NULL = default stream); no synchronisation. */
#define JG_NOALLOC_MAX_CELLS 65536
int jg_relax_csr_noalloc(int ncv, const int *nbocv_i, const int *nbocv_v, const double *A, const double *rhs,
                         double *dq, int sweeps, void *stream);

/* Restart files: the reference's binary restart format (Ugp::writeRestart,
 * Ugp::readRestart, src/common/Ugp.cpp:9792-13240; header Ugp.h:3423-3446),
 * so that a solution can move between the reference and this library in
 * either direction.  Host-only code, no GPU needed except for the two state
 * calls.  A jg_restart_t holds a whole file in host memory: the mesh (node
 * coordinates x_no[nno][3]; face nodes noofa_i[nfa+1] / noofa_v, ordered so
 * that the face normal points from cvofa[f][0] to cvofa[f][1]; cvofa[nfa][2]
 * with -1 for a boundary face and -(partner)-2 for a periodic one; the face
 * zones, each a contiguous face range, in face order; the partition cv_part)
 * and the data records in the order they were read or put.  Cells, faces and
 * nodes are numbered in the file's global order.  jg_restart_write lays the
 * records out as the reference does with one process: the file the reference
 * wrote is written back byte for byte.  Names are at most 51 characters. */
typedef struct jg_restart jg_restart_t;
/* data record kinds: the reference's UGP_IO_* ids (Ugp.cpp:9797-9820) */
enum { JG_RS_I0 = 11, JG_RS_D0 = 12, JG_RS_FA_D1 = 24, JG_RS_NO_D1 = 32, JG_RS_NO_D3 = 33,
       JG_RS_CV_D1 = 42, JG_RS_CV_D3 = 43, JG_RS_CV_D33 = 44 };
/* face zone kinds: FA_ZONE_* (Ugp.h:41-55) */
enum { JG_FA_ZONE_BOUNDARY = 1, JG_FA_ZONE_PERIODIC_CART = 2, JG_FA_ZONE_INTERNAL = 6 };
int jg_restart_new(jg_restart_t **out);
int jg_restart_free(jg_restart_t *r);
/* whole file; byte-swapped files are recognised and swapped.  JG_ERR_IO on a
 * missing, truncated or malformed file (the message says which record). */
int jg_restart_read(const char *path, jg_restart_t **out);
int jg_restart_write(const jg_restart_t *r, const char *path);
int jg_restart_counts(const jg_restart_t *r, int *nno, int *nfa, int *ncv, int *noofa_count, int *nzones,
                      int *nrecords);
/* any pointer may be NULL; sizes from jg_restart_counts */
int jg_restart_get_mesh(const jg_restart_t *r, double *x_no, int *noofa_i, int *noofa_v, int *cvofa, int *cv_part);
/* name: 52 bytes; periodic[3] (FaZone::getPeriodicData) may be NULL */
int jg_restart_get_zone(const jg_restart_t *r, int izone, char *name, int *kind, int *ifa_f, int *ifa_l,
                        double *periodic);
/* replaces the mesh (and clears the zones; one partition); records already
 * held must fit the new counts */
int jg_restart_set_mesh(jg_restart_t *r, int nno, int nfa, int ncv, const double *x_no, const int *noofa_i,
                        const int *noofa_v, const int *cvofa);
/* appends a zone; zones are added in face order and must end up covering every face */
int jg_restart_add_zone(jg_restart_t *r, const char *name, int kind, int ifa_f, int ifa_l, const double *periodic);
/* irec = -1 when no record has that name */
int jg_restart_find(const jg_restart_t *r, const char *name, int *irec);
/* count = items (cells, nodes or faces; 0 for I0 / D0), width = doubles per
 * item (1, 3, 9); data[count*width] may be NULL; any other pointer may be NULL */
int jg_restart_get_record(const jg_restart_t *r, int irec, char *name, int *kind, int *count, int *width,
                          double *data, int *ivalue, double *dvalue);
/* replaces the record of that name in place, or appends it; array kinds take
 * one item per cell / node / face of the mesh */
int jg_restart_put_record(jg_restart_t *r, const char *name, int kind, const double *data, int ivalue,
                          double dvalue);
/* the handle's state into the restart (its mesh must have the handle's cells, in
 * the handle's caller order): STEP, RHO, RHOE, the model's scalars (nuSA; kine,
 * omega) and RHOU; the other records are left as they are. */
int jg_restart_save_state(jg_restart_t *r, jg_case_t *h);
/* the handle's state from the restart as readRestart + initialHook leave the
 * reference (JoeWithModels.cpp:20-31, 201-213): RHO, RHOU, RHOE, the model's
 * scalars, and STEP (0 when absent) with the CFL back at jg_params.cfl, as
 * runBackwardEuler resumes after a restart (JoeWithModels.cpp:975-978). */
int jg_restart_load_state(jg_case_t *h, const jg_restart_t *r);

/* Per-face Euler fluxes and implicit matrices, batched over n faces on the
 * GPU: kind = JG_FLUX_HLLC, ROE, AUSM (HLLC matrices), HAENEL or AUSMDV (the
 * AUSMDV blend with the expansion-fan entropy fix, no shock fix: that needs
 * the cells' sonic flags); calcEulerFlux_* and calcEulerFluxMatrices_*
 * (src/joe/UgpWithCvCompFlow.cpp:120-709, 879-1505, 3281-3641).  JST needs
 * its cells' sensors and is not offered per face.  L/R[n][6] = (rho, u, v,
 * w, p, gamma), area[n], nvec[n][3] unit normals; F[n][5]; AL/AR[n][5][5] may
 * be NULL. */
int jg_euler_flux_faces(int kind, int n, const double *L, const double *R, const double *area, const double *nvec,
                        double *F, double *AL, double *AR);
/* Per-face viscous fluxes and implicit blocks, batched over n faces on the GPU:
 * addViscFlux (src/joe/UgpWithCvCompFlow.cpp:1521-1763), laminar (no turbulent
 * viscosity).  S0/S1[n][8] = (rho, u, v, w, h, T, R, gamma) of the two sides,
 * gu0/gu1[n][3][3] velocity gradients, gh0/gh1[n][3] enthalpy gradients,
 * mul/lamOcp[n] at the face, u_fa[n][3], area[n], nvec/svec[n][3] the unit
 * normal and unit cell-to-cell vector, smag[n] the distance; F[n][4] = (Frhou,
 * FrhoE); A0/A1[n][5][5] (may be NULL): the blocks calcViscousFluxNS
 * subtracts from the first cell's row (JoeWithModels.cpp:3678-3696). */
int jg_visc_flux_faces(int n, const double *S0, const double *S1, const double *gu0, const double *gu1,
                       const double *gh0, const double *gh1, const double *mul, const double *lamOcp,
                       const double *u_fa, const double *area, const double *nvec, const double *svec,
                       const double *smag, double *F, double *A0, double *A1);

#ifdef __cplusplus
}
#endif
#endif /* JOE_B200_H */
