/*
 * joe_oracle.h -- CPU restatement of the reference's implicit finite-volume
 * iteration (Joe: JoeWithModels / UgpWithCvCompFlow / UgpWithCv), used as the
 * checker for the GPU library.  TEST INFRASTRUCTURE ONLY: nothing in the
 * product links or calls it.  Every function cites the reference lines it
 * restates; the restatement is pinned against dumps of the reference solver
 * itself (oracle/_ref/ref_harness) by tests/test_oracle_vs_reference.py.
 */
#ifndef JOE_ORACLE_H
#define JOE_ORACLE_H
#include "../include/joe_b200.h"

typedef struct jo_case jo_case;

jo_case *jo_create(const jg_mesh *m, const jg_params *p);
void jo_destroy(jo_case *h);
void jo_set_state(jo_case *h, const double *rho, const double *rhou, const double *rhoE);
void jo_get_state(jo_case *h, double *rho, double *rhou, double *rhoE);
/* calcStateVariables + calcMaterialProperties + setBC (+ mut = 0); returns 0 or -1 */
int jo_calc_state(jo_case *h);
double jo_calc_dt(jo_case *h, double cfl);
/* calcRhs; A (nbocv_s*25) may be NULL when implicit == 0 */
void jo_calc_rhs(jo_case *h, double *rhs_rho, double *rhs_rhou, double *rhs_rhoE, double *A, int implicit);
/* solveCoupledLinSysNS (BCGSTAB / LUSGS) plus the GPU's point relaxations; returns iterations */
int jo_solve(jo_case *h, double *dq, const double *A, const double *rhs, double zeroAbs, double zeroRel,
             int maxIter, int solver);
/* nsteps iterations of the runBackwardEuler loop body; resid[5] = last L1 residual */
int jo_step(jo_case *h, int nsteps, double *resid);
/* named internal arrays: "vel","press","temp","enthalpy","sos","rho_bfa","T_bfa","vel_bfa","p_bfa",
 * "h_bfa","gam_bfa","RoM_bfa","mul_fa","lamOcp_fa","mut_fa","grad_u","grad_rho","grad_p",
 * "grad_enthalpy","alpha_rho","local_dt" */
double *jo_array(jo_case *h, const char *name);
/* initializeLinelet's lines: off[nlines+1], cv[off[nlines]]; returns nlines (NULL arrays: count only) */
int jo_linelets(jo_case *h, int *off, int *cv);
void jo_build_linelets(jo_case *h);
/* the lines of the LINE relaxation (initializeLinelet's rule, crossing prism/hexahedron interfaces) */
int jo_relax_lines(jo_case *h, int *off, int *cv);
double jo_cfl(jo_case *h);
int jo_step_count(jo_case *h);

/* per-face flux kernels, batched over n faces: states L/R [n][6] = (rho,u,v,w,p,gamma),
 * area[n], nvec[n][3]; F[n][5]; AL/AR[n][25] (may be NULL) */
void jo_euler_flux_faces(int kind, int n, const double *L, const double *R, const double *area,
                         const double *nvec, double *F, double *AL, double *AR);
void jo_visc_flux_faces(int n, const double *S0, const double *S1, const double *gu0, const double *gu1,
                        const double *gh0, const double *gh1, const double *mul, const double *lamOcp,
                        const double *u_fa, const double *area, const double *nV, const double *sV,
                        const double *smag, double *F, double *A0, double *A1);

/* Coupled path with a turbulence model (jg_params.turb_model SA: nscal 1, block
 * 6; SST: nscal 2 (kine, omega), block 7): scalars phi[ncv][nscal] in/out,
 * wall distance (calcWallDistance), the coupled preamble (state + material +
 * BC + scalar BC + calcRansTurbViscMuet), calcRhsCoupled (rhs[ncv][B],
 * A[nbocv_s][B][B] accumulated), block relaxation of a B x B system (sgs 0:
 * Jacobi, 1: multicolour Gauss-Seidel) and the coupled step.  Named arrays:
 * "phi","phi_bfa","grad_phi","diff" (scalar 0), "phi1",... (scalar 1),
 * "wallDist","strMag","vortMag","diverg","crossDiff","blendFuncF1","blendFuncF2". */
void jo_set_scalars(jo_case *h, const double *phi);
void jo_get_scalars(jo_case *h, double *phi);
void jo_wall_distance(jo_case *h);
int jo_calc_state_coupled(jo_case *h);
void jo_calc_rhs_coupled(jo_case *h, double *rhs, double *A, int implicit);
int jo_solve_blocks(jo_case *h, int B, double *x, const double *A, const double *rhs, int sweeps, int sgs);
/* LINE relaxation (the GPU's JG_LS_LINE): block line-Jacobi sweeps from x = 0 */
int jo_line_relax(jo_case *h, int B, double *x, const double *A, const double *rhs, int sweeps);
int jo_step_coupled(jo_case *h, int nsteps, double *resid);
double *jo_sa_array(jo_case *h, const char *name);
void jo_sa_release(jo_case *h);
#endif
