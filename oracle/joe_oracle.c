/*
 * joe_oracle.c -- CPU restatement of the reference's implicit finite-volume
 * iteration.  TEST INFRASTRUCTURE ONLY (the checker for libjoe_b200.so).
 *
 * Reference files cited below are paths inside the reference project:
 *   src/joe/JoeWithModels.cpp, src/joe/UgpWithCvCompFlow.{h,cpp},
 *   src/common/UgpWithCv.{h,cpp}, src/common/tc_vec3d.h
 * Scope: the segregated Navier-Stokes path without transported scalars
 * (inviscid or laminar), ideal gas, LSQ gradients, the smooth Barth-Jespersen
 * limiter, HLLC / Roe / AUSM fluxes with their implicit matrices, the
 * viscous flux, boundary conditions, local time step, BiCGSTAB / LU-SGS.
 */
#include "joe_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct jo_case {
  jg_mesh m;
  jg_params p;
  int ncv, nfa, nfa_b, nbs;
  double *rho, *rhou, *rhoE;
  double *vel, *press, *temp, *enthalpy, *sos, *gam, *RoM;
  double *rho_bfa, *T_bfa, *vel_bfa, *p_bfa, *h_bfa, *gam_bfa, *RoM_bfa;
  double *mul_fa, *lamOcp_fa, *mut_fa;
  double *grad_u, *grad_rho, *grad_p, *grad_h, *alpha_rho;
  double *local_dt;
  double *fscale;   /* [N][5] sum over the cell's faces of |F| (rounding scale of the residual) */
  double cfl;
  int step;
  int dt_fixed_done;
  double dt_fixed;
  double *kine;     /* turbulent kinetic energy per cell (SST), NULL otherwise */
  int nlines;       /* linelets (initializeLinelet): cells line_cv[line_off[l] .. line_off[l+1]) */
  int *line_off, *line_cv;
  unsigned char *linelet;  /* [N] the reference's Linelet flag: the cell is on a line of >= 2 cells */
  int rnlines;      /* the LINE relaxation's lines (crossing prism/hexahedron interfaces) */
  int *rline_off, *rline_cv;
  /* JST: per cell {PressSensor, Lambda, NeighborCV, Conserv_Und_Lapl[5]}, BoundaryCV, p1/p2_Und_Lapl */
  double *jst;
  unsigned char *bcv;
  double *p1_lapl, *p2_lapl;
};

static double *dalloc(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }
static double dot3(const double *a, const double *b) {
  /* vecDotVec3d, tc_vec3d.h:14-22 (sequential sum from 0.0) */
  double d = 0.0;
  for (int i = 0; i < 3; i++) d += a[i] * b[i];
  return d;
}
static double norm3(double *n, const double *v) {
  /* normVec3d(vNorm, v), tc_vec3d.h:36-46 */
  double mag = sqrt(dot3(v, v));
  for (int i = 0; i < 3; i++) n[i] = v[i] / mag;
  return mag;
}
static double dmin(double a, double b) { return a < b ? a : b; }
static double dmax(double a, double b) { return a > b ? a : b; }

jo_case *jo_create(const jg_mesh *m, const jg_params *p) {
  jo_case *h = (jo_case *)calloc(1, sizeof(jo_case));
  h->m = *m;
  h->p = *p;
  h->ncv = m->ncv; h->nfa = m->nfa; h->nfa_b = m->nfa_b; h->nbs = m->nbocv_s;
  int n = h->ncv, nf = h->nfa, nb = h->nfa_b;
  h->rho = dalloc(n); h->rhou = dalloc(3 * n); h->rhoE = dalloc(n);
  h->vel = dalloc(3 * n); h->press = dalloc(n); h->temp = dalloc(n); h->enthalpy = dalloc(n);
  h->sos = dalloc(n); h->gam = dalloc(n); h->RoM = dalloc(n);
  h->rho_bfa = dalloc(nb); h->T_bfa = dalloc(nb); h->vel_bfa = dalloc(3 * nb); h->p_bfa = dalloc(nb);
  h->h_bfa = dalloc(nb); h->gam_bfa = dalloc(nb); h->RoM_bfa = dalloc(nb);
  h->mul_fa = dalloc(nf); h->lamOcp_fa = dalloc(nf); h->mut_fa = dalloc(nf);
  h->grad_u = dalloc(9 * n); h->grad_rho = dalloc(3 * n); h->grad_p = dalloc(3 * n);
  h->grad_h = dalloc(3 * n); h->alpha_rho = dalloc(n); h->local_dt = dalloc(n);
  h->fscale = dalloc(5 * n);
  h->jst = dalloc(8 * n);
  h->p1_lapl = dalloc(n);
  h->p2_lapl = dalloc(n);
  h->bcv = (unsigned char *)calloc(n ? n : 1, 1);
  /* calcJSTCoeff_Const (JoeWithModels.cpp:13380-13395): BoundaryCV is set on the first cell of every
   * internal face (as the reference writes it), NeighborCV counts the internal faces of each cell */
  for (int f = m->nfa_b; f < m->nfa; f++) {
    h->bcv[m->cvofa[2 * f]] = 1;
    h->jst[8 * m->cvofa[2 * f] + 2] += 1.0;
    h->jst[8 * m->cvofa[2 * f + 1] + 2] += 1.0;
  }
  /* initialHookScalarRansCombModel: RoM = R_gas, gamma = GAMMA (UgpWithCvCompFlow.h:1630-1640) */
  for (int i = 0; i < n; i++) { h->gam[i] = p->gamma; h->RoM[i] = p->R_gas; }
  h->cfl = p->cfl;
  return h;
}

void jo_destroy(jo_case *h) {
  if (!h) return;
  double *arrs[] = {h->rho, h->rhou, h->rhoE, h->vel, h->press, h->temp, h->enthalpy, h->sos, h->gam, h->RoM,
                    h->rho_bfa, h->T_bfa, h->vel_bfa, h->p_bfa, h->h_bfa, h->gam_bfa, h->RoM_bfa, h->mul_fa,
                    h->lamOcp_fa, h->mut_fa, h->grad_u, h->grad_rho, h->grad_p, h->grad_h, h->alpha_rho,
                    h->local_dt, h->fscale, h->jst, h->p1_lapl, h->p2_lapl};
  for (size_t i = 0; i < sizeof(arrs) / sizeof(arrs[0]); i++) free(arrs[i]);
  free(h->bcv);
  free(h->line_off);
  free(h->line_cv);
  free(h->linelet);
  free(h->rline_off);
  free(h->rline_cv);
  free(h);
}

void jo_set_state(jo_case *h, const double *rho, const double *rhou, const double *rhoE) {
  memcpy(h->rho, rho, sizeof(double) * h->ncv);
  memcpy(h->rhou, rhou, sizeof(double) * 3 * h->ncv);
  memcpy(h->rhoE, rhoE, sizeof(double) * h->ncv);
}

void jo_get_state(jo_case *h, double *rho, double *rhou, double *rhoE) {
  memcpy(rho, h->rho, sizeof(double) * h->ncv);
  memcpy(rhou, h->rhou, sizeof(double) * 3 * h->ncv);
  memcpy(rhoE, h->rhoE, sizeof(double) * h->ncv);
}

double *jo_array(jo_case *h, const char *name) {
  struct { const char *n; double *p; } t[] = {
      {"vel", h->vel}, {"press", h->press}, {"temp", h->temp}, {"enthalpy", h->enthalpy}, {"sos", h->sos},
      {"rho_bfa", h->rho_bfa}, {"T_bfa", h->T_bfa}, {"vel_bfa", h->vel_bfa}, {"p_bfa", h->p_bfa},
      {"h_bfa", h->h_bfa}, {"gam_bfa", h->gam_bfa}, {"RoM_bfa", h->RoM_bfa}, {"mul_fa", h->mul_fa},
      {"lamOcp_fa", h->lamOcp_fa}, {"mut_fa", h->mut_fa}, {"grad_u", h->grad_u}, {"grad_rho", h->grad_rho},
      {"grad_p", h->grad_p}, {"grad_enthalpy", h->grad_h}, {"alpha_rho", h->alpha_rho},
      {"local_dt", h->local_dt}, {"flux_scale", h->fscale}, {"rho", h->rho}, {"rhou", h->rhou}, {"rhoE", h->rhoE}};
  for (size_t i = 0; i < sizeof(t) / sizeof(t[0]); i++)
    if (strcmp(t[i].n, name) == 0) return t[i].p;
  return NULL;
}
double jo_cfl(jo_case *h) { return h->cfl; }
int jo_step_count(jo_case *h) { return h->step; }

/* ------------------------------------------------------------------------ */
/* thermodynamics                                                            */
/* ------------------------------------------------------------------------ */

static double mu_law(const jg_params *p, double T) {
  /* calcMuLam / ComputeBCProperties_T, UgpWithCvCompFlow.h:1601-1621, 1796-1805 */
  if (p->mu_mode == JG_MU_SUTHERLAND)
    return p->mu_ref * pow(T / p->SL_Tref, 1.5) * (p->SL_Tref + p->SL_Sref) / (T + p->SL_Sref);
  return p->mu_ref * pow(T / p->T_ref, p->mu_power_law);
}

/* calcStateVariables, UgpWithCvCompFlow.h:1662-1694 (no kine) */
static void calc_state_variables(jo_case *h) {
  for (int c = 0; c < h->ncv; c++) {
    double r = h->rho[c];
    double *ru = &h->rhou[3 * c];
    for (int i = 0; i < 3; i++) h->vel[3 * c + i] = ru[i] / r;
    double kinecv = 0.0;
    if (h->kine) kinecv = h->kine[c];
    double pr = (h->gam[c] - 1.0) * (h->rhoE[c] - 0.5 * dot3(ru, ru) / r - r * kinecv);
    if (pr > 0.0) h->press[c] = pr;  /* negative pressure: keep the old value */
    h->temp[c] = h->press[c] / (r * h->RoM[c]);
    h->enthalpy[c] = h->gam[c] * h->RoM[c] / (h->gam[c] - 1.0) * h->temp[c];
    h->sos[c] = sqrt(h->gam[c] * h->press[c] / r);
  }
}

/* calcMaterialProperties, UgpWithCvCompFlow.h:1701-1753 (internal faces) */
static void calc_material_properties(jo_case *h) {
  const jg_params *p = &h->p;
  if (!(p->mu_ref > 0.0)) return;
  for (int f = h->nfa_b; f < h->nfa; f++) {
    int c0 = h->m.cvofa[2 * f], c1 = h->m.cvofa[2 * f + 1];
    double dx0[3], dx1[3];
    for (int i = 0; i < 3; i++) {
      dx0[i] = h->m.x_fa[3 * f + i] - h->m.x_cv[3 * c0 + i];
      dx1[i] = h->m.x_fa[3 * f + i] - h->m.x_cv[3 * c1 + i];
    }
    double w0 = sqrt(dot3(dx0, dx0));
    double w1 = sqrt(dot3(dx1, dx1));
    double T = (w1 * h->temp[c0] + w0 * h->temp[c1]) / (w0 + w1);
    h->mul_fa[f] = mu_law(p, T);
    h->lamOcp_fa[f] = h->mul_fa[f] / p->Pr;
  }
}

/* ComputeBCProperties_T, UgpWithCvCompFlow.h:1783-1812 */
static void bc_props_T(jo_case *h, int f0, int f1) {
  const jg_params *p = &h->p;
  for (int f = f0; f <= f1; f++) {
    h->gam_bfa[f] = p->gamma;
    h->RoM_bfa[f] = p->R_gas;
    h->h_bfa[f] = p->gamma * p->R_gas / (p->gamma - 1.0) * h->T_bfa[f];
  }
  if (p->mu_ref > 0.0)
    for (int f = f0; f <= f1; f++) {
      h->mul_fa[f] = mu_law(p, h->T_bfa[f]);
      h->lamOcp_fa[f] = h->mul_fa[f] / p->Pr;
    }
}

/* ComputeBCProperties_H, UgpWithCvCompFlow.h:1815-1839 */
static void bc_props_H(jo_case *h, int f0, int f1) {
  const jg_params *p = &h->p;
  for (int f = f0; f <= f1; f++) {
    h->gam_bfa[f] = p->gamma;
    h->RoM_bfa[f] = p->R_gas;
    h->T_bfa[f] = h->h_bfa[f] * (p->gamma - 1.0) / (p->gamma * p->R_gas);
  }
  if (p->mu_ref > 0.0)
    for (int f = f0; f <= f1; f++) {
      h->mul_fa[f] = mu_law(p, h->T_bfa[f]);
      h->lamOcp_fa[f] = h->mul_fa[f] / p->Pr;
    }
}

/* setBC, JoeWithModels.cpp:3857-4300 */
static int set_bc(jo_case *h) {
  const jg_params *p = &h->p;
  for (int z = 0; z < h->m.nzones; z++) {
    const jg_zone *zn = &h->m.zones[z];
    int f0 = zn->ifa_f, f1 = zn->ifa_l;
    const double *v = zn->v;
    switch (zn->kind) {
      case JG_BC_CBC: {
        const double *u_bc = v; double T_bc = v[3], p_bc = v[4];
        for (int f = f0; f <= f1; f++) {
          int c0 = h->m.cvofa[2 * f];
          double nV[3];
          norm3(nV, &h->m.fa_normal[3 * f]);
          if (dot3(u_bc, nV) > 0.0) {
            double un = dot3(&h->vel[3 * c0], nV);
            double mach = fabs(un) / h->sos[c0];
            h->T_bfa[f] = h->temp[c0];
            for (int i = 0; i < 3; i++) h->vel_bfa[3 * f + i] = h->vel[3 * c0 + i];
            h->p_bfa[f] = (mach >= 1.0) ? h->press[c0] : p_bc;
          } else {
            h->T_bfa[f] = T_bc;
            for (int i = 0; i < 3; i++) h->vel_bfa[3 * f + i] = u_bc[i];
            h->p_bfa[f] = p_bc;
          }
        }
        bc_props_T(h, f0, f1);
      } break;
      case JG_BC_CBC_SUBSONIC_INLET: {
        const double *ang = v; double Ttot = v[3], ptot = v[4];
        for (int f = f0; f <= f1; f++) {
          int c0 = h->m.cvofa[2 * f];
          double r = h->rho[c0];
          double u[3] = {h->rhou[3 * c0] / r, h->rhou[3 * c0 + 1] / r, h->rhou[3 * c0 + 2] / r};
          double vm = sqrt(dot3(u, u));
          for (int i = 0; i < 3; i++) h->vel_bfa[3 * f + i] = ang[i] * vm;
          h->T_bfa[f] = Ttot;
          h->p_bfa[f] = ptot;
        }
        bc_props_T(h, f0, f1);
        for (int f = f0; f <= f1; f++) {
          double w2 = dot3(&h->vel_bfa[3 * f], &h->vel_bfa[3 * f]);
          h->h_bfa[f] -= 0.5 * w2;
        }
        bc_props_H(h, f0, f1);
        for (int f = f0; f <= f1; f++)
          h->p_bfa[f] = ptot * pow(h->T_bfa[f] / Ttot, h->gam_bfa[f] / (h->gam_bfa[f] - 1.0));
      } break;
      case JG_BC_CBC_SUBSONIC_OUTLET: {
        double p_bc = v[0];
        for (int f = f0; f <= f1; f++) {
          int c0 = h->m.cvofa[2 * f];
          h->p_bfa[f] = p_bc;
          for (int i = 0; i < 3; i++) h->vel_bfa[3 * f + i] = h->rhou[3 * c0 + i] / h->rho[c0];
          h->T_bfa[f] = h->temp[c0];
        }
        bc_props_T(h, f0, f1);
      } break;
      case JG_BC_SYMMETRY: {
        for (int f = f0; f <= f1; f++) {
          int c0 = h->m.cvofa[2 * f];
          double nV[3];
          norm3(nV, &h->m.fa_normal[3 * f]);
          double *u0 = &h->vel[3 * c0];
          double un = dot3(nV, u0);
          for (int i = 0; i < 3; i++) h->vel_bfa[3 * f + i] = u0[i] - 1.0 * un * nV[i];
          h->T_bfa[f] = h->temp[c0];
          h->p_bfa[f] = h->press[c0];
        }
        bc_props_T(h, f0, f1);
      } break;
      case JG_BC_NEUMANN: {
        for (int f = f0; f <= f1; f++) {
          int c0 = h->m.cvofa[2 * f];
          for (int i = 0; i < 3; i++) h->vel_bfa[3 * f + i] = h->rhou[3 * c0 + i] / h->rho[c0];
          h->T_bfa[f] = h->temp[c0];
          h->p_bfa[f] = h->press[c0];
        }
        bc_props_T(h, f0, f1);
      } break;
      case JG_BC_WALL: {
        double T_bc = v[0];
        for (int f = f0; f <= f1; f++) {
          int c0 = h->m.cvofa[2 * f];
          for (int i = 0; i < 3; i++) h->vel_bfa[3 * f + i] = 0.0;
          h->T_bfa[f] = (T_bc > 0.0) ? T_bc : h->temp[c0];
          h->p_bfa[f] = h->press[c0];
        }
        bc_props_T(h, f0, f1);
      } break;
      case JG_BC_FARFIELD: {
        const double *u_bc = v; double p_bc = v[3], rho_bc = v[4], gamma_bc = v[5];
        double gm1 = gamma_bc - 1.0;
        double ovgm1 = 1.0 / gm1;
        double c_bc = sqrt(gamma_bc * p_bc / rho_bc);
        double s_bc = pow(rho_bc, gamma_bc) / p_bc;
        for (int f = f0; f <= f1; f++) {
          int c0 = h->m.cvofa[2 * f];
          double nV[3];
          norm3(nV, &h->m.fa_normal[3 * f]);
          double qn_bc = dot3(nV, u_bc);
          double vn_bc = qn_bc;
          double qne = dot3(nV, &h->vel[3 * c0]);
          double ce = sqrt(h->gam[c0] * h->press[c0] / h->rho[c0]);
          double ac1 = (vn_bc > -c_bc) ? qne + 2.0 * ovgm1 * ce : qn_bc + 2.0 * ovgm1 * c_bc;
          double ac2 = (vn_bc > c_bc) ? qne - 2.0 * ovgm1 * ce : qn_bc - 2.0 * ovgm1 * c_bc;
          double qnf = 0.5 * (ac1 + ac2);
          double cf = 0.25 * (ac1 - ac2) * gm1;
          double velf[3], sf;
          if (vn_bc > 0) {
            for (int i = 0; i < 3; i++) velf[i] = h->vel[3 * c0 + i] + (qnf - qne) * nV[i];
            sf = pow(h->rho[c0], h->gam[c0]) / h->press[c0];
          } else {
            for (int i = 0; i < 3; i++) velf[i] = u_bc[i] + (qnf - qn_bc) * nV[i];
            sf = s_bc;
          }
          h->rho_bfa[f] = pow((sf * cf * cf / h->gam[c0]), ovgm1);
          for (int i = 0; i < 3; i++) h->vel_bfa[3 * f + i] = velf[i];
          h->p_bfa[f] = h->rho_bfa[f] * cf * cf / h->gam[c0];
          h->T_bfa[f] = h->p_bfa[f] / (p->R_gas * h->rho_bfa[f]);
        }
        bc_props_T(h, f0, f1);
      } break;
      default:
        return -1;
    }
  }
  /* density from the equation of state, JoeWithModels.cpp:4291-4293 */
  for (int f = 0; f < h->nfa_b; f++) h->rho_bfa[f] = h->p_bfa[f] / (h->RoM_bfa[f] * h->T_bfa[f]);
  return 0;
}

int jo_calc_state(jo_case *h) {
  calc_state_variables(h);
  calc_material_properties(h);
  int e = set_bc(h);
  /* calcRansTurbViscMuet without a turbulence model: mut_fa = 0 (UgpWithCvCompFlow.h:1568-1580) */
  for (int f = 0; f < h->nfa; f++) h->mut_fa[f] = 0.0;
  return e;
}

/* ------------------------------------------------------------------------ */
/* local time step, UgpWithCvCompFlow.cpp:5-110                              */
/* ------------------------------------------------------------------------ */
double jo_calc_dt(jo_case *h, double cfl_target) {
  const jg_params *p = &h->p;
  if (p->time_step_mode == JG_TS_DT) {
    if (!h->dt_fixed_done) {
      h->dt_fixed = p->dt;
      for (int c = 0; c < h->ncv; c++) h->local_dt[c] = p->dt;
      h->dt_fixed_done = 1;
    }
    return h->dt_fixed;
  }
  double dt_min = 1.0e20;
  for (int c = 0; c < h->ncv; c++) {
    double r = h->rho[c];
    double cs = sqrt(h->gam[c] * h->press[c] / r);
    const double *ru = &h->rhou[3 * c];
    double dt_cv;
    if (p->time_step == JG_DT_MAX_BASED) {
      double lambdaMax = 0.0;
      for (int k = h->m.faocv_i[c]; k < h->m.faocv_i[c + 1]; k++) {
        int f = h->m.faocv_v[k];
        double nV[3];
        double area = norm3(nV, &h->m.fa_normal[3 * f]);
        double Uk = dot3(ru, nV) / r;
        double lambda = (fabs(Uk) + cs) * area;
        double lamdiff = 4.0 * (h->mul_fa[f] + h->mut_fa[f]) / r * area * area / h->m.cv_volume[c];
        lambda = dmax(lambda, lamdiff);
        lambdaMax = dmax(lambdaMax, lambda);
      }
      dt_cv = cfl_target * h->m.cv_volume[c] / lambdaMax;
    } else {
      double lc = 0.0, ld = 0.0;
      for (int k = h->m.faocv_i[c]; k < h->m.faocv_i[c + 1]; k++) {
        int f = h->m.faocv_v[k];
        double nV[3];
        double area = norm3(nV, &h->m.fa_normal[3 * f]);
        double Uk = dot3(ru, nV) / r;
        int c0 = h->m.cvofa[2 * f], c1 = h->m.cvofa[2 * f + 1];
        double vol = (c0 >= 0 && c1 >= 0) ? 0.5 * (h->m.cv_volume[c0] + h->m.cv_volume[c1]) : 0.5 * h->m.cv_volume[c];
        lc += (fabs(Uk) + cs) * area;
        if (p->mu_ref > 0.0) {
          double kv = (4.0 / 3.0) * (h->mul_fa[f] + h->mut_fa[f]) / r;
          ld += area * area * kv / vol;
        } else
          ld = 0.0;
      }
      double dt_conv = cfl_target * h->m.cv_volume[c] / lc;
      double dt_visc = (p->mu_ref > 0.0) ? 0.25 * cfl_target * h->m.cv_volume[c] / ld : 1.0e20;
      dt_cv = dmin(dt_conv, dt_visc);
    }
    dt_min = dmin(dt_min, dt_cv);
    h->local_dt[c] = dt_cv;
  }
  if (p->time_step_mode == JG_TS_CFL_MIN)
    for (int c = 0; c < h->ncv; c++) h->local_dt[c] = dt_min;
  return dt_min;
}

/* ------------------------------------------------------------------------ */
/* gradients + limiters, UgpWithCv.h:803-1083                                */
/* ------------------------------------------------------------------------ */
#define SDWLS_CLIP_SCALAR 1.0e-8 /* SDWLSClippingScalar, UgpWithCv.h:20 */

/* distance weights of face f (GG_WITH_DIST): w0 = |x_fa - x_cv0|, w1 = |x_fa - x_cv1| */
static void gg_weights(const jg_mesh *m, int f, double *w0, double *w1) {
  int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
  double d0[3], d1[3];
  for (int i = 0; i < 3; i++) {
    d0[i] = m->x_fa[3 * f + i] - m->x_cv[3 * c0 + i];
    d1[i] = m->x_fa[3 * f + i] - m->x_cv[3 * c1 + i];
  }
  *w0 = sqrt(dot3(d0, d0));
  *w1 = sqrt(dot3(d1, d1));
}

/* calcCvScalarGradGreenGauss (UgpWithCv.h:1091-1128) with GG_WITH_DIST */
static void grad_scalar_gg(jo_case *h, double *g, const double *phi, const double *phi_bfa) {
  const jg_mesh *m = &h->m;
  for (int k = 0; k < 3 * h->ncv; k++) g[k] = 0.0;
  for (int f = h->nfa_b; f < h->nfa; f++) {
    int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
    double w0, w1;
    gg_weights(m, f, &w0, &w1);
    double fv = (w1 * phi[c0] + w0 * phi[c1]) / (w0 + w1);
    for (int i = 0; i < 3; i++) {
      g[3 * c0 + i] += fv * m->fa_normal[3 * f + i];
      g[3 * c1 + i] -= fv * m->fa_normal[3 * f + i];
    }
  }
  for (int f = 0; f < h->nfa_b; f++) {
    int c = m->cvofa[2 * f];
    for (int i = 0; i < 3; i++) g[3 * c + i] += phi_bfa[f] * m->fa_normal[3 * f + i];
  }
  for (int c = 0; c < h->ncv; c++)
    for (int i = 0; i < 3; i++) g[3 * c + i] /= m->cv_volume[c];
}

/* calcCvVectorGradGreenGauss (UgpWithCv.h:1133-1184) with GG_WITH_DIST */
static void grad_vector_gg(jo_case *h, double *g, const double *u, const double *u_bfa) {
  const jg_mesh *m = &h->m;
  for (int k = 0; k < 9 * h->ncv; k++) g[k] = 0.0;
  for (int f = h->nfa_b; f < h->nfa; f++) {
    int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
    double w0, w1;
    gg_weights(m, f, &w0, &w1);
    for (int i = 0; i < 3; i++) {
      double fv = (w1 * u[3 * c0 + i] + w0 * u[3 * c1 + i]) / (w0 + w1);
      for (int j = 0; j < 3; j++) {
        g[9 * c0 + 3 * i + j] += fv * m->fa_normal[3 * f + j];
        g[9 * c1 + 3 * i + j] -= fv * m->fa_normal[3 * f + j];
      }
    }
  }
  for (int f = 0; f < h->nfa_b; f++) {
    int c = m->cvofa[2 * f];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) g[9 * c + 3 * i + j] += u_bfa[3 * f + i] * m->fa_normal[3 * f + j];
  }
  for (int c = 0; c < h->ncv; c++)
    for (int k = 0; k < 9; k++) g[9 * c + k] /= m->cv_volume[c];
}

/* SDWLS weight of one neighbour or boundary face: 1 / (|dx|^2 (limiterWeight(d) + e)) with the van
 * Leer weight limiterWeight(a) = |a| and geomWeighting's |dx|^2 (UgpWithCv.h:16-23) */
static double sdwls_weight(const double dx[3], double dphi_abs, double e) {
  double dist2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
  return 1.0 / (dist2 * (dphi_abs + e));
}

/* the weighted moments sw[6] = {xx, yy, zz, xy, xz, yz} */
static void sdwls_moment_add(double sw[6], double w, const double dx[3]) {
  sw[0] += w * dx[0] * dx[0];
  sw[1] += w * dx[1] * dx[1];
  sw[2] += w * dx[2] * dx[2];
  sw[3] += w * dx[0] * dx[1];
  sw[4] += w * dx[0] * dx[2];
  sw[5] += w * dx[1] * dx[2];
}

/* the determinant of the moment matrix */
static double sdwls_denom(const double sw[6]) {
  return 2.0 * sw[3] * sw[4] * sw[5] + sw[0] * sw[1] * sw[2] - sw[0] * sw[5] * sw[5] - sw[1] * sw[4] * sw[4] -
         sw[2] * sw[3] * sw[3];
}

/* row j of the adjugate of the moment matrix applied to dx */
static double sdwls_row(const double sw[6], int j, const double dx[3]) {
  if (j == 0)
    return (sw[1] * sw[2] - sw[5] * sw[5]) * dx[0] + (sw[4] * sw[5] - sw[3] * sw[2]) * dx[1] +
           (sw[3] * sw[5] - sw[4] * sw[1]) * dx[2];
  if (j == 1)
    return (sw[4] * sw[5] - sw[3] * sw[2]) * dx[0] + (sw[0] * sw[2] - sw[4] * sw[4]) * dx[1] +
           (sw[3] * sw[4] - sw[5] * sw[0]) * dx[2];
  return (sw[3] * sw[5] - sw[4] * sw[1]) * dx[0] + (sw[3] * sw[4] - sw[5] * sw[0]) * dx[1] +
         (sw[0] * sw[1] - sw[3] * sw[3]) * dx[2];
}

/* calcCvScalarGradSDWLS (UgpWithCv.h:1418-1585): per cell, least squares over the neighbours and the
 * boundary faces with solution-dependent weights; e = max(EPS ref, SDWLSClippingScalar); no limiter */
static void grad_scalar_sdwls(jo_case *h, double *g, const double *phi, const double *phi_bfa, const double *ref) {
  const jg_mesh *m = &h->m;
  for (int c = 0; c < h->ncv; c++) {
    double sw[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double e = dmax(h->p.eps * ref[c], SDWLS_CLIP_SCALAR);
    const int nf = m->nbocv_i[c], nl = m->nbocv_i[c + 1] - 1;
    for (int pass = 0; pass < 2; pass++) {
      double denom = pass ? sdwls_denom(sw) : 0.0;
      if (pass)
        for (int i = 0; i < 3; i++) g[3 * c + i] = 0.0;
      for (int k = nf + 1; k <= nl; k++) {
        int nb = m->nbocv_v[k];
        double dp = phi[nb] - phi[c], dx[3];
        for (int i = 0; i < 3; i++) dx[i] = m->x_cv[3 * nb + i] - m->x_cv[3 * c + i];
        double w = sdwls_weight(dx, fabs(dp), e);
        if (!pass) sdwls_moment_add(sw, w, dx);
        else
          for (int i = 0; i < 3; i++) g[3 * c + i] += dp * w * sdwls_row(sw, i, dx) / denom;
      }
      for (int k = m->faocv_i[c]; k < m->faocv_i[c + 1]; k++) {
        int f = m->faocv_v[k];
        if (f >= h->nfa_b) continue;
        double dp = phi_bfa[f] - phi[c], dx[3];
        for (int i = 0; i < 3; i++) dx[i] = m->x_fa[3 * f + i] - m->x_cv[3 * c + i];
        double w = sdwls_weight(dx, fabs(dp), e);
        if (!pass) sdwls_moment_add(sw, w, dx);
        else
          for (int i = 0; i < 3; i++) g[3 * c + i] += dp * w * sdwls_row(sw, i, dx) / denom;
      }
    }
  }
}

/* calcCvVectorGradSDWLS (UgpWithCv.h:1589-1800): the weight from |du|, e = EPS ref (no clipping) */
static void grad_vector_sdwls(jo_case *h, double *g, const double *u, const double *u_bfa, const double *ref) {
  const jg_mesh *m = &h->m;
  for (int c = 0; c < h->ncv; c++) {
    double sw[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    const double e = h->p.eps * ref[c];
    const int nf = m->nbocv_i[c], nl = m->nbocv_i[c + 1] - 1;
    for (int pass = 0; pass < 2; pass++) {
      double denom = pass ? sdwls_denom(sw) : 0.0;
      if (pass)
        for (int k = 0; k < 9; k++) g[9 * c + k] = 0.0;
      for (int k = nf + 1; k <= nl; k++) {
        int nb = m->nbocv_v[k];
        double du[3], du2 = 0.0, dx[3];
        for (int i = 0; i < 3; i++) {
          du[i] = u[3 * nb + i] - u[3 * c + i];
          du2 += du[i] * du[i];
        }
        for (int i = 0; i < 3; i++) dx[i] = m->x_cv[3 * nb + i] - m->x_cv[3 * c + i];
        double w = sdwls_weight(dx, fabs(sqrt(du2)), e);
        if (!pass) sdwls_moment_add(sw, w, dx);
        else
          for (int j = 0; j < 3; j++) {
            double t = w * sdwls_row(sw, j, dx) / denom;
            for (int i = 0; i < 3; i++) g[9 * c + 3 * i + j] += du[i] * t;
          }
      }
      for (int k = m->faocv_i[c]; k < m->faocv_i[c + 1]; k++) {
        int f = m->faocv_v[k];
        if (f >= h->nfa_b) continue;
        double du[3], du2 = 0.0, dx[3];
        for (int i = 0; i < 3; i++) {
          du[i] = u_bfa[3 * f + i] - u[3 * c + i];
          du2 += du[i] * du[i];
        }
        for (int i = 0; i < 3; i++) dx[i] = m->x_fa[3 * f + i] - m->x_cv[3 * c + i];
        double w = sdwls_weight(dx, fabs(sqrt(du2)), e);
        if (!pass) sdwls_moment_add(sw, w, dx);
        else
          for (int j = 0; j < 3; j++) {
            double t = w * sdwls_row(sw, j, dx) / denom;
            for (int i = 0; i < 3; i++) g[9 * c + 3 * i + j] += du[i] * t;
          }
      }
    }
  }
}

static void grad_scalar(jo_case *h, double *g, const double *phi, const double *phi_bfa, int limit,
                        const double *ref, double *alpha) {
  const jg_mesh *m = &h->m;
  /* calcCvScalarGrad(grad, phi) + boundary part, UgpWithCv.h:1009-1056 (or Green-Gauss); SDWLS
   * takes no limiter (calcCvScalarGrad's GRAD_SDWLS case, UgpWithCv.h:826-828) */
  if (h->p.grad_scheme == JG_GRAD_SDWLS) {
    grad_scalar_sdwls(h, g, phi, phi_bfa, ref);
    if (alpha)
      for (int c = 0; c < h->ncv; c++) alpha[c] = 1.0;
    return;
  }
  if (h->p.grad_scheme == JG_GRAD_GREENGAUSS) grad_scalar_gg(h, g, phi, phi_bfa);
  else
  for (int c = 0; c < h->ncv; c++) {
    int nf = m->nbocv_i[c], nl = m->nbocv_i[c + 1] - 1;
    for (int i = 0; i < 3; i++) g[3 * c + i] = m->nbocv_lsg_coeff[3 * nf + i] * phi[c];
    for (int k = nf + 1; k <= nl; k++) {
      int nb = m->nbocv_v[k];
      for (int i = 0; i < 3; i++) g[3 * c + i] += m->nbocv_lsg_coeff[3 * k + i] * phi[nb];
    }
  }
  if (h->p.grad_scheme != JG_GRAD_GREENGAUSS)
    for (int f = 0; f < h->nfa_b; f++) {
      int c = m->cvofa[2 * f];
      for (int i = 0; i < 3; i++) g[3 * c + i] += m->boundary_fa_lsg_coeff[3 * f + i] * phi_bfa[f];
    }
  if (!limit) return;
  /* limitCvScalarGradBJ (smooth form), UgpWithCv.h:881-938 */
  for (int c = 0; c < h->ncv; c++) {
    double pmax = phi[c], pmin = pmax;
    for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++) {
      int nb = m->nbocv_v[k];
      pmax = dmax(pmax, phi[nb]);
      pmin = dmin(pmin, phi[nb]);
    }
    double alfa = 1.0;
    if ((pmax - pmin) > 1.0e-12) {
      for (int k = m->faocv_i[c]; k < m->faocv_i[c + 1]; k++) {
        int f = m->faocv_v[k];
        if (f >= h->nfa_b) {
          double r0[3];
          for (int i = 0; i < 3; i++) r0[i] = m->x_fa[3 * f + i] - m->x_cv[3 * c + i];
          double phifa = phi[c] + dot3(r0, &g[3 * c]);
          double eps2 = dmax(h->p.eps * fabs(ref[c]), SDWLS_CLIP_SCALAR);
          eps2 = pow(eps2, 2.0);
          double dm = phifa - phi[c];
          double dp = ((phifa - phi[c]) >= 0.0) ? pmax - phi[c] : pmin - phi[c];
          alfa = dmin(alfa, (dp * dp + 2.0 * dm * dp + eps2) / (dp * dp + 2 * dm * dm + dm * dp + eps2));
        }
      }
    } else
      alfa = 0.0;
    for (int i = 0; i < 3; i++) g[3 * c + i] *= alfa;
    if (alpha) alpha[c] = alfa;
  }
}

static void grad_vector(jo_case *h, double *g, const double *u, const double *u_bfa, int limit, const double *ref) {
  const jg_mesh *m = &h->m;
  /* calcCvVectorGrad(grad, u) + boundary part, UgpWithCv.h:1031-1083; g[c][i][j] = d u_i / d x_j */
  if (h->p.grad_scheme == JG_GRAD_SDWLS) {
    grad_vector_sdwls(h, g, u, u_bfa, ref);
    return;
  }
  if (h->p.grad_scheme == JG_GRAD_GREENGAUSS) grad_vector_gg(h, g, u, u_bfa);
  else
  for (int c = 0; c < h->ncv; c++) {
    int nf = m->nbocv_i[c], nl = m->nbocv_i[c + 1] - 1;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) g[9 * c + 3 * i + j] = m->nbocv_lsg_coeff[3 * nf + j] * u[3 * c + i];
    for (int k = nf + 1; k <= nl; k++) {
      int nb = m->nbocv_v[k];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) g[9 * c + 3 * i + j] += m->nbocv_lsg_coeff[3 * k + j] * u[3 * nb + i];
    }
  }
  if (h->p.grad_scheme != JG_GRAD_GREENGAUSS)
    for (int f = 0; f < h->nfa_b; f++) {
      int c = m->cvofa[2 * f];
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) g[9 * c + 3 * i + j] += m->boundary_fa_lsg_coeff[3 * f + j] * u_bfa[3 * f + i];
    }
  if (!limit) return;
  /* limitCvVectorGradBJ, UgpWithCv.h:943-1000 */
  for (int c = 0; c < h->ncv; c++) {
    for (int i = 0; i < 3; i++) {
      double pmax = u[3 * c + i], pmin = pmax;
      for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++) {
        int nb = m->nbocv_v[k];
        pmax = dmax(pmax, u[3 * nb + i]);
        pmin = dmin(pmin, u[3 * nb + i]);
      }
      double alfa = 1.0;
      if ((pmax - pmin) > 1.0e-8) {
        for (int k = m->faocv_i[c]; k < m->faocv_i[c + 1]; k++) {
          int f = m->faocv_v[k];
          if (f >= h->nfa_b) {
            double r0[3];
            for (int j = 0; j < 3; j++) r0[j] = m->x_fa[3 * f + j] - m->x_cv[3 * c + j];
            double phifa = u[3 * c + i] + dot3(r0, &g[9 * c + 3 * i]);
            double eps2 = pow(h->p.eps * ref[c], 2.0);
            double dm = phifa - u[3 * c + i];
            double dp = ((phifa - u[3 * c + i]) >= 0.0) ? pmax - u[3 * c + i] : pmin - u[3 * c + i];
            alfa = dmin(alfa, (dp * dp + 2.0 * dm * dp + eps2) / (dp * dp + 2 * dm * dm + dm * dp + eps2));
          }
        }
      } else
        alfa = 0.0;
      for (int j = 0; j < 3; j++) g[9 * c + 3 * i + j] *= alfa;
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Euler fluxes and their implicit matrices                                  */
/* ------------------------------------------------------------------------ */
typedef struct { double rho, u[3], p, gam, k, h; } fstate;  /* h: static enthalpy */

/* calcEulerFlux_HLLC, UgpWithCvCompFlow.cpp:120-235 */
static void flux_hllc(double F[5], const fstate *L, const fstate *R, double area, const double *nV) {
  double surfv = 0.0;
  double unL = dot3(L->u, nV) - surfv, unLr = unL - surfv;
  double uLuL = dot3(L->u, L->u);
  double cL = sqrt(L->gam * L->p / L->rho);
  double hL = L->gam / (L->gam - 1.0) * L->p / L->rho + 0.5 * uLuL + L->k;
  double eL = hL * L->rho - L->p;
  double unR = dot3(R->u, nV) - surfv, unRr = unR - surfv;
  double uRuR = dot3(R->u, R->u);
  double cR = sqrt(R->gam * R->p / R->rho);
  double hR = R->gam / (R->gam - 1.0) * R->p / R->rho + 0.5 * uRuR + R->k;
  double eR = hR * R->rho - R->p;
  double Rrho = sqrt(R->rho / L->rho);
  double tmp = 1.0 / (1.0 + Rrho);
  double velRoe[3];
  for (int i = 0; i < 3; i++) velRoe[i] = tmp * (L->u[i] + R->u[i] * Rrho);
  double uRoe = dot3(velRoe, nV);
  double gamPdivRho = tmp * ((L->gam * L->p / L->rho + 0.5 * (L->gam - 1.0) * uLuL) +
                             (R->gam * R->p / R->rho + 0.5 * (R->gam - 1.0) * uRuR) * Rrho);
  double cRoe = sqrt(gamPdivRho - ((L->gam + R->gam) * 0.5 - 1.0) * 0.5 * dot3(velRoe, velRoe));
  double sL = dmin(uRoe - cRoe, unLr - cL);
  double sR = dmax(uRoe + cRoe, unRr + cR);
  double sM = (L->p - R->p - L->rho * unL * (sL - unL) + R->rho * unR * (sR - unR)) /
              (R->rho * (sR - unR) - L->rho * (sL - unL));
  double pStar = R->rho * (unR - sR) * (unR - sM) + R->p;
  if (sM >= 0.0) {
    if (sL > 0.0) {
      F[0] = L->rho * unLr;
      for (int i = 0; i < 3; i++) F[1 + i] = L->rho * L->u[i] * unLr + L->p * nV[i];
      F[4] = eL * unLr + L->p * unL;
    } else {
      double inv = 1.0 / (sL - sM);
      double sLmuL = sL - unL;
      double rhoSL = L->rho * sLmuL * inv;
      double rhouSL[3];
      for (int i = 0; i < 3; i++) rhouSL[i] = (L->rho * L->u[i] * sLmuL + (pStar - L->p) * nV[i]) * inv;
      double eSL = (sLmuL * eL - L->p * unL + pStar * sM) * inv;
      F[0] = rhoSL * sM;
      for (int i = 0; i < 3; i++) F[1 + i] = rhouSL[i] * sM + pStar * nV[i];
      F[4] = (eSL + pStar) * sM;
    }
  } else {
    if (sR >= 0.0) {
      double inv = 1.0 / (sR - sM);
      double sRmuR = sR - unR;
      double rhoSR = R->rho * sRmuR * inv;
      double rhouSR[3];
      for (int i = 0; i < 3; i++) rhouSR[i] = (R->rho * R->u[i] * sRmuR + (pStar - R->p) * nV[i]) * inv;
      double eSR = (sRmuR * eR - R->p * unR + pStar * sM) * inv;
      F[0] = rhoSR * sM;
      for (int i = 0; i < 3; i++) F[1 + i] = rhouSR[i] * sM + pStar * nV[i];
      F[4] = (eSR + pStar) * sM;
    } else {
      F[0] = R->rho * unRr;
      for (int i = 0; i < 3; i++) F[1 + i] = R->rho * R->u[i] * unRr + R->p * nV[i];
      F[4] = eR * unRr + R->p * unR;
    }
  }
  for (int i = 0; i < 5; i++) F[i] *= area;
}

/* calcJacobianA, UgpWithCvCompFlow.cpp:666-709 (nV carries the area) */
static void jacobian_A(double A[5][5], const double *vel, double pp, double rrho, const double *nV, double gamma,
                       double surfVeloc) {
  double kapm1 = (gamma - 1.0);
  double nVel[3] = {vel[0] * nV[0], vel[1] * nV[1], vel[2] * nV[2]};
  double U_k = nVel[0] + nVel[1] + nVel[2];
  double vSquHlf = 0.5 * dot3(vel, vel);
  double c = sqrt(gamma * pp / rrho);
  double inv_kap_m1 = 1.0 / kapm1;
  A[0][0] = -surfVeloc; A[0][1] = nV[0]; A[0][2] = nV[1]; A[0][3] = nV[2]; A[0][4] = 0.0;
  A[1][0] = -vel[0] * (nVel[1] + nVel[2]) + nV[0] * (kapm1 * vSquHlf - vel[0] * vel[0]);
  A[1][1] = (2. - gamma) * nVel[0] + U_k - surfVeloc;
  A[1][2] = vel[0] * nV[1] - kapm1 * vel[1] * nV[0];
  A[1][3] = vel[0] * nV[2] - kapm1 * vel[2] * nV[0];
  A[1][4] = kapm1 * nV[0];
  A[2][0] = -vel[1] * (nVel[0] + nVel[2]) + nV[1] * (kapm1 * vSquHlf - vel[1] * vel[1]);
  A[2][1] = -kapm1 * vel[0] * nV[1] + vel[1] * nV[0];
  A[2][2] = (2. - gamma) * nVel[1] + U_k - surfVeloc;
  A[2][3] = vel[1] * nV[2] - kapm1 * vel[2] * nV[1];
  A[2][4] = kapm1 * nV[1];
  A[3][0] = -vel[2] * (nVel[0] + nVel[1]) + nV[2] * (kapm1 * vSquHlf - vel[2] * vel[2]);
  A[3][1] = -kapm1 * vel[0] * nV[2] + vel[2] * nV[0];
  A[3][2] = -kapm1 * vel[1] * nV[2] + vel[2] * nV[1];
  A[3][3] = (2. - gamma) * nVel[2] + U_k - surfVeloc;
  A[3][4] = kapm1 * nV[2];
  A[4][0] = U_k * ((gamma - 2.) * vSquHlf - c * c * inv_kap_m1);
  A[4][1] = c * c * inv_kap_m1 * nV[0] - kapm1 * vel[0] * (nVel[1] + nVel[2]) - (kapm1 * vel[0] * vel[0] - vSquHlf) * nV[0];
  A[4][2] = c * c * inv_kap_m1 * nV[1] - kapm1 * vel[1] * (nVel[0] + nVel[2]) - (kapm1 * vel[1] * vel[1] - vSquHlf) * nV[1];
  A[4][3] = c * c * inv_kap_m1 * nV[2] - kapm1 * vel[2] * (nVel[0] + nVel[1]) - (kapm1 * vel[2] * vel[2] - vSquHlf) * nV[2];
  A[4][4] = gamma * U_k - surfVeloc;
}

/* calcSubSonicJacobeanHLLC, UgpWithCvCompFlow.cpp:605-659 */
static void subsonic_jac_hllc(double (*AL)[5], double (*AR)[5], double rhoL, const double *uL, double pL, double eL,
                              double qL, double psiL, double SL, double rhoSL, const double *rhouSL, double eSL,
                              const double *dSMdUL, const double *dSMdUR, const double *dpsdUL, const double *dpsdUR,
                              double SM, double pS, double gamma, const double *nV) {
  double gm1 = (gamma - 1.0);
  double omL = 1.0 / (SL - SM);
  if (AL) {
    AL[0][0] = SL + rhoSL * dSMdUL[0];
    AL[0][1] = -nV[0] + rhoSL * dSMdUL[1];
    AL[0][2] = -nV[1] + rhoSL * dSMdUL[2];
    AL[0][3] = -nV[2] + rhoSL * dSMdUL[3];
    AL[0][4] = +rhoSL * dSMdUL[4];
    AL[1][0] = qL * uL[0] - nV[0] * psiL * gm1 / 2.0 + nV[0] * dpsdUL[0] + rhouSL[0] * dSMdUL[0];
    AL[1][1] = SL - qL + nV[0] * (gamma - 2.0) * uL[0] + nV[0] * dpsdUL[1] + rhouSL[0] * dSMdUL[1];
    AL[1][2] = -uL[0] * nV[1] + nV[0] * gm1 * uL[1] + nV[0] * dpsdUL[2] + rhouSL[0] * dSMdUL[2];
    AL[1][3] = -uL[0] * nV[2] + nV[0] * gm1 * uL[2] + nV[0] * dpsdUL[3] + rhouSL[0] * dSMdUL[3];
    AL[1][4] = -gm1 * nV[0] + nV[0] * dpsdUL[4] + rhouSL[0] * dSMdUL[4];
    AL[2][0] = qL * uL[1] - nV[1] * psiL * gm1 / 2.0 + nV[1] * dpsdUL[0] + rhouSL[1] * dSMdUL[0];
    AL[2][1] = -uL[1] * nV[0] + nV[1] * gm1 * uL[0] + nV[1] * dpsdUL[1] + rhouSL[1] * dSMdUL[1];
    AL[2][2] = SL - qL + nV[1] * (gamma - 2.0) * uL[1] + nV[1] * dpsdUL[2] + rhouSL[1] * dSMdUL[2];
    AL[2][3] = -uL[1] * nV[2] + nV[1] * gm1 * uL[2] + nV[1] * dpsdUL[3] + rhouSL[1] * dSMdUL[3];
    AL[2][4] = -gm1 * nV[1] + nV[1] * dpsdUL[4] + rhouSL[1] * dSMdUL[4];
    AL[3][0] = qL * uL[2] - nV[2] * psiL * gm1 / 2.0 + nV[2] * dpsdUL[0] + rhouSL[2] * dSMdUL[0];
    AL[3][1] = -uL[2] * nV[0] + nV[2] * gm1 * uL[0] + nV[2] * dpsdUL[1] + rhouSL[2] * dSMdUL[1];
    AL[3][2] = -uL[2] * nV[1] + nV[2] * gm1 * uL[1] + nV[2] * dpsdUL[2] + rhouSL[2] * dSMdUL[2];
    AL[3][3] = SL - qL + nV[2] * (gamma - 2.0) * uL[2] + nV[2] * dpsdUL[3] + rhouSL[2] * dSMdUL[3];
    AL[3][4] = -gm1 * nV[2] + nV[2] * dpsdUL[4] + rhouSL[2] * dSMdUL[4];
    AL[4][0] = qL * (eL + pL) / rhoL - qL * psiL * (gamma - 1.0) / 2.0 + SM * dpsdUL[0] + (pS + eSL) * dSMdUL[0];
    AL[4][1] = -nV[0] * (eL + pL) / rhoL + gm1 * uL[0] * qL + SM * dpsdUL[1] + (pS + eSL) * dSMdUL[1];
    AL[4][2] = -nV[1] * (eL + pL) / rhoL + gm1 * uL[1] * qL + SM * dpsdUL[2] + (pS + eSL) * dSMdUL[2];
    AL[4][3] = -nV[2] * (eL + pL) / rhoL + gm1 * uL[2] * qL + SM * dpsdUL[3] + (pS + eSL) * dSMdUL[3];
    AL[4][4] = SL - qL * gamma + SM * dpsdUL[4] + (pS + eSL) * dSMdUL[4];
    for (int i = 0; i < 5; i++)
      for (int j = 0; j < 5; j++) AL[i][j] *= omL;
  }
  if (AR) {
    for (int i = 0; i < 5; i++) AR[0][i] = omL * rhoSL * dSMdUR[i];
    for (int i = 0; i < 5; i++) AR[1][i] = omL * (nV[0] * dpsdUR[i] + rhouSL[0] * dSMdUR[i]);
    for (int i = 0; i < 5; i++) AR[2][i] = omL * (nV[1] * dpsdUR[i] + rhouSL[1] * dSMdUR[i]);
    for (int i = 0; i < 5; i++) AR[3][i] = omL * (nV[2] * dpsdUR[i] + rhouSL[2] * dSMdUR[i]);
    for (int i = 0; i < 5; i++) AR[4][i] = omL * (dpsdUR[i] * SM + (pS + eSL) * dSMdUR[i]);
  }
}

/* calcEulerFluxMatrices_HLLC, UgpWithCvCompFlow.cpp:242-595 (no scalars) */
static void matrices_hllc(double (*A_L)[5], double (*A_R)[5], const fstate *L, const fstate *R, double area,
                          const double *nV) {
  double rhoL = L->rho, pL = L->p, gammaL = L->gam;
  double rhoR = R->rho, pR = R->p, gammaR = R->gam;
  const double *uL = L->u, *uR = R->u;
  double unL = dot3(uL, nV);
  double uLuL = dot3(uL, uL);
  double cL = sqrt(gammaL * pL / rhoL);
  double hL = gammaL / (gammaL - 1.0) * pL / rhoL + 0.5 * uLuL + L->k;
  double eL = hL * rhoL - pL;
  double unR = dot3(uR, nV);
  double uRuR = dot3(uR, uR);
  double cR = sqrt(gammaR * pR / rhoR);
  double hR = gammaR / (gammaR - 1.0) * pR / rhoR + 0.5 * uRuR + R->k;
  double eR = hR * rhoR - pR;
  double Rrho = sqrt(rhoR / rhoL);
  double tmp = 1.0 / (1.0 + Rrho);
  double velRoe[3];
  for (int i = 0; i < 3; i++) velRoe[i] = tmp * (uL[i] + uR[i] * Rrho);
  double uRoe = dot3(velRoe, nV);
  double gamPdivRho = tmp * ((gammaL * pL / rhoL + 0.5 * (gammaL - 1.0) * uLuL) + (gammaR * pR / rhoR + 0.5 * (gammaR - 1.0) * uRuR) * Rrho);
  double cRoe = sqrt(gamPdivRho - ((gammaL + gammaR) * 0.5 - 1.0) * 0.5 * dot3(velRoe, velRoe));
  double sL = dmin(uRoe - cRoe, unL - cL);
  double sR = dmax(uRoe + cRoe, unR + cR);
  double sM = (pL - pR - rhoL * unL * (sL - unL) + rhoR * unR * (sR - unR)) / (rhoR * (sR - unR) - rhoL * (sL - unL));
  double pStar = rhoR * (unR - sR) * (unR - sM) + pR;
  double gmean = 0.5 * (gammaL + gammaR);
  if (sM >= 0.0) {
    if (sL > 0.0) {
      if (A_L) {
        double nA[3];
        for (int i = 0; i < 3; i++) nA[i] = nV[i] * area;
        jacobian_A(A_L, uL, pL, rhoL, nA, gmean, 0.0);
      }
      if (A_R)
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) A_R[i][j] = 0.0;
    } else {
      double invSLmSs = 1.0 / (sL - sM);
      double sLmuL = sL - unL;
      double rhoSL = rhoL * sLmuL * invSLmSs;
      double rhouSL[3];
      for (int i = 0; i < 3; i++) rhouSL[i] = (rhoL * uL[i] * sLmuL + (pStar - pL) * nV[i]) * invSLmSs;
      double eSL = (sLmuL * eL - pL * unL + pStar * sM) * invSLmSs;
      double gLm1 = gammaL - 1.0, gRm1 = gammaR - 1.0;
      double invrhotld = 1.0 / (rhoR * (sR - unR) - rhoL * (sL - unL));
      double dSMdUL[5] = {0}, dSMdUR[5] = {0}, dpsdUL[5] = {0}, dpsdUR[5] = {0};
      if (A_L) {
        dSMdUL[0] = -unL * unL + uLuL * gLm1 / 2.0 + sM * sL;
        dSMdUL[1] = nV[0] * (2.0 * unL - sL - sM) - gLm1 * uL[0];
        dSMdUL[2] = nV[1] * (2.0 * unL - sL - sM) - gLm1 * uL[1];
        dSMdUL[3] = nV[2] * (2.0 * unL - sL - sM) - gLm1 * uL[2];
        dSMdUL[4] = gLm1;
        for (int i = 0; i < 5; i++) { dSMdUL[i] *= invrhotld; dpsdUL[i] = rhoR * (sR - unR) * dSMdUL[i]; }
      }
      if (A_R) {
        dSMdUR[0] = unR * unR - uRuR * gRm1 / 2.0 - sM * sR;
        dSMdUR[1] = -nV[0] * (2.0 * unR - sR - sM) + gRm1 * uR[0];
        dSMdUR[2] = -nV[1] * (2.0 * unR - sR - sM) + gRm1 * uR[1];
        dSMdUR[3] = -nV[2] * (2.0 * unR - sR - sM) + gRm1 * uR[2];
        dSMdUR[4] = -gRm1;
        for (int i = 0; i < 5; i++) { dSMdUR[i] *= invrhotld; dpsdUR[i] = rhoL * (sL - unL) * dSMdUR[i]; }
      }
      subsonic_jac_hllc(A_L, A_R, rhoL, uL, pL, eL, unL, uLuL, sL, rhoSL, rhouSL, eSL, dSMdUL, dSMdUR, dpsdUL,
                        dpsdUR, sM, pStar, gmean, nV);
      if (A_L) {
        for (int i = 0; i < 5; i++) A_L[0][i] = A_L[0][i] * sM + dSMdUL[i] * rhoSL;
        for (int i = 0; i < 5; i++) A_L[1][i] = A_L[1][i] * sM + dSMdUL[i] * rhouSL[0] + dpsdUL[i] * nV[0];
        for (int i = 0; i < 5; i++) A_L[2][i] = A_L[2][i] * sM + dSMdUL[i] * rhouSL[1] + dpsdUL[i] * nV[1];
        for (int i = 0; i < 5; i++) A_L[3][i] = A_L[3][i] * sM + dSMdUL[i] * rhouSL[2] + dpsdUL[i] * nV[2];
        for (int i = 0; i < 5; i++) A_L[4][i] = (A_L[4][i] + dpsdUL[i]) * sM + (eSL + pStar) * dSMdUL[i];
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) A_L[i][j] *= area;
      }
      if (A_R) {
        for (int i = 0; i < 5; i++) A_R[0][i] = A_R[0][i] * sM + dSMdUR[i] * rhoSL;
        for (int i = 0; i < 5; i++) A_R[1][i] = A_R[1][i] * sM + dSMdUR[i] * rhouSL[0] + dpsdUR[i] * nV[0];
        for (int i = 0; i < 5; i++) A_R[2][i] = A_R[2][i] * sM + dSMdUR[i] * rhouSL[1] + dpsdUR[i] * nV[1];
        for (int i = 0; i < 5; i++) A_R[3][i] = A_R[3][i] * sM + dSMdUR[i] * rhouSL[2] + dpsdUR[i] * nV[2];
        for (int i = 0; i < 5; i++) A_R[4][i] = (A_R[4][i] + dpsdUR[i]) * sM + (eSL + pStar) * dSMdUR[i];
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) A_R[i][j] *= area;
      }
    }
  } else {
    if (sR >= 0.0) {
      double invSRmSs = 1.0 / (sR - sM);
      double sRmuR = sR - unR;
      double rhoSR = rhoR * sRmuR * invSRmSs;
      double rhouSR[3];
      for (int i = 0; i < 3; i++) rhouSR[i] = (rhoR * uR[i] * sRmuR + (pStar - pR) * nV[i]) * invSRmSs;
      double eSR = (sRmuR * eR - pR * unR + pStar * sM) * invSRmSs;
      double gLm1 = gammaL - 1.0, gRm1 = gammaR - 1.0;
      double invrhotld = 1.0 / (rhoR * (sR - unR) - rhoL * (sL - unL));
      double dSMdUL[5] = {0}, dSMdUR[5] = {0}, dpsdUL[5] = {0}, dpsdUR[5] = {0};
      if (A_L) {
        dSMdUL[0] = -unL * unL + uLuL * gLm1 / 2.0 + sM * sL;
        dSMdUL[1] = nV[0] * (2.0 * unL - sL - sM) - gLm1 * uL[0];
        dSMdUL[2] = nV[1] * (2.0 * unL - sL - sM) - gLm1 * uL[1];
        dSMdUL[3] = nV[2] * (2.0 * unL - sL - sM) - gLm1 * uL[2];
        dSMdUL[4] = gLm1;
        for (int i = 0; i < 5; i++) { dSMdUL[i] *= invrhotld; dpsdUL[i] = rhoR * (sR - unR) * dSMdUL[i]; }
      }
      if (A_R) {
        dSMdUR[0] = unR * unR - uRuR * gRm1 / 2.0 - sM * sR;
        dSMdUR[1] = -nV[0] * (2.0 * unR - sR - sM) + gRm1 * uR[0];
        dSMdUR[2] = -nV[1] * (2.0 * unR - sR - sM) + gRm1 * uR[1];
        dSMdUR[3] = -nV[2] * (2.0 * unR - sR - sM) + gRm1 * uR[2];
        dSMdUR[4] = -gRm1;
        for (int i = 0; i < 5; i++) { dSMdUR[i] *= invrhotld; dpsdUR[i] = rhoL * (sL - unL) * dSMdUR[i]; }
      }
      subsonic_jac_hllc(A_R, A_L, rhoR, uR, pR, eR, unR, uRuR, sR, rhoSR, rhouSR, eSR, dSMdUR, dSMdUL, dpsdUR,
                        dpsdUL, sM, pStar, gmean, nV);
      if (A_L) {
        for (int i = 0; i < 5; i++) A_L[0][i] = A_L[0][i] * sM + dSMdUL[i] * rhoSR;
        for (int i = 0; i < 5; i++) A_L[1][i] = A_L[1][i] * sM + dSMdUL[i] * rhouSR[0] + dpsdUL[i] * nV[0];
        for (int i = 0; i < 5; i++) A_L[2][i] = A_L[2][i] * sM + dSMdUL[i] * rhouSR[1] + dpsdUL[i] * nV[1];
        for (int i = 0; i < 5; i++) A_L[3][i] = A_L[3][i] * sM + dSMdUL[i] * rhouSR[2] + dpsdUL[i] * nV[2];
        for (int i = 0; i < 5; i++) A_L[4][i] = (A_L[4][i] + dpsdUL[i]) * sM + (eSR + pStar) * dSMdUL[i];
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) A_L[i][j] *= area;
      }
      if (A_R) {
        for (int i = 0; i < 5; i++) A_R[0][i] = A_R[0][i] * sM + dSMdUR[i] * rhoSR;
        for (int i = 0; i < 5; i++) A_R[1][i] = A_R[1][i] * sM + dSMdUR[i] * rhouSR[0] + dpsdUR[i] * nV[0];
        for (int i = 0; i < 5; i++) A_R[2][i] = A_R[2][i] * sM + dSMdUR[i] * rhouSR[1] + dpsdUR[i] * nV[1];
        for (int i = 0; i < 5; i++) A_R[3][i] = A_R[3][i] * sM + dSMdUR[i] * rhouSR[2] + dpsdUR[i] * nV[2];
        for (int i = 0; i < 5; i++) A_R[4][i] = (A_R[4][i] + dpsdUR[i]) * sM + (eSR + pStar) * dSMdUR[i];
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) A_R[i][j] *= area;
      }
    } else {
      if (A_R) {
        double nA[3];
        for (int i = 0; i < 3; i++) nA[i] = nV[i] * area;
        jacobian_A(A_R, uR, pR, rhoR, nA, gmean, 0.0);
      }
      if (A_L)
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) A_L[i][j] = 0.0;
    }
  }
}

/* calcEulerFlux_Roe, UgpWithCvCompFlow.cpp:3281-3380 (no entropy fix; when the
 * Roe-averaged c^2 < 1e-12 the reference returns with only the central part) */
static void flux_roe(double F[5], const fstate *L, const fstate *R, double area, const double *nV) {
  double rho0 = L->rho, rho1 = R->rho;
  const double *u0 = L->u, *u1 = R->u;
  double p0 = L->p, p1 = R->p;
  double gamma = 0.5 * (L->gam + R->gam);
  double gm1 = gamma - 1.0;
  double rhoun0 = rho0 * dot3(u0, nV);
  double rhoun1 = rho1 * dot3(u1, nV);
  double rhoE0 = p0 / gm1 + 0.5 * rho0 * dot3(u0, u0);
  double rhoE1 = p1 / gm1 + 0.5 * rho1 * dot3(u1, u1);
  double H0 = (rhoE0 + p0) / rho0, H1 = (rhoE1 + p1) / rho1;
  F[0] = 0.5 * area * (rhoun0 + rhoun1);
  F[1] = 0.5 * area * (rhoun0 * u0[0] + rhoun1 * u1[0] + (p0 + p1) * nV[0]);
  F[2] = 0.5 * area * (rhoun0 * u0[1] + rhoun1 * u1[1] + (p0 + p1) * nV[1]);
  F[3] = 0.5 * area * (rhoun0 * u0[2] + rhoun1 * u1[2] + (p0 + p1) * nV[2]);
  F[4] = 0.5 * area * (rhoun0 * H0 + rhoun1 * H1);
  double sqrt_rho0 = sqrt(rho0), sqrt_rho1 = sqrt(rho1);
  double tmp = 1.0 / (sqrt_rho0 + sqrt_rho1);
  double uAvg = tmp * (u0[0] * sqrt_rho0 + u1[0] * sqrt_rho1);
  double vAvg = tmp * (u0[1] * sqrt_rho0 + u1[1] * sqrt_rho1);
  double wAvg = tmp * (u0[2] * sqrt_rho0 + u1[2] * sqrt_rho1);
  double hAvg = tmp * (H0 * sqrt_rho0 + H1 * sqrt_rho1);
  double alphaAvg = 0.5 * (uAvg * uAvg + vAvg * vAvg + wAvg * wAvg);
  double a2Avg = gm1 * (hAvg - alphaAvg);
  if (a2Avg < 1.0E-12) return;
  double aAvg = sqrt(a2Avg);
  double unAvg = uAvg * nV[0] + vAvg * nV[1] + wAvg * nV[2];
  double dr = rho1 - rho0;
  double dru = rho1 * u1[0] - rho0 * u0[0];
  double drv = rho1 * u1[1] - rho0 * u0[1];
  double drw = rho1 * u1[2] - rho0 * u0[2];
  double drE = rhoE1 - rhoE0;
  double lam1 = fabs(unAvg), lam2 = fabs(unAvg + aAvg), lam3 = fabs(unAvg - aAvg);
  double abv1 = 0.5 * (lam2 + lam3);
  double abv2 = 0.5 * (lam2 - lam3);
  double abv3 = abv1 - lam1;
  double abv4 = gm1 * (alphaAvg * dr - uAvg * dru - vAvg * drv - wAvg * drw + drE);
  double abv5 = unAvg * dr - nV[0] * dru - nV[1] * drv - nV[2] * drw;
  double abv6 = abv3 * abv4 / a2Avg - abv2 * abv5 / aAvg;
  double abv7 = abv3 * abv5 - abv2 * abv4 / aAvg;
  F[0] -= 0.5 * area * (lam1 * dr + abv6);
  F[1] -= 0.5 * area * (lam1 * dru + uAvg * abv6 - nV[0] * abv7);
  F[2] -= 0.5 * area * (lam1 * drv + vAvg * abv6 - nV[1] * abv7);
  F[3] -= 0.5 * area * (lam1 * drw + wAvg * abv6 - nV[2] * abv7);
  F[4] -= 0.5 * area * (lam1 * drE + hAvg * abv6 - unAvg * abv7);
}

/* calcPMatrix / calcInvPMatrix, UgpWithCvCompFlow.cpp:3480-3559 */
static void p_matrix(double P[5][5], const double *vel, double c, double rrho, const double *nV, double gamma) {
  double kapm1 = (gamma - 1.0);
  double rhooc = rrho / c, rhoxc = rrho * c;
  double vSqu = dot3(vel, vel);
  P[0][0] = nV[0]; P[0][1] = nV[1]; P[0][2] = nV[2]; P[0][3] = 0.5 * rhooc; P[0][4] = 0.5 * rhooc;
  P[1][0] = vel[0] * nV[0]; P[1][1] = vel[0] * nV[1] - rrho * nV[2]; P[1][2] = vel[0] * nV[2] + rrho * nV[1];
  P[1][3] = 0.5 * (vel[0] * rhooc + rrho * nV[0]); P[1][4] = 0.5 * (vel[0] * rhooc - rrho * nV[0]);
  P[2][0] = vel[1] * nV[0] + rrho * nV[2]; P[2][1] = vel[1] * nV[1]; P[2][2] = vel[1] * nV[2] - rrho * nV[0];
  P[2][3] = 0.5 * (vel[1] * rhooc + rrho * nV[1]); P[2][4] = 0.5 * (vel[1] * rhooc - rrho * nV[1]);
  P[3][0] = vel[2] * nV[0] - rrho * nV[1]; P[3][1] = vel[2] * nV[1] + rrho * nV[0]; P[3][2] = vel[2] * nV[2];
  P[3][3] = 0.5 * (vel[2] * rhooc + rrho * nV[2]); P[3][4] = 0.5 * (vel[2] * rhooc - rrho * nV[2]);
  P[4][0] = 0.5 * vSqu * nV[0] + rrho * vel[1] * nV[2] - rrho * vel[2] * nV[1];
  P[4][1] = 0.5 * vSqu * nV[1] - rrho * vel[0] * nV[2] + rrho * vel[2] * nV[0];
  P[4][2] = 0.5 * vSqu * nV[2] + rrho * vel[0] * nV[1] - rrho * vel[1] * nV[0];
  P[4][3] = 0.5 * (0.5 * vSqu * rhooc + rrho * (vel[0] * nV[0] + vel[1] * nV[1] + vel[2] * nV[2]) + rhoxc / kapm1);
  P[4][4] = 0.5 * (0.5 * vSqu * rhooc - rrho * (vel[0] * nV[0] + vel[1] * nV[1] + vel[2] * nV[2]) + rhoxc / kapm1);
}

static void inv_p_matrix(double iP[5][5], const double *vel, double c, double rrho, const double *nV, double gamma) {
  double kapm1 = (gamma - 1.0);
  double rhoxc = rrho * c, c2 = c * c;
  double vSqu = dot3(vel, vel);
  iP[0][0] = nV[0] - nV[2] * vel[1] / rrho + nV[1] * vel[2] / rrho - nV[0] * 0.5 * kapm1 * vSqu / c2;
  iP[0][1] = nV[0] * kapm1 * vel[0] / c2;
  iP[0][2] = nV[2] / rrho + nV[0] * kapm1 * vel[1] / c2;
  iP[0][3] = -nV[1] / rrho + nV[0] * kapm1 * vel[2] / c2;
  iP[0][4] = -nV[0] * kapm1 / c2;
  iP[1][0] = nV[1] + nV[2] * vel[0] / rrho - nV[0] * vel[2] / rrho - nV[1] * 0.5 * kapm1 * vSqu / c2;
  iP[1][1] = -nV[2] / rrho + nV[1] * kapm1 * vel[0] / c2;
  iP[1][2] = nV[1] * kapm1 * vel[1] / c2;
  iP[1][3] = nV[0] / rrho + nV[1] * kapm1 * vel[2] / c2;
  iP[1][4] = -nV[1] * kapm1 / c2;
  iP[2][0] = nV[2] - nV[1] * vel[0] / rrho + nV[0] * vel[1] / rrho - nV[2] * 0.5 * kapm1 * vSqu / c2;
  iP[2][1] = nV[1] / rrho + nV[2] * kapm1 * vel[0] / c2;
  iP[2][2] = -nV[0] / rrho + nV[2] * kapm1 * vel[1] / c2;
  iP[2][3] = nV[2] * kapm1 * vel[2] / c2;
  iP[2][4] = -nV[2] * kapm1 / c2;
  iP[3][0] = -(nV[0] * vel[0] + nV[1] * vel[1] + nV[2] * vel[2]) / rrho + 0.5 * kapm1 * vSqu / rhoxc;
  iP[3][1] = nV[0] / rrho - kapm1 * vel[0] / rhoxc;
  iP[3][2] = nV[1] / rrho - kapm1 * vel[1] / rhoxc;
  iP[3][3] = nV[2] / rrho - kapm1 * vel[2] / rhoxc;
  iP[3][4] = kapm1 / rhoxc;
  iP[4][0] = (nV[0] * vel[0] + nV[1] * vel[1] + nV[2] * vel[2]) / rrho + 0.5 * kapm1 * vSqu / rhoxc;
  iP[4][1] = -nV[0] / rrho - kapm1 * vel[0] / rhoxc;
  iP[4][2] = -nV[1] / rrho - kapm1 * vel[1] / rhoxc;
  iP[4][3] = -nV[2] / rrho - kapm1 * vel[2] / rhoxc;
  iP[4][4] = kapm1 / rhoxc;
}

/* calcEulerFluxMatrices_Roe, UgpWithCvCompFlow.cpp:3382-3476 */
static void matrices_roe(double (*A_L)[5], double (*A_R)[5], const fstate *L, const fstate *R, double area,
                         const double *nV) {
  double rhoL = L->rho, pL = L->p, gammaL = L->gam;
  double rhoR = R->rho, pR = R->p, gammaR = R->gam;
  const double *uL = L->u, *uR = R->u;
  double uLuL = dot3(uL, uL), uRuR = dot3(uR, uR);
  double Rrho = sqrt(rhoR / rhoL);
  double rhoRoe = Rrho * rhoL;
  double tmp = 1.0 / (1.0 + Rrho);
  double velRoe[3];
  for (int i = 0; i < 3; i++) velRoe[i] = tmp * (uL[i] + uR[i] * Rrho);
  double uRoe = dot3(velRoe, nV);
  double gamPdivRho = tmp * ((gammaL * pL / rhoL + 0.5 * (gammaL - 1.0) * uLuL) + (gammaR * pR / rhoR + 0.5 * (gammaR - 1.0) * uRuR) * Rrho);
  double cRoe = sqrt(gamPdivRho - ((gammaL + gammaR) * 0.5 - 1.0) * 0.5 * dot3(velRoe, velRoe));
  double nA[3];
  for (int i = 0; i < 3; i++) nA[i] = nV[i] * area;
  double Lambda[5] = {uRoe, uRoe, uRoe, uRoe + cRoe, uRoe - cRoe};
  double P[5][5], iP[5][5];
  double gmean = 0.5 * (gammaL + gammaR);
  p_matrix(P, velRoe, cRoe, rhoRoe, nV, gmean);
  inv_p_matrix(iP, velRoe, cRoe, rhoRoe, nV, gmean);
  if (A_L) jacobian_A(A_L, uL, pL, rhoL, nA, gmean, 0.0);
  if (A_R) jacobian_A(A_R, uR, pR, rhoR, nA, gmean, 0.0);
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) {
      double pm = 0.0;
      for (int k = 0; k < 5; k++) pm += P[i][k] * fabs(Lambda[k]) * iP[k][j];
      if (A_L) A_L[i][j] = 0.5 * A_L[i][j] + 0.5 * pm * area;
      if (A_R) A_R[i][j] = 0.5 * A_R[i][j] - 0.5 * pm * area;
    }
}

/* calcEulerFlux_AUSM, UgpWithCvCompFlow.cpp:3566-3641 */
static void flux_ausm(double F[5], const fstate *L, const fstate *R, double area, const double *nV) {
  double rhoL = L->rho, pL = L->p, gammaL = L->gam;
  double rhoR = R->rho, pR = R->p, gammaR = R->gam;
  const double *uL = L->u, *uR = R->u;
  double unL = dot3(uL, nV), uLuL = dot3(uL, uL);
  double cL = sqrt(gammaL * pL / rhoL);
  double hL = (gammaL / (gammaL - 1.0)) * (pL / rhoL) + 0.5 * uLuL + L->k;
  double mL = unL / cL;
  double unR = dot3(uR, nV), uRuR = dot3(uR, uR);
  double cR = sqrt(gammaR * pR / rhoR);
  double hR = (gammaR / (gammaR - 1.0)) * (pR / rhoR) + 0.5 * uRuR + R->k;
  double mR = unR / cR;
  double mLP = (fabs(mL) <= 1.0) ? 0.25 * (mL + 1.0) * (mL + 1.0) : 0.5 * (mL + fabs(mL));
  double mRM = (fabs(mR) <= 1.0) ? -0.25 * (mR - 1.0) * (mR - 1.0) : 0.5 * (mR - fabs(mR));
  double mF = mLP + mRM;
  double pLP = (fabs(mL) <= 1.0) ? 0.25 * pL * (mL + 1.0) * (mL + 1.0) * (2.0 - mL) : 0.5 * pL * (mL + fabs(mL)) / mL;
  double pRM = (fabs(mR) <= 1.0) ? 0.25 * pR * (mR - 1.0) * (mR - 1.0) * (2.0 + mR) : 0.5 * pR * (mR - fabs(mR)) / mR;
  double pF = pLP + pRM;
  double Phi = fabs(mF);
  F[0] = 0.5 * (mF * ((rhoL * cL) + (rhoR * cR)) - Phi * ((rhoR * cR) - (rhoL * cL)));
  for (int i = 0; i < 3; i++)
    F[1 + i] = 0.5 * (mF * ((rhoL * cL * uL[i]) + (rhoR * cR * uR[i])) - Phi * ((rhoR * cR * uR[i]) - (rhoL * cL * uL[i]))) + nV[i] * pF;
  F[4] = 0.5 * (mF * ((rhoL * cL * hL) + (rhoR * cR * hR)) - Phi * ((rhoR * cR * hR) - (rhoL * cL * hL)));
  for (int i = 0; i < 5; i++) F[i] *= area;
}

/* Haenel & Schwane: calcEulerFlux_HAENEL and calcEulerFluxMatrices_HAENEL
 * (UgpWithCvCompFlow.cpp:1329-1505) with p_plusminus, u_plusminus (alpha 1),
 * drhou_plusminus_dQ and dp_plusminus_dQ (753-877) */
static double hs_p_pm(double p, double un, double c, double sign) {
  double M = sign * un / c;
  if (1.0 <= M) return p;
  else if (-1.0 <= M) return 0.25 * p * (M + 1.0) * (M + 1.0) * (2.0 - M);
  return 0.0;
}
static double hs_u_pm(double alpha, double un, double c, double sign) {
  double M = sign * un / c;
  if (1.0 <= M) return un;
  else if (0.0 <= M) return sign * alpha * c * 0.25 * (M + 1.0) * (M + 1.0) + (1.0 - alpha) * un;
  else if (-1.0 <= M) return sign * alpha * c * 0.25 * (M + 1.0) * (M + 1.0);
  return 0.0;
}
static void hs_drhou_pm(double *b, double alpha, double un, double c, const double *n, double sign) {
  double M = sign * un / c;
  if (1.0 <= M) {
    b[0] = 0.0;
    for (int i = 0; i < 3; i++) b[1 + i] = n[i];
  } else if (0.0 <= M) {
    b[0] = sign * 0.25 * alpha * c * (1.0 - M * M);
    for (int i = 0; i < 3; i++) b[1 + i] = n[i] * (0.5 * alpha * (M + 1.0) + (1.0 - alpha));
  } else if (-1.0 <= M) {
    b[0] = sign * 0.25 * alpha * c * (1.0 - M * M);
    for (int i = 0; i < 3; i++) b[1 + i] = n[i] * (0.5 * alpha * (M + 1.0));
  } else {
    b[0] = 0.0;
    for (int i = 0; i < 3; i++) b[1 + i] = 0.0;
  }
  b[4] = 0.0;
}
static void hs_dp_pm(double *d, const double *u, double rho, double p, double un, double uu, double ht, double c,
                     double gam, const double *n, double sign) {
  double M = sign * un / c;
  double dpdrho = gam * p / rho + (1.0 - gam) * (ht - uu);
  if (1.0 <= M) {
    d[0] = dpdrho;
    for (int i = 0; i < 3; i++) d[1 + i] = (1.0 - gam) * u[i];
    d[4] = (gam - 1.0);
  } else if (-1.0 <= M) {
    d[0] = 0.25 * (M + 1.0) * (M + 1.0) * (2.0 - M) * dpdrho - 0.75 * p / rho * (1.0 + M) * (1.0 - M) * M;
    for (int i = 0; i < 3; i++)
      d[1 + i] = 0.25 * (M + 1.0) * (M + 1.0) * (2.0 - M) * (1.0 - gam) * u[i] +
                 0.75 * p / (rho * c) * (1.0 + M) * (1.0 - M) * sign * n[i];
    d[4] = 0.25 * (M + 1.0) * (M + 1.0) * (2.0 - M) * (gam - 1.0);
  } else {
    for (int i = 0; i < 5; i++) d[i] = 0.0;
  }
}
static void flux_haenel(double F[5], const fstate *L, const fstate *R, double area, const double *nV) {
  double unL = dot3(L->u, nV), uLuL = dot3(L->u, L->u), cL = sqrt(L->gam * L->p / L->rho);
  double hL = L->h + 0.5 * uLuL + L->k;
  double unR = dot3(R->u, nV), uRuR = dot3(R->u, R->u), cR = sqrt(R->gam * R->p / R->rho);
  double hR = R->h + 0.5 * uRuR + R->k;
  double cLR = dmax(cL, cR);
  double p_half = hs_p_pm(L->p, unL, cLR, +1.0) + hs_p_pm(R->p, unR, cLR, -1.0);
  double uLp = hs_u_pm(1.0, unL, cLR, +1.0), uRm = hs_u_pm(1.0, unR, cLR, -1.0);
  F[0] = L->rho * uLp + R->rho * uRm;
  for (int i = 0; i < 3; i++) F[1 + i] = L->rho * uLp * L->u[i] + R->rho * uRm * R->u[i] + p_half * nV[i];
  F[4] = L->rho * uLp * hL + R->rho * uRm * hR;
  for (int i = 0; i < 5; i++) F[i] *= area;
}
static void haenel_side(double (*A)[5], const fstate *S, double uu, double hS, double upm, const double *beta,
                        const double *delta, double area, const double *nV) {
  for (int j = 0; j < 5; j++) {
    A[0][j] = beta[j];
    for (int i = 0; i < 3; i++) A[1 + i][j] = beta[j] * S->u[i] + delta[j] * nV[i];
    A[4][j] = beta[j] * hS;
  }
  for (int i = 0; i < 3; i++) {
    A[1 + i][0] += -upm * S->u[i];
    A[1 + i][1 + i] += upm;
  }
  A[4][0] += upm * ((S->gam - 1.0) * uu - S->gam * hS + S->gam * S->p / S->rho);
  for (int j = 0; j < 3; j++) A[4][1 + j] += upm * (1.0 - S->gam) * S->u[j];
  A[4][4] += upm * S->gam;
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) A[i][j] *= area;
}
static void matrices_haenel(double (*AL)[5], double (*AR)[5], const fstate *L, const fstate *R, double area,
                            const double *nV) {
  double unL = dot3(L->u, nV), uLuL = dot3(L->u, L->u), cL = sqrt(L->gam * L->p / L->rho);
  double hL = L->h + 0.5 * uLuL + L->k;
  double unR = dot3(R->u, nV), uRuR = dot3(R->u, R->u), cR = sqrt(R->gam * R->p / R->rho);
  double hR = R->h + 0.5 * uRuR + R->k;
  double cLR = dmax(cL, cR);
  double uLp = hs_u_pm(1.0, unL, cLR, 1.0), uRm = hs_u_pm(1.0, unR, cLR, -1.0);
  double bp[5], bm[5], dp[5], dm[5];
  hs_drhou_pm(bp, 1.0, unL, cLR, nV, +1.0);
  hs_drhou_pm(bm, 1.0, unR, cLR, nV, -1.0);
  hs_dp_pm(dp, L->u, L->rho, L->p, unL, uLuL, hL, cLR, L->gam, nV, +1.0);
  hs_dp_pm(dm, R->u, R->rho, R->p, unR, uRuR, hR, cLR, R->gam, nV, -1.0);
  if (AL) haenel_side(AL, L, uLuL, hL, uLp, bp, dp, area, nV);
  if (AR) haenel_side(AR, R, uRuR, hR, uRm, bm, dm, area, nV);
}

/* AUSMDV options of one face: the blend (JG_AUSM_*), the entropy fix, the face's shock fix
 * (JG_SHOCK_FIX_*: HAENEL selects the Haenel & Schwane flux, ALPHA_LR alpha from the densities) */
typedef struct { int type, efix, shock; } ausm_opt;

/* alpha_LR_L (UgpWithCvCompFlow.cpp:753-759) */
static double ausm_alpha_L(double pL, double rhoL, double pR, double rhoR, int shock) {
  if (shock == JG_SHOCK_FIX_ALPHA_LR) return 2.0 * (1.0 / rhoL) / ((1.0 / rhoL) + (1.0 / rhoR));
  return 2.0 * (pL / rhoL) / ((pL / rhoL) + (pR / rhoR));
}

static double ausm_s(double pL, double pR, int type) {
  if (type == JG_AUSM_DV) return 0.5 * dmin(1.0, (10.0 * fabs(pR - pL)) / dmin(pL, pR));
  if (type == JG_AUSM_V) return 0.5;
  return -0.5;
}

/* calcEulerFlux_AUSMDV (UgpWithCvCompFlow.cpp:879-971) */
static void flux_ausmdv(double F[5], const fstate *L, const fstate *R, double area, const double *nV, ausm_opt o) {
  double unL = dot3(L->u, nV), uLuL = dot3(L->u, L->u), cL = sqrt(L->gam * L->p / L->rho);
  double hL = L->h + 0.5 * uLuL + L->k;
  double alphaL = ausm_alpha_L(L->p, L->rho, R->p, R->rho, o.shock);
  double unR = dot3(R->u, nV), uRuR = dot3(R->u, R->u), cR = sqrt(R->gam * R->p / R->rho);
  double hR = R->h + 0.5 * uRuR + R->k;
  double alphaR = 2.0 - alphaL;
  double cLR = dmax(cL, cR);
  double p_half = hs_p_pm(L->p, unL, cLR, +1.0) + hs_p_pm(R->p, unR, cLR, -1.0);
  double unL_plus = hs_u_pm(alphaL, unL, cLR, +1.0);
  double unR_minus = hs_u_pm(alphaR, unR, cLR, -1.0);
  double rhou_half = L->rho * unL_plus + R->rho * unR_minus;
  double s = ausm_s(L->p, R->p, o.type);
  F[0] = rhou_half;
  if (rhou_half >= 0.0) {
    for (int i = 0; i < 3; i++)
      F[1 + i] = rhou_half * (L->u[i] - unL * nV[i]) +
                 nV[i] * (p_half + (0.5 + s) * (L->rho * unL * unL_plus + R->rho * unR * unR_minus) +
                          (0.5 - s) * rhou_half * unL);
    F[4] = rhou_half * hL;
  } else {
    for (int i = 0; i < 3; i++)
      F[1 + i] = rhou_half * (R->u[i] - unR * nV[i]) +
                 nV[i] * (p_half + (0.5 + s) * (L->rho * unL * unL_plus + R->rho * unR * unR_minus) +
                          (0.5 - s) * rhou_half * unR);
    F[4] = rhou_half * hR;
  }
  if (o.efix) {
    double dl;
    if ((unL <= -cL) && (unR >= cR)) dl = 0.0;
    else if (((unL - cL) < 0.0) && ((unR - cR) > 0.0)) dl = 0.125 * ((unR - cR) - (unL - cL));
    else if (((unL + cL) < 0.0) && ((unR + cR) > 0.0)) dl = 0.125 * ((unR + cR) - (unL + cL));
    else dl = 0.0;
    if (dl != 0.0) {
      F[0] -= dl * (R->rho - L->rho);
      for (int i = 0; i < 3; i++) F[1 + i] -= dl * (R->rho * R->u[i] - L->rho * L->u[i]);
      F[4] -= dl * (R->rho * hR - L->rho * hL);
    }
  }
  for (int i = 0; i < 5; i++) F[i] *= area;
}

/* one side of calcEulerFluxMatrices_AUSMDV (UgpWithCvCompFlow.cpp:978-1183): S this side, own: the
 * side is upwind (rho u_half's sign), ut / hu the upwind side's tangential velocity and total
 * enthalpy, un_o the other side's normal velocity */
static void ausmdv_side(double (*A)[5], const fstate *S, int own, double un, double uu, double hS, double upm,
                        double rhou_half, double s, const double *beta, const double *delta, const double *ut,
                        double hu, double un_o, const double *nV) {
  double unstar, dun[4];
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) A[i][j] = 0.0;
  if (own) {
    double eS = hS - S->p / S->rho;
    A[0][0] += beta[0];
    for (int j = 0; j < 3; j++) A[0][1 + j] += beta[1 + j];
    for (int i = 0; i < 3; i++) {
      A[1 + i][0] += beta[0] * ut[i] - rhou_half * ut[i] / S->rho;
      for (int j = 0; j < 3; j++) A[1 + i][1 + j] += beta[1 + j] * ut[i] - rhou_half * nV[i] * nV[j] / S->rho;
      A[1 + i][1 + i] += rhou_half / S->rho;
    }
    A[4][0] += beta[0] * hS + rhou_half * ((S->gam - 1.0) * uu - S->gam * eS) / S->rho;
    for (int j = 0; j < 3; j++) A[4][1 + j] += beta[1 + j] * hS - rhou_half * (S->gam - 1.0) * S->u[j] / S->rho;
    A[4][4] += rhou_half * S->gam / S->rho;
    unstar = un;
    dun[0] = -un / S->rho;
    for (int j = 0; j < 3; j++) dun[1 + j] = nV[j] / S->rho;
  } else {
    A[0][0] += beta[0];
    for (int j = 0; j < 3; j++) A[0][1 + j] += beta[1 + j];
    for (int i = 0; i < 3; i++) {
      A[1 + i][0] += beta[0] * ut[i];
      for (int j = 0; j < 3; j++) A[1 + i][1 + j] += beta[1 + j] * ut[i];
    }
    A[4][0] += beta[0] * hu;
    for (int j = 0; j < 3; j++) A[4][1 + j] += beta[1 + j] * hu;
    unstar = un_o;
    for (int j = 0; j < 4; j++) dun[j] = 0.0;
  }
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 4; j++)
      A[1 + i][j] += nV[i] * (beta[j] * ((0.5 + s) * un + (0.5 - s) * unstar) + (0.5 - s) * rhou_half * dun[j]);
    A[1 + i][0] += -nV[i] * (0.5 + s) * upm * un;
    for (int j = 0; j < 3; j++) A[1 + i][1 + j] += nV[i] * (0.5 + s) * upm * nV[j];
    for (int j = 0; j < 5; j++) A[1 + i][j] += nV[i] * delta[j];
  }
}

/* the entropy fix's part of one side (UgpWithCvCompFlow.cpp:1185-1283): sg = +1 for A_L, -1 for A_R */
static void ausmdv_efix_side(double (*A)[5], const fstate *S, const fstate *L, const fstate *R, double sg, double dl,
                             double un, double uu, double hS, double hL, double hR, const double *nV) {
  if (sg > 0.0) {
    A[0][0] += 0.125 * (dl + un / S->rho * (L->rho - R->rho));
    for (int i = 0; i < 3; i++) A[1 + i][0] += 0.125 * un / S->rho * (L->rho * L->u[i] - R->rho * R->u[i]);
    A[4][0] += 0.125 * (dl * ((1.0 - S->gam) * (hS - uu) + S->gam * S->p / S->rho) +
                        un / S->rho * (L->rho * hL - R->rho * hR));
    for (int j = 0; j < 3; j++) {
      A[0][1 + j] += -0.125 * nV[j] / S->rho * (L->rho - R->rho);
      A[1 + j][1 + j] += 0.125 * dl;
      for (int i = 0; i < 3; i++) A[1 + i][1 + j] += -0.125 * nV[j] / S->rho * (L->rho * L->u[i] - R->rho * R->u[i]);
      A[4][1 + j] += 0.125 * (dl * (1.0 - S->gam) * S->u[j] - nV[j] / S->rho * (L->rho * hL - R->rho * hR));
    }
    A[4][4] += 0.125 * dl * S->gam;
  } else {
    A[0][0] -= 0.125 * (dl + un / S->rho * (L->rho - R->rho));
    for (int i = 0; i < 3; i++) A[1 + i][0] -= 0.125 * un / S->rho * (L->rho * L->u[i] - R->rho * R->u[i]);
    A[4][0] -= 0.125 * (dl * ((1.0 - S->gam) * (hS - uu) + S->gam * S->p / S->rho) +
                        un / S->rho * (L->rho * hL - R->rho * hR));
    for (int j = 0; j < 3; j++) {
      A[0][1 + j] -= -0.125 * nV[j] / S->rho * (L->rho - R->rho);
      A[1 + j][1 + j] -= 0.125 * dl;
      for (int i = 0; i < 3; i++) A[1 + i][1 + j] -= -0.125 * nV[j] / S->rho * (L->rho * L->u[i] - R->rho * R->u[i]);
      A[4][1 + j] -= 0.125 * (dl * (1.0 - S->gam) * S->u[j] - nV[j] / S->rho * (L->rho * hL - R->rho * hR));
    }
    A[4][4] -= 0.125 * dl * S->gam;
  }
}

/* calcEulerFluxMatrices_AUSMDV (UgpWithCvCompFlow.cpp:978-1322) */
static void matrices_ausmdv(double (*AL)[5], double (*AR)[5], const fstate *L, const fstate *R, double area,
                            const double *nV, ausm_opt o) {
  double unL = dot3(L->u, nV), uLuL = dot3(L->u, L->u), cL = sqrt(L->gam * L->p / L->rho);
  double hL = L->h + 0.5 * uLuL + L->k;
  double alphaL = ausm_alpha_L(L->p, L->rho, R->p, R->rho, o.shock);
  double utL[3], utR[3];
  for (int i = 0; i < 3; i++) utL[i] = L->u[i] - unL * nV[i];
  double unR = dot3(R->u, nV), uRuR = dot3(R->u, R->u), cR = sqrt(R->gam * R->p / R->rho);
  double hR = R->h + 0.5 * uRuR + R->k;
  double alphaR = 2.0 - alphaL;
  for (int i = 0; i < 3; i++) utR[i] = R->u[i] - unR * nV[i];
  double cLR = dmax(cL, cR);
  double unL_plus = hs_u_pm(alphaL, unL, cLR, +1.0);
  double unR_minus = hs_u_pm(alphaR, unR, cLR, -1.0);
  double rhou_half = L->rho * unL_plus + R->rho * unR_minus;
  double s = ausm_s(L->p, R->p, o.type);
  double bp[5], bm[5], dp[5], dm[5];
  hs_drhou_pm(bp, alphaL, unL, cLR, nV, +1.0);
  hs_drhou_pm(bm, alphaR, unR, cLR, nV, -1.0);
  hs_dp_pm(dp, L->u, L->rho, L->p, unL, uLuL, hL, cLR, L->gam, nV, +1.0);
  hs_dp_pm(dm, R->u, R->rho, R->p, unR, uRuR, hR, cLR, R->gam, nV, -1.0);
  int ownL = rhou_half >= 0.0;
  if (AL) ausmdv_side(AL, L, ownL, unL, uLuL, hL, unL_plus, rhou_half, s, bp, dp, ownL ? utL : utR, hR, unR, nV);
  if (AR) ausmdv_side(AR, R, !ownL, unR, uRuR, hR, unR_minus, rhou_half, s, bm, dm, !ownL ? utR : utL, hL, unL, nV);
  if (o.efix) {
    double dl;
    if ((unL <= -cL) && (unR >= cR)) dl = 0.0;
    else if (((unL - cL) < 0.0) && ((unR - cR) > 0.0)) dl = ((unR - cR) - (unL - cL));
    else if (((unL + cL) < 0.0) && ((unR + cR) > 0.0)) dl = ((unR + cR) - (unL + cL));
    else dl = 0.0;
    if (dl != 0.0) {
      if (AL) ausmdv_efix_side(AL, L, L, R, +1.0, dl, unL, uLuL, hL, hL, hR, nV);
      if (AR) ausmdv_efix_side(AR, R, L, R, -1.0, dl, unR, uRuR, hR, hL, hR, nV);
    }
  }
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) {
      if (AL) AL[i][j] *= area;
      if (AR) AR[i][j] *= area;
    }
}

/* calcEulerFlux_JST (UgpWithCvCompFlow.cpp:4050-4160): central flux of the mean state plus the
 * blended second / fourth difference dissipation; J = {PressSensor, Lambda, NeighborCV,
 * Conserv_Und_Lapl[5]} of each side's cell (transported scalars: none) */
static void flux_jst(double F[5], const fstate *L, const fstate *R, double area, const double *nV, const double *JL,
                     const double *JR) {
  double Param_p = 0.3, Param_Kappa_2 = 0.5, Param_Kappa_4 = 0.02;
  double unL = dot3(L->u, nV), uLuL = dot3(L->u, L->u), cL = sqrt(L->gam * L->p / L->rho);
  double hL = L->gam / (L->gam - 1.0) * L->p / L->rho + 0.5 * uLuL + L->k;
  double unR = dot3(R->u, nV), uRuR = dot3(R->u, R->u), cR = sqrt(R->gam * R->p / R->rho);
  double hR = R->gam / (R->gam - 1.0) * R->p / R->rho + 0.5 * uRuR + R->k;
  double md = 0.5 * (L->rho + R->rho), mp = 0.5 * (L->p + R->p), mh = 0.5 * (hL + hR), mv[3];
  for (int i = 0; i < 3; i++) mv[i] = 0.5 * (L->u[i] + R->u[i]);
  double ru = md * mv[0], rv = md * mv[1], rw = md * mv[2], pf[5];
  pf[0] = ru * nV[0];
  pf[1] = (ru * mv[0] + mp) * nV[0];
  pf[2] = ru * mv[1] * nV[0];
  pf[3] = ru * mv[2] * nV[0];
  pf[4] = ru * mh * nV[0];
  pf[0] += rv * nV[1];
  pf[1] += rv * mv[0] * nV[1];
  pf[2] += (rv * mv[1] + mp) * nV[1];
  pf[3] += rv * mv[2] * nV[1];
  pf[4] += rv * mh * nV[1];
  pf[0] += rw * nV[2];
  pf[1] += rw * mv[0] * nV[2];
  pf[2] += rw * mv[1] * nV[2];
  pf[3] += (rw * mv[2] + mp) * nV[2];
  pf[4] += rw * mh * nV[2];
  for (int i = 0; i < 5; i++) F[i] = pf[i] * area;
  double dU[5], dL[5];
  dU[0] = L->rho - R->rho;
  for (int i = 0; i < 3; i++) dU[1 + i] = L->rho * L->u[i] - R->rho * R->u[i];
  dU[4] = L->rho * hL - R->rho * hR;
  for (int i = 0; i < 5; i++) dL[i] = JL[3 + i] - JR[3 + i];
  double lamL = (fabs(unL) + cL) * area, lamR = (fabs(unR) + cR) * area;
  double mlam = 0.5 * (lamL + lamR);
  double phiL = pow(JL[1] / (4.0 * mlam), Param_p), phiR = pow(JR[1] / (4.0 * mlam), Param_p);
  double stretch = 4.0 * phiL * phiR / (phiL + phiR);
  int nL = (int)JL[2], nR = (int)JR[2];
  double sc2 = 3.0 * ((double)nL + (double)nR) / ((double)nL * (double)nR);
  double sc4 = sc2 * sc2 / 4.0;
  double e2 = Param_Kappa_2 * 0.5 * (JL[0] + JR[0]) * sc2;
  double e4 = dmax(0.0, Param_Kappa_4 - e2) * sc4;
  for (int i = 0; i < 5; i++) F[i] += (e2 * dU[i] - e4 * dL[i]) * stretch * mlam;
}

/* calcJSTCoeff_Var (JoeWithModels.cpp:13435-13492): spectral radii, the pressure sensor and the
 * undivided Laplacian of the conserved state (rhoE + p for the energy) over the internal faces */
static void calc_jst_var(jo_case *h) {
  const jg_mesh *m = &h->m;
  for (int c = 0; c < h->ncv; c++) {
    h->p1_lapl[c] = 0.0;
    h->p2_lapl[c] = 0.0;
    for (int k = 0; k < 5; k++) h->jst[8 * c + 3 + k] = 0.0;
    h->jst[8 * c + 1] = 0.0;
  }
  for (int f = h->nfa_b; f < h->nfa; f++) {
    int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
    double nV[3];
    double area = norm3(nV, &m->fa_normal[3 * f]);
    double P0 = h->press[c0], P1 = h->press[c1];
    double a0 = sqrt(h->gam[c0] * P0 / h->rho[c0]), a1 = sqrt(h->gam[c1] * P1 / h->rho[c1]);
    double u0[3], u1[3];
    for (int i = 0; i < 3; i++) {
      u0[i] = h->rhou[3 * c0 + i] / h->rho[c0];
      u1[i] = h->rhou[3 * c1 + i] / h->rho[c1];
    }
    double l0 = 0.5 * (fabs(dot3(u0, nV)) + a0) * area, l1 = 0.5 * (fabs(dot3(u1, nV)) + a1) * area;
    h->jst[8 * c0 + 1] += l0;
    h->jst[8 * c0 + 1] += l1;
    h->jst[8 * c1 + 1] += l0;
    h->jst[8 * c1 + 1] += l1;
    h->p1_lapl[c0] += (P1 - P0);
    h->p1_lapl[c1] += (P0 - P1);
    h->p2_lapl[c0] += (P0 + P1);
    h->p2_lapl[c1] += (P0 + P1);
    double d[5];
    d[0] = h->rho[c0] - h->rho[c1];
    for (int i = 0; i < 3; i++) d[1 + i] = h->rhou[3 * c0 + i] - h->rhou[3 * c1 + i];
    d[4] = (h->rhoE[c0] + P0) - (h->rhoE[c1] + P1);
    int b0 = h->bcv[c0], b1 = h->bcv[c1];
    if ((!b0 && !b1) || (b0 && b1)) {
      for (int k = 0; k < 5; k++) h->jst[8 * c0 + 3 + k] -= d[k];
      for (int k = 0; k < 5; k++) h->jst[8 * c1 + 3 + k] += d[k];
    }
    if (!b0 && b1)
      for (int k = 0; k < 5; k++) h->jst[8 * c0 + 3 + k] -= d[k];
    if (b0 && !b1)
      for (int k = 0; k < 5; k++) h->jst[8 * c1 + 3 + k] += d[k];
  }
  for (int c = 0; c < h->ncv; c++) h->jst[8 * c] = fabs(h->p1_lapl[c]) / h->p2_lapl[c];
}

/* the face options: fo.shock = JG_SHOCK_FIX_HAENEL selects calcEulerFlux_HAENEL
 * (JoeWithModels.cpp:2970-2979, 3041-3050) */
static void euler_flux_o(int kind, double F[5], const fstate *L, const fstate *R, double area, const double *nV,
                         ausm_opt o, const double *JL, const double *JR) {
  if (kind == JG_FLUX_JST) flux_jst(F, L, R, area, nV, JL, JR);
  else if (kind == JG_FLUX_ROE) flux_roe(F, L, R, area, nV);
  else if (kind == JG_FLUX_AUSM) flux_ausm(F, L, R, area, nV);
  else if (kind == JG_FLUX_HAENEL) flux_haenel(F, L, R, area, nV);
  else if (kind == JG_FLUX_AUSMDV) {
    if (o.shock == JG_SHOCK_FIX_HAENEL) flux_haenel(F, L, R, area, nV);
    else flux_ausmdv(F, L, R, area, nV, o);
  } else flux_hllc(F, L, R, area, nV);
}

/* implicit matrices per flux choice: AUSM uses the HLLC matrices (JoeWithModels.cpp:3057-3061) */
static void euler_matrices_o(int kind, double (*AL)[5], double (*AR)[5], const fstate *L, const fstate *R,
                             double area, const double *nV, ausm_opt o) {
  if (kind == JG_FLUX_ROE) matrices_roe(AL, AR, L, R, area, nV);
  else if (kind == JG_FLUX_HAENEL) matrices_haenel(AL, AR, L, R, area, nV);
  else if (kind == JG_FLUX_AUSMDV) {
    if (o.shock == JG_SHOCK_FIX_HAENEL) matrices_haenel(AL, AR, L, R, area, nV);
    else matrices_ausmdv(AL, AR, L, R, area, nV, o);
  } else matrices_hllc(AL, AR, L, R, area, nV);
}

/* boundary faces and the per-face entry: AUSMDV without the shock fix */
static ausm_opt bnd_opt(const jg_params *p) {
  ausm_opt o = {p->ausm_type, p->entropy_fix, JG_SHOCK_FIX_NONE};
  return o;
}

/* boundary faces: JST takes the sensors of the boundary cell on both sides (JoeWithModels.cpp:3169-3178) */
static void euler_flux(int kind, double F[5], const fstate *L, const fstate *R, double area, const double *nV,
                       const jg_params *p, const double *J) {
  euler_flux_o(kind, F, L, R, area, nV, bnd_opt(p), J, J);
}

static void euler_matrices(int kind, double (*AL)[5], double (*AR)[5], const fstate *L, const fstate *R, double area,
                           const double *nV, const jg_params *p) {
  euler_matrices_o(kind, AL, AR, L, R, area, nV, bnd_opt(p));
}

/* AUSMDV's sonic test of an internal face at its cells' centre states (JoeWithModels.cpp:2765-2776) */
static int face_sonic(jo_case *h, int f) {
  const jg_mesh *m = &h->m;
  int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
  double nV[3];
  norm3(nV, &m->fa_normal[3 * f]);
  double unL = dot3(&h->vel[3 * c0], nV), unR = dot3(&h->vel[3 * c1], nV);
  double cL = sqrt(h->gam[c0] * h->press[c0] / h->rho[c0]), cR = sqrt(h->gam[c1] * h->press[c1] / h->rho[c1]);
  return (((unL - cL) > 0.0) && ((unR - cR) < 0.0)) || (((unL + cL) > 0.0) && ((unR + cR) < 0.0));
}

void jo_euler_flux_faces(int kind, int n, const double *L, const double *R, const double *area, const double *nvec,
                         double *F, double *AL, double *AR) {
  for (int f = 0; f < n; f++) {
    fstate sl = {L[6 * f], {L[6 * f + 1], L[6 * f + 2], L[6 * f + 3]}, L[6 * f + 4], L[6 * f + 5], 0.0, 0.0};
    fstate sr = {R[6 * f], {R[6 * f + 1], R[6 * f + 2], R[6 * f + 3]}, R[6 * f + 4], R[6 * f + 5], 0.0, 0.0};
    /* ideal-gas enthalpy from the state */
    sl.h = sl.gam * sl.p / ((sl.gam - 1.0) * sl.rho);
    sr.h = sr.gam * sr.p / ((sr.gam - 1.0) * sr.rho);
    /* kind 4: AUSMDV with the entropy fix, no shock fix */
    ausm_opt o = {JG_AUSM_DV, 1, JG_SHOCK_FIX_NONE};
    euler_flux_o(kind, &F[5 * f], &sl, &sr, area[f], &nvec[3 * f], o, NULL, NULL);
    if (AL || AR)
      euler_matrices_o(kind, AL ? (double(*)[5]) & AL[25 * f] : NULL, AR ? (double(*)[5]) & AR[25 * f] : NULL, &sl,
                       &sr, area[f], &nvec[3 * f], o);
  }
}

/* ------------------------------------------------------------------------ */
/* calcEulerFlux, JoeWithModels.cpp:2621-3589 (nScal == 0)                   */
/* ------------------------------------------------------------------------ */
static int csr_slot(const jg_mesh *m, int row, int col) {
  /* getImplDependencyIndex, UgpWithCv.h:745-755 */
  int k = m->nbocv_i[row];
  while (m->nbocv_v[++k] != col) {}
  return k;
}

static fstate cell_state(jo_case *h, int c) {
  fstate s = {h->rho[c], {h->vel[3 * c], h->vel[3 * c + 1], h->vel[3 * c + 2]}, h->press[c], h->gam[c], 0.0,
              h->enthalpy[c]};
  return s;
}
static fstate bfa_state(jo_case *h, int f) {
  fstate s = {h->rho_bfa[f], {h->vel_bfa[3 * f], h->vel_bfa[3 * f + 1], h->vel_bfa[3 * f + 2]}, h->p_bfa[f],
              h->gam_bfa[f], 0.0, h->h_bfa[f]};
  return s;
}

/* reconstruct rho, p, u at x_fa from cell c (JoeWithModels.cpp:2832-2921); returns 1 on first-order fallback */
static int reconstruct(jo_case *h, int c, int f, fstate *s) {
  double r0[3];
  for (int i = 0; i < 3; i++) r0[i] = h->m.x_fa[3 * f + i] - h->m.x_cv[3 * c + i];
  double rho0 = h->rho[c] + dot3(r0, &h->grad_rho[3 * c]);
  double p0 = h->press[c] + dot3(r0, &h->grad_p[3 * c]);
  int fallback = (p0 <= 0.0) || (rho0 <= 0.0);
  if (fallback) {
    s->rho = h->rho[c];
    s->p = h->press[c];
  } else {
    s->rho = rho0;
    s->p = p0;
    for (int i = 0; i < 3; i++) s->u[i] = h->vel[3 * c + i] + dot3(r0, &h->grad_u[9 * c + 3 * i]);
  }
  /* calcThermoProp_p at the face (ideal gas: gamma = GAMMA, R = R_gas) */
  s->gam = h->p.gamma;
  double T = s->p / (s->rho * h->p.R_gas);
  s->h = h->p.gamma * h->p.R_gas / (h->p.gamma - 1.0) * T;
  return fallback;
}

static void add_block(double *A, int slot, double (*B)[5], double sgn) {
  double *a = &A[25 * slot];
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) a[5 * i + j] += sgn * B[i][j];
}

static void calc_euler_flux(jo_case *h, double *rr, double *ru, double *rE, double *A, int implicit) {
  const jg_mesh *m = &h->m;
  const jg_params *p = &h->p;
  int kind = p->flux;
  /* JST: its coefficients of the current state first (JoeWithModels.cpp:2663-2664) */
  if (kind == JG_FLUX_JST) calc_jst_var(h);
  if (p->second_order) {
    grad_vector(h, h->grad_u, h->vel, h->vel_bfa, p->limiter, h->sos);
    for (int c = 0; c < h->ncv; c++) h->alpha_rho[c] = 1.0;
    grad_scalar(h, h->grad_rho, h->rho, h->rho_bfa, p->limiter, h->rho, h->alpha_rho);
    grad_scalar(h, h->grad_p, h->press, h->p_bfa, p->limiter, h->press, NULL);
  }
  /* AUSMDV shock sensor: flag the cells beside a sonic internal face (JoeWithModels.cpp:2753-2781) */
  double *flag = NULL;
  if (kind == JG_FLUX_AUSMDV && p->shock_fix != JG_SHOCK_FIX_NONE) {
    flag = dalloc(h->ncv);
    for (int f = h->nfa_b; f < h->nfa; f++)
      if (face_sonic(h, f)) {
        flag[m->cvofa[2 * f]] = 1.0;
        flag[m->cvofa[2 * f + 1]] = 1.0;
      }
  }
  const double flag_sum = p->shock_flag == JG_SHOCK_FLAG_TET ? 0.9 : 1.1;
  double Apl[5][5], Ami[5][5], F[5];
  for (int f = h->nfa_b; f < h->nfa; f++) {
    int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
    double nV[3];
    double area = norm3(nV, &m->fa_normal[3 * f]);
    fstate L = cell_state(h, c0), R = cell_state(h, c1);
    if (p->second_order) {
      reconstruct(h, c0, f, &L);
      reconstruct(h, c1, f, &R);
    }
    /* the face's shock fix (JoeWithModels.cpp:2933-2957): both (or either) cells flagged; with
     * SHOCKFIX_ACROSS_SHOCK defined (JoeWithModels.cpp:4) also on the sonic faces themselves */
    ausm_opt o = bnd_opt(p);
    if (flag && (flag[c0] + flag[c1]) > flag_sum) o.shock = p->shock_fix;
    euler_flux_o(kind, F, &L, &R, area, nV, o, &h->jst[8 * c0], &h->jst[8 * c1]);
    rr[c0] -= F[0]; for (int i = 0; i < 3; i++) ru[3 * c0 + i] -= F[1 + i]; rE[c0] -= F[4];
    rr[c1] += F[0]; for (int i = 0; i < 3; i++) ru[3 * c1 + i] += F[1 + i]; rE[c1] += F[4];
    for (int i = 0; i < 5; i++) { h->fscale[5 * c0 + i] += fabs(F[i]); h->fscale[5 * c1 + i] += fabs(F[i]); }
    if (implicit) {
      fstate L0 = cell_state(h, c0), R0 = cell_state(h, c1);
      euler_matrices_o(kind, Apl, Ami, &L0, &R0, area, nV, o);
      int n00 = m->nbocv_i[c0], n01 = csr_slot(m, c0, c1), n11 = m->nbocv_i[c1], n10 = csr_slot(m, c1, c0);
      add_block(A, n00, Apl, 1.0);
      add_block(A, n01, Ami, 1.0);
      add_block(A, n11, Ami, -1.0);
      add_block(A, n10, Apl, -1.0);
    }
  }
  for (int z = 0; z < m->nzones; z++) {
    const jg_zone *zn = &m->zones[z];
    for (int f = zn->ifa_f; f <= zn->ifa_l; f++) {
      int c0 = m->cvofa[2 * f];
      double nV[3];
      double area = norm3(nV, &m->fa_normal[3 * f]);
      int n00 = m->nbocv_i[c0];
      if (zn->kind == JG_BC_SYMMETRY) {
        fstate B = bfa_state(h, f);
        euler_flux(kind, F, &B, &B, area, nV, p, &h->jst[8 * c0]);
        for (int i = 0; i < 5; i++) h->fscale[5 * c0 + i] += fabs(F[i]);
        if (p->symm_bc == JG_SYMM_ANALYTICAL) {
          for (int i = 0; i < 3; i++) ru[3 * c0 + i] -= h->p_bfa[f] * nV[i] * area;
        } else {
          rr[c0] -= F[0]; for (int i = 0; i < 3; i++) ru[3 * c0 + i] -= F[1 + i]; rE[c0] -= F[4];
        }
        if (implicit) {
          euler_matrices(kind, Apl, Ami, &B, &B, area, nV, p);
          if (p->symm_bc == JG_SYMM_ORIGINAL_NUMERIC) add_block(A, n00, Apl, 1.0);
          else if (p->symm_bc == JG_SYMM_NEW_NUMERIC) {
            double S[5][5];
            for (int i = 0; i < 5; i++)
              for (int j = 0; j < 5; j++) S[i][j] = Apl[i][j] + Ami[i][j];
            add_block(A, n00, S, 1.0);
          }
          else {
            /* analytical pressure Jacobian, JoeWithModels.cpp:3231-3251 */
            double S[5][5];
            const double *vb = &h->vel_bfa[3 * f];
            double a2 = h->gam_bfa[f] - 1.0;
            double phi = 0.5 * a2 * (vb[0] * vb[0] + vb[1] * vb[1] + vb[2] * vb[2]);
            for (int i = 0; i < 5; i++) { S[0][i] = 0.0; S[4][i] = 0.0; }
            for (int i = 0; i < 3; i++) {
              S[i + 1][0] = phi * nV[i] * area;
              for (int j = 0; j < 3; j++) S[i + 1][j + 1] = -a2 * vb[j] * nV[i] * area;
              S[i + 1][4] = a2 * nV[i] * area;
            }
            add_block(A, n00, S, 1.0);
          }
        }
      } else if (zn->kind == JG_BC_WALL) {
        fstate B = bfa_state(h, f);
        euler_flux(kind, F, &B, &B, area, nV, p, &h->jst[8 * c0]);
        rr[c0] -= F[0]; for (int i = 0; i < 3; i++) ru[3 * c0 + i] -= F[1 + i]; rE[c0] -= F[4];
        for (int i = 0; i < 5; i++) h->fscale[5 * c0 + i] += fabs(F[i]);
        if (implicit) {
          euler_matrices(kind, Apl, NULL, &B, &B, area, nV, p);
          add_block(A, n00, Apl, 1.0);
        }
      } else {
        fstate L = cell_state(h, c0);
        if (p->second_order) reconstruct(h, c0, f, &L);
        fstate B = bfa_state(h, f);
        euler_flux(kind, F, &L, &B, area, nV, p, &h->jst[8 * c0]);
        rr[c0] -= F[0]; for (int i = 0; i < 3; i++) ru[3 * c0 + i] -= F[1 + i]; rE[c0] -= F[4];
        for (int i = 0; i < 5; i++) h->fscale[5 * c0 + i] += fabs(F[i]);
        if (implicit) {
          fstate L0 = cell_state(h, c0);
          euler_matrices(kind, Apl, NULL, &L0, &B, area, nV, p);
          add_block(A, n00, Apl, 1.0);
        }
      }
    }
  }
  free(flag);
}

/* ------------------------------------------------------------------------ */
/* viscous flux: addViscFlux, UgpWithCvCompFlow.cpp:1521-1763                */
/* ------------------------------------------------------------------------ */
static void add_visc_flux(jo_case *h, double Fu[3], double *FE, double (*A0)[5], double (*A1)[5], double rho0,
                          const double *u0, const double *gu0, double h0, const double *gh0, double T0, double R0,
                          double gam0, double rho1, const double *u1, const double *gu1, double h1, const double *gh1,
                          double T1, double R1, double gam1, double mul, double mut, double lamOcp,
                          const double *u_fa, double area, const double *nV, double smag, const double *sV) {
  double alpha = dot3(nV, sV);
  double g[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) g[i][j] = 0.5 * (gu0[3 * i + j] + gu1[3 * i + j]);
  double fC[3] = {nV[0] - alpha * sV[0], nV[1] - alpha * sV[1], nV[2] - alpha * sV[2]};
  double tl[3], tt[3], tau[3];
  double nonL = 0.0;
  for (int i = 0; i < 3; i++)
    tl[i] = mul * (alpha * (u1[i] - u0[i]) / smag + g[i][0] * fC[0] + g[0][i] * nV[0] + g[i][1] * fC[1] +
                   g[1][i] * nV[1] + g[i][2] * fC[2] + g[2][i] * nV[2]);
  double tmp = 2.0 / 3.0 * mul * (g[0][0] + g[1][1] + g[2][2]);
  for (int i = 0; i < 3; i++) tl[i] -= tmp * nV[i];
  for (int i = 0; i < 3; i++)
    tt[i] = (1.0 - nonL) * mut * (alpha * (u1[i] - u0[i]) / smag + g[i][0] * fC[0] + g[0][i] * nV[0] + g[i][1] * fC[1] +
                                  g[1][i] * nV[1] + g[i][2] * fC[2] + g[2][i] * nV[2]);
  tmp = (1.0 - nonL) * 2.0 / 3.0 * mut * (g[0][0] + g[1][1] + g[2][2]);
  for (int i = 0; i < 3; i++) tt[i] -= tmp * nV[i];
  /* Reynolds-stress terms vanish (nonLinear = 0, rij = 0) */
  for (int i = 0; i < 3; i++) tau[i] = tl[i] + tt[i];
  for (int i = 0; i < 3; i++) Fu[i] = -area * tau[i];
  double keff = lamOcp + mut / h->p.PrTurb;
  double enth = keff * (alpha * (h1 - h0) / smag +
                        0.5 * ((gh0[0] + gh1[0]) * fC[0] + (gh0[1] + gh1[1]) * fC[1] + (gh0[2] + gh1[2]) * fC[2]));
  double psi = 0.0;
  *FE = -area * (enth + tau[0] * u_fa[0] + tau[1] * u_fa[1] + tau[2] * u_fa[2] + psi);

  for (int side = 0; side < 2; side++) {
    double (*Ax)[5] = side == 0 ? A0 : A1;
    if (!Ax) continue;
    double fU[5][5] = {{0}}, UQ[5][5] = {{0}};
    double d = (side == 0) ? -(mul + mut) * alpha / smag * area : (mul + mut) * alpha / smag * area;
    fU[1][1] = d; fU[2][2] = d; fU[3][3] = d;
    fU[4][1] = area * tau[0] * 0.5 + u_fa[0] * fU[1][1];
    fU[4][2] = area * tau[1] * 0.5 + u_fa[1] * fU[2][2];
    fU[4][3] = area * tau[2] * 0.5 + u_fa[2] * fU[3][3];
    fU[4][4] = (side == 0) ? -area * keff * alpha / smag : area * keff * alpha / smag;
    double r = side == 0 ? rho0 : rho1;
    const double *u = side == 0 ? u0 : u1;
    double hh = side == 0 ? h0 : h1, TT = side == 0 ? T0 : T1, RR = side == 0 ? R0 : R1, gg = side == 0 ? gam0 : gam1;
    double kine = 0.0;
    double invRho = 1.0 / r;
    UQ[1][0] = -u[0] * invRho;
    UQ[2][0] = -u[1] * invRho;
    UQ[3][0] = -u[2] * invRho;
    UQ[4][0] = gg * invRho * (-hh - kine + RR * TT + 0.5 * dot3(u, u));
    UQ[1][1] = invRho; UQ[4][1] = -gg * u[0] * invRho;
    UQ[2][2] = invRho; UQ[4][2] = -gg * u[1] * invRho;
    UQ[3][3] = invRho; UQ[4][3] = -gg * u[2] * invRho;
    UQ[4][4] = gg * invRho;
    /* dFdU_times_dUdQ, UgpWithCvCompFlow.cpp:717-745 (rows 1..4; column 4 only in row 4) */
    for (int i = 1; i < 4; i++) Ax[i][0] = fU[i][1] * UQ[1][0] + fU[i][2] * UQ[2][0] + fU[i][3] * UQ[3][0];
    Ax[4][0] = fU[4][1] * UQ[1][0] + fU[4][2] * UQ[2][0] + fU[4][3] * UQ[3][0] + fU[4][4] * UQ[4][0];
    for (int i = 1; i < 4; i++) Ax[i][1] = fU[i][1] * UQ[1][1];
    Ax[4][1] = fU[4][1] * UQ[1][1] + fU[4][4] * UQ[4][1];
    for (int i = 1; i < 4; i++) Ax[i][2] = fU[i][2] * UQ[2][2];
    Ax[4][2] = fU[4][2] * UQ[2][2] + fU[4][4] * UQ[4][2];
    for (int i = 1; i < 4; i++) Ax[i][3] = fU[i][3] * UQ[3][3];
    Ax[4][3] = fU[4][3] * UQ[3][3] + fU[4][4] * UQ[4][3];
    Ax[4][4] = fU[4][1] * UQ[1][4] + fU[4][2] * UQ[2][4] + fU[4][3] * UQ[3][4] + fU[4][4] * UQ[4][4];
  }
}

/* addViscFlux per face, batched (test entry): S0/S1[n][8] = (rho, u, v, w, h, T, R, gamma) of the two
 * sides, gu0/gu1[n][9] velocity gradients, gh0/gh1[n][3] enthalpy gradients, mul/lamOcp[n] at the
 * face, u_fa[n][3], area[n], nV/sV[n][3] unit normal and unit cell-to-cell vector, smag[n];
 * F[n][4] = (Frhou, FrhoE), A0/A1[n][5][5] (may be NULL).  No turbulent viscosity. */
void jo_visc_flux_faces(int n, const double *S0, const double *S1, const double *gu0, const double *gu1,
                        const double *gh0, const double *gh1, const double *mul, const double *lamOcp,
                        const double *u_fa, const double *area, const double *nV, const double *sV,
                        const double *smag, double *F, double *A0, double *A1) {
  jo_case tmp;
  memset(&tmp, 0, sizeof(tmp));
  tmp.p.PrTurb = 0.9;
  for (int f = 0; f < n; f++) {
    const double *a = &S0[8 * f], *b = &S1[8 * f];
    double Fu[3], FE;
    add_visc_flux(&tmp, Fu, &FE, A0 ? (double(*)[5]) & A0[25 * f] : NULL, A1 ? (double(*)[5]) & A1[25 * f] : NULL,
                  a[0], &a[1], &gu0[9 * f], a[4], &gh0[3 * f], a[5], a[6], a[7], b[0], &b[1], &gu1[9 * f], b[4],
                  &gh1[3 * f], b[5], b[6], b[7], mul[f], 0.0, lamOcp[f], &u_fa[3 * f], area[f], &nV[3 * f], smag[f],
                  &sV[3 * f]);
    for (int i = 0; i < 3; i++) F[4 * f + i] = Fu[i];
    F[4 * f + 3] = FE;
  }
}

/* calcViscousFluxNS, JoeWithModels.cpp:3591-3855 */
static void calc_viscous_flux(jo_case *h, double *ru, double *rE, double *A, int implicit) {
  const jg_mesh *m = &h->m;
  const jg_params *p = &h->p;
  if (p->visc_limiter) {
    if (!p->second_order) grad_vector(h, h->grad_u, h->vel, h->vel_bfa, p->limiter, h->sos);
    grad_scalar(h, h->grad_h, h->enthalpy, h->h_bfa, p->limiter, h->enthalpy, NULL);
  } else {
    grad_vector(h, h->grad_u, h->vel, h->vel_bfa, 0, h->sos);
    grad_scalar(h, h->grad_h, h->enthalpy, h->h_bfa, 0, h->enthalpy, NULL);
  }
  double A0[5][5] = {{0}}, A1[5][5] = {{0}};
  double Fu[3], FE;
  for (int f = h->nfa_b; f < h->nfa; f++) {
    int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
    double nV[3];
    double area = norm3(nV, &m->fa_normal[3 * f]);
    double sV[3];
    for (int i = 0; i < 3; i++) sV[i] = m->x_cv[3 * c1 + i] - m->x_cv[3 * c0 + i];
    double smag = norm3(sV, sV);
    double ufa[3] = {0.5 * (h->vel[3 * c0] + h->vel[3 * c1]), 0.5 * (h->vel[3 * c0 + 1] + h->vel[3 * c1 + 1]),
                     0.5 * (h->vel[3 * c0 + 2] + h->vel[3 * c1 + 2])};
    add_visc_flux(h, Fu, &FE, implicit ? A0 : NULL, implicit ? A1 : NULL, h->rho[c0], &h->vel[3 * c0],
                  &h->grad_u[9 * c0], h->enthalpy[c0], &h->grad_h[3 * c0], h->temp[c0], h->RoM[c0], h->gam[c0],
                  h->rho[c1], &h->vel[3 * c1], &h->grad_u[9 * c1], h->enthalpy[c1], &h->grad_h[3 * c1], h->temp[c1],
                  h->RoM[c1], h->gam[c1], h->mul_fa[f], h->mut_fa[f], h->lamOcp_fa[f], ufa, area, nV, smag, sV);
    if (implicit) {
      int n00 = m->nbocv_i[c0], n01 = csr_slot(m, c0, c1), n11 = m->nbocv_i[c1], n10 = csr_slot(m, c1, c0);
      for (int i = 1; i < 5; i++)
        for (int j = 0; j < 5; j++) {
          A[25 * n00 + 5 * i + j] -= A0[i][j];
          A[25 * n01 + 5 * i + j] -= A1[i][j];
          A[25 * n11 + 5 * i + j] += A1[i][j];
          A[25 * n10 + 5 * i + j] += A0[i][j];
        }
    }
    for (int i = 0; i < 3; i++) ru[3 * c0 + i] -= Fu[i];
    rE[c0] -= FE;
    for (int i = 0; i < 3; i++) ru[3 * c1 + i] += Fu[i];
    rE[c1] += FE;
    for (int i = 0; i < 3; i++) { h->fscale[5 * c0 + 1 + i] += fabs(Fu[i]); h->fscale[5 * c1 + 1 + i] += fabs(Fu[i]); }
    h->fscale[5 * c0 + 4] += fabs(FE); h->fscale[5 * c1 + 4] += fabs(FE);
  }
  for (int z = 0; z < m->nzones; z++) {
    const jg_zone *zn = &m->zones[z];
    if (zn->kind == JG_BC_SYMMETRY) continue; /* nothing without a turbulence model */
    for (int f = zn->ifa_f; f <= zn->ifa_l; f++) {
      int c0 = m->cvofa[2 * f];
      double nV[3];
      double area = norm3(nV, &m->fa_normal[3 * f]);
      double sV[3];
      for (int i = 0; i < 3; i++) sV[i] = m->x_fa[3 * f + i] - m->x_cv[3 * c0 + i];
      double smag;
      const double *sVec;
      double mut;
      if (zn->kind == JG_BC_WALL) {
        smag = fabs(dot3(sV, nV));  /* project onto the wall normal, use nVec as sVec */
        sVec = nV;
        mut = 0.0;
      } else {
        smag = norm3(sV, sV);
        sVec = sV;
        mut = h->mut_fa[f];
      }
      add_visc_flux(h, Fu, &FE, implicit ? A0 : NULL, NULL, h->rho[c0], &h->vel[3 * c0], &h->grad_u[9 * c0],
                    h->enthalpy[c0], &h->grad_h[3 * c0], h->temp[c0], h->RoM[c0], h->gam[c0], h->rho_bfa[f],
                    &h->vel_bfa[3 * f], &h->grad_u[9 * c0], h->h_bfa[f], &h->grad_h[3 * c0], h->T_bfa[f],
                    h->RoM_bfa[f], h->gam_bfa[f], h->mul_fa[f], mut, h->lamOcp_fa[f], &h->vel_bfa[3 * f], area, nV,
                    smag, sVec);
      if (implicit) {
        int n00 = m->nbocv_i[c0];
        for (int i = 1; i < 5; i++)
          for (int j = 0; j < 5; j++) A[25 * n00 + 5 * i + j] -= A0[i][j];
      }
      for (int i = 0; i < 3; i++) ru[3 * c0 + i] -= Fu[i];
      rE[c0] -= FE;
      for (int i = 0; i < 3; i++) h->fscale[5 * c0 + 1 + i] += fabs(Fu[i]);
      h->fscale[5 * c0 + 4] += fabs(FE);
    }
  }
}

void jo_calc_rhs(jo_case *h, double *rr, double *ru, double *rE, double *A, int implicit) {
  /* calcRhs, JoeWithModels.cpp:2564-2619 */
  memset(rr, 0, sizeof(double) * h->ncv);
  memset(ru, 0, sizeof(double) * 3 * h->ncv);
  memset(rE, 0, sizeof(double) * h->ncv);
  memset(h->fscale, 0, sizeof(double) * 5 * h->ncv);
  calc_euler_flux(h, rr, ru, rE, A, implicit);
  if (h->p.mu_ref > 0.0) calc_viscous_flux(h, ru, rE, A, implicit);
  /* sourceHook: gravity (JoeWithModels.h:111-129) */
  const double *g = h->p.gravity;
  for (int c = 0; c < h->ncv; c++) {
    double vol = h->m.cv_volume[c];
    ru[3 * c + 0] += vol * h->rho[c] * g[0];
    ru[3 * c + 1] += vol * h->rho[c] * g[1];
    ru[3 * c + 2] += vol * h->rho[c] * g[2];
    rE[c] += vol * (g[0] * h->rhou[3 * c + 0] + g[1] * h->rhou[3 * c + 1] + g[2] * h->rhou[3 * c + 2]);
    if (A && implicit) {
      double *a = &A[25 * (size_t)h->m.nbocv_i[c]];
      a[5 * 1 + 0] -= vol * g[0];
      a[5 * 2 + 0] -= vol * g[1];
      a[5 * 3 + 0] -= vol * g[2];
      a[5 * 4 + 1] -= vol * g[0];
      a[5 * 4 + 2] -= vol * g[1];
      a[5 * 4 + 3] -= vol * g[2];
    }
  }
}

/* ------------------------------------------------------------------------ */
/* linear solvers, UgpWithCv.cpp:2489-2876, 3172-3329                        */
/* ------------------------------------------------------------------------ */
static void ludeco(double (*A)[5], int order) {
  for (int jc = 1; jc < order; jc++) A[0][jc] /= A[0][0];
  int jrjc = 0;
  for (;;) {
    jrjc++;
    int jrjcm1 = jrjc - 1, jrjcp1 = jrjc + 1;
    for (int jr = jrjc; jr < order; jr++) {
      double sum = A[jr][jrjc];
      for (int jm = 0; jm <= jrjcm1; jm++) sum -= A[jr][jm] * A[jm][jrjc];
      A[jr][jrjc] = sum;
    }
    if (jrjc == (order - 1)) return;
    for (int jc = jrjcp1; jc < order; jc++) {
      double sum = A[jrjc][jc];
      for (int jm = 0; jm <= jrjcm1; jm++) sum -= A[jrjc][jm] * A[jm][jc];
      A[jrjc][jc] = sum / A[jrjc][jrjc];
    }
  }
}

static void lusolv(double (*A)[5], double *c, int order) {
  c[0] = c[0] / A[0][0];
  for (int jr = 1; jr < order; jr++) {
    double sum = c[jr];
    for (int jm = 0; jm <= jr - 1; jm++) sum -= A[jr][jm] * c[jm];
    c[jr] = sum / A[jr][jr];
  }
  for (int jrjr = 1; jrjr < order; jrjr++) {
    int jr = (order - 1) - jrjr;
    int jrp1 = jr + 1;
    double sum = c[jr];
    for (int jmjm = jrp1; jmjm < order; jmjm++) {
      int jm = (order - 1) - jmjm + jrp1;
      sum -= A[jr][jm] * c[jm];
    }
    c[jr] = sum;
  }
}

static void matvec(jo_case *h, double *res, const double *A, const double *x) {
  /* matTimesVecOverCVs, UgpWithCv.cpp:2580-2596 */
  const jg_mesh *m = &h->m;
  for (int c = 0; c < h->ncv; c++) {
    for (int i = 0; i < 5; i++) res[5 * c + i] = 0.0;
    for (int k = m->nbocv_i[c]; k < m->nbocv_i[c + 1]; k++) {
      int nb = m->nbocv_v[k];
      for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) res[5 * c + i] += A[25 * k + 5 * i + j] * x[5 * nb + j];
    }
  }
}

/* findFace (JoeWithModels.cpp:7572-7587): the first face of cell a's list that cell b also has */
static int find_face(const jg_mesh *m, int a, int b) {
  if (a == b) return -1;
  for (int i = m->faocv_i[a]; i < m->faocv_i[a + 1]; i++)
    for (int j = m->faocv_i[b]; j < m->faocv_i[b + 1]; j++)
      if (m->faocv_v[i] == m->faocv_v[j]) return m->faocv_v[i];
  return -1;
}

/* initializeLinelet (JoeWithModels.cpp:7471-7559).  Sources are the cells of
 * the WALL faces; as in the reference, each WALL zone replaces the sources of
 * the previous one (only the last WALL zone starts lines) while every WALL
 * zone's cells are taken out of later lines.  From each source a line grows
 * to the one unused neighbour (not the cell it came from) whose weight
 * 0.5 |A_f| (1/V_cell + 1/V_nb) exceeds half the cell's largest neighbour
 * weight; two or more candidates (an isotropic region) or none end it.
 * With `relaxed` (the lines of the LINE relaxation, not the reference's),
 * every WALL zone's cells start lines, and a
 * line also goes on when several candidates pass but the strongest is more
 * than 1.1 times the next: so it crosses from a prism row into the hexahedron
 * above, whose other lower neighbour is the second prism of the quad. */
static void build_lines(jo_case *h, int relaxed, int *nlines_out, int **off_out, int **cv_out) {
  const jg_mesh *m = &h->m;
  const int N = h->ncv;
  unsigned char *check = (unsigned char *)malloc(N ? N : 1);
  memset(check, 1, N);
  int nsrc = 0, *src = NULL;
  for (int z = 0; z < m->nzones; z++) {
    if (m->zones[z].kind != JG_BC_WALL) continue;
    int nz = m->zones[z].ifa_l - m->zones[z].ifa_f + 1;
    int base = relaxed ? nsrc : 0;  /* relaxed: every WALL zone's cells are sources */
    src = (int *)realloc(src, sizeof(int) * (base + nz + 1));
    nsrc = base + nz;
    for (int f = m->zones[z].ifa_f, i = base; f <= m->zones[z].ifa_l; f++, i++) {
      src[i] = m->cvofa[2 * f];
      check[src[i]] = 0;
    }
  }
  int cap = nsrc + 16, len = 0;
  int *cv = (int *)malloc(sizeof(int) * cap);
  int *off = (int *)malloc(sizeof(int) * (nsrc + 1));
  off[0] = 0;
  for (int l = 0; l < nsrc; l++) {
    if (len + 1 > cap) { cap *= 2; cv = (int *)realloc(cv, sizeof(int) * cap); }
    cv[len++] = src[l];
    int index_cv = 0, add;
    do {
      int icv = cv[off[l] + index_cv];
      double max_weight = 0.0, nv[3];
      for (int k = m->nbocv_i[icv] + 1; k < m->nbocv_i[icv + 1]; k++) {
        int ino = m->nbocv_v[k];
        int f = find_face(m, icv, ino);
        double area = norm3(nv, &m->fa_normal[3 * f]);
        double w = 0.5 * area * ((1.0 / m->cv_volume[icv]) + (1.0 / m->cv_volume[ino]));
        max_weight = dmax(max_weight, w);
      }
      add = 0;
      int counter = 0, next_cv = -1, best = -1;
      double best_w = 0.0, second_w = 0.0;
      for (int k = m->nbocv_i[icv] + 1; k < m->nbocv_i[icv + 1]; k++) {
        int ino = m->nbocv_v[k];
        int f = find_face(m, icv, ino);
        double area = norm3(nv, &m->fa_normal[3 * f]);
        double w = 0.5 * area * ((1.0 / m->cv_volume[icv]) + (1.0 / m->cv_volume[ino]));
        if (check[ino] && w / max_weight > 0.5 && (index_cv == 0 || ino != cv[off[l] + index_cv - 1])) {
          add = 1;
          next_cv = ino;
          counter++;
          if (w > best_w) {
            second_w = best_w;
            best_w = w;
            best = ino;
          } else if (w > second_w) {
            second_w = w;
          }
        }
      }
      if (counter > 1) {
        add = relaxed && best_w > 1.1 * second_w;
        next_cv = best;
      }
      if (add) {
        if (len + 1 > cap) { cap *= 2; cv = (int *)realloc(cv, sizeof(int) * cap); }
        cv[len++] = next_cv;
        check[next_cv] = 0;
        index_cv++;
      }
    } while (add);
    off[l + 1] = len;
  }
  *nlines_out = nsrc;
  *off_out = off;
  *cv_out = cv;
  free(src);
  free(check);
}

void jo_build_linelets(jo_case *h) {
  free(h->line_off); free(h->line_cv); free(h->linelet);
  build_lines(h, 0, &h->nlines, &h->line_off, &h->line_cv);
  const int N = h->ncv;
  h->linelet = (unsigned char *)calloc(N ? N : 1, 1);
  for (int l = 0; l < h->nlines; l++)
    if (h->line_off[l + 1] - h->line_off[l] >= 2)
      for (int i = h->line_off[l]; i < h->line_off[l + 1]; i++) h->linelet[h->line_cv[i]] = 1;
}

int jo_relax_lines(jo_case *h, int *off, int *cv) {
  if (!h->rline_off) build_lines(h, 1, &h->rnlines, &h->rline_off, &h->rline_cv);
  if (off) memcpy(off, h->rline_off, sizeof(int) * (h->rnlines + 1));
  if (cv) memcpy(cv, h->rline_cv, sizeof(int) * h->rline_off[h->rnlines]);
  return h->rnlines;
}

int jo_linelets(jo_case *h, int *off, int *cv) {
  if (!h->line_off) jo_build_linelets(h);
  if (off) memcpy(off, h->line_off, sizeof(int) * (h->nlines + 1));
  if (cv) memcpy(cv, h->line_cv, sizeof(int) * h->line_off[h->nlines]);
  return h->nlines;
}

/* luinv (UgpWithCv.cpp:2542-2577): the inverse from the ludeco factors, column by column */
static void luinv(double (*A)[5], double Ainv[5][5]) {
  for (int i = 0; i < 5; i++) {
    double c[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    c[i] = 1.0;
    c[0] = c[0] / A[0][0];
    for (int jr = 1; jr < 5; jr++) {
      double sum = c[jr];
      for (int jm = 0; jm <= jr - 1; jm++) sum -= A[jr][jm] * c[jm];
      c[jr] = sum / A[jr][jr];
    }
    for (int jrjr = 1; jrjr < 5; jrjr++) {
      int jr = 4 - jrjr;
      double sum = c[jr];
      for (int jmjm = jr + 1; jmjm < 5; jmjm++) {
        int jm = 4 - jmjm + jr + 1;
        sum -= A[jr][jm] * c[jm];
      }
      c[jr] = sum;
    }
    for (int r = 0; r < 5; r++) Ainv[r][i] = c[r];
  }
}

/* getMultMatrix (UgpWithCv.cpp:3994-4026): c = a b, sums from 0.0 in k order */
static void mat_mul(double c[5][5], const double *a, const double b[5][5]) {
  for (int i = 0; i < 5; i++)
    for (int j = 0; j < 5; j++) {
      c[i][j] = 0.0;
      for (int k = 0; k < 5; k++) c[i][j] += a[5 * i + k] * b[k][j];
    }
}
static void mat_vec(double c[5], const double *a, const double *b) {
  for (int i = 0; i < 5; i++) {
    c[i] = 0.0;
    for (int j = 0; j < 5; j++) c[i] += a[5 * i + j] * b[j];
  }
}

/* getImplDependencyIndex (UgpWithCv.h:745-755): CSR entry of column b in row a */
static int csr_entry(const jg_mesh *m, int a, int b) {
  int k = m->nbocv_i[a];
  while (m->nbocv_v[++k] != b);
  return k;
}

/* the LINE IMPLICIT preconditioner of solveCvVectorR5BcgstabLine
 * (UgpWithCv.cpp:3729-3810): the block diagonal (LU) off the lines, a
 * block-tridiagonal Thomas solve along each line (every line, single cells
 * included, overwrites its cells) */
static void line_precond(jo_case *h, const double *A, const double *LU, const double *pv, double *phat,
                         double (*bhat)[5][5], double (*invbhat)[5][5], double (*vhat)[5]) {
  const jg_mesh *m = &h->m;
  for (int c = 0; c < h->ncv; c++)
    if (!h->linelet[c]) {
      memcpy(&phat[5 * c], &pv[5 * c], 5 * sizeof(double));
      lusolv((double(*)[5]) & LU[25 * c], &phat[5 * c], 5);
    }
  double LUb[5][5], mhat[5][5], aux0[5][5], aux1[5], aux2[5];
  for (int l = 0; l < h->nlines; l++) {
    const int *cv = &h->line_cv[h->line_off[l]];
    int n = h->line_off[l + 1] - h->line_off[l];
    for (int i = 0; i < 5; i++) {
      vhat[0][i] = pv[5 * cv[0] + i];
      for (int j = 0; j < 5; j++) bhat[0][i][j] = A[25 * m->nbocv_i[cv[0]] + 5 * i + j];
    }
    for (int i = 1; i < n; i++) {
      int noc01 = csr_entry(m, cv[i - 1], cv[i]), noc11 = m->nbocv_i[cv[i]], noc10 = csr_entry(m, cv[i], cv[i - 1]);
      memcpy(LUb, bhat[i - 1], sizeof(LUb));
      ludeco(LUb, 5);
      luinv(LUb, invbhat[i - 1]);
      mat_mul(mhat, &A[25 * noc10], invbhat[i - 1]);
      double a01[5][5];
      memcpy(a01, &A[25 * noc01], sizeof(a01));
      mat_mul(aux0, &mhat[0][0], a01);
      for (int r = 0; r < 5; r++)
        for (int c = 0; c < 5; c++) bhat[i][r][c] = A[25 * noc11 + 5 * r + c] - aux0[r][c];
      mat_vec(aux1, &mhat[0][0], vhat[i - 1]);
      for (int r = 0; r < 5; r++) vhat[i][r] = pv[5 * cv[i] + r] - aux1[r];
    }
    memcpy(LUb, bhat[n - 1], sizeof(LUb));
    ludeco(LUb, 5);
    luinv(LUb, invbhat[n - 1]);
    mat_vec(&phat[5 * cv[n - 1]], &invbhat[n - 1][0][0], vhat[n - 1]);
    for (int i = n - 2; i >= 0; i--) {
      int noc01 = csr_entry(m, cv[i], cv[i + 1]);
      mat_vec(aux2, &A[25 * noc01], &phat[5 * cv[i + 1]]);
      for (int r = 0; r < 5; r++) aux1[r] = vhat[i][r] - aux2[r];
      mat_vec(&phat[5 * cv[i]], &invbhat[i][0][0], aux1);
    }
  }
}

static int solve_bcgstab(jo_case *h, double *phi, const double *A, const double *rhs, double zeroAbs, double zeroRel,
                         int maxiter, int line) {
  /* solveCvVectorR5Bcgstab, UgpWithCv.cpp:2660-2876; with `line` its
   * line-implicit twin solveCvVectorR5BcgstabLine, UgpWithCv.cpp:3627-3992 */
  int n = h->ncv;
  const jg_mesh *m = &h->m;
  double *res = dalloc(5 * n), *res0 = dalloc(5 * n), *pv = dalloc(5 * n), *v = dalloc(5 * n), *t = dalloc(5 * n),
         *s = dalloc(5 * n), *phat = dalloc(5 * n), *shat = dalloc(5 * n), *LU = dalloc(25 * n);
  for (int c = 0; c < n; c++) {
    memcpy(&LU[25 * c], &A[25 * m->nbocv_i[c]], 25 * sizeof(double));
    ludeco((double(*)[5]) & LU[25 * c], 5);
  }
  int lmax = 1;
  if (line) {
    if (!h->line_off) jo_build_linelets(h);
    for (int l = 0; l < h->nlines; l++) lmax = lmax > h->line_off[l + 1] - h->line_off[l] ? lmax : h->line_off[l + 1] - h->line_off[l];
  }
  double(*bhat)[5][5] = (double(*)[5][5])dalloc(25 * (size_t)lmax);
  double(*invbhat)[5][5] = (double(*)[5][5])dalloc(25 * (size_t)lmax);
  double(*vhat)[5] = (double(*)[5])dalloc(5 * (size_t)lmax);
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  matvec(h, res, A, phi);
  for (int k = 0; k < 5 * n; k++) { res[k] = rhs[k] - res[k]; res0[k] = res[k]; }
  double res0_max = 0.0;
  for (int c = 0; c < n; c++) {
    double tmp[5];
    memcpy(tmp, &res[5 * c], sizeof(tmp));
    lusolv((double(*)[5]) & LU[25 * c], tmp, 5);
    for (int i = 0; i < 5; i++) res0_max = dmax(res0_max, fabs(tmp[i]));
  }
  int iter = 0, done = 0;
  double res_max = 0.0;
  while (done == 0) {
    iter++;
    double rho_prime = -omega * rho;
    double my_rho = 0.0;
    for (int k = 0; k < 5 * n; k++) my_rho += res[k] * res0[k];
    rho = my_rho;
    if (fabs(rho_prime) < 1.0E-20) rho_prime = 1.0E-20;
    double beta = alpha * rho / rho_prime;
    for (int k = 0; k < 5 * n; k++) pv[k] = res[k] - beta * (pv[k] - omega * v[k]);
    if (line) {
      line_precond(h, A, LU, pv, phat, bhat, invbhat, vhat);
    } else {
      for (int c = 0; c < n; c++) {
        memcpy(&phat[5 * c], &pv[5 * c], 5 * sizeof(double));
        lusolv((double(*)[5]) & LU[25 * c], &phat[5 * c], 5);
      }
    }
    matvec(h, v, A, phat);
    double gamma = 0.0;
    for (int k = 0; k < 5 * n; k++) gamma += v[k] * res0[k];
    if (fabs(gamma) < 1.0E-20) gamma = 1.0E-20;
    alpha = rho / gamma;
    for (int k = 0; k < 5 * n; k++) s[k] = res[k] - alpha * v[k];
    if (line) {
      line_precond(h, A, LU, s, shat, bhat, invbhat, vhat);
    } else {
      for (int c = 0; c < n; c++) {
        memcpy(&shat[5 * c], &s[5 * c], 5 * sizeof(double));
        lusolv((double(*)[5]) & LU[25 * c], &shat[5 * c], 5);
      }
    }
    matvec(h, t, A, shat);
    double b0 = 0.0, b1 = 0.0;
    for (int k = 0; k < 5 * n; k++) { b0 += s[k] * t[k]; b1 += t[k] * t[k]; }
    omega = b0 / (b1 + 1.0E-20);
    for (int k = 0; k < 5 * n; k++) phi[k] += alpha * phat[k] + omega * shat[k];
    matvec(h, res, A, phi);
    for (int k = 0; k < 5 * n; k++) res[k] = rhs[k] - res[k];
    res_max = 0.0;
    for (int c = 0; c < n; c++) {
      double tmp[5];
      memcpy(tmp, &res[5 * c], sizeof(tmp));
      lusolv((double(*)[5]) & LU[25 * c], tmp, 5);
      for (int i = 0; i < 5; i++) res_max = dmax(res_max, fabs(tmp[i]));
    }
    if ((res_max <= zeroAbs) || (res_max / (res0_max + 1.0E-12) <= zeroRel)) done = 1;
    else if (iter > maxiter) done = 2;
  }
  free(res); free(res0); free(pv); free(v); free(t); free(s); free(phat); free(shat); free(LU);
  free(bhat); free(invbhat); free(vhat);
  return iter;
}

static int solve_lusgs(jo_case *h, double *phi, const double *A, const double *rhs) {
  /* solveCvVectorR5Lusgs, UgpWithCv.cpp:3172-3239: (D+L) x* = b with L applied to the input phi,
   * then D x1 = D x* - U x* */
  int n = h->ncv;
  const jg_mesh *m = &h->m;
  double *LU = dalloc(25 * n), *xn = dalloc(5 * n), *aux = dalloc(5 * n);
  for (int c = 0; c < n; c++) {
    memcpy(&LU[25 * c], &A[25 * m->nbocv_i[c]], 25 * sizeof(double));
    ludeco((double(*)[5]) & LU[25 * c], 5);
  }
  for (int c = 0; c < n; c++) {
    double low[5] = {0}, tmp[5];
    for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++) {
      int nb = m->nbocv_v[k];
      if (nb < c)
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) low[i] += A[25 * k + 5 * i + j] * phi[5 * nb + j];
    }
    for (int i = 0; i < 5; i++) tmp[i] = rhs[5 * c + i] - low[i];
    lusolv((double(*)[5]) & LU[25 * c], tmp, 5);
    memcpy(&xn[5 * c], tmp, sizeof(tmp));
  }
  for (int c = 0; c < n; c++) {
    double dg[5] = {0}, up[5] = {0};
    int kd = m->nbocv_i[c];
    for (int i = 0; i < 5; i++)
      for (int j = 0; j < 5; j++) dg[i] += A[25 * kd + 5 * i + j] * xn[5 * c + j];
    for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++) {
      int nb = m->nbocv_v[k];
      if (nb > c)
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) up[i] += A[25 * k + 5 * i + j] * xn[5 * nb + j];
    }
    for (int i = 0; i < 5; i++) aux[5 * c + i] = dg[i] - up[i];
  }
  for (int c = 0; c < n; c++) lusolv((double(*)[5]) & LU[25 * c], &aux[5 * c], 5);
  memcpy(phi, aux, sizeof(double) * 5 * n);
  free(LU); free(xn); free(aux);
  return 1;
}

/* Block point relaxation as the GPU runs it (not in the reference): sweeps of
 * block Jacobi, x <- D^-1 (b - O x) with D^-1 from ludeco + luinv. */
static int solve_jacobi(jo_case *h, double *phi, const double *A, const double *rhs, int sweeps) {
  int n = h->ncv;
  const jg_mesh *m = &h->m;
  double *LU = dalloc(25 * n), *xn = dalloc(5 * n);
  for (int c = 0; c < n; c++) {
    memcpy(&LU[25 * c], &A[25 * m->nbocv_i[c]], 25 * sizeof(double));
    ludeco((double(*)[5]) & LU[25 * c], 5);
  }
  for (int s = 0; s < sweeps; s++) {
    for (int c = 0; c < n; c++) {
      double b[5];
      for (int i = 0; i < 5; i++) b[i] = rhs[5 * c + i];
      for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++) {
        int nb = m->nbocv_v[k];
        for (int i = 0; i < 5; i++)
          for (int j = 0; j < 5; j++) b[i] -= A[25 * k + 5 * i + j] * phi[5 * nb + j];
      }
      lusolv((double(*)[5]) & LU[25 * c], b, 5);
      memcpy(&xn[5 * c], b, sizeof(b));
    }
    memcpy(phi, xn, sizeof(double) * 5 * n);
  }
  free(LU); free(xn);
  return sweeps;
}

/* Multicolour block Gauss-Seidel as the GPU runs it (not in the reference):
 * greedy colouring of the cell graph in cell order; each pass updates the
 * colours in turn (forward, then backward on the next pass) from x = 0. */
static int solve_sgs(jo_case *h, double *phi, const double *A, const double *rhs, int sweeps) {
  int n = h->ncv;
  const jg_mesh *m = &h->m;
  double *LU = dalloc(25 * n);
  int *color = (int *)calloc(n, sizeof(int));
  int ncol = 1;
  int mark[256];
  for (int k = 0; k < 256; k++) mark[k] = -1;
  for (int c = 0; c < n; c++) {
    for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++)
      if (m->nbocv_v[k] < c) mark[color[m->nbocv_v[k]]] = c;
    int q = 0;
    while (q < 255 && mark[q] == c) q++;
    color[c] = q;
    if (q + 1 > ncol) ncol = q + 1;
  }
  for (int c = 0; c < n; c++) {
    memcpy(&LU[25 * c], &A[25 * m->nbocv_i[c]], 25 * sizeof(double));
    ludeco((double(*)[5]) & LU[25 * c], 5);
  }
  memset(phi, 0, sizeof(double) * 5 * n);
  for (int s = 0; s < sweeps; s++)
    for (int q = 0; q < ncol; q++) {
      int col = (s % 2 == 0) ? q : ncol - 1 - q;
      for (int c = 0; c < n; c++) {
        if (color[c] != col) continue;
        double b[5];
        for (int i = 0; i < 5; i++) b[i] = rhs[5 * c + i];
        for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++) {
          int nb = m->nbocv_v[k];
          for (int i = 0; i < 5; i++)
            for (int j = 0; j < 5; j++) b[i] -= A[25 * k + 5 * i + j] * phi[5 * nb + j];
        }
        lusolv((double(*)[5]) & LU[25 * c], b, 5);
        memcpy(&phi[5 * c], b, sizeof(b));
      }
    }
  free(LU);
  free(color);
  return sweeps;
}

int jo_solve(jo_case *h, double *dq, const double *A, const double *rhs, double zeroAbs, double zeroRel, int maxIter,
             int solver) {
  switch (solver) {
    case JG_LS_BCGSTAB: return solve_bcgstab(h, dq, A, rhs, zeroAbs, zeroRel, maxIter, 0);
    case JG_LS_BCGSTAB_LINELET: return solve_bcgstab(h, dq, A, rhs, zeroAbs, zeroRel, maxIter, 1);
    case JG_LS_LINE: return jo_line_relax(h, 5, dq, A, rhs, maxIter);
    case JG_LS_LUSGS: return solve_lusgs(h, dq, A, rhs);
    case JG_LS_JACOBI: return solve_jacobi(h, dq, A, rhs, maxIter);
    case JG_LS_SGS: return solve_sgs(h, dq, A, rhs, maxIter);
    default: return -1;
  }
}

/* ------------------------------------------------------------------------ */
/* runBackwardEuler loop body, JoeWithModels.cpp:975-1159                    */
/* ------------------------------------------------------------------------ */
int jo_step(jo_case *h, int nsteps, double *resid) {
  const jg_params *p = &h->p;
  int n = h->ncv, nbs = h->nbs;
  double *A = dalloc(25 * (size_t)nbs), *dq = dalloc(5 * n), *rhs = dalloc(5 * n);
  double *rr = dalloc(n), *ru = dalloc(3 * n), *rE = dalloc(n);
  int err = 0;
  for (int it = 0; it < nsteps; it++) {
    h->step++;
    if ((h->step >= p->cfl_after) && (h->step % p->cfl_interval == 0) && (h->cfl < p->cfl_max)) h->cfl *= p->cfl_factor;
    jo_calc_dt(h, h->cfl);
    memset(A, 0, sizeof(double) * 25 * nbs);
    memset(dq, 0, sizeof(double) * 5 * n);
    jo_calc_rhs(h, rr, ru, rE, A, 1);
    for (int c = 0; c < n; c++) {
      rhs[5 * c + 0] = p->under_relax * rr[c];
      rhs[5 * c + 1] = p->under_relax * ru[3 * c];
      rhs[5 * c + 2] = p->under_relax * ru[3 * c + 1];
      rhs[5 * c + 3] = p->under_relax * ru[3 * c + 2];
      rhs[5 * c + 4] = p->under_relax * rE[c];
      double tmp = h->m.cv_volume[c] / (h->local_dt[c]);
      for (int i = 0; i < 5; i++) A[25 * h->m.nbocv_i[c] + 6 * i] += tmp;
    }
    jo_solve(h, dq, A, rhs, p->ls_abs, p->ls_rel, p->ls_max_iter, p->lin_solver);
    for (int c = 0; c < n; c++) {
      h->rho[c] += dq[5 * c];
      for (int i = 0; i < 3; i++) h->rhou[3 * c + i] += dq[5 * c + 1 + i];
      h->rhoE[c] += dq[5 * c + 4];
    }
    if (jo_calc_state(h) != 0) err = -1;
    double r[5] = {0, 0, 0, 0, 0};
    for (int c = 0; c < n; c++) {
      r[0] += fabs(rr[c]);
      for (int i = 0; i < 3; i++) r[1 + i] += fabs(ru[3 * c + i]);
      r[4] += fabs(rE[c]);
    }
    if (resid) memcpy(resid, r, sizeof(r));
  }
  free(A); free(dq); free(rhs); free(rr); free(ru); free(rE);
  return err;
}


/* ======================================================================== */
/* Coupled path with a turbulence model: runBackwardEulerCoupled /           */
/* calcRhsCoupled / calcFluxCoupled, JoeWithModels.cpp:4326-5826;           */
/* UgpWithCvCompFlow.cpp:1808-2292, 3040-3276; Scalars.cpp:289-360;          */
/* UgpWithCvCompFlow.h:1305-1552.  SA (TurbModel_SA.h): one scalar, nuSA,    */
/* block size 6.  SST (TurbModel_KOMSST.h): kine and omega, block size 7;    */
/* kine also enters the pressure, the HLLC energy and the viscous terms.    */
/* Row/column 5+s of every block is rho*phi_s.                               */
/* ======================================================================== */
#define MAXS 2
#define MAXB 7
/* RansTurbSA defaults (TurbModel_SA.h:21-36) */
#define SA_CV1_3 357.911
#define SA_CW1 3.239067817
#define SA_CW2 0.3
#define SA_CW3_6 64.0
#define SA_SIGMA 0.6666666
#define SA_CB1 0.1355
#define SA_CB2 0.622
#define SA_K2 0.1681
/* RansTurbKOmSST defaults (TurbModel_KOMSST.h:19-54) */
#define SST_SK1 0.85
#define SST_SK2 1.0
#define SST_SO1 0.5
#define SST_SO2 0.856
#define SST_B1 0.075
#define SST_B2 0.0828
#define SST_BS 0.09
#define SST_A1 0.31

typedef struct {
  int model, ns;
  double *phi[MAXS], *phi_bfa[MAXS], *grad_phi[MAXS], *diff[MAXS];
  double *wallDist, *strMag, *vortMag, *diverg, *crossDiff, *F1, *F2;
  double lower[MAXS], upper[MAXS];
} jo_turb;

typedef struct turb_node { jo_case *h; jo_turb t; struct turb_node *next; } turb_node;
static turb_node *g_turb = NULL;

static jo_turb *turb_of(jo_case *h) {
  for (turb_node *n = g_turb; n; n = n->next)
    if (n->h == h) return &n->t;
  turb_node *n = (turb_node *)calloc(1, sizeof(turb_node));
  n->h = h;
  jo_turb *t = &n->t;
  int c = h->ncv, nb = h->nfa_b, nf = h->nfa;
  t->model = h->p.turb_model;
  t->ns = h->p.nscal;
  for (int s = 0; s < t->ns; s++) {
    t->phi[s] = dalloc(c); t->phi_bfa[s] = dalloc(nb); t->grad_phi[s] = dalloc(3 * c); t->diff[s] = dalloc(nf);
  }
  t->wallDist = dalloc(c); t->strMag = dalloc(c); t->vortMag = dalloc(c); t->diverg = dalloc(c);
  t->crossDiff = dalloc(c); t->F1 = dalloc(c); t->F2 = dalloc(c);
  if (t->model == JG_TURB_SA) {
    t->lower[0] = 1.0e-10; t->upper[0] = 1.0;
  } else {
    t->lower[0] = 1.0e-10; t->upper[0] = 1.0e10;  /* kine */
    t->lower[1] = 1.0e-4; t->upper[1] = 1.0e15;   /* omega */
    h->kine = t->phi[0];
  }
  n->next = g_turb;
  g_turb = n;
  return t;
}

void jo_sa_release(jo_case *h) {
  turb_node **pp = &g_turb;
  while (*pp) {
    if ((*pp)->h == h) {
      turb_node *n = *pp;
      *pp = n->next;
      jo_turb *t = &n->t;
      for (int s = 0; s < t->ns; s++) {
        free(t->phi[s]); free(t->phi_bfa[s]); free(t->grad_phi[s]); free(t->diff[s]);
      }
      free(t->wallDist); free(t->strMag); free(t->vortMag); free(t->diverg); free(t->crossDiff);
      free(t->F1); free(t->F2);
      h->kine = NULL;
      free(n);
      return;
    }
    pp = &(*pp)->next;
  }
}

/* transported scalars in/out: phi[ncv][ns] */
void jo_set_scalars(jo_case *h, const double *phi) {
  jo_turb *t = turb_of(h);
  for (int c = 0; c < h->ncv; c++)
    for (int s = 0; s < t->ns; s++) t->phi[s][c] = phi[t->ns * c + s];
}
void jo_get_scalars(jo_case *h, double *phi) {
  jo_turb *t = turb_of(h);
  for (int c = 0; c < h->ncv; c++)
    for (int s = 0; s < t->ns; s++) phi[t->ns * c + s] = t->phi[s][c];
}

double *jo_sa_array(jo_case *h, const char *name) {
  jo_turb *t = turb_of(h);
  struct { const char *n; double *p; } tab[] = {
      {"phi", t->phi[0]}, {"phi_bfa", t->phi_bfa[0]}, {"grad_phi", t->grad_phi[0]}, {"diff", t->diff[0]},
      {"phi1", t->phi[1]}, {"phi1_bfa", t->phi_bfa[1]}, {"grad_phi1", t->grad_phi[1]}, {"diff1", t->diff[1]},
      {"wallDist", t->wallDist}, {"strMag", t->strMag}, {"vortMag", t->vortMag}, {"diverg", t->diverg},
      {"crossDiff", t->crossDiff}, {"blendFuncF1", t->F1}, {"blendFuncF2", t->F2}};
  for (size_t i = 0; i < sizeof(tab) / sizeof(tab[0]); i++)
    if (strcmp(tab[i].n, name) == 0) return tab[i].p;
  return NULL;
}

/* calcWallDistance, UgpWithCvCompFlow.h:1395-1535: nearest WALL face
 * centroid, then the normal projection when the cell sits over that face */
void jo_wall_distance(jo_case *h) {
  const jg_mesh *m = &h->m;
  jo_turb *t = turb_of(h);
  int nw = 0;
  for (int z = 0; z < m->nzones; z++)
    if (m->zones[z].kind == JG_BC_WALL) nw += m->zones[z].ifa_l - m->zones[z].ifa_f + 1;
  int *wf = (int *)malloc(sizeof(int) * (nw ? nw : 1));
  nw = 0;
  for (int z = 0; z < m->nzones; z++)
    if (m->zones[z].kind == JG_BC_WALL)
      for (int f = m->zones[z].ifa_f; f <= m->zones[z].ifa_l; f++) wf[nw++] = f;
  for (int c = 0; c < h->ncv; c++) {
    double minDist = 1.0e20;
    int save = 0;
    const double *x = &m->x_cv[3 * c];
    for (int k = 0; k < nw; k++) {
      const double *xf = &m->x_fa[3 * wf[k]];
      double dist = sqrt(pow(x[0] - xf[0], 2.0) + pow(x[1] - xf[1], 2.0) + pow(x[2] - xf[2], 2.0));
      if (dist < minDist) { save = k; minDist = dist; }
    }
    int f = wf[save];
    double n[3], sh[3];
    double nmag = norm3(n, &m->fa_normal[3 * f]);
    for (int i = 0; i < 3; i++) sh[i] = m->x_fa[3 * f + i] - x[i];
    double sMag2 = dot3(sh, sh);
    double dNorm2 = dot3(sh, n) * dot3(sh, n);
    double dTang2 = sMag2 - dNorm2;
    double specRadius2 = 0.5 * nmag;
    t->wallDist[c] = (dTang2 > specRadius2) ? minDist : fabs(dot3(sh, n));
  }
  free(wf);
}

/* setScalarBC (Scalars.cpp:289-360) with the SST omega wall hook
 * (boundaryHookScalarRansTurb, TurbModel_KOMSST.h:342-358) */
static void set_scalar_bc(jo_case *h) {
  const jg_mesh *m = &h->m;
  jo_turb *t = turb_of(h);
  for (int z = 0; z < m->nzones; z++) {
    const jg_zone *zn = &m->zones[z];
    for (int s = 0; s < t->ns; s++)
      for (int f = zn->ifa_f; f <= zn->ifa_l; f++) {
        int c0 = m->cvofa[2 * f];
        if (zn->scal_bc & (1 << (4 + s))) {
          if (t->model == JG_TURB_SST && s == 1 && zn->kind == JG_BC_WALL) {
            double muLamCV = mu_law(&h->p, h->temp[c0]);
            t->phi_bfa[s][f] = 60.0 * muLamCV / (h->rho[c0] * SST_B1 * t->wallDist[c0] * t->wallDist[c0]);
          }
        } else if (zn->scal_bc & (1 << s)) {
          t->phi_bfa[s][f] = (dot3(&h->vel_bfa[3 * f], &m->fa_normal[3 * f]) > 1.0e-8) ? t->phi[s][c0] : zn->v[6 + s];
        } else {
          t->phi_bfa[s][f] = t->phi[s][c0];
        }
      }
  }
}

/* InterpolateAtCellCenterFromFaceValues, UgpWithCvCompFlow.h:1538-1552 */
static double face_avg(jo_case *h, const double *phi, int c) {
  double v = 0.0;
  int f0 = h->m.faocv_i[c], f1 = h->m.faocv_i[c + 1] - 1;
  for (int k = f0; k <= f1; k++) v += phi[h->m.faocv_v[k]];
  return v / (double)(f1 - f0 + 1);
}

static void face_weights(jo_case *h, int f, int c0, int c1, double *w0, double *w1) {
  double dx0[3], dx1[3];
  for (int i = 0; i < 3; i++) {
    dx0[i] = h->m.x_fa[3 * f + i] - h->m.x_cv[3 * c0 + i];
    dx1[i] = h->m.x_fa[3 * f + i] - h->m.x_cv[3 * c1 + i];
  }
  *w0 = sqrt(dot3(dx0, dx0));
  *w1 = sqrt(dot3(dx1, dx1));
}

/* calcRansTurbViscMuet of the model (TurbModel_SA.h:74-128; TurbModel_KOMSST.h:109-167 with
 * calcMenterBlendingFunctions 360-386), calcGradVel / calcStrainRate(AndDivergence) / calcVorticity */
static void turb_visc(jo_case *h) {
  const jg_mesh *m = &h->m;
  jo_turb *t = turb_of(h);
  grad_vector(h, h->grad_u, h->vel, h->vel_bfa, h->p.limiter, h->sos);
  for (int c = 0; c < h->ncv; c++) {
    const double *g = &h->grad_u[9 * c];
    double sm = 0.0, vm = 0.0;
    double div = g[0] + g[4] + g[8];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        if (i == j) sm += pow(0.5 * (g[3 * i + j] + g[3 * j + i]) - 1. / 3. * div, 2.0);
        else sm += pow(0.5 * (g[3 * i + j] + g[3 * j + i]), 2.0);
      }
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) vm += pow(0.5 * (g[3 * i + j] - g[3 * j + i]), 2.0);
    t->strMag[c] = sqrt(2.0 * sm);
    t->vortMag[c] = sqrt(2.0 * vm);
    t->diverg[c] = div;
  }
  if (t->model == JG_TURB_SA) {
    const double *nu = t->phi[0];
    for (int f = h->nfa_b; f < h->nfa; f++) {
      int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
      double w0, w1;
      face_weights(h, f, c0, c1, &w0, &w1);
      double rho_fa = (w1 * h->rho[c0] + w0 * h->rho[c1]) / (w0 + w1);
      double nu_fa = (w1 * nu[c0] + w0 * nu[c1]) / (w0 + w1);
      double muSA = rho_fa * nu_fa;
      double chi_3 = pow(muSA / h->mul_fa[f], 3.0);
      double fv1 = chi_3 / (chi_3 + SA_CV1_3);
      h->mut_fa[f] = dmax(muSA * fv1, 0.0);
    }
    for (int z = 0; z < m->nzones; z++) {
      const jg_zone *zn = &m->zones[z];
      for (int f = zn->ifa_f; f <= zn->ifa_l; f++) {
        if (zn->kind == JG_BC_WALL) { h->mut_fa[f] = 0.0; continue; }
        int c0 = m->cvofa[2 * f];
        double muSA = h->rho[c0] * nu[c0];
        double mul0 = face_avg(h, h->mul_fa, c0);
        double chi_3 = pow(muSA / mul0, 3.0);
        double fv1 = chi_3 / (chi_3 + SA_CV1_3);
        h->mut_fa[f] = dmax(muSA * fv1, 0.0);
      }
    }
    return;
  }
  /* SST: Menter blending functions, then mut with the shear-stress limiter (vorticity) */
  const double *k = t->phi[0], *om = t->phi[1];
  grad_scalar(h, t->grad_phi[0], k, t->phi_bfa[0], h->p.limiter, k, NULL);
  grad_scalar(h, t->grad_phi[1], om, t->phi_bfa[1], h->p.limiter, om, NULL);
  for (int c = 0; c < h->ncv; c++) {
    double d = t->wallDist[c];
    double mue = face_avg(h, h->mul_fa, c);
    t->crossDiff[c] = dmax(2.0 * h->rho[c] * SST_SO2 / om[c] * dot3(&t->grad_phi[0][3 * c], &t->grad_phi[1][3 * c]),
                           1.0e-20);
    double gamma1 = 500.0 * mue / (pow(d, 2.0) * h->rho[c] * om[c]);
    double gamma2 = 4.0 * SST_SO2 * h->rho[c] * k[c] / (d * d * t->crossDiff[c]);
    double gamma3 = sqrt(k[c]) / (SST_BS * om[c] * d);
    double gamma = dmin(dmax(gamma1, gamma3), gamma2);
    t->F1[c] = tanh(pow(gamma, 4.0));
    gamma = dmax(2.0 * gamma3, gamma1);
    t->F2[c] = tanh(pow(gamma, 2.0));
  }
  const double *lim = t->vortMag;
  for (int f = h->nfa_b; f < h->nfa; f++) {
    int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
    double w0, w1;
    face_weights(h, f, c0, c1, &w0, &w1);
    double rho_fa = (w1 * h->rho[c0] + w0 * h->rho[c1]) / (w0 + w1);
    double kine_fa = (w1 * k[c0] + w0 * k[c1]) / (w0 + w1);
    double om_fa = (w1 * om[c0] + w0 * om[c1]) / (w0 + w1);
    double lim_fa = (w1 * lim[c0] + w0 * lim[c1]) / (w0 + w1);
    double F2_fa = (w1 * t->F2[c0] + w0 * t->F2[c1]) / (w0 + w1);
    double zeta = dmin(1.0 / om_fa, SST_A1 / (lim_fa * F2_fa));
    h->mut_fa[f] = dmin(dmax(rho_fa * kine_fa * zeta, 0.0), 1.0);
  }
  for (int z = 0; z < m->nzones; z++) {
    const jg_zone *zn = &m->zones[z];
    for (int f = zn->ifa_f; f <= zn->ifa_l; f++) {
      if (zn->kind == JG_BC_WALL) { h->mut_fa[f] = 0.0; continue; }
      int c0 = m->cvofa[2 * f];
      double zeta = dmin(1.0 / om[c0], SST_A1 / (lim[c0] * t->F2[c0]));
      h->mut_fa[f] = dmin(dmax(h->rho[c0] * k[c0] * zeta, 0.0), 1.0);
    }
  }
}

/* state + material + BC (NS and scalars) + turbulent viscosity: the preamble of
 * runBackwardEulerCoupled, JoeWithModels.cpp:4379-4401 */
int jo_calc_state_coupled(jo_case *h) {
  turb_of(h);
  calc_state_variables(h);
  calc_material_properties(h);
  int e = set_bc(h);
  set_scalar_bc(h);
  turb_visc(h);
  return e;
}

/* ---- coupled HLLC (UgpWithCvCompFlow.cpp:1808-2289), nScal scalars, ConvTerm = 1, dp/dscal = 0 ---- */
typedef struct { double rho, u[3], p, T, h, R, gam, sc[MAXS], k; } cstate;

static void flux_hllc_coupled(double *F, int ns, const cstate *L, const cstate *R, double area, const double *nV,
                              int only_pressure) {
  int B = 5 + ns;
  if (only_pressure) {
    F[0] = 0.0;
    for (int i = 1; i < 4; i++) F[i] = L->p * nV[i - 1];
    for (int i = 4; i < B; i++) F[i] = 0.0;
  } else {
    double unL = dot3(L->u, nV), uLuL = dot3(L->u, L->u), cL = sqrt(L->gam * L->p / L->rho);
    double rhoeL = (L->h + 0.5 * uLuL + L->k) * L->rho - L->p;
    double unR = dot3(R->u, nV), uRuR = dot3(R->u, R->u), cR = sqrt(R->gam * R->p / R->rho);
    double rhoeR = (R->h + 0.5 * uRuR + R->k) * R->rho - R->p;
    double Rrho = sqrt(R->rho / L->rho);
    double tmp = 1.0 / (1.0 + Rrho);
    double velRoe[3];
    for (int i = 0; i < 3; i++) velRoe[i] = tmp * (L->u[i] + R->u[i] * Rrho);
    double uRoe = dot3(velRoe, nV);
    double gamPdivRho = tmp * ((L->gam * L->p / L->rho + 0.5 * (L->gam - 1.0) * uLuL) +
                               (R->gam * R->p / R->rho + 0.5 * (R->gam - 1.0) * uRuR) * Rrho);
    double cRoe = sqrt(gamPdivRho - ((L->gam + R->gam) * 0.5 - 1.0) * 0.5 * dot3(velRoe, velRoe));
    double sL = dmin(uRoe - cRoe, unL - cL);
    double sR = dmax(uRoe + cRoe, unR + cR);
    double sM = (L->p - R->p - L->rho * unL * (sL - unL) + R->rho * unR * (sR - unR)) /
                (R->rho * (sR - unR) - L->rho * (sL - unL));
    double pStar = R->rho * (unR - sR) * (unR - sM) + R->p;
    const cstate *S;
    if (sM >= 0.0) {
      S = L;
      if (sL > 0.0) {
        F[0] = L->rho * unL;
        for (int i = 0; i < 3; i++) F[1 + i] = L->rho * L->u[i] * unL + L->p * nV[i];
        F[4] = (rhoeL + L->p) * unL;
      } else {
        double inv = 1.0 / (sL - sM), sLmuL = sL - unL;
        double rhoS = L->rho * sLmuL * inv, rhouS[3];
        for (int i = 0; i < 3; i++) rhouS[i] = (L->rho * L->u[i] * sLmuL + (pStar - L->p) * nV[i]) * inv;
        double rhoeS = (sLmuL * rhoeL - L->p * unL + pStar * sM) * inv;
        F[0] = rhoS * sM;
        for (int i = 0; i < 3; i++) F[1 + i] = rhouS[i] * sM + pStar * nV[i];
        F[4] = (rhoeS + pStar) * sM;
      }
    } else {
      S = R;
      if (sR >= 0.0) {
        double inv = 1.0 / (sR - sM), sRmuR = sR - unR;
        double rhoS = R->rho * sRmuR * inv, rhouS[3];
        for (int i = 0; i < 3; i++) rhouS[i] = (R->rho * R->u[i] * sRmuR + (pStar - R->p) * nV[i]) * inv;
        double rhoeS = (sRmuR * rhoeR - R->p * unR + pStar * sM) * inv;
        F[0] = rhoS * sM;
        for (int i = 0; i < 3; i++) F[1 + i] = rhouS[i] * sM + pStar * nV[i];
        F[4] = (rhoeS + pStar) * sM;
      } else {
        F[0] = R->rho * unR;
        for (int i = 0; i < 3; i++) F[1 + i] = R->rho * R->u[i] * unR + R->p * nV[i];
        F[4] = (rhoeR + R->p) * unR;
      }
    }
    for (int s = 0; s < ns; s++) F[5 + s] = 1.0 * F[0] * S->sc[s];
  }
  for (int i = 0; i < B; i++) F[i] *= area;
}

/* calcJacobianCoupled_HLLC (:2180-2244), row-major A[B][B] */
static void jac_coupled(double *A, int ns, const double *vel, double pp, double rrho, double hh, const double *sc,
                        const double *nV, double gamma) {
  int B = 5 + ns;
  double kapm1 = gamma - 1.0;
  double nVel[3] = {vel[0] * nV[0], vel[1] * nV[1], vel[2] * nV[2]};
  double U_k = nVel[0] + nVel[1] + nVel[2];
  double vSquHlf = 0.5 * dot3(vel, vel);
  A[0] = 0.0; A[1] = nV[0]; A[2] = nV[1]; A[3] = nV[2]; A[4] = 0.0;
  for (int s = 0; s < ns; s++) A[5 + s] = 0.0;
  for (int r = 0; r < 3; r++) {
    double *a = A + B * (1 + r);
    a[0] = -vel[r] * U_k + nV[r] * (kapm1 * vSquHlf + gamma * pp / rrho - kapm1 * hh);
    for (int c = 0; c < 3; c++)
      a[1 + c] = (r == c) ? (2.0 - gamma) * nVel[r] + U_k : vel[r] * nV[c] - kapm1 * vel[c] * nV[r];
    a[4] = kapm1 * nV[r];
    for (int s = 0; s < ns; s++) a[5 + s] = 0.0 * nV[r];
  }
  double *a4 = A + 4 * B;
  a4[0] = U_k * ((gamma - 2.0) * vSquHlf - gamma * (hh - pp / rrho));
  for (int c = 0; c < 3; c++) a4[1 + c] = (hh + vSquHlf) * nV[c] - kapm1 * vel[c] * U_k;
  a4[4] = gamma * U_k;
  for (int s = 0; s < ns; s++) a4[5 + s] = 0.0 * U_k;
  for (int s = 0; s < ns; s++) {
    double *a = A + B * (5 + s);
    a[0] = 0.0;
    for (int c = 0; c < 3; c++) a[1 + c] = sc[s] * nV[c];
    a[4] = 0.0;
    for (int q = 0; q < ns; q++) a[5 + q] = 0.0;
    a[5 + s] = rrho * U_k;
  }
}

/* calcdSMdU_HLLC (:2247-2266) */
static void dsmdu(double *d, int ns, const double *vel, double pp, double rrho, double hh, const double *nV,
                  double gamma, double SM, double S, double invertrho, double Factor) {
  double kapm1 = gamma - 1.0;
  double U_k = vel[0] * nV[0] + vel[1] * nV[1] + vel[2] * nV[2];
  double vSquHlf = 0.5 * dot3(vel, vel);
  d[0] = Factor * invertrho * (-U_k * U_k + kapm1 * vSquHlf + gamma * pp / rrho - kapm1 * hh + SM * S);
  for (int i = 0; i < 3; i++) d[1 + i] = Factor * invertrho * ((2 * U_k - S - SM) * nV[i] - kapm1 * vel[i]);
  d[4] = Factor * invertrho * kapm1;
  for (int s = 0; s < ns; s++) d[5 + s] = Factor * invertrho * 0.0;
}

/* calcSubSonicJacobianCoupled_HLLC (:2270-2289) */
static void subsonic_coupled(double *A, int ns, const double *d, double rhoS, const double *rhouS, double rhoeS,
                             const double *sc, double pS, double Omega, double sM, double rhoSmq, const double *nV,
                             double area) {
  int B = 5 + ns;
  double OmSM = Omega * sM, OmSMp1 = OmSM + 1.0;
  for (int i = 0; i < B; i++) {
    A[i] = -OmSM * A[i] + area * OmSMp1 * d[i] * rhoS;
    A[B + i] = -OmSM * A[B + i] + area * OmSMp1 * d[i] * (rhouS[0] + rhoSmq * nV[0]);
    A[2 * B + i] = -OmSM * A[2 * B + i] + area * OmSMp1 * d[i] * (rhouS[1] + rhoSmq * nV[1]);
    A[3 * B + i] = -OmSM * A[3 * B + i] + area * OmSMp1 * d[i] * (rhouS[2] + rhoSmq * nV[2]);
    A[4 * B + i] = -OmSM * A[4 * B + i] + area * OmSMp1 * d[i] * (rhoeS + pS + rhoSmq * sM);
    for (int s = 0; s < ns; s++)
      A[(5 + s) * B + i] = -OmSM * A[(5 + s) * B + i] + area * OmSMp1 * d[i] * rhoS * sc[s];
  }
}

/* calcEulerFluxMatricesCoupled_HLLC (:1934-2176): ALL_TERMS / ONLY_PRESSURE, then dU/dQ of the scalar columns */
static void matrices_hllc_coupled(double *AL, double *AR, int ns, const cstate *L, const cstate *R, double area,
                                  const double *nV, int only_pressure) {
  int B = 5 + ns, BB = B * B;
  if (!only_pressure) {
    double dL[MAXB], dR[MAXB];
    double unL = dot3(L->u, nV), uLuL = dot3(L->u, L->u), cL = sqrt(L->gam * L->p / L->rho);
    double hL = L->h + L->k;
    double rhoeL = (hL + 0.5 * uLuL) * L->rho - L->p;
    double unR = dot3(R->u, nV), uRuR = dot3(R->u, R->u), cR = sqrt(R->gam * R->p / R->rho);
    double hR = R->h + R->k;
    double rhoeR = (hR + 0.5 * uRuR) * R->rho - R->p;
    double Rrho = sqrt(R->rho / L->rho);
    double tmp = 1.0 / (1.0 + Rrho);
    double velRoe[3];
    for (int i = 0; i < 3; i++) velRoe[i] = tmp * (L->u[i] + R->u[i] * Rrho);
    double uRoe = dot3(velRoe, nV);
    double gamPdivRho = tmp * ((L->gam * L->p / L->rho + 0.5 * (L->gam - 1.0) * uLuL) +
                               (R->gam * R->p / R->rho + 0.5 * (R->gam - 1.0) * uRuR) * Rrho);
    double cRoe = sqrt(gamPdivRho - ((L->gam + R->gam) * 0.5 - 1.0) * 0.5 * dot3(velRoe, velRoe));
    double sL = dmin(uRoe - cRoe, unL - cL);
    double sR = dmax(uRoe + cRoe, unR + cR);
    double invrhotld = 1.0 / (R->rho * (sR - unR) - L->rho * (sL - unL));
    double sM = (L->p - R->p - L->rho * unL * (sL - unL) + R->rho * unR * (sR - unR)) /
                (R->rho * (sR - unR) - L->rho * (sL - unL));
    double pStar = R->rho * (unR - sR) * (unR - sM) + R->p;
    double nA[3] = {nV[0] * area, nV[1] * area, nV[2] * area};
    if (sM >= 0.0) {
      if (sL > 0.0) {
        if (AL) jac_coupled(AL, ns, L->u, L->p, L->rho, hL, L->sc, nA, L->gam);
        if (AR) memset(AR, 0, sizeof(double) * BB);
      } else {
        double Om = 1.0 / (sL - sM), sLmuL = sL - unL;
        double rhoS = L->rho * sLmuL * Om, rhouS[3];
        for (int i = 0; i < 3; i++) rhouS[i] = (L->rho * L->u[i] * sLmuL + (pStar - L->p) * nV[i]) * Om;
        double rhoeS = (sLmuL * rhoeL - L->p * unL + pStar * sM) * Om;
        if (AL) {
          dsmdu(dL, ns, L->u, L->p, L->rho, hL, nV, L->gam, sM, sL, invrhotld, 1.0);
          jac_coupled(AL, ns, L->u, L->p, L->rho, hL, L->sc, nA, L->gam);
          subsonic_coupled(AL, ns, dL, rhoS, rhouS, rhoeS, L->sc, pStar, Om, sM, R->rho * (sR - unR), nV, area);
          for (int i = 0; i < 5; i++) AL[(B + 1) * i] += area * Om * sM * sL;
          for (int s = 0; s < ns; s++) {
            AL[(5 + s) * B] += area * Om * sM * sL * L->sc[s];
            AL[(5 + s) * B + 5 + s] += area * Om * sM * sL * L->rho;
          }
        }
        if (AR) {
          dsmdu(dR, ns, R->u, R->p, R->rho, hR, nV, R->gam, sM, sR, invrhotld, -1.0);
          memset(AR, 0, sizeof(double) * BB);
          subsonic_coupled(AR, ns, dR, rhoS, rhouS, rhoeS, L->sc, pStar, Om, sM, L->rho * (sL - unL), nV, area);
        }
      }
    } else {
      if (sR >= 0.0) {
        double Om = 1.0 / (sR - sM), sRmuR = sR - unR;
        double rhoS = R->rho * sRmuR * Om, rhouS[3];
        for (int i = 0; i < 3; i++) rhouS[i] = (R->rho * R->u[i] * sRmuR + (pStar - R->p) * nV[i]) * Om;
        double rhoeS = (sRmuR * rhoeR - R->p * unR + pStar * sM) * Om;
        if (AR) {
          dsmdu(dR, ns, R->u, R->p, R->rho, hR, nV, R->gam, sM, sR, invrhotld, -1.0);
          jac_coupled(AR, ns, R->u, R->p, R->rho, hR, R->sc, nA, R->gam);
          subsonic_coupled(AR, ns, dR, rhoS, rhouS, rhoeS, R->sc, pStar, Om, sM, L->rho * (sL - unL), nV, area);
          for (int i = 0; i < 5; i++) AR[(B + 1) * i] += area * Om * sM * sR;
          for (int s = 0; s < ns; s++) {
            AR[(5 + s) * B] += area * Om * sM * sR * R->sc[s];
            AR[(5 + s) * B + 5 + s] += area * Om * sM * sR * R->rho;
          }
        }
        if (AL) {
          dsmdu(dL, ns, L->u, L->p, L->rho, hL, nV, L->gam, sM, sL, invrhotld, 1.0);
          memset(AL, 0, sizeof(double) * BB);
          subsonic_coupled(AL, ns, dL, rhoS, rhouS, rhoeS, R->sc, pStar, Om, sM, R->rho * (sR - unR), nV, area);
        }
      } else {
        if (AR) jac_coupled(AR, ns, R->u, R->p, R->rho, hR, R->sc, nA, R->gam);
        if (AL) memset(AL, 0, sizeof(double) * BB);
      }
    }
  } else {
    if (AL) {
      double uLuL = dot3(L->u, L->u), hL = L->h + L->k, g = L->gam;
      for (int j = 0; j < B; j++) AL[j] = 0.0;
      double dpdrho = 0.5 * (g - 1.0) * uLuL - (g - 1.0) * hL + g * L->p / L->rho;
      for (int r = 0; r < 3; r++) {
        double *a = AL + B * (1 + r);
        a[0] = dpdrho * nV[r] * area;
        for (int c = 0; c < 3; c++) a[1 + c] = -(g - 1.0) * L->u[c] * nV[r] * area;
        a[4] = (g - 1.0) * nV[r] * area;
        for (int s = 0; s < ns; s++) a[5 + s] = 0.0 * nV[r] * area;
      }
      for (int e = 4 * B; e < BB; e++) AL[e] = 0.0;
    }
    if (AR) memset(AR, 0, sizeof(double) * BB);
  }
  for (int side = 0; side < 2; side++) {
    double *A = side ? AR : AL;
    const cstate *S = side ? R : L;
    if (!A) continue;
    for (int j = 0; j < B; j++)
      for (int s = 0; s < ns; s++) {
        A[B * j] -= S->sc[s] / S->rho * A[B * j + 5 + s];
        A[B * j + 5 + s] /= S->rho;
      }
  }
}

/* ---- coupled AUSMDV and Haenel & Schwane (UgpWithCvCompFlow.cpp:2293-3036), ConvTerm = 1,
 * dp/dscal = 0 (no model here sets dpress_dphi).  The five flow entries are the segregated
 * schemes' (their total enthalpy h + u.u/2 + k in the same order); the scalars ride on the mass
 * flux of the upwind side (AUSMDV) or of each split part (HAENEL), and the entropy fix acts on
 * them as on the density. ---- */
static fstate fstate_of(const cstate *c) {
  fstate f = {c->rho, {c->u[0], c->u[1], c->u[2]}, c->p, c->gam, c->k, c->h};
  return f;
}

/* the AUSMDV mass flux rho u_1/2 and the entropy fix's unscaled wave-speed jump (0: no fix) */
static void ausmdv_mass(const cstate *L, const cstate *R, const double *nV, ausm_opt o, double *rhou_half,
                        double *dl, double *unL_o, double *unR_o, double *alphaL_o, double *cLR_o) {
  double unL = dot3(L->u, nV), cL = sqrt(L->gam * L->p / L->rho);
  double alphaL = ausm_alpha_L(L->p, L->rho, R->p, R->rho, o.shock);
  double unR = dot3(R->u, nV), cR = sqrt(R->gam * R->p / R->rho);
  double alphaR = 2.0 - alphaL;
  double cLR = dmax(cL, cR);
  *rhou_half = L->rho * hs_u_pm(alphaL, unL, cLR, +1.0) + R->rho * hs_u_pm(alphaR, unR, cLR, -1.0);
  double d = 0.0;
  if (o.efix) {
    if ((unL <= -cL) && (unR >= cR)) d = 0.0;
    else if (((unL - cL) < 0.0) && ((unR - cR) > 0.0)) d = ((unR - cR) - (unL - cL));
    else if (((unL + cL) < 0.0) && ((unR + cR) > 0.0)) d = ((unR + cR) - (unL + cL));
  }
  *dl = d;
  *unL_o = unL;
  *unR_o = unR;
  *alphaL_o = alphaL;
  *cLR_o = cLR;
}

/* calcEulerFluxCoupled_AUSMDV (:2293-2399) and calcEulerFluxCoupled_HAENEL (:2802-2850);
 * haenel selects the latter */
static void flux_ausm_coupled(double *F, int ns, const cstate *L, const cstate *R, double area, const double *nV,
                              int only_pressure, int haenel, ausm_opt o) {
  if (only_pressure) {
    flux_hllc_coupled(F, ns, L, R, area, nV, 1);  /* the same pressure-only flux */
    return;
  }
  fstate fL = fstate_of(L), fR = fstate_of(R);
  double F5[5];
  if (haenel) {
    flux_haenel(F5, &fL, &fR, area, nV);
    double unL = dot3(L->u, nV), cL = sqrt(L->gam * L->p / L->rho);
    double unR = dot3(R->u, nV), cR = sqrt(R->gam * R->p / R->rho);
    double cLR = dmax(cL, cR);
    double uLp = hs_u_pm(1.0, unL, cLR, 1.0), uRm = hs_u_pm(1.0, unR, cLR, -1.0);
    for (int s = 0; s < ns; s++) F[5 + s] = (L->rho * uLp * L->sc[s] + R->rho * uRm * R->sc[s]) * area;
  } else {
    flux_ausmdv(F5, &fL, &fR, area, nV, o);
    double rh, dl, unL, unR, aL, cLR;
    ausmdv_mass(L, R, nV, o, &rh, &dl, &unL, &unR, &aL, &cLR);
    dl *= 0.125;
    for (int s = 0; s < ns; s++) {
      double fs = 1.0 * rh * (rh >= 0.0 ? L->sc[s] : R->sc[s]);
      if (dl != 0.0) fs -= dl * (R->rho * R->sc[s] - L->rho * L->sc[s]);
      F[5 + s] = fs * area;
    }
  }
  for (int i = 0; i < 5; i++) F[i] = F5[i];
}

/* calcEulerFluxMatricesCoupled_AUSMDV (:2405-2796) and calcEulerFluxMatricesCoupled_HAENEL
 * (:2858-3034), then dQ/dU of the scalar columns */
static void matrices_ausm_coupled(double *AL, double *AR, int ns, const cstate *L, const cstate *R, double area,
                                  const double *nV, int only_pressure, int haenel, ausm_opt o) {
  int B = 5 + ns, BB = B * B;
  if (only_pressure) {
    if (AL) {
      double uLuL = dot3(L->u, L->u), g = L->gam;
      double hL = L->h + 0.5 * uLuL + L->k;
      double dpdrho = (1.0 - g) * (hL - uLuL) + g * L->p / L->rho;
      for (int e = 0; e < BB; e++) AL[e] = 0.0;
      for (int r = 0; r < 3; r++) {
        double *a = AL + B * (1 + r);
        a[0] = dpdrho * nV[r];
        for (int c = 0; c < 3; c++) a[1 + c] = (1.0 - g) * L->u[c] * nV[r];
        a[4] = (g - 1.0) * nV[r];
      }
      for (int e = 0; e < BB; e++) AL[e] *= area;
    }
    if (AR) memset(AR, 0, sizeof(double) * BB);
  } else {
    fstate fL = fstate_of(L), fR = fstate_of(R);
    double L5[5][5], R5[5][5];
    if (haenel) matrices_haenel(AL ? L5 : NULL, AR ? R5 : NULL, &fL, &fR, area, nV);
    else matrices_ausmdv(AL ? L5 : NULL, AR ? R5 : NULL, &fL, &fR, area, nV, o);
    double unL = dot3(L->u, nV), cL = sqrt(L->gam * L->p / L->rho);
    double unR = dot3(R->u, nV), cR = sqrt(R->gam * R->p / R->rho);
    double cLR = dmax(cL, cR);
    double bp[5], bm[5];
    double rh = 0.0, dl = 0.0, uLp, uRm;
    if (haenel) {
      uLp = hs_u_pm(1.0, unL, cLR, 1.0);
      uRm = hs_u_pm(1.0, unR, cLR, -1.0);
      hs_drhou_pm(bp, 1.0, unL, cLR, nV, +1.0);
      hs_drhou_pm(bm, 1.0, unR, cLR, nV, -1.0);
    } else {
      double aL;
      ausmdv_mass(L, R, nV, o, &rh, &dl, &unL, &unR, &aL, &cLR);
      uLp = uRm = 0.0;
      hs_drhou_pm(bp, aL, unL, cLR, nV, +1.0);
      hs_drhou_pm(bm, 2.0 - aL, unR, cLR, nV, -1.0);
    }
    for (int side = 0; side < 2; side++) {
      double *A = side ? AR : AL;
      if (!A) continue;
      const cstate *S = side ? R : L, *O = side ? L : R;
      double (*A5)[5] = side ? R5 : L5;
      const double *beta = side ? bm : bp;
      for (int e = 0; e < BB; e++) A[e] = 0.0;
      for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) A[B * i + j] = A5[i][j];
      for (int q = 0; q < ns; q++) {
        double *a = A + B * (5 + q);
        if (haenel) {
          for (int j = 0; j < 5; j++) a[j] = beta[j] * S->sc[q] * area;
          a[5 + q] = S->rho * (side ? uRm : uLp) * area;
        } else {
          /* upwind side: d(rho u_1/2)/dQ phi + rho u_1/2 on the diagonal; else the other side's phi */
          int own = side ? (rh < 0.0) : (rh >= 0.0);
          double ph = own ? S->sc[q] : O->sc[q];
          double v0 = beta[0] * ph, v[3], vd = own ? rh : 0.0;
          for (int j = 0; j < 3; j++) v[j] = beta[1 + j] * ph;
          if (dl != 0.0) {
            double jump = L->rho * L->sc[q] - R->rho * R->sc[q];
            double un = side ? unR : unL;
            if (!side) {
              v0 += 0.125 * (dl * S->sc[q] + un / S->rho * jump);
              for (int j = 0; j < 3; j++) v[j] += -0.125 * nV[j] / S->rho * jump;
              vd += 0.125 * dl * S->rho;
            } else {
              v0 -= 0.125 * (dl * S->sc[q] + un / S->rho * jump);
              for (int j = 0; j < 3; j++) v[j] -= -0.125 * nV[j] / S->rho * jump;
              vd -= 0.125 * dl * S->rho;
            }
          }
          a[0] = v0 * area;
          for (int j = 0; j < 3; j++) a[1 + j] = v[j] * area;
          a[5 + q] = vd * area;
        }
      }
    }
  }
  for (int side = 0; side < 2; side++) {
    double *A = side ? AR : AL;
    const cstate *S = side ? R : L;
    if (!A) continue;
    for (int j = 0; j < B; j++)
      for (int s = 0; s < ns; s++) {
        A[B * j] -= S->sc[s] / S->rho * A[B * j + 5 + s];
        A[B * j + 5 + s] /= S->rho;
      }
  }
}

/* the coupled path's flux choice (calcFluxCoupled, JoeWithModels.cpp:4987-5057 and the boundary
 * branches 5139-5799): HLLC, AUSMDV (the face's shock fix o.shock; HAENEL there selects the Haenel &
 * Schwane scheme) or HAENEL */
static void cflux(const jg_params *p, ausm_opt o, double *F, int ns, const cstate *L, const cstate *R, double area,
                  const double *nV, int only_pressure) {
  if (p->flux == JG_FLUX_HLLC) flux_hllc_coupled(F, ns, L, R, area, nV, only_pressure);
  else flux_ausm_coupled(F, ns, L, R, area, nV, only_pressure,
                         p->flux == JG_FLUX_HAENEL || o.shock == JG_SHOCK_FIX_HAENEL, o);
}
static void cmatrices(const jg_params *p, ausm_opt o, double *AL, double *AR, int ns, const cstate *L,
                      const cstate *R, double area, const double *nV, int only_pressure) {
  if (p->flux == JG_FLUX_HLLC) matrices_hllc_coupled(AL, AR, ns, L, R, area, nV, only_pressure);
  else matrices_ausm_coupled(AL, AR, ns, L, R, area, nV, only_pressure,
                             p->flux == JG_FLUX_HAENEL || o.shock == JG_SHOCK_FIX_HAENEL, o);
}

/* calcViscousFluxCoupled (UgpWithCvCompFlow.cpp:3040-3276), turbulence model on */
typedef struct {
  double rho, u[3], h, T, R, gam, sc[MAXS], k;
  const double *gu, *gh, *gs[MAXS];
} vstate;

static void visc_coupled(double *Fv, double *A0, double *A1, int ns, const vstate *a, const vstate *b, double mul,
                         double mut, double lamOcp, double PrTurb, double kine_fa, const double *u_fa,
                         const double *diff, const double *diffTerm, double area, const double *nV, double smag,
                         const double *sV, double alpha) {
  int B = 5 + ns;
  double g[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) g[i][j] = 0.5 * (a->gu[3 * i + j] + b->gu[3 * i + j]);
  double fC[3] = {nV[0] - alpha * sV[0], nV[1] - alpha * sV[1], nV[2] - alpha * sV[2]};
  double muT = mul + mut;
  double tn[3];
  Fv[0] = 0.0;
  for (int i = 0; i < 3; i++)
    tn[i] = muT * (alpha * (b->u[i] - a->u[i]) / smag + g[i][0] * fC[0] + g[0][i] * nV[0] + g[i][1] * fC[1] +
                   g[1][i] * nV[1] + g[i][2] * fC[2] + g[2][i] * nV[2]);
  double tmp = 2.0 / 3.0 * muT * (g[0][0] + g[1][1] + g[2][2]);
  tmp += 1.0 / 3.0 * (a->rho + b->rho) * kine_fa;
  for (int i = 0; i < 3; i++) tn[i] -= tmp * nV[i];
  for (int i = 0; i < 3; i++) Fv[1 + i] = -area * tn[i];
  double keff = lamOcp + mut / PrTurb;
  double enth = keff * (alpha * (b->h - a->h) / smag + 0.5 * ((a->gh[0] + b->gh[0]) * fC[0] +
                                                             (a->gh[1] + b->gh[1]) * fC[1] +
                                                             (a->gh[2] + b->gh[2]) * fC[2]));
  double psi = muT * (alpha * (b->k - a->k) / smag);
  Fv[4] = -area * (enth + tn[0] * u_fa[0] + tn[1] * u_fa[1] + tn[2] * u_fa[2] + psi);
  static const double zero3[3] = {0.0, 0.0, 0.0};
  for (int s = 0; s < ns; s++) {
    const double *g0 = a->gs[s] ? a->gs[s] : zero3, *g1 = b->gs[s] ? b->gs[s] : zero3;
    Fv[5 + s] = -area * diffTerm[s] * diff[s] * (alpha * (b->sc[s] - a->sc[s]) / smag +
                                                 0.5 * ((g0[0] + g1[0]) * fC[0] + (g0[1] + g1[1]) * fC[1] +
                                                        (g0[2] + g1[2]) * fC[2]));
  }
  double aas = area * alpha / smag;
  for (int side = 0; side < 2; side++) {
    double *A = side ? A1 : A0;
    if (!A) continue;
    const vstate *v = side ? b : a;
    double sg = side ? -1.0 : 1.0;
    double d11 = sg * muT * aas;
    double d41 = -area * tn[0] * 0.5 + u_fa[0] * d11;
    double d42 = -area * tn[1] * 0.5 + u_fa[1] * d11;
    double d43 = -area * tn[2] * 0.5 + u_fa[2] * d11;
    double d44 = sg * keff * aas;
    double iR = 1.0 / v->rho;
    double q10 = -iR * v->u[0], q20 = -iR * v->u[1], q30 = -iR * v->u[2];
    double q40 = iR * v->gam * (-v->h - v->k + v->R * v->T + 0.5 * dot3(v->u, v->u));
    double q41 = -iR * v->u[0] * v->gam, q42 = -iR * v->u[1] * v->gam, q43 = -iR * v->u[2] * v->gam;
    double q44 = iR * v->gam;
    A[B + 0] = d11 * q10; A[B + 1] = d11 * iR;
    A[2 * B + 0] = d11 * q20; A[2 * B + 2] = d11 * iR;
    A[3 * B + 0] = d11 * q30; A[3 * B + 3] = d11 * iR;
    A[4 * B + 0] = d41 * q10 + d42 * q20 + d43 * q30 + d44 * q40;
    A[4 * B + 1] = d41 * iR + d44 * q41;
    A[4 * B + 2] = d42 * iR + d44 * q42;
    A[4 * B + 3] = d43 * iR + d44 * q43;
    A[4 * B + 4] = d44 * q44;
    for (int s = 0; s < ns; s++) {
      double dss = sg * diffTerm[s] * diff[s] * aas;
      A[4 * B + 5 + s] = d44 * (iR * iR * 0.0);
      A[(5 + s) * B + 0] = dss * (-iR * v->sc[s]);
      A[(5 + s) * B + 5 + s] = dss * iR;
    }
  }
}

static void add_blk(double *A, int B, int slot, const double *M, double sgn) {
  double *a = &A[(size_t)B * B * slot];
  for (int e = 0; e < B * B; e++) a[e] += sgn * M[e];
}

static cstate cell_cstate(jo_case *h, const jo_turb *t, int c) {
  cstate s = {h->rho[c], {h->vel[3 * c], h->vel[3 * c + 1], h->vel[3 * c + 2]}, h->press[c], h->temp[c],
              h->enthalpy[c], h->RoM[c], h->gam[c], {0.0, 0.0}, 0.0};
  for (int q = 0; q < t->ns; q++) s.sc[q] = t->phi[q][c];
  return s;
}
static cstate bfa_cstate(jo_case *h, const jo_turb *t, int f) {
  cstate s = {h->rho_bfa[f], {h->vel_bfa[3 * f], h->vel_bfa[3 * f + 1], h->vel_bfa[3 * f + 2]}, h->p_bfa[f],
              h->T_bfa[f], h->h_bfa[f], h->RoM_bfa[f], h->gam_bfa[f], {0.0, 0.0}, 0.0};
  for (int q = 0; q < t->ns; q++) s.sc[q] = t->phi_bfa[q][f];
  return s;
}
static vstate cell_vstate(jo_case *h, const jo_turb *t, int c) {
  vstate v = {h->rho[c], {h->vel[3 * c], h->vel[3 * c + 1], h->vel[3 * c + 2]}, h->enthalpy[c], h->temp[c],
              h->RoM[c], h->gam[c], {0.0, 0.0}, 0.0, &h->grad_u[9 * c], &h->grad_h[3 * c], {NULL, NULL}};
  for (int q = 0; q < t->ns; q++) {
    v.sc[q] = t->phi[q][c];
    v.gs[q] = &t->grad_phi[q][3 * c];
  }
  if (t->model == JG_TURB_SST) v.k = t->phi[0][c];
  return v;
}
static vstate bfa_vstate(jo_case *h, const jo_turb *t, int f, int c) {
  vstate v = {h->rho_bfa[f], {h->vel_bfa[3 * f], h->vel_bfa[3 * f + 1], h->vel_bfa[3 * f + 2]}, h->h_bfa[f],
              h->T_bfa[f], h->RoM_bfa[f], h->gam_bfa[f], {0.0, 0.0}, 0.0, &h->grad_u[9 * c], &h->grad_h[3 * c],
              {NULL, NULL}};
  return v;
}

/* face reconstruction with the scalars (JoeWithModels.cpp:4837-4921), then calcThermoProp_p */
static void reconstruct_c(jo_case *h, const jo_turb *t, int c, int f, cstate *s) {
  double r0[3];
  for (int i = 0; i < 3; i++) r0[i] = h->m.x_fa[3 * f + i] - h->m.x_cv[3 * c + i];
  double rho0 = h->rho[c] + dot3(r0, &h->grad_rho[3 * c]);
  double p0 = h->press[c] + dot3(r0, &h->grad_p[3 * c]);
  if ((p0 <= 0.0) || (rho0 <= 0.0)) {
    s->p = h->press[c];
    s->rho = h->rho[c];
  } else {
    s->rho = rho0;
    s->p = p0;
    for (int i = 0; i < 3; i++) s->u[i] = h->vel[3 * c + i] + dot3(r0, &h->grad_u[9 * c + 3 * i]);
    for (int q = 0; q < t->ns; q++) s->sc[q] += dot3(r0, &t->grad_phi[q][3 * c]);
  }
  s->R = h->p.R_gas;
  s->gam = h->p.gamma;
  s->T = s->p / (s->rho * s->R);
  s->h = s->gam * s->R / (s->gam - 1.0) * s->T;
}

/* scalar diffusivities (diffusivityHookScalarRansTurb: TurbModel_SA.h:130-173, TurbModel_KOMSST.h:169-256) */
static void turb_diffusivity(jo_case *h, jo_turb *t) {
  const jg_mesh *m = &h->m;
  for (int f = h->nfa_b; f < h->nfa; f++) {
    int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
    double w0, w1;
    face_weights(h, f, c0, c1, &w0, &w1);
    if (t->model == JG_TURB_SA) {
      double rho_fa = (w1 * h->rho[c0] + w0 * h->rho[c1]) / (w0 + w1);
      double nu_fa = (w1 * t->phi[0][c0] + w0 * t->phi[0][c1]) / (w0 + w1);
      t->diff[0][f] = (1.0 / SA_SIGMA) * (h->mul_fa[f] + rho_fa * nu_fa);
    } else {
      double f1_fa = (w1 * t->F1[c0] + w0 * t->F1[c1]) / (w0 + w1);
      t->diff[0][f] = h->mul_fa[f] + (SST_SK1 * f1_fa + (1. - f1_fa) * SST_SK2) * h->mut_fa[f];
      t->diff[1][f] = h->mul_fa[f] + (SST_SO1 * f1_fa + (1. - f1_fa) * SST_SO2) * h->mut_fa[f];
    }
  }
  for (int z = 0; z < m->nzones; z++) {
    const jg_zone *zn = &m->zones[z];
    for (int f = zn->ifa_f; f <= zn->ifa_l; f++) {
      int c0 = m->cvofa[2 * f];
      if (t->model == JG_TURB_SA) {
        t->diff[0][f] = (zn->kind == JG_BC_WALL) ? (1.0 / SA_SIGMA) * h->mul_fa[f]
                                                 : (1.0 / SA_SIGMA) * (h->mul_fa[f] + h->rho_bfa[f] * t->phi_bfa[0][f]);
      } else if (zn->kind == JG_BC_WALL) {
        t->diff[0][f] = h->mul_fa[f];
        t->diff[1][f] = h->mul_fa[f];
      } else {
        double F1 = t->F1[c0];
        t->diff[0][f] = h->mul_fa[f] + (SST_SK1 * F1 + (1. - F1) * SST_SK2) * h->mut_fa[f];
        t->diff[1][f] = h->mul_fa[f] + (SST_SO1 * F1 + (1. - F1) * SST_SO2) * h->mut_fa[f];
      }
    }
  }
}

/* calcRhsCoupled (JoeWithModels.cpp:4597-4611): rhs[ncv][B], A[nbocv_s][B][B] (accumulated), B = 5 + nscal */
void jo_calc_rhs_coupled(jo_case *h, double *rhs, double *A, int implicit) {
  const jg_mesh *m = &h->m;
  const jg_params *p = &h->p;
  jo_turb *t = turb_of(h);
  const int ns = t->ns, B = 5 + ns, BB = B * B;
  const int sst = t->model == JG_TURB_SST;
  int visc = p->mu_ref > 0.0;
  int only_p = p->symm_bc == JG_SYMM_ANALYTICAL;
  memset(rhs, 0, sizeof(double) * B * h->ncv);
  /* gradients, JoeWithModels.cpp:4683-4754 */
  if (p->second_order || visc) grad_vector(h, h->grad_u, h->vel, h->vel_bfa, p->limiter, h->sos);
  if (p->second_order) {
    grad_scalar(h, h->grad_rho, h->rho, h->rho_bfa, p->limiter, h->rho, NULL);
    grad_scalar(h, h->grad_p, h->press, h->p_bfa, p->limiter, h->press, NULL);
  }
  if (visc) grad_scalar(h, h->grad_h, h->enthalpy, h->h_bfa, p->limiter, h->enthalpy, NULL);
  if (p->second_order || visc)
    for (int q = 0; q < ns; q++) grad_scalar(h, t->grad_phi[q], t->phi[q], t->phi_bfa[q], p->limiter, t->phi[q], NULL);
  if (visc) turb_diffusivity(h, t);
  double F[MAXB], Fv[MAXB], Apl[MAXB * MAXB], Ami[MAXB * MAXB], A0[MAXB * MAXB], A1[MAXB * MAXB];
  memset(A0, 0, sizeof(A0));
  memset(A1, 0, sizeof(A1));
  double ones[MAXS] = {1.0, 1.0}, dterm[MAXS], dfa[MAXS];
  /* AUSMDV shock sensor at the cell-centre states (JoeWithModels.cpp:4763-4792) */
  double *flag = NULL;
  if (p->flux == JG_FLUX_AUSMDV && p->shock_fix != JG_SHOCK_FIX_NONE) {
    flag = dalloc(h->ncv);
    for (int f = h->nfa_b; f < h->nfa; f++)
      if (face_sonic(h, f)) {
        flag[m->cvofa[2 * f]] = 1.0;
        flag[m->cvofa[2 * f + 1]] = 1.0;
      }
  }
  const double flag_sum = p->shock_flag == JG_SHOCK_FLAG_TET ? 0.9 : 1.1;
  const ausm_opt ob = bnd_opt(p);  /* boundary faces: AUSMDV without the shock fix */
  /* internal faces, JoeWithModels.cpp:4797-5132 */
  for (int f = h->nfa_b; f < h->nfa; f++) {
    int c0 = m->cvofa[2 * f], c1 = m->cvofa[2 * f + 1];
    double nV[3];
    double area = norm3(nV, &m->fa_normal[3 * f]);
    cstate L = cell_cstate(h, t, c0), R = cell_cstate(h, t, c1);
    if (p->second_order) {
      reconstruct_c(h, t, c0, f, &L);
      reconstruct_c(h, t, c1, f, &R);
    }
    double kine_fa = 0.0;
    if (sst) {
      L.k = L.sc[0];  /* face value (reconstructed in second order) */
      R.k = R.sc[0];
      double w0, w1;
      face_weights(h, f, c0, c1, &w0, &w1);
      kine_fa = (w1 * t->phi[0][c0] + w0 * t->phi[0][c1]) / (w0 + w1);
    }
    /* the face's shock fix (JoeWithModels.cpp:4956-4982) */
    ausm_opt o = bnd_opt(p);
    if (flag && (flag[c0] + flag[c1]) > flag_sum) o.shock = p->shock_fix;
    cflux(p, o, F, ns, &L, &R, area, nV, 0);
    for (int i = 0; i < B; i++) { rhs[B * c0 + i] -= F[i]; rhs[B * c1 + i] += F[i]; }
    int n00 = m->nbocv_i[c0], n01 = csr_slot(m, c0, c1), n11 = m->nbocv_i[c1], n10 = csr_slot(m, c1, c0);
    if (implicit) {
      cstate L0 = cell_cstate(h, t, c0), R0 = cell_cstate(h, t, c1);
      if (sst) { L0.k = t->phi[0][c0]; R0.k = t->phi[0][c1]; }
      cmatrices(p, o, Apl, Ami, ns, &L0, &R0, area, nV, 0);
      add_blk(A, B, n00, Apl, 1.0);
      add_blk(A, B, n01, Ami, 1.0);
      add_blk(A, B, n11, Ami, -1.0);
      add_blk(A, B, n10, Apl, -1.0);
    }
    if (visc) {
      double sV[3];
      for (int i = 0; i < 3; i++) sV[i] = m->x_cv[3 * c1 + i] - m->x_cv[3 * c0 + i];
      double smag = norm3(sV, sV);
      double alpha = dot3(nV, sV);
      double uf[3];
      for (int i = 0; i < 3; i++) uf[i] = 0.5 * (h->vel[3 * c0 + i] + h->vel[3 * c1 + i]);
      vstate v0 = cell_vstate(h, t, c0), v1 = cell_vstate(h, t, c1);
      for (int q = 0; q < ns; q++) dfa[q] = t->diff[q][f];
      visc_coupled(Fv, implicit ? A0 : NULL, implicit ? A1 : NULL, ns, &v0, &v1, h->mul_fa[f], h->mut_fa[f],
                   h->lamOcp_fa[f], p->PrTurb, kine_fa, uf, dfa, ones, area, nV, smag, sV, alpha);
      for (int i = 0; i < B; i++) { rhs[B * c0 + i] -= Fv[i]; rhs[B * c1 + i] += Fv[i]; }
      if (implicit) {
        add_blk(A, B, n00, A0, 1.0);
        add_blk(A, B, n01, A1, 1.0);
        add_blk(A, B, n11, A1, -1.0);
        add_blk(A, B, n10, A0, -1.0);
      }
    }
  }
  /* boundary faces, JoeWithModels.cpp:5139-5799 */
  for (int z = 0; z < m->nzones; z++) {
    const jg_zone *zn = &m->zones[z];
    for (int q = 0; q < ns; q++) dterm[q] = (zn->scal_bc & ((1 << q) | (1 << (4 + q)))) ? 1.0 : 0.0;
    for (int f = zn->ifa_f; f <= zn->ifa_l; f++) {
      int c0 = m->cvofa[2 * f];
      int n00 = m->nbocv_i[c0];
      double nV[3];
      double area = norm3(nV, &m->fa_normal[3 * f]);
      cstate Bs = bfa_cstate(h, t, f);
      for (int q = 0; q < ns; q++) dfa[q] = t->diff[q][f];
      if (zn->kind == JG_BC_SYMMETRY || zn->kind == JG_BC_NEUMANN) {
        if (sst) Bs.k = t->phi_bfa[0][f];
        int op = (zn->kind == JG_BC_SYMMETRY) ? only_p : 0;
        cflux(p, ob, F, ns, &Bs, &Bs, area, nV, op);
        for (int i = 0; i < B; i++) rhs[B * c0 + i] -= F[i];
        if (implicit) {
          if (zn->kind == JG_BC_NEUMANN || p->symm_bc == JG_SYMM_NEW_NUMERIC) {
            cmatrices(p, ob, Apl, Ami, ns, &Bs, &Bs, area, nV, 0);
            for (int e = 0; e < BB; e++)
              A[(size_t)BB * n00 + e] += (p->symm_bc == JG_SYMM_NEW_NUMERIC) ? Apl[e] + Ami[e] : Apl[e];
          } else {
            cmatrices(p, ob, Apl, NULL, ns, &Bs, &Bs, area, nV, only_p);
            add_blk(A, B, n00, Apl, 1.0);
          }
        }
        if (visc && zn->kind == JG_BC_SYMMETRY) {
          const double *g = &h->grad_u[9 * c0];
          double tmp = 2.0 / 3.0 * ((h->mul_fa[f] + h->mut_fa[f]) * (g[0] + g[4] + g[8]) + h->rho_bfa[f] * Bs.k);
          for (int i = 0; i < 3; i++) rhs[B * c0 + 1 + i] -= area * tmp * nV[i];
        }
        if (visc && zn->kind == JG_BC_NEUMANN) {
          double sV[3];
          for (int i = 0; i < 3; i++) sV[i] = m->x_fa[3 * f + i] - m->x_cv[3 * c0 + i];
          double smag = fabs(dot3(sV, nV));
          vstate vb = bfa_vstate(h, t, f, c0);
          for (int q = 0; q < ns; q++) vb.sc[q] = t->phi_bfa[q][f];
          vb.k = Bs.k;
          visc_coupled(Fv, implicit ? A0 : NULL, implicit ? A1 : NULL, ns, &vb, &vb, h->mul_fa[f], h->mut_fa[f],
                       h->lamOcp_fa[f], p->PrTurb, Bs.k, &h->vel_bfa[3 * f], dfa, ones, area, nV, smag, nV, 1.0);
          for (int i = 0; i < B; i++) rhs[B * c0 + i] -= Fv[i];
          if (implicit) add_blk(A, B, n00, A0, 1.0);
        }
      } else if (zn->kind == JG_BC_WALL) {
        /* the wall branch keeps the face kinetic energy at 0 (JoeWithModels.cpp:5448-5452) */
        cflux(p, ob, F, ns, &Bs, &Bs, area, nV, only_p);
        for (int i = 0; i < B; i++) rhs[B * c0 + i] -= F[i];
        if (implicit) {
          if (p->symm_bc == JG_SYMM_NEW_NUMERIC) {
            cmatrices(p, ob, Apl, Ami, ns, &Bs, &Bs, area, nV, 0);
            for (int e = 0; e < BB; e++) A[(size_t)BB * n00 + e] += Apl[e] + Ami[e];
          } else {
            cmatrices(p, ob, Apl, NULL, ns, &Bs, &Bs, area, nV, only_p);
            add_blk(A, B, n00, Apl, 1.0);
          }
        }
        if (visc) {
          double sV[3];
          for (int i = 0; i < 3; i++) sV[i] = m->x_fa[3 * f + i] - m->x_cv[3 * c0 + i];
          double smag = fabs(dot3(sV, nV));
          vstate v0 = cell_vstate(h, t, c0);
          vstate vb = bfa_vstate(h, t, f, c0);
          for (int q = 0; q < ns; q++) {
            vb.sc[q] = t->phi_bfa[q][f];
            vb.gs[q] = &t->grad_phi[q][3 * c0];
          }
          vb.k = 0.0;
          visc_coupled(Fv, implicit ? A0 : NULL, NULL, ns, &v0, &vb, h->mul_fa[f], 0.0, h->lamOcp_fa[f], p->PrTurb,
                       0.0, &h->vel_bfa[3 * f], dfa, dterm, area, nV, smag, nV, 1.0);
          for (int i = 0; i < B; i++) rhs[B * c0 + i] -= Fv[i];
          if (implicit) add_blk(A, B, n00, A0, 1.0);
        }
      } else {
        /* CBC, CBC_SUBSONIC_INLET/OUTLET, FARFIELD: JoeWithModels.cpp:5624-5788 */
        cstate L = cell_cstate(h, t, c0);
        if (p->second_order) reconstruct_c(h, t, c0, f, &L);
        if (sst) { L.k = L.sc[0]; Bs.k = t->phi_bfa[0][f]; }
        cflux(p, ob, F, ns, &L, &Bs, area, nV, 0);
        for (int i = 0; i < B; i++) rhs[B * c0 + i] -= F[i];
        if (implicit) {
          cstate L0 = cell_cstate(h, t, c0);
          if (sst) L0.k = t->phi[0][c0];
          cmatrices(p, ob, Apl, NULL, ns, &L0, &Bs, area, nV, 0);
          add_blk(A, B, n00, Apl, 1.0);
        }
        if (visc) {
          double sV[3];
          for (int i = 0; i < 3; i++) sV[i] = m->x_fa[3 * f + i] - m->x_cv[3 * c0 + i];
          double smag = norm3(sV, sV);
          double alpha = dot3(nV, sV);
          vstate v0 = cell_vstate(h, t, c0);
          vstate vb = bfa_vstate(h, t, f, c0);
          /* the outer state carries the reconstructed face scalars, as the reference passes them */
          for (int q = 0; q < ns; q++) {
            vb.sc[q] = L.sc[q];
            vb.gs[q] = &t->grad_phi[q][3 * c0];
          }
          vb.k = Bs.k;
          visc_coupled(Fv, implicit ? A0 : NULL, NULL, ns, &v0, &vb, h->mul_fa[f], h->mut_fa[f], h->lamOcp_fa[f],
                       p->PrTurb, Bs.k, &h->vel_bfa[3 * f], dfa, dterm, area, nV, smag, sV, alpha);
          for (int i = 0; i < B; i++) rhs[B * c0 + i] -= Fv[i];
          if (implicit) add_blk(A, B, n00, A0, 1.0);
        }
      }
    }
  }
  free(flag);
  /* sourceHookCoupled: gravity (JoeWithModels.h:134-152) */
  {
    const double *g = p->gravity;
    for (int c = 0; c < h->ncv; c++) {
      double vol = m->cv_volume[c];
      rhs[B * c + 1] += vol * h->rho[c] * g[0];
      rhs[B * c + 2] += vol * h->rho[c] * g[1];
      rhs[B * c + 3] += vol * h->rho[c] * g[2];
      rhs[B * c + 4] += vol * (g[0] * h->rhou[3 * c + 0] + g[1] * h->rhou[3 * c + 1] + g[2] * h->rhou[3 * c + 2]);
      if (implicit) {
        double *a = &A[(size_t)BB * m->nbocv_i[c]];
        a[B * 1 + 0] -= vol * g[0];
        a[B * 2 + 0] -= vol * g[1];
        a[B * 3 + 0] -= vol * g[2];
        a[B * 4 + 1] -= vol * g[0];
        a[B * 4 + 2] -= vol * g[1];
        a[B * 4 + 3] -= vol * g[2];
      }
    }
  }
  /* source terms: sourceHookRansTurbCoupled (TurbModel_SA.h:359-434; TurbModel_KOMSST.h:306-340) */
  for (int c = 0; c < h->ncv; c++) {
    size_t d0 = (size_t)BB * m->nbocv_i[c];
    double vol = m->cv_volume[c], rho = h->rho[c];
    if (t->model == JG_TURB_SA) {
      double mue = face_avg(h, h->mul_fa, c);
      double Om = dmax(t->vortMag[c], 1.e-8);
      double Strainrate = dmax(t->strMag[c], 1.e-8);
      double d = t->wallDist[c];
      double nu = t->phi[0][c];
      double chi = nu * rho / mue;
      double chi_3 = pow(chi, 3.0);
      double inv_K2d2 = 1.0 / (SA_K2 * d * d);
      double fv1 = chi_3 / (chi_3 + SA_CV1_3);
      double fv2 = 1.0 - chi / (1.0 + chi * fv1);
      double S = dmax(Om + dmin(0.0, Strainrate - Om) * 0.0, 0.0);
      double Shat = S + nu * fv2 * inv_K2d2;
      double inv_Shat = 1.0 / dmax(Shat, 1.0e-8);
      double r = dmin(nu * inv_Shat * inv_K2d2, 10.0);
      double g = r + SA_CW2 * (pow(r, 6.0) - r);
      double g_6 = pow(g, 6.0);
      double fw = g * pow((1.0 + SA_CW3_6) / (g_6 + SA_CW3_6), 1.0 / 6.0);
      double H1 = SA_CB1 * Shat * nu;
      double H2 = -SA_CW1 * fw * nu * nu / pow(d, 2.0);
      double H3 = SA_CB2 / SA_SIGMA * dot3(&t->grad_phi[0][3 * c], &t->grad_phi[0][3 * c]);
      rhs[B * c + 5] += rho * vol * (H1 + H2 + H3);
      if (implicit) {
        double d_H1 = 0.0;
        double d_H2 = -2.0 * SA_CW1 * fw * nu / pow(d, 2.0);
        A[d0 + B * 5 + 5] -= (d_H1 + d_H2) * vol;
      }
    } else {
      double k = t->phi[0][c], om = t->phi[1][c];
      double F1 = t->F1[c];
      double alfa_1 = SST_B1 / SST_BS - SST_SO1 * pow(0.41, 2.0) / sqrt(SST_BS);
      double alfa_2 = SST_B2 / SST_BS - SST_SO2 * pow(0.41, 2.0) / sqrt(SST_BS);
      double alfa = F1 * alfa_1 + (1.0 - F1) * alfa_2;
      double beta = F1 * SST_B1 + (1.0 - F1) * SST_B2;
      double zeta = dmin(1.0 / om, SST_A1 / (t->vortMag[c] * t->F2[c]));
      double mut = dmin(dmax(rho * k * zeta, 1.0e-8), 1.0e5);
      double Pk = dmax(mut * t->strMag[c] * t->strMag[c] - 2. / 3. * rho * k * t->diverg[c], 0.0);
      Pk = dmin(Pk, 20.0 * SST_BS * rho * k * om);
      rhs[B * c + 5] += (Pk - SST_BS * rho * om * k) * vol;
      zeta = dmax(om, t->vortMag[c] * t->F2[c] / SST_A1);
      Pk = dmax(t->strMag[c] * t->strMag[c] - 2. / 3. * zeta * t->diverg[c], 0.0);
      rhs[B * c + 6] += (alfa * rho * Pk + (1.0 - F1) * t->crossDiff[c] - beta * rho * om * om) * vol;
      if (implicit) {
        A[d0 + B * 5 + 5] -= -SST_BS * om * vol;
        A[d0 + B * 6 + 6] -= -2.0 * beta * om * vol;
      }
    }
  }
}

/* n x n LU without pivoting (ludeco / lusolv, UgpWithCv.cpp:2489-2577, any order) */
static void ludeco_n(double *A, int n) {
  for (int jc = 1; jc < n; jc++) A[jc] /= A[0];
  int jrjc = 0;
  for (;;) {
    jrjc++;
    int jrjcm1 = jrjc - 1, jrjcp1 = jrjc + 1;
    for (int jr = jrjc; jr < n; jr++) {
      double sum = A[n * jr + jrjc];
      for (int jm = 0; jm <= jrjcm1; jm++) sum -= A[n * jr + jm] * A[n * jm + jrjc];
      A[n * jr + jrjc] = sum;
    }
    if (jrjc == (n - 1)) return;
    for (int jc = jrjcp1; jc < n; jc++) {
      double sum = A[n * jrjc + jc];
      for (int jm = 0; jm <= jrjcm1; jm++) sum -= A[n * jrjc + jm] * A[n * jm + jc];
      A[n * jrjc + jc] = sum / A[n * jrjc + jrjc];
    }
  }
}
static void lusolv_n(const double *A, double *c, int n) {
  c[0] = c[0] / A[0];
  for (int jr = 1; jr < n; jr++) {
    double sum = c[jr];
    for (int jm = 0; jm <= jr - 1; jm++) sum -= A[n * jr + jm] * c[jm];
    c[jr] = sum / A[n * jr + jr];
  }
  for (int jrjr = 1; jrjr < n; jrjr++) {
    int jr = (n - 1) - jrjr, jrp1 = jr + 1;
    double sum = c[jr];
    for (int jmjm = jrp1; jmjm < n; jmjm++) {
      int jm = (n - 1) - jmjm + jrp1;
      sum -= A[n * jr + jm] * c[jm];
    }
    c[jr] = sum;
  }
}

/* LINE relaxation as the GPU runs it (no reference counterpart): `sweeps`
 * block line-Jacobi sweeps of the B x B system from x = 0.  On the lines of
 * build_lines' relaxed rule (two or more cells) the block-tridiagonal system is
 * solved exactly by block Thomas elimination; the other cells take a block
 * Jacobi step; every coupling that is not between line neighbours uses the
 * previous sweep's x. */
int jo_line_relax(jo_case *h, int B, double *x, const double *A, const double *rhs, int sweeps) {
  const jg_mesh *m = &h->m;
  const int n = h->ncv, BB = B * B;
  if (!h->rline_off) build_lines(h, 1, &h->rnlines, &h->rline_off, &h->rline_cv);
  int *prev = (int *)malloc(sizeof(int) * n), *next = (int *)malloc(sizeof(int) * n);
  char *on = (char *)calloc(n, 1);
  for (int c = 0; c < n; c++) prev[c] = next[c] = -1;
  int ncl = 0;
  for (int l = 0; l < h->rnlines; l++) {
    int a = h->rline_off[l], b = h->rline_off[l + 1];
    if (b - a < 2) continue;
    for (int k = a; k < b; k++) {
      int c = h->rline_cv[k];
      on[c] = 1;
      ncl++;
      if (k > a) prev[c] = h->rline_cv[k - 1];
      if (k + 1 < b) next[c] = h->rline_cv[k + 1];
    }
  }
  double *LU = dalloc((size_t)BB * n), *xn = dalloc((size_t)B * n), *r = dalloc((size_t)B * n);
  double *inv = dalloc((size_t)BB * n), *low = dalloc((size_t)BB * n), *vv = dalloc((size_t)B * n);
  for (int c = 0; c < n; c++) {
    memcpy(&LU[(size_t)BB * c], &A[(size_t)BB * m->nbocv_i[c]], sizeof(double) * BB);
    ludeco_n(&LU[(size_t)BB * c], B);
  }
  /* line factors: inv_i of the eliminated diagonal, low_i = A(c_i, c_{i-1}) inv_{i-1}, indexed by cell */
  double bh[MAXB * MAXB], lu[MAXB * MAXB], col[MAXB];
  for (int l = 0; l < h->rnlines; l++) {
    int a = h->rline_off[l], b = h->rline_off[l + 1];
    if (b - a < 2) continue;
    memcpy(bh, &A[(size_t)BB * m->nbocv_i[h->rline_cv[a]]], sizeof(double) * BB);
    for (int k = a; k < b; k++) {
      int c = h->rline_cv[k];
      memcpy(lu, bh, sizeof(double) * BB);
      ludeco_n(lu, B);
      for (int j = 0; j < B; j++) {
        for (int i = 0; i < B; i++) col[i] = (i == j) ? 1.0 : 0.0;
        lusolv_n(lu, col, B);
        for (int i = 0; i < B; i++) inv[(size_t)BB * c + B * i + j] = col[i];
      }
      if (k + 1 == b) break;
      int cn = h->rline_cv[k + 1];
      const double *Alo = &A[(size_t)BB * csr_entry(m, cn, c)];
      const double *Aup = &A[(size_t)BB * csr_entry(m, c, cn)];
      for (int i = 0; i < B; i++)
        for (int j = 0; j < B; j++) {
          double t = 0.0;
          for (int q = 0; q < B; q++) t += Alo[B * i + q] * inv[(size_t)BB * c + B * q + j];
          low[(size_t)BB * cn + B * i + j] = t;
        }
      const double *Dn = &A[(size_t)BB * m->nbocv_i[cn]];
      for (int i = 0; i < B; i++)
        for (int j = 0; j < B; j++) {
          double t = 0.0;
          for (int q = 0; q < B; q++) t += low[(size_t)BB * cn + B * i + q] * Aup[B * q + j];
          bh[B * i + j] = Dn[B * i + j] - t;
        }
    }
  }
  memset(x, 0, sizeof(double) * B * n);
  for (int s = 0; s < sweeps; s++) {
    for (int c = 0; c < n; c++) {
      double *rc = &r[(size_t)B * c];
      for (int i = 0; i < B; i++) rc[i] = rhs[(size_t)B * c + i];
      for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++) {
        int nb = m->nbocv_v[k];
        if (nb == prev[c] || nb == next[c]) continue;
        for (int i = 0; i < B; i++)
          for (int j = 0; j < B; j++) rc[i] -= A[(size_t)BB * k + B * i + j] * x[(size_t)B * nb + j];
      }
      if (!on[c]) {
        memcpy(&xn[(size_t)B * c], rc, sizeof(double) * B);
        lusolv_n(&LU[(size_t)BB * c], &xn[(size_t)B * c], B);
      }
    }
    for (int l = 0; l < h->rnlines; l++) {
      int a = h->rline_off[l], b = h->rline_off[l + 1];
      if (b - a < 2) continue;
      for (int k = a; k < b; k++) {
        int c = h->rline_cv[k];
        for (int i = 0; i < B; i++) {
          double t = 0.0;
          if (k > a)
            for (int q = 0; q < B; q++) t += low[(size_t)BB * c + B * i + q] * vv[(size_t)B * h->rline_cv[k - 1] + q];
          vv[(size_t)B * c + i] = r[(size_t)B * c + i] - t;
        }
      }
      for (int k = b - 1; k >= a; k--) {
        int c = h->rline_cv[k];
        double a1[MAXB];
        for (int i = 0; i < B; i++) {
          double t = 0.0;
          if (k + 1 < b) {
            int cn = h->rline_cv[k + 1];
            const double *Aup = &A[(size_t)BB * csr_entry(m, c, cn)];
            for (int q = 0; q < B; q++) t += Aup[B * i + q] * xn[(size_t)B * cn + q];
          }
          a1[i] = vv[(size_t)B * c + i] - t;
        }
        for (int i = 0; i < B; i++) {
          double t = 0.0;
          for (int q = 0; q < B; q++) t += inv[(size_t)BB * c + B * i + q] * a1[q];
          xn[(size_t)B * c + i] = t;
        }
      }
    }
    memcpy(x, xn, sizeof(double) * B * n);
  }
  (void)ncl;
  free(prev); free(next); free(on); free(LU); free(xn); free(r); free(inv); free(low); free(vv);
  return sweeps;
}

/* block Jacobi (sgs = 0) or multicolour block Gauss-Seidel (sgs = 1) sweeps
 * of the B x B system from x = 0, as the GPU runs them */
int jo_solve_blocks(jo_case *h, int B, double *x, const double *A, const double *rhs, int sweeps, int sgs) {
  int n = h->ncv;
  const jg_mesh *m = &h->m;
  double *LU = dalloc((size_t)B * B * n), *xn = dalloc((size_t)B * n);
  int *color = (int *)calloc(n, sizeof(int));
  int ncol = 1, mark[256];
  for (int k = 0; k < 256; k++) mark[k] = -1;
  for (int c = 0; c < n; c++) {
    for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++)
      if (m->nbocv_v[k] < c) mark[color[m->nbocv_v[k]]] = c;
    int q = 0;
    while (q < 255 && mark[q] == c) q++;
    color[c] = q;
    if (q + 1 > ncol) ncol = q + 1;
  }
  if (!sgs) ncol = 1;
  for (int c = 0; c < n; c++) {
    memcpy(&LU[(size_t)B * B * c], &A[(size_t)B * B * m->nbocv_i[c]], sizeof(double) * B * B);
    ludeco_n(&LU[(size_t)B * B * c], B);
  }
  memset(x, 0, sizeof(double) * B * n);
  double b[MAXB];
  for (int s = 0; s < sweeps; s++)
    for (int q = 0; q < ncol; q++) {
      int col = (s % 2 == 0) ? q : ncol - 1 - q;
      for (int c = 0; c < n; c++) {
        if (sgs && color[c] != col) continue;
        for (int i = 0; i < B; i++) b[i] = rhs[B * c + i];
        for (int k = m->nbocv_i[c] + 1; k < m->nbocv_i[c + 1]; k++) {
          int nb = m->nbocv_v[k];
          for (int i = 0; i < B; i++)
            for (int j = 0; j < B; j++) b[i] -= A[(size_t)B * B * k + B * i + j] * x[B * nb + j];
        }
        lusolv_n(&LU[(size_t)B * B * c], b, B);
        memcpy(sgs ? &x[B * c] : &xn[B * c], b, sizeof(double) * B);
      }
      if (!sgs) memcpy(x, xn, sizeof(double) * B * n);
    }
  free(LU); free(xn); free(color);
  return sweeps;
}

/* runBackwardEulerCoupled loop body (JoeWithModels.cpp:4416-4529) with the
 * GPU's block relaxation for the linear solve; resid[B] = last L1 residual */
int jo_step_coupled(jo_case *h, int nsteps, double *resid) {
  const jg_params *p = &h->p;
  jo_turb *t = turb_of(h);
  const int ns = t->ns, B = 5 + ns;
  int n = h->ncv, nbs = h->nbs;
  double *A = dalloc((size_t)B * B * nbs), *dq = dalloc((size_t)B * n), *rhs = dalloc((size_t)B * n);
  int err = 0;
  for (int it = 0; it < nsteps; it++) {
    h->step++;
    if ((h->step >= p->cfl_after) && (h->step % p->cfl_interval == 0) && (h->cfl < p->cfl_max)) h->cfl *= p->cfl_factor;
    jo_calc_dt(h, h->cfl);
    memset(A, 0, sizeof(double) * B * B * nbs);
    jo_calc_rhs_coupled(h, rhs, A, 1);
    double r[MAXB] = {0, 0, 0, 0, 0, 0, 0};
    for (int c = 0; c < n; c++)
      for (int i = 0; i < B; i++) r[i] += fabs(rhs[B * c + i]);
    for (int c = 0; c < n; c++) {
      for (int i = 0; i < B; i++) rhs[B * c + i] *= p->under_relax;
      double tmp = h->m.cv_volume[c] / (h->local_dt[c]);
      for (int i = 0; i < B; i++) A[(size_t)B * B * h->m.nbocv_i[c] + (B + 1) * i] += tmp;
    }
    if (p->lin_solver == JG_LS_LINE) jo_line_relax(h, B, dq, A, rhs, p->ls_max_iter);
    else jo_solve_blocks(h, B, dq, A, rhs, p->ls_max_iter, p->lin_solver == JG_LS_SGS);
    for (int c = 0; c < n; c++) {
      h->rho[c] += dq[B * c];
      for (int i = 0; i < 3; i++) h->rhou[3 * c + i] += dq[B * c + 1 + i];
      h->rhoE[c] += dq[B * c + 4];
    }
    for (int q = 0; q < ns; q++)
      for (int c = 0; c < n; c++)
        t->phi[q][c] = dmin(dmax((t->phi[q][c] * (h->rho[c] - dq[B * c]) + dq[B * c + 5 + q]) / h->rho[c], t->lower[q]),
                            t->upper[q]);
    if (jo_calc_state_coupled(h) != 0) err = -1;
    if (resid) memcpy(resid, r, sizeof(double) * B);
  }
  free(A); free(dq); free(rhs);
  return err;
}
