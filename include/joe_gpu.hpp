/* joe_gpu.hpp -- the drop-in binding on the reference's side: a case class that
 * keeps the reference's mesh reading, geometry, LSQ coefficients, initial
 * condition and output, and runs runBackwardEuler's loop
 * (src/joe/JoeWithModels.cpp:881-1198) on the GPU through the C ABI of
 * joe_b200.h.
 *
 * The reference's extension point is a case-local joe.cpp whose classes derive
 * from JoeWithModels (reference README:45-60, src/joe/joe.cpp:925-1019).
 * runBackwardEuler, calcRhs and solveCoupledLinSysNS are not virtual
 * (JoeWithModels.h, UgpWithCvCompFlow.h:899), so the drop-in is a subclass
 * whose run() calls the GPU loop.  Include this header in the case's joe.cpp
 * after the reference's own headers, compile it with the reference's flags
 * and -I<repo>/include, and link with -L<repo>/myjoe_b200 -ljoe_b200:
 *
 *   #include "JoeWithModels.h"
 *   #include "joe_gpu.hpp"
 *   int main(int argc, char *argv[]) {
 *     MPI_Init(&argc, &argv); initMpiStuff();
 *     JoeGpu *joe = new JoeGpu((char *)"Joe.in");
 *     joe->run();
 *     delete joe; MPI_Finalize(); return 0;
 *   }
 *
 * JoeGpuCase<Base> takes the reference class it extends (JoeWithModels; with a
 * turbulence mixin the case uses the coupled path: jg_params.turb_model). One
 * MPI rank (the GPU holds the whole case). */
#pragma once
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "joe_b200.h"

template <class Base>
class JoeGpuCase : public Base {
 public:
  JoeGpuCase(char *name) : Base(name), UgpWithCvCompFlow(name) {}

  /* GPU settings beside the reference's Joe.in (no reference keys): the form and the
   * linear solver's alternatives.  Defaults are the plain FP64 drop-in. */
  int gpu_precision = JG_PREC_FP64;
  int gpu_renumber = JG_RENUMBER_NONE;

  /* the zone table from the reference's own BC parameters (setBC, JoeWithModels.cpp:3857-4300) */
  std::vector<jg_zone> gpuZones() {
    std::vector<jg_zone> z;
    for (std::list<FaZone>::iterator zone = this->faZoneList.begin(); zone != this->faZoneList.end(); zone++) {
      if (zone->getKind() != FA_ZONE_BOUNDARY) continue;
      Param *p;
      if (!this->getParam(p, zone->getName())) {
        std::cerr << "no boundary condition for zone " << zone->getName() << std::endl;
        throw(-1);
      }
      jg_zone q = {};
      q.ifa_f = zone->ifa_f;
      q.ifa_l = zone->ifa_l;
      const std::string k = p->getString();
      if (k == "SYMMETRY") {
        q.kind = JG_BC_SYMMETRY;
      } else if (k == "WALL") {
        q.kind = JG_BC_WALL;
        const int i = p->findString("TEMP");
        q.v[0] = i ? p->getDouble(i + 1) : 0.0;
      } else if (k == "CBC") {  /* u_bc[3], T_bc, p_bc */
        q.kind = JG_BC_CBC;
        for (int i = 0; i < 5; i++) q.v[i] = p->getDouble(i + 2);
      } else if (k == "CBC_SUBSONIC_INLET") {  /* angleU[3], Ttot, ptot */
        q.kind = JG_BC_CBC_SUBSONIC_INLET;
        for (int i = 0; i < 5; i++) q.v[i] = p->getDouble(i + 2);
      } else if (k == "CBC_SUBSONIC_OUTLET") {
        q.kind = JG_BC_CBC_SUBSONIC_OUTLET;
        q.v[0] = p->getDouble(2);
      } else if (k == "NEUMANN") {
        q.kind = JG_BC_NEUMANN;
      } else if (k == "FARFIELD") {  /* u_bc[3], p_bc, rho_bc, gamma_bc */
        q.kind = JG_BC_FARFIELD;
        for (int i = 0; i < 6; i++) q.v[i] = p->getDouble(i + 2);
      } else {
        std::cerr << "boundary condition " << k << " of zone " << zone->getName() << " is not on the GPU path"
                  << std::endl;
        throw(-1);
      }
      z.push_back(q);
    }
    return z;
  }

  /* the hot path's Joe.in settings, as UgpWithCvCompFlow's constructor and runBackwardEuler
   * read them (UgpWithCvCompFlow.h:57-502, JoeWithModels.cpp:881-924) */
  jg_params gpuParams() {
    jg_params q = {};
    q.gamma = this->GAMMA;
    q.R_gas = this->R_gas;
    q.Pr = this->Pr;
    q.PrTurb = this->PrTurb;
    q.mu_mode = this->viscMode == "SUTHERLAND" ? JG_MU_SUTHERLAND : JG_MU_POWERLAW;
    q.mu_ref = this->mu_ref;
    q.mu_power_law = this->mu_power_law;
    q.SL_Tref = this->SL_Tref;
    q.SL_Sref = this->SL_Sref;
    q.T_ref = this->T_ref;
    const std::string f = this->getStringParam("SPACE_INTEGRATION", "HLLC");
    q.flux = f == "ROE" ? JG_FLUX_ROE : f == "AUSM" ? JG_FLUX_AUSM : f == "HAENEL" ? JG_FLUX_HAENEL
           : (f == "AUSMDV" || f == "AUSMD" || f == "AUSMV") ? JG_FLUX_AUSMDV : f == "JST" ? JG_FLUX_JST : JG_FLUX_HLLC;
    if (q.flux == JG_FLUX_AUSMDV) {
      q.ausm_type = this->AUSM_Type == "V" ? JG_AUSM_V : this->AUSM_Type == "D" ? JG_AUSM_D : JG_AUSM_DV;
      q.shock_fix = this->Shock_Fix_Type == "HAENEL" ? JG_SHOCK_FIX_HAENEL
                  : this->Shock_Fix_Type == "ALPHA_LR" ? JG_SHOCK_FIX_ALPHA_LR : JG_SHOCK_FIX_NONE;
      q.shock_flag = this->Shock_Fix_Flag == "CELL_FLAG_TET" ? JG_SHOCK_FLAG_TET : JG_SHOCK_FLAG_HEX;
      q.entropy_fix = this->Entropy_Fix == "EXPANSION_FAN";
    }
    q.second_order = this->sndOrder;
    q.limiter = this->limiterNavierS != UgpWithCv::NOLIMITER;
    q.eps = this->epsilonSDWLS;  /* GRAD_RECONSTRUCTION EPS, the limiter's and SDWLS's epsilon */
    q.grad_scheme = this->gradreconstruction == UgpWithCv::GRAD_GG ? JG_GRAD_GREENGAUSS
                  : this->gradreconstruction == UgpWithCv::GRAD_SDWLS ? JG_GRAD_SDWLS : JG_GRAD_LSQ;
    q.visc_limiter = this->getStringParam("VISC_LIMITER", "YES") == "YES";
    const std::string s = this->getStringParam("SYMM_BC", "ORIGINAL_NUMERIC");
    q.symm_bc = s == "ANALYTICAL" ? JG_SYMM_ANALYTICAL : s == "NEW_NUMERIC" ? JG_SYMM_NEW_NUMERIC
              : JG_SYMM_ORIGINAL_NUMERIC;
    q.time_step_mode = this->timeStepMode == "DT" ? JG_TS_DT : this->timeStepMode == "CFL_MIN" ? JG_TS_CFL_MIN
                     : JG_TS_CFL;
    q.time_step = this->getStringParam("TIME_STEP", "MAX_BASED") == "SUM_BASED" ? JG_DT_SUM_BASED : JG_DT_MAX_BASED;
    q.cfl = this->cfl;
    q.dt = this->timeStepMode == "DT" ? this->getDoubleParam("DT") : 0.0;
    if (!this->checkParam("CFL_RAMP"))  /* runBackwardEuler's default: no increase */
      ParamMap::add("CFL_RAMP AFTER_ITER=100  INTERVAL_ITER=10  FACTOR_CFL=1.0  MAX_CFL=100.0");
    Param *r = this->getParam("CFL_RAMP");
    q.cfl_after = r->getInt("AFTER_ITER");
    q.cfl_interval = r->getInt("INTERVAL_ITER");
    q.cfl_factor = r->getDouble("FACTOR_CFL");
    q.cfl_max = r->getDouble("MAX_CFL");
    q.under_relax = this->getDoubleParam("UNDER_RELAXATION", "0.3");
    const std::string ls = this->getStringParam("LINEAR_SOLVER_NS", "BCGSTAB");
    q.lin_solver = ls == "LUSGS" ? JG_LS_LUSGS : ls == "BCGSTAB_LINELET" ? JG_LS_BCGSTAB_LINELET
                 : ls == "JACOBI" ? JG_LS_JACOBI : ls == "SGS" ? JG_LS_SGS : ls == "LINE" ? JG_LS_LINE
                 : JG_LS_BCGSTAB;
    if (!this->checkParam("LINEAR_SOLVER_NS_TRESHOLDS"))
      ParamMap::add("LINEAR_SOLVER_NS_TRESHOLDS  MAX_ITER=30  ABS_RESID=1.0e-8  REL_RESID=1.0e-2");
    Param *t = this->getParam("LINEAR_SOLVER_NS_TRESHOLDS");
    q.ls_max_iter = t->getInt("MAX_ITER");
    q.ls_abs = t->getDouble("ABS_RESID");
    q.ls_rel = t->getDouble("REL_RESID");
    for (int i = 0; i < 3; i++) q.gravity[i] = this->gravity[i];  /* GX, GY, GZ of sourceHook */
    q.precision = gpu_precision;
    q.renumber = gpu_renumber;
    q.jac_lag = 1;
    return q;
  }

  /* runBackwardEuler on the GPU: the reference's state in, steps until doneSolver, the state out
   * (with the reference's own state, material and boundary passes, so its output sees it) */
  void runBackwardEulerGpu() {
    std::vector<jg_zone> zl = gpuZones();
    jg_mesh m = {this->ncv, this->nfa, this->nfa_b, this->nbocv_s, (int)zl.size(), &this->cvofa[0][0],
                 this->faocv_i, this->faocv_v, this->nbocv_i, this->nbocv_v, &this->x_cv[0][0], &this->x_fa[0][0],
                 &this->fa_normal[0][0], this->cv_volume, &this->nbocv_lsg_coeff[0][0],
                 &this->boundary_fa_lsg_coeff[0][0], zl.data()};
    jg_params q = gpuParams();
    jg_case_t *h = NULL;
    if (jg_create(&m, &q, &h) != JG_OK) {
      std::cerr << jg_last_error() << std::endl;
      throw(-1);
    }
    if (jg_set_state(h, this->rho, &this->rhou[0][0], this->rhoE) != JG_OK ||
        jg_set_cfl_step(h, this->cfl, this->step) != JG_OK) {
      std::cerr << jg_last_error() << std::endl;
      jg_destroy(h);
      throw(-1);
    }
    double res[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    int done = this->doneSolver(1.0e20);
    while (done != 1) {  /* one GPU step per pass, the reference's stopping rule */
      if (jg_step(h, 1, res) != JG_OK) {
        std::cerr << jg_last_error() << std::endl;
        break;
      }
      this->step++;
      if (this->step % this->check_interval == 0) this->showResidue(res);
      done = this->doneSolver(res[4]);
    }
    double cfl;
    int step;
    jg_get_cfl_step(h, &cfl, &step);
    this->cfl = cfl;
    jg_get_state(h, this->rho, &this->rhou[0][0], this->rhoE);
    jg_destroy(h);
    this->calcStateVariables();
    this->calcMaterialProperties();
    this->setBC();
  }

  /* JoeWithModels::run (JoeWithModels.cpp:20-60) with the GPU loop */
  void run() {
    this->initializeFromRestartFile(this->getStringParam("RESTART"));
    this->initialHook();
    this->initialHookScalarRansTurbModel();
    this->initialHookScalarRansCombModel();
    runBackwardEulerGpu();
    this->finalHook();
    this->writeRestart();
  }
};

typedef JoeGpuCase<JoeWithModels> JoeGpu;
