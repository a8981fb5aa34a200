// Test harness over the reference solver (Joe, MUM suite), compiled from the
// reference's own sources by oracle/Makefile into oracle/_ref/.  This is the
// reference's documented extension point (a case-local main that derives from
// JoeWithModels, reference README:45-60, src/joe/joe.cpp:925-1019); it is test
// infrastructure only: it dumps the reference's arrays so the oracle and the
// GPU path can be checked against them, and it times the reference's own
// runBackwardEuler as the CPU baseline.
//
// usage: ref_harness <Joe.in> <run 0|1|2> <dump|coupled|run> <outdir>
//        joe_gpu_case <Joe.in> 0 gpu <outdir>   (the same harness built with the drop-in binding)
//   run 0 : JoeWithModels (laminar / inviscid); run 1 : + RansTurbSA; run 2 : + RansTurbKOmSST
//   dump    : init -> state/material/BC -> calcDt -> calcRhs(implicit) -> one
//             linear solve (solveCoupledLinSysNS); every array written to outdir
//   coupled : init -> state/material/BC/turbulent viscosity -> calcDt ->
//             calcRhsCoupled(implicit): the (5+nScal) residual and block
//             Jacobian of runBackwardEulerCoupled, plus the turbulence arrays
//   run     : init -> runBackwardEuler (NSTEPS from the input); prints the
//             wall-clock of the iteration loop and writes the final state
//   gpu     : as run, with include/joe_gpu.hpp's JoeGpu in place of JoeWithModels:
//             the loop on the GPU through libjoe_b200.so
//
// Extra input keys read only by this harness:
//   HARNESS_PERTURB = a   smooth perturbation of the uniform initial state
//                         (same formula as myjoe_b200.case.perturbed_state);
//                         transported scalars get the factor of scal_perturb
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "JoeWithModels.h"
#include "turbModels/TurbModel_SA.h"
#include "turbModels/TurbModel_KOMSST.h"
#ifdef JOE_GPU_BINDING
// the drop-in binding (include/joe_gpu.hpp), built into oracle/_ref/joe_gpu_case with the
// library linked: mode "gpu" runs the same case path as "run" with the loop on the GPU
#include "joe_gpu.hpp"
#endif

static std::string g_out;

static void dumpRaw(const char *name, const void *p, size_t bytes) {
  std::string fn = g_out + "/" + name;
  FILE *f = fopen(fn.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", fn.c_str()); exit(3); }
  if (bytes) fwrite(p, 1, bytes, f);
  fclose(f);
}
#define DUMPD(name, ptr, n) dumpRaw(name ".f64", (const void *)(ptr), sizeof(double) * (size_t)(n))
#define DUMPI(name, ptr, n) dumpRaw(name ".i32", (const void *)(ptr), sizeof(int) * (size_t)(n))

// Perturbation used by both sides (harness and myjoe_b200.case).
static void perturb(double x, double y, double z, double a, double f[5]) {
  f[0] = 1.0 + a * sin(2.1 * x + 0.3) * cos(1.7 * y + 0.2) * (1.0 + 0.3 * sin(3.1 * z));
  f[1] = a * cos(1.3 * x + 0.1) * sin(2.3 * y + 0.4);
  f[2] = a * sin(1.9 * x + 0.7) * cos(0.9 * y + 0.5);
  f[3] = 0.5 * a * sin(2.7 * z + 0.2) * cos(1.1 * x);
  f[4] = 1.0 + 0.5 * a * cos(1.5 * x + 0.6) * sin(1.2 * y + 0.8);
}

// Perturbation factor of transported scalars (same formula in myjoe_b200.case).
static double scal_perturb(double x, double y, double z, double a) {
  return 1.0 + a * sin(1.3 * x + 0.4) * cos(0.7 * y + 0.1) * (1.0 + 0.2 * cos(2.3 * z));
}

// the reference's case-local SA / SST classes (src/joe/joe.cpp:286-313 pattern)
class JoeSA : public JoeWithModels, public RansTurbSA {
public:
  JoeSA(char *name) : JoeWithModels(name), UgpWithCvCompFlow(name) {}
};
class JoeSST : public JoeWithModels, public RansTurbKOmSST {
public:
  JoeSST(char *name) : JoeWithModels(name), UgpWithCvCompFlow(name) {}
};

template <class Base>
class Harness : public Base {
public:
  Harness(char *name) : Base(name), UgpWithCvCompFlow(name) {}

  void initialHook() {
    JoeWithModels::initialHook();
    if (this->checkParam("HARNESS_PERTURB")) {
      double a = this->getDoubleParam("HARNESS_PERTURB");
      double uref[3] = {0.0, 0.0, 0.0};
      Param *p;
      if (this->getParam(p, "U_INITIAL")) { uref[0] = p->getDouble(1); uref[1] = p->getDouble(2); uref[2] = p->getDouble(3); }
      double umag = sqrt(uref[0] * uref[0] + uref[1] * uref[1] + uref[2] * uref[2]) + 1.0;
      for (int icv = 0; icv < this->ncv; icv++) {
        double f[5];
        perturb(this->x_cv[icv][0], this->x_cv[icv][1], this->x_cv[icv][2], a, f);
        double r0 = this->rho[icv];
        double u[3] = {this->rhou[icv][0] / r0, this->rhou[icv][1] / r0, this->rhou[icv][2] / r0};
        double p0 = (this->gamma[icv] - 1.0) * (this->rhoE[icv] - 0.5 * r0 * (u[0] * u[0] + u[1] * u[1] + u[2] * u[2]));
        double r = r0 * f[0];
        double v[3] = {u[0] + umag * f[1], u[1] + umag * f[2], u[2] + umag * f[3]};
        double pp = p0 * f[4];
        this->rho[icv] = r;
        for (int i = 0; i < 3; i++) this->rhou[icv][i] = r * v[i];
        this->rhoE[icv] = pp / (this->gamma[icv] - 1.0) + 0.5 * r * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      }
      for (size_t s = 0; s < this->scalarTranspEqVector.size(); s++) {
        double *phi = this->scalarTranspEqVector[s].phi;
        for (int icv = 0; icv < this->ncv; icv++)
          phi[icv] *= scal_perturb(this->x_cv[icv][0], this->x_cv[icv][1], this->x_cv[icv][2], a);
      }
    }
  }

  bool lines = false;

  // JoeWithModels::run's preamble (JoeWithModels.cpp:20-31), up to the time integration
  void setup() {
    this->initializeFromRestartFile(this->getStringParam("RESTART"));
    this->initialHook();
    this->initialHookScalarRansTurbModel();
    this->initialHookScalarRansCombModel();
    if (this->getStringParam("LINEAR_SOLVER_NS") == "BCGSTAB_LINELET") {
      this->initializeLinelet();
      lines = true;
    }
  }

  // the lines initializeLinelet built: line_off[nSources+1], line_cv (cells of the lines in order)
  void dumpLinelets() {
    if (!lines) return;
    std::vector<int> off(1, 0), cv;
    for (int l = 0; l < this->nSources; l++) {
      for (size_t i = 0; i < this->linelet_cv[l].size(); i++) cv.push_back(this->linelet_cv[l][i]);
      off.push_back((int)cv.size());
    }
    DUMPI("line_off", off.data(), off.size());
    DUMPI("line_cv", cv.data(), cv.size());
  }

  void writeMeta() {
    std::string fn = g_out + "/meta.txt";
    FILE *f = fopen(fn.c_str(), "w");
    int nScal = this->scalarTranspEqVector.size();
    fprintf(f, "ncv %d\nncv_g %d\nnfa %d\nnfa_b %d\nnbocv_s %d\nfaocv_s %d\nnScal %d\n", this->ncv, this->ncv_g,
            this->nfa, this->nfa_b, this->nbocv_s, this->faocv_i[this->ncv], nScal);
    fprintf(f, "R_gas %.17e\nGAMMA %.17e\n", this->R_gas, this->GAMMA);
    for (list<FaZone>::iterator zone = this->faZoneList.begin(); zone != this->faZoneList.end(); zone++)
      if (zone->getKind() == FA_ZONE_BOUNDARY)
        fprintf(f, "zone %s %d %d\n", zone->getName(), zone->ifa_f, zone->ifa_l);
    fclose(f);
  }

  void dumpState(const char *tag) {
    char nm[64];
    sprintf(nm, "%s_rho.f64", tag);  dumpRaw(nm, this->rho, sizeof(double) * this->ncv);
    sprintf(nm, "%s_rhou.f64", tag); dumpRaw(nm, this->rhou, sizeof(double) * 3 * this->ncv);
    sprintf(nm, "%s_rhoE.f64", tag); dumpRaw(nm, this->rhoE, sizeof(double) * this->ncv);
  }

  // the JST arrays runBackwardEuler allocates before its loop (JoeWithModels.cpp:932-937),
  // so that calcRhs can run outside it
  void prepareJST() {
    if (this->getStringParam("SPACE_INTEGRATION", "HLLC") != "JST") return;
    int n = this->ncv_g;
    this->PressSensor = new double[n];
    this->Conserv_Und_Lapl = new double[n][5];
    this->Lambda = new double[n];
    this->BoundaryCV = new bool[n];
    this->NeighborCV = new int[n];
    this->p1_Und_Lapl = new double[n];
    this->p2_Und_Lapl = new double[n];
    this->calcJSTCoeff_Const(0);
  }

  void dumpAll() {
    int ncv = this->ncv, nfa = this->nfa, nfa_b = this->nfa_b, nbocv_s = this->nbocv_s;
    prepareJST();
    writeMeta();
    DUMPI("cvofa", this->cvofa, 2 * nfa);
    DUMPI("faocv_i", this->faocv_i, ncv + 1);
    DUMPI("faocv_v", this->faocv_v, this->faocv_i[ncv]);
    DUMPI("nbocv_i", this->nbocv_i, ncv + 1);
    DUMPI("nbocv_v", this->nbocv_v, nbocv_s);
    DUMPD("x_cv", this->x_cv, 3 * ncv);
    DUMPD("x_fa", this->x_fa, 3 * nfa);
    DUMPD("fa_normal", this->fa_normal, 3 * nfa);
    DUMPD("cv_volume", this->cv_volume, ncv);
    dumpLinelets();
    DUMPD("nbocv_lsg_coeff", this->nbocv_lsg_coeff, 3 * nbocv_s);
    DUMPD("boundary_fa_lsg_coeff", this->boundary_fa_lsg_coeff, 3 * nfa_b);
    dumpState("init");

    this->calcStateVariables();
    this->calcMaterialProperties();
    this->setBC();
    this->calcRansTurbViscMuet();

    DUMPD("vel", this->vel, 3 * ncv);
    DUMPD("press", this->press, ncv);
    DUMPD("temp", this->temp, ncv);
    DUMPD("enthalpy", this->enthalpy, ncv);
    DUMPD("sos", this->sos, ncv);
    DUMPD("rho_bfa", this->rho_bfa, nfa_b);
    DUMPD("T_bfa", this->T_bfa, nfa_b);
    DUMPD("vel_bfa", this->vel_bfa, 3 * nfa_b);
    DUMPD("p_bfa", this->p_bfa, nfa_b);
    DUMPD("h_bfa", this->h_bfa, nfa_b);
    DUMPD("gam_bfa", this->gam_bfa, nfa_b);
    DUMPD("RoM_bfa", this->RoM_bfa, nfa_b);
    DUMPD("mul_fa", this->mul_fa, nfa);
    DUMPD("lamOcp_fa", this->lamOcp_fa, nfa);
    DUMPD("mut_fa", this->mut_fa, nfa);

    double dt_min = this->calcDt(this->cfl);
    DUMPD("local_dt", this->local_dt, ncv);
    DUMPD("dt_min", &dt_min, 1);

    double *RHSrho = new double[ncv];
    double(*RHSrhou)[3] = new double[ncv][3];
    double *RHSrhoE = new double[ncv];
    double(*A)[5][5] = new double[nbocv_s][5][5];
    for (int noc = 0; noc < nbocv_s; noc++)
      for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) A[noc][i][j] = 0.0;
    this->calcRhs(RHSrho, RHSrhou, RHSrhoE, NULL, A, NULL, true);
    DUMPD("rhs_rho", RHSrho, ncv);
    DUMPD("rhs_rhou", RHSrhou, 3 * ncv);
    DUMPD("rhs_rhoE", RHSrhoE, ncv);
    DUMPD("A", A, 25 * nbocv_s);
    DUMPD("grad_u", this->grad_u, 9 * ncv);
    if (this->grad_rho) DUMPD("grad_rho", this->grad_rho, 3 * ncv);
    if (this->grad_p) DUMPD("grad_p", this->grad_p, 3 * ncv);
    if (this->grad_enthalpy) DUMPD("grad_enthalpy", this->grad_enthalpy, 3 * ncv);
    if (this->alpha_rho) DUMPD("alpha_rho", this->alpha_rho, ncv);

    // one linear solve exactly as runBackwardEuler prepares it
    double underRelax = this->getDoubleParam("UNDER_RELAXATION", "0.3");
    if (!this->checkParam("LINEAR_SOLVER_NS_TRESHOLDS"))
      ParamMap::add("LINEAR_SOLVER_NS_TRESHOLDS  MAX_ITER=30  ABS_RESID=1.0e-8  REL_RESID=1.0e-2");
    int maxIterLS = this->getParam("LINEAR_SOLVER_NS_TRESHOLDS")->getInt("MAX_ITER");
    double zeroAbsLS = this->getParam("LINEAR_SOLVER_NS_TRESHOLDS")->getDouble("ABS_RESID");
    double zeroRelLS = this->getParam("LINEAR_SOLVER_NS_TRESHOLDS")->getDouble("REL_RESID");
    double(*rhs)[5] = new double[ncv][5];
    double(*dq)[5] = new double[this->ncv_g][5];
    for (int icv = 0; icv < ncv; icv++) {
      rhs[icv][0] = underRelax * RHSrho[icv];
      rhs[icv][1] = underRelax * RHSrhou[icv][0];
      rhs[icv][2] = underRelax * RHSrhou[icv][1];
      rhs[icv][3] = underRelax * RHSrhou[icv][2];
      rhs[icv][4] = underRelax * RHSrhoE[icv];
      double tmp = this->cv_volume[icv] / (this->local_dt[icv]);
      for (int i = 0; i < 5; i++) A[this->nbocv_i[icv]][i][i] += tmp;
    }
    for (int icv = 0; icv < this->ncv_g; icv++)
      for (int i = 0; i < 5; i++) dq[icv][i] = 0.0;
    DUMPD("A_sys", A, 25 * nbocv_s);
    DUMPD("rhs_sys", rhs, 5 * ncv);
    this->solveCoupledLinSysNS(dq, A, rhs, zeroAbsLS, zeroRelLS, maxIterLS);
    DUMPD("dq", dq, 5 * ncv);
  }

  // calcRhsCoupled as runBackwardEulerCoupled calls it (JoeWithModels.cpp:4326-4611)
  void dumpCoupled() {
    int ncv = this->ncv, nfa = this->nfa, nfa_b = this->nfa_b, nbocv_s = this->nbocv_s;
    int nScal = this->scalarTranspEqVector.size();
    int B = 5 + nScal;
    writeMeta();
    DUMPI("cvofa", this->cvofa, 2 * nfa);
    DUMPI("faocv_i", this->faocv_i, ncv + 1);
    DUMPI("faocv_v", this->faocv_v, this->faocv_i[ncv]);
    DUMPI("nbocv_i", this->nbocv_i, ncv + 1);
    DUMPI("nbocv_v", this->nbocv_v, nbocv_s);
    DUMPD("x_cv", this->x_cv, 3 * ncv);
    DUMPD("x_fa", this->x_fa, 3 * nfa);
    DUMPD("fa_normal", this->fa_normal, 3 * nfa);
    DUMPD("cv_volume", this->cv_volume, ncv);
    DUMPD("nbocv_lsg_coeff", this->nbocv_lsg_coeff, 3 * nbocv_s);
    DUMPD("boundary_fa_lsg_coeff", this->boundary_fa_lsg_coeff, 3 * nfa_b);
    dumpState("init");
    for (int s = 0; s < nScal; s++) {
      char nm[64];
      sprintf(nm, "init_scal%d.f64", s);
      dumpRaw(nm, this->scalarTranspEqVector[s].phi, sizeof(double) * ncv);
    }

    for (int iScal = 0; iScal < nScal; iScal++) this->scalarTranspEqVector[iScal].coupling = "COUPLED";
    this->calcStateVariables();
    this->calcMaterialProperties();
    this->setBC();
    this->calcRansTurbViscMuet();
    DUMPD("mul_fa", this->mul_fa, nfa);
    DUMPD("lamOcp_fa", this->lamOcp_fa, nfa);
    DUMPD("mut_fa", this->mut_fa, nfa);
    DUMPD("rho_bfa", this->rho_bfa, nfa_b);
    DUMPD("vel_bfa", this->vel_bfa, 3 * nfa_b);
    DUMPD("p_bfa", this->p_bfa, nfa_b);
    DUMPD("T_bfa", this->T_bfa, nfa_b);
    DUMPD("h_bfa", this->h_bfa, nfa_b);
    for (int s = 0; s < nScal; s++) {
      char nm[64];
      sprintf(nm, "scal%d_bfa.f64", s);
      dumpRaw(nm, this->scalarTranspEqVector[s].phi_bfa, sizeof(double) * nfa_b);
    }
    const char *cvnames[] = {"wallDist", "strMag", "vortMag", "diverg", "crossDiff", "blendFuncF1", "blendFuncF2"};
    for (const char *nm : cvnames)
      if (this->getScalarData(nm)) {
        char fn[64];
        sprintf(fn, "%s.f64", nm);
        dumpRaw(fn, *(this->getScalarData(nm)->ptr), sizeof(double) * ncv);
      }

    double dt_min = this->calcDt(this->cfl);
    DUMPD("local_dt", this->local_dt, ncv);
    DUMPD("dt_min", &dt_min, 1);

    // A[nbocv_s][B][B] and rhs[ncv][B] as the pointer tables calcRhsCoupled takes
    std::vector<double> Abuf((size_t)nbocv_s * B * B, 0.0), rbuf((size_t)ncv * B, 0.0);
    std::vector<double *> Arows((size_t)nbocv_s * B), rrows(ncv);
    std::vector<double **> Ablk(nbocv_s);
    for (int noc = 0; noc < nbocv_s; noc++) {
      for (int i = 0; i < B; i++) Arows[(size_t)noc * B + i] = &Abuf[((size_t)noc * B + i) * B];
      Ablk[noc] = &Arows[(size_t)noc * B];
    }
    for (int icv = 0; icv < ncv; icv++) rrows[icv] = &rbuf[(size_t)icv * B];
    double ***A = Ablk.data();
    double **rhs = rrows.data();
    for (int noc = 0; noc < nbocv_s; noc++)
      for (int i = 0; i < B; i++)
        for (int j = 0; j < B; j++) A[noc][i][j] = 0.0;
    this->calcRhsCoupled(rhs, A, nScal, true);
    std::vector<double> flat((size_t)nbocv_s * B * B), r((size_t)ncv * B);
    for (int noc = 0; noc < nbocv_s; noc++)
      for (int i = 0; i < B; i++)
        for (int j = 0; j < B; j++) flat[((size_t)noc * B + i) * B + j] = A[noc][i][j];
    for (int icv = 0; icv < ncv; icv++)
      for (int i = 0; i < B; i++) r[(size_t)icv * B + i] = rhs[icv][i];
    DUMPD("A_coupled", flat.data(), flat.size());
    DUMPD("rhs_coupled", r.data(), r.size());
    DUMPD("grad_u", this->grad_u, 9 * ncv);
    if (this->grad_rho) DUMPD("grad_rho", this->grad_rho, 3 * ncv);
    if (this->grad_p) DUMPD("grad_p", this->grad_p, 3 * ncv);
    if (this->grad_enthalpy) DUMPD("grad_enthalpy", this->grad_enthalpy, 3 * ncv);
    for (int s = 0; s < nScal; s++) {
      char nm[64];
      sprintf(nm, "scal%d_grad.f64", s);
      dumpRaw(nm, this->scalarTranspEqVector[s].grad_phi, sizeof(double) * 3 * ncv);
      sprintf(nm, "scal%d_diff.f64", s);
      dumpRaw(nm, this->scalarTranspEqVector[s].diff, sizeof(double) * nfa);
    }
  }

  // mode "gpu" (Base = JoeGpu): the binding's GPU loop in place of runBackwardEuler
  void runTimedGpu() {
    writeMeta();
    DUMPD("x_cv", this->x_cv, 3 * this->ncv);
    dumpState("init");
    auto t0 = std::chrono::steady_clock::now();
    this->runBackwardEulerGpu();
    auto t1 = std::chrono::steady_clock::now();
    double secs = std::chrono::duration<double>(t1 - t0).count();
    dumpState("final");
    printf("HARNESS_STEPS %d\nHARNESS_SECONDS %.6f\n", this->step, secs);
  }

  void runTimed() {
    writeMeta();
    DUMPD("x_cv", this->x_cv, 3 * this->ncv);
    dumpState("init");
    auto t0 = std::chrono::steady_clock::now();
    this->runBackwardEuler();
    auto t1 = std::chrono::steady_clock::now();
    double secs = std::chrono::duration<double>(t1 - t0).count();
    dumpState("final");
    printf("HARNESS_STEPS %d\nHARNESS_SECONDS %.6f\n", this->step, secs);
  }
};

int main(int argc, char *argv[]) {
  if (argc < 5) {
    fprintf(stderr, "usage: %s <Joe.in> <run 0|1|2> <dump|run> <outdir>\n", argv[0]);
    return 2;
  }
  MPI_Init(&argc, &argv);
  initMpiStuff();
  g_out = argv[4];
  int run = atoi(argv[2]);
  std::string mode = argv[3];
  try {
#ifdef JOE_GPU_BINDING
    if (mode == "gpu" && run == 0) {
      Harness<JoeGpu> *j = new Harness<JoeGpu>(argv[1]);
      j->setup();
      j->runTimedGpu();
      MPI_Finalize();
      return 0;
    }
#endif
    if (run == 0) {
      Harness<JoeWithModels> *j = new Harness<JoeWithModels>(argv[1]);
      j->setup();
      if (mode == "dump") j->dumpAll(); else if (mode == "coupled") j->dumpCoupled(); else j->runTimed();
    } else if (run == 1) {
      Harness<JoeSA> *j = new Harness<JoeSA>(argv[1]);
      j->setup();
      if (mode == "dump") j->dumpAll(); else if (mode == "coupled") j->dumpCoupled(); else j->runTimed();
    } else if (run == 2) {
      Harness<JoeSST> *j = new Harness<JoeSST>(argv[1]);
      j->setup();
      if (mode == "dump") j->dumpAll(); else if (mode == "coupled") j->dumpCoupled(); else j->runTimed();
    } else {
      fprintf(stderr, "run %d not built into this harness yet\n", run);
      return 2;
    }
  } catch (int e) {
    fprintf(stderr, "reference threw %d\n", e);
    return 1;
  }
  MPI_Finalize();
  return 0;
}
