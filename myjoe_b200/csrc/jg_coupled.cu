// jg_coupled.cu -- the coupled (5+ns)x(5+ns) path with a turbulence model:
// runBackwardEulerCoupled / calcRhsCoupled / calcFluxCoupled
// (src/joe/JoeWithModels.cpp:4326-5826) with RansTurbSA
// (src/joe/turbModels/TurbModel_SA.h, ns = 1: nuSA, 6x6 blocks) or
// RansTurbKOmSST (TurbModel_KOMSST.h, ns = 2: kine and omega, 7x7 blocks).
//
// Same structure as the 5x5 path: one thread per cell walks its faces in the
// reference's faocv order, evaluates every face in the face's own orientation
// (bit-identical on both sides), owns its residual, its diagonal block and
// its row of off-diagonal blocks (sliced ELL, B*B components).  Row/column
// 5+s of every block is rho*phi_s.  Gradients, strain/vorticity, blending
// functions, turbulent viscosity and scalar diffusivities are computed once
// after each update from the new state (the reference recomputes them from
// the same state inside the next calcFluxCoupled; the values are identical).
#include <cuda_runtime.h>
#include <math.h>

#include "jg_cell.cuh"
#include "jg_flux.cuh"
#include "jg_internal.h"

namespace jg {

// RansTurbSA defaults (TurbModel_SA.h:21-36)
constexpr double SA_CV1_3 = 357.911, SA_CW1 = 3.239067817, SA_CW2 = 0.3, SA_CW3_6 = 64.0;
constexpr double SA_SIGMA = 0.6666666, SA_CB1 = 0.1355, SA_CB2 = 0.622, SA_K2 = 0.1681;
// RansTurbKOmSST defaults (TurbModel_KOMSST.h:19-54)
constexpr double SST_SK1 = 0.85, SST_SK2 = 1.0, SST_SO1 = 0.5, SST_SO2 = 0.856;
constexpr double SST_B1 = 0.075, SST_B2 = 0.0828, SST_BS = 0.09, SST_A1 = 0.31;

template <int MODEL>
struct TM {
  static constexpr int NS = (MODEL == JG_TURB_SST) ? 2 : 1;
  static constexpr int B = 5 + NS;
  static constexpr int BB = B * B;
};

__device__ __forceinline__ void unit_normal_c(const Mesh& m, int f, double nV[3], double& area) {
  unit_normal(m, f, nV, area);
}
__device__ __forceinline__ double sq(double x) { return x * x; }  // pow(x, 2.0) of the reference, exactly

// ---------------------------------------------------------------------------
// calcWallDistance (UgpWithCvCompFlow.h:1395-1535): nearest WALL face centroid
// (first in zone order on ties), then the normal distance when the cell lies
// over that face.  Wall-face centroids are staged through shared memory.
// Cells [c0, c1) against the WALL faces wall_f[w0 .. w1) (a batch: one case).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_wall_dist(Mesh m, Turb t, int c0, int c1, int w0, int w1) {
  __shared__ double sx[256][3];
  const int c = c0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int nwall = w1 - w0;
  double x[3] = {0.0, 0.0, 0.0};
  if (c < c1)
    for (int i = 0; i < 3; i++) x[i] = m.x_cv[3 * c + i];
  double minD = 1.0e20;
  int save = 0;
  for (int k0 = 0; k0 < nwall; k0 += 256) {
    int k = k0 + threadIdx.x;
    if (k < nwall)
      for (int i = 0; i < 3; i++) sx[threadIdx.x][i] = m.x_fa[3 * t.wall_f[w0 + k] + i];
    __syncthreads();
    int n = min(256, nwall - k0);
    for (int j = 0; j < n; j++) {
      double d = sqrt(sq(x[0] - sx[j][0]) + sq(x[1] - sx[j][1]) + sq(x[2] - sx[j][2]));
      if (d < minD) {
        minD = d;
        save = k0 + j;
      }
    }
    __syncthreads();
  }
  if (c >= c1 || nwall == 0) return;
  int f = t.wall_f[w0 + save];
  double n[3], sh[3], nmag;
  unit_normal_c(m, f, n, nmag);
  for (int i = 0; i < 3; i++) sh[i] = m.x_fa[3 * f + i] - x[i];
  double sMag2 = dot3(sh, sh);
  double dNorm2 = dot3(sh, n) * dot3(sh, n);
  double dTang2 = sMag2 - dNorm2;
  double specRadius2 = 0.5 * nmag;
  t.wd[c] = (dTang2 > specRadius2) ? minD : fabs(dot3(sh, n));
}

__device__ __forceinline__ double mu_lam(const Params& p, double T) {
  // calcMuLam, UgpWithCvCompFlow.h:1596-1616
  if (p.mu_mode == JG_MU_SUTHERLAND) return p.mu_ref * pow(T / p.SL_T, 1.5) * (p.SL_T + p.SL_S) / (T + p.SL_S);
  return p.mu_ref * pow(T / p.T_ref, p.mu_pow);
}

// setScalarBC (Scalars.cpp:289-360): Dirichlet value on inflow, the model's
// hook (SST omega on a wall, TurbModel_KOMSST.h:342-358), else zero flux
__global__ void k_scalar_bc(Mesh m, Params p, State st, Turb t) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nfa_b) return;
  const DevZone z = m.zones[m.bzone[f]];
  const int c0 = m.cvofa[2 * f], N = m.ncv, nb = m.nfa_b;
  const double* vb = &st.bfa[8 * f + 1];
  for (int s = 0; s < t.ns; s++) {
    double v;
    if (z.scal_bc & (1 << (4 + s))) {
      if (t.model == JG_TURB_SST && s == 1 && z.kind == JG_BC_WALL) {
        double muLamCV = mu_lam(p, st.prim[8 * c0 + 4]);
        double d = t.wd[c0];
        v = 60.0 * muLamCV / (st.q[5 * c0] * SST_B1 * d * d);
      } else {
        v = t.phi_bfa[s * nb + f];  // a hook the model does not define leaves the value as it is
      }
    } else if (z.scal_bc & (1 << s)) {
      double un = vb[0] * m.fa_n[3 * f] + vb[1] * m.fa_n[3 * f + 1] + vb[2] * m.fa_n[3 * f + 2];
      v = (un > 1.0e-8) ? t.phi[s * N + c0] : z.v[6 + s];
    } else {
      v = t.phi[s * N + c0];
    }
    t.phi_bfa[s * nb + f] = v;
  }
}

// calcCvScalarGrad + limitCvScalarGradBJ (UgpWithCv.h:881-938, 1009-1056) of every scalar
__global__ void k_grad_phi(Mesh m, Params p, Turb t) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  const int N = m.ncv, nb = m.nfa_b;
  for (int s = 0; s < t.ns; s++) {
    const double* phi = t.phi + (size_t)s * N;
    const double* pb = t.phi_bfa + (size_t)s * nb;
    const double pc = phi[c];
    double g[3];
    int k0 = m.nb_i[c], k1 = m.nb_i[c + 1];
    for (int j = 0; j < 3; j++) g[j] = m.lsq[3 * k0 + j] * pc;
    double pmax = pc, pmin = pc;
    for (int k = k0 + 1; k < k1; k++) {
      double pn = phi[m.nb_v[k]];
      for (int j = 0; j < 3; j++) g[j] += m.lsq[3 * k + j] * pn;
      pmax = fmax(pmax, pn);
      pmin = fmin(pmin, pn);
    }
    for (int k = m.bf_i[c]; k < m.bf_i[c + 1]; k++) {
      int f = m.bf_v[k];
      for (int j = 0; j < 3; j++) g[j] += m.blsq[3 * f + j] * pb[f];
    }
    if (p.limiter) {
      double alfa = 1.0;
      if ((pmax - pmin) > 1.0e-12) {
        double e2 = sq(fmax(p.eps * fabs(pc), 1.0e-8));
        for (int k = m.slot_i[c]; k < m.slot_i[c + 1]; k++) {
          Slot sl = m.slots[k];
          if (sl.nb < 0) continue;
          double r0[3];
          for (int j = 0; j < 3; j++) r0[j] = m.x_fa[3 * sl.f + j] - m.x_cv[3 * c + j];
          double phifa = pc + dot3(r0, g);
          double dm = phifa - pc;
          double dp = ((phifa - pc) >= 0.0) ? pmax - pc : pmin - pc;
          alfa = fmin(alfa, (dp * dp + 2.0 * dm * dp + e2) / (dp * dp + 2 * dm * dm + dm * dp + e2));
        }
      } else {
        alfa = 0.0;
      }
      for (int j = 0; j < 3; j++) g[j] *= alfa;
    }
    for (int j = 0; j < 3; j++) t.grad_phi[((size_t)s * N + c) * 3 + j] = g[j];
  }
}

// InterpolateAtCellCenterFromFaceValues (UgpWithCvCompFlow.h:1538-1552)
__device__ __forceinline__ double face_avg_c(const Mesh& m, const double* phi, int c) {
  double v = 0.0;
  int k0 = m.slot_i[c], k1 = m.slot_i[c + 1];
  for (int k = k0; k < k1; k++) v += phi[m.slots[k].f];
  return v / (double)(k1 - k0);
}

// calcStrainRate(AndDivergence) + calcVorticity (UgpWithCvCompFlow.h:1310-1393)
// from the limited grad_u; SST: calcMenterBlendingFunctions (TurbModel_KOMSST.h:360-386)
__global__ void k_turb_cell(Mesh m, State st, Turb t) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  const double* g = &st.gu[9 * c];
  double div = g[0] + g[4] + g[8];
  double sm = 0.0, vm = 0.0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      if (i == j) sm += sq(0.5 * (g[3 * i + j] + g[3 * j + i]) - 1. / 3. * div);
      else sm += sq(0.5 * (g[3 * i + j] + g[3 * j + i]));
    }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) vm += sq(0.5 * (g[3 * i + j] - g[3 * j + i]));
  t.strMag[c] = sqrt(2.0 * sm);
  t.vortMag[c] = sqrt(2.0 * vm);
  if (t.model != JG_TURB_SST) return;
  t.diverg[c] = div;
  const int N = m.ncv;
  double rho = st.q[5 * c], k = t.phi[c], om = t.phi[N + c];
  double d = t.wd[c];
  double mue = face_avg_c(m, st.mul_fa, c);
  const double* gk = &t.grad_phi[3 * c];
  const double* go = &t.grad_phi[3 * ((size_t)N + c)];
  double cd = fmax(2.0 * rho * SST_SO2 / om * dot3(gk, go), 1.0e-20);
  t.crossDiff[c] = cd;
  double gamma1 = 500.0 * mue / (sq(d) * rho * om);
  double gamma2 = 4.0 * SST_SO2 * rho * k / (d * d * cd);
  double gamma3 = sqrt(k) / (SST_BS * om * d);
  double gamma = fmin(fmax(gamma1, gamma3), gamma2);
  t.F1[c] = tanh(pow(gamma, 4.0));
  gamma = fmax(2.0 * gamma3, gamma1);
  t.F2[c] = tanh(sq(gamma));
}

// calcRansTurbViscMuet (TurbModel_SA.h:74-128; TurbModel_KOMSST.h:109-167) and the
// scalar diffusivities (diffusivityHookScalarRansTurb, SA :130-173, SST :169-256)
__global__ void k_turb_face(Mesh m, State st, Turb t) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nfa) return;
  const int N = m.ncv, nf = m.nfa, nb = m.nfa_b;
  const double mul = st.mul_fa[f];
  const bool sst = t.model == JG_TURB_SST;
  if (f >= m.nfa_b) {
    int c0 = m.cvofa[2 * f], c1 = m.cvofa[2 * f + 1];
    double d0[3], d1[3];
    for (int i = 0; i < 3; i++) {
      d0[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c0 + i];
      d1[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c1 + i];
    }
    double w0 = sqrt(dot3(d0, d0)), w1 = sqrt(dot3(d1, d1));
    double rho_fa = (w1 * st.q[5 * c0] + w0 * st.q[5 * c1]) / (w0 + w1);
    if (!sst) {
      double nu_fa = (w1 * t.phi[c0] + w0 * t.phi[c1]) / (w0 + w1);
      double muSA = rho_fa * nu_fa;
      double chi_3 = pow(muSA / mul, 3.0);
      double fv1 = chi_3 / (chi_3 + SA_CV1_3);
      st.mut_fa[f] = fmax(muSA * fv1, 0.0);
      t.diff[f] = (1.0 / SA_SIGMA) * (mul + rho_fa * nu_fa);
    } else {
      double kine_fa = (w1 * t.phi[c0] + w0 * t.phi[c1]) / (w0 + w1);
      double om_fa = (w1 * t.phi[N + c0] + w0 * t.phi[N + c1]) / (w0 + w1);
      double lim_fa = (w1 * t.vortMag[c0] + w0 * t.vortMag[c1]) / (w0 + w1);
      double F2_fa = (w1 * t.F2[c0] + w0 * t.F2[c1]) / (w0 + w1);
      double zeta = fmin(1.0 / om_fa, SST_A1 / (lim_fa * F2_fa));
      double mut = fmin(fmax(rho_fa * kine_fa * zeta, 0.0), 1.0);
      st.mut_fa[f] = mut;
      double f1_fa = (w1 * t.F1[c0] + w0 * t.F1[c1]) / (w0 + w1);
      t.diff[f] = mul + (SST_SK1 * f1_fa + (1. - f1_fa) * SST_SK2) * mut;
      t.diff[nf + f] = mul + (SST_SO1 * f1_fa + (1. - f1_fa) * SST_SO2) * mut;
    }
  } else {
    const DevZone z = m.zones[m.bzone[f]];
    const int c0 = m.cvofa[2 * f];
    const double rho0 = st.q[5 * c0];
    if (!sst) {
      if (z.kind == JG_BC_WALL) {
        st.mut_fa[f] = 0.0;
        t.diff[f] = (1.0 / SA_SIGMA) * mul;
      } else {
        double muSA = rho0 * t.phi[c0];
        double mul0 = face_avg_c(m, st.mul_fa, c0);
        double chi_3 = pow(muSA / mul0, 3.0);
        double fv1 = chi_3 / (chi_3 + SA_CV1_3);
        st.mut_fa[f] = fmax(muSA * fv1, 0.0);
        t.diff[f] = (1.0 / SA_SIGMA) * (mul + st.bfa[8 * f] * t.phi_bfa[f]);
      }
    } else {
      if (z.kind == JG_BC_WALL) {
        st.mut_fa[f] = 0.0;
        t.diff[f] = mul;
        t.diff[nf + f] = mul;
      } else {
        double zeta = fmin(1.0 / t.phi[N + c0], SST_A1 / (t.vortMag[c0] * t.F2[c0]));
        double mut = fmin(fmax(rho0 * t.phi[c0] * zeta, 0.0), 1.0);
        st.mut_fa[f] = mut;
        double F1 = t.F1[c0];
        t.diff[f] = mul + (SST_SK1 * F1 + (1. - F1) * SST_SK2) * mut;
        t.diff[nf + f] = mul + (SST_SO1 * F1 + (1. - F1) * SST_SO2) * mut;
      }
    }
  }
  (void)nb;
}

// ---------------------------------------------------------------------------
// coupled HLLC flux and matrices (UgpWithCvCompFlow.cpp:1808-2289; ConvTerm =
// 1, dp/dscal = 0); k is the kinetic energy of the state (SST), else 0
// ---------------------------------------------------------------------------
template <int NS>
struct CState {
  double rho, u[3], p, T, h, gam, sc[NS], k;
};

template <int NS>
__device__ void flux_hllc_c(double* F, const CState<NS>& L, const CState<NS>& R, double area, const double* nV,
                            bool only_p) {
  constexpr int B = 5 + NS;
  if (only_p) {
    F[0] = 0.0;
    for (int i = 1; i < 4; i++) F[i] = L.p * nV[i - 1];
    for (int i = 4; i < B; i++) F[i] = 0.0;
  } else {
    double unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u), cL = sqrt(L.gam * L.p / L.rho);
    double rhoeL = (L.h + 0.5 * uLuL + L.k) * L.rho - L.p;
    double unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u), cR = sqrt(R.gam * R.p / R.rho);
    double rhoeR = (R.h + 0.5 * uRuR + R.k) * R.rho - R.p;
    double Rrho = sqrt(R.rho / L.rho);
    double tmp = 1.0 / (1.0 + Rrho);
    double vR[3];
    for (int i = 0; i < 3; i++) vR[i] = tmp * (L.u[i] + R.u[i] * Rrho);
    double uRoe = dot3(vR, nV);
    double gpr = tmp * ((L.gam * L.p / L.rho + 0.5 * (L.gam - 1.0) * uLuL) +
                        (R.gam * R.p / R.rho + 0.5 * (R.gam - 1.0) * uRuR) * Rrho);
    double cRoe = sqrt(gpr - ((L.gam + R.gam) * 0.5 - 1.0) * 0.5 * dot3(vR, vR));
    double sL = fmin(uRoe - cRoe, unL - cL);
    double sR = fmax(uRoe + cRoe, unR + cR);
    double sM = (L.p - R.p - L.rho * unL * (sL - unL) + R.rho * unR * (sR - unR)) /
                (R.rho * (sR - unR) - L.rho * (sL - unL));
    double pS = R.rho * (unR - sR) * (unR - sM) + R.p;
    const double* sc;
    if (sM >= 0.0) {
      sc = L.sc;
      if (sL > 0.0) {
        F[0] = L.rho * unL;
        for (int i = 0; i < 3; i++) F[1 + i] = L.rho * L.u[i] * unL + L.p * nV[i];
        F[4] = (rhoeL + L.p) * unL;
      } else {
        double inv = 1.0 / (sL - sM), d = sL - unL;
        F[0] = (L.rho * d * inv) * sM;
        for (int i = 0; i < 3; i++) F[1 + i] = ((L.rho * L.u[i] * d + (pS - L.p) * nV[i]) * inv) * sM + pS * nV[i];
        F[4] = ((d * rhoeL - L.p * unL + pS * sM) * inv + pS) * sM;
      }
    } else {
      sc = R.sc;
      if (sR >= 0.0) {
        double inv = 1.0 / (sR - sM), d = sR - unR;
        F[0] = (R.rho * d * inv) * sM;
        for (int i = 0; i < 3; i++) F[1 + i] = ((R.rho * R.u[i] * d + (pS - R.p) * nV[i]) * inv) * sM + pS * nV[i];
        F[4] = ((d * rhoeR - R.p * unR + pS * sM) * inv + pS) * sM;
      } else {
        F[0] = R.rho * unR;
        for (int i = 0; i < 3; i++) F[1 + i] = R.rho * R.u[i] * unR + R.p * nV[i];
        F[4] = (rhoeR + R.p) * unR;
      }
    }
    for (int s = 0; s < NS; s++) F[5 + s] = 1.0 * F[0] * sc[s];
  }
  for (int i = 0; i < B; i++) F[i] *= area;
}

// calcJacobianCoupled_HLLC (:2180-2244); nA = n * area
template <int NS>
__device__ void jac_c(double* A, const double* vel, double pp, double rrho, double hh, const double* sc,
                      const double* nA, double gamma) {
  constexpr int B = 5 + NS;
  double kapm1 = gamma - 1.0;
  double nVel[3] = {vel[0] * nA[0], vel[1] * nA[1], vel[2] * nA[2]};
  double U_k = nVel[0] + nVel[1] + nVel[2];
  double vSquHlf = 0.5 * dot3(vel, vel);
  A[0] = 0.0; A[1] = nA[0]; A[2] = nA[1]; A[3] = nA[2]; A[4] = 0.0;
  for (int s = 0; s < NS; s++) A[5 + s] = 0.0;
  for (int r = 0; r < 3; r++) {
    double* a = A + B * (1 + r);
    a[0] = -vel[r] * U_k + nA[r] * (kapm1 * vSquHlf + gamma * pp / rrho - kapm1 * hh);
    for (int c = 0; c < 3; c++)
      a[1 + c] = (r == c) ? (2.0 - gamma) * nVel[r] + U_k : vel[r] * nA[c] - kapm1 * vel[c] * nA[r];
    a[4] = kapm1 * nA[r];
    for (int s = 0; s < NS; s++) a[5 + s] = 0.0 * nA[r];
  }
  double* a4 = A + 4 * B;
  a4[0] = U_k * ((gamma - 2.0) * vSquHlf - gamma * (hh - pp / rrho));
  for (int c = 0; c < 3; c++) a4[1 + c] = (hh + vSquHlf) * nA[c] - kapm1 * vel[c] * U_k;
  a4[4] = gamma * U_k;
  for (int s = 0; s < NS; s++) a4[5 + s] = 0.0 * U_k;
  for (int s = 0; s < NS; s++) {
    double* a = A + B * (5 + s);
    a[0] = 0.0;
    for (int c = 0; c < 3; c++) a[1 + c] = sc[s] * nA[c];
    a[4] = 0.0;
    for (int q = 0; q < NS; q++) a[5 + q] = 0.0;
    a[5 + s] = rrho * U_k;
  }
}

// calcdSMdU_HLLC (:2247-2266)
template <int NS>
__device__ void dsmdu_c(double* d, const double* vel, double pp, double rrho, double hh, const double* nV,
                        double gamma, double SM, double S, double invertrho, double Factor) {
  double kapm1 = gamma - 1.0;
  double U_k = vel[0] * nV[0] + vel[1] * nV[1] + vel[2] * nV[2];
  double vSquHlf = 0.5 * dot3(vel, vel);
  d[0] = Factor * invertrho * (-U_k * U_k + kapm1 * vSquHlf + gamma * pp / rrho - kapm1 * hh + SM * S);
  for (int i = 0; i < 3; i++) d[1 + i] = Factor * invertrho * ((2 * U_k - S - SM) * nV[i] - kapm1 * vel[i]);
  d[4] = Factor * invertrho * kapm1;
  for (int s = 0; s < NS; s++) d[5 + s] = Factor * invertrho * 0.0;
}

// calcSubSonicJacobianCoupled_HLLC (:2270-2289)
template <int NS>
__device__ void subsonic_c(double* A, const double* d, double rhoS, const double* rhouS, double rhoeS,
                           const double* sc, double pS, double Om, double sM, double rhoSmq, const double* nV,
                           double area) {
  constexpr int B = 5 + NS;
  double OmSM = Om * sM, OmSMp1 = OmSM + 1.0;
  double rr[B];
  rr[0] = rhoS;
  for (int i = 0; i < 3; i++) rr[1 + i] = rhouS[i] + rhoSmq * nV[i];
  rr[4] = rhoeS + pS + rhoSmq * sM;
  for (int s = 0; s < NS; s++) rr[5 + s] = rhoS * sc[s];
  for (int i = 0; i < B; i++)
    for (int r = 0; r < B; r++) A[B * r + i] = -OmSM * A[B * r + i] + area * OmSMp1 * d[i] * rr[r];
}

// calcEulerFluxMatricesCoupled_HLLC (:1934-2176), then dU/dQ of the scalar columns
template <int NS>
__device__ void matrices_hllc_c(double* AL, double* AR, const CState<NS>& L, const CState<NS>& R, double area,
                                const double* nV, bool only_p) {
  constexpr int B = 5 + NS, BB = B * B;
  if (!only_p) {
    double dd[B];
    double unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u), cL = sqrt(L.gam * L.p / L.rho);
    double hL = L.h + L.k, rhoeL = (hL + 0.5 * uLuL) * L.rho - L.p;
    double unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u), cR = sqrt(R.gam * R.p / R.rho);
    double hR = R.h + R.k, rhoeR = (hR + 0.5 * uRuR) * R.rho - R.p;
    double Rrho = sqrt(R.rho / L.rho);
    double tmp = 1.0 / (1.0 + Rrho);
    double vR[3];
    for (int i = 0; i < 3; i++) vR[i] = tmp * (L.u[i] + R.u[i] * Rrho);
    double uRoe = dot3(vR, nV);
    double gpr = tmp * ((L.gam * L.p / L.rho + 0.5 * (L.gam - 1.0) * uLuL) +
                        (R.gam * R.p / R.rho + 0.5 * (R.gam - 1.0) * uRuR) * Rrho);
    double cRoe = sqrt(gpr - ((L.gam + R.gam) * 0.5 - 1.0) * 0.5 * dot3(vR, vR));
    double sL = fmin(uRoe - cRoe, unL - cL);
    double sR = fmax(uRoe + cRoe, unR + cR);
    double invrhotld = 1.0 / (R.rho * (sR - unR) - L.rho * (sL - unL));
    double sM = (L.p - R.p - L.rho * unL * (sL - unL) + R.rho * unR * (sR - unR)) /
                (R.rho * (sR - unR) - L.rho * (sL - unL));
    double pS = R.rho * (unR - sR) * (unR - sM) + R.p;
    double nA[3] = {nV[0] * area, nV[1] * area, nV[2] * area};
    if (sM >= 0.0) {
      if (sL > 0.0) {
        if (AL) jac_c<NS>(AL, L.u, L.p, L.rho, hL, L.sc, nA, L.gam);
        if (AR)
          for (int e = 0; e < BB; e++) AR[e] = 0.0;
      } else {
        double Om = 1.0 / (sL - sM), d = sL - unL;
        double rhoS = L.rho * d * Om, rhouS[3];
        for (int i = 0; i < 3; i++) rhouS[i] = (L.rho * L.u[i] * d + (pS - L.p) * nV[i]) * Om;
        double rhoeS = (d * rhoeL - L.p * unL + pS * sM) * Om;
        if (AL) {
          dsmdu_c<NS>(dd, L.u, L.p, L.rho, hL, nV, L.gam, sM, sL, invrhotld, 1.0);
          jac_c<NS>(AL, L.u, L.p, L.rho, hL, L.sc, nA, L.gam);
          subsonic_c<NS>(AL, dd, rhoS, rhouS, rhoeS, L.sc, pS, Om, sM, R.rho * (sR - unR), nV, area);
          for (int i = 0; i < 5; i++) AL[(B + 1) * i] += area * Om * sM * sL;
          for (int s = 0; s < NS; s++) {
            AL[(5 + s) * B] += area * Om * sM * sL * L.sc[s];
            AL[(5 + s) * B + 5 + s] += area * Om * sM * sL * L.rho;
          }
        }
        if (AR) {
          dsmdu_c<NS>(dd, R.u, R.p, R.rho, hR, nV, R.gam, sM, sR, invrhotld, -1.0);
          for (int e = 0; e < BB; e++) AR[e] = 0.0;
          subsonic_c<NS>(AR, dd, rhoS, rhouS, rhoeS, L.sc, pS, Om, sM, L.rho * (sL - unL), nV, area);
        }
      }
    } else {
      if (sR >= 0.0) {
        double Om = 1.0 / (sR - sM), d = sR - unR;
        double rhoS = R.rho * d * Om, rhouS[3];
        for (int i = 0; i < 3; i++) rhouS[i] = (R.rho * R.u[i] * d + (pS - R.p) * nV[i]) * Om;
        double rhoeS = (d * rhoeR - R.p * unR + pS * sM) * Om;
        if (AR) {
          dsmdu_c<NS>(dd, R.u, R.p, R.rho, hR, nV, R.gam, sM, sR, invrhotld, -1.0);
          jac_c<NS>(AR, R.u, R.p, R.rho, hR, R.sc, nA, R.gam);
          subsonic_c<NS>(AR, dd, rhoS, rhouS, rhoeS, R.sc, pS, Om, sM, L.rho * (sL - unL), nV, area);
          for (int i = 0; i < 5; i++) AR[(B + 1) * i] += area * Om * sM * sR;
          for (int s = 0; s < NS; s++) {
            AR[(5 + s) * B] += area * Om * sM * sR * R.sc[s];
            AR[(5 + s) * B + 5 + s] += area * Om * sM * sR * R.rho;
          }
        }
        if (AL) {
          dsmdu_c<NS>(dd, L.u, L.p, L.rho, hL, nV, L.gam, sM, sL, invrhotld, 1.0);
          for (int e = 0; e < BB; e++) AL[e] = 0.0;
          subsonic_c<NS>(AL, dd, rhoS, rhouS, rhoeS, R.sc, pS, Om, sM, R.rho * (sR - unR), nV, area);
        }
      } else {
        if (AR) jac_c<NS>(AR, R.u, R.p, R.rho, hR, R.sc, nA, R.gam);
        if (AL)
          for (int e = 0; e < BB; e++) AL[e] = 0.0;
      }
    }
  } else {
    if (AL) {
      double uLuL = dot3(L.u, L.u), hL = L.h + L.k, g = L.gam;
      for (int j = 0; j < B; j++) AL[j] = 0.0;
      double dpdrho = 0.5 * (g - 1.0) * uLuL - (g - 1.0) * hL + g * L.p / L.rho;
      for (int r = 0; r < 3; r++) {
        double* a = AL + B * (1 + r);
        a[0] = dpdrho * nV[r] * area;
        for (int c = 0; c < 3; c++) a[1 + c] = -(g - 1.0) * L.u[c] * nV[r] * area;
        a[4] = (g - 1.0) * nV[r] * area;
        for (int s = 0; s < NS; s++) a[5 + s] = 0.0 * nV[r] * area;
      }
      for (int e = 4 * B; e < BB; e++) AL[e] = 0.0;
    }
    if (AR)
      for (int e = 0; e < BB; e++) AR[e] = 0.0;
  }
  if (AL)
    for (int j = 0; j < B; j++)
      for (int s = 0; s < NS; s++) {
        AL[B * j] -= L.sc[s] / L.rho * AL[B * j + 5 + s];
        AL[B * j + 5 + s] /= L.rho;
      }
  if (AR)
    for (int j = 0; j < B; j++)
      for (int s = 0; s < NS; s++) {
        AR[B * j] -= R.sc[s] / R.rho * AR[B * j + 5 + s];
        AR[B * j + 5 + s] /= R.rho;
      }
}

// ---------------------------------------------------------------------------
// coupled AUSMDV / AUSMV / AUSMD and Haenel & Schwane (UgpWithCvCompFlow.cpp:2293-3036;
// ConvTerm = 1, dp/dscal = 0): the flow part is the segregated scheme of jg_flux.cuh with the
// state's k in the total enthalpy; the scalars ride on the mass flux of the upwind side (AUSMDV,
// with the entropy fix acting on them as on the density) or of each split part (HAENEL).
// fo: the face's AUSMDV options (FO_*); haenel: the Haenel & Schwane scheme (SPACE_INTEGRATION
// HAENEL, or AUSMDV's HAENEL shock fix on this face)
// ---------------------------------------------------------------------------
template <int NS>
__device__ __forceinline__ FState fstate_c(const CState<NS>& s) {
  FState f;
  f.rho = s.rho;
  for (int i = 0; i < 3; i++) f.u[i] = s.u[i];
  f.p = s.p;
  f.gam = s.gam;
  f.h = s.h + s.k;
  return f;
}

template <int NS>
__device__ void flux_ausm_c(double* F, const CState<NS>& L, const CState<NS>& R, double area, const double* nV,
                            bool only_p, bool haenel, int fo) {
  if (only_p) {
    flux_hllc_c<NS>(F, L, R, area, nV, true);  // the same pressure-only flux
    return;
  }
  const FState fL = fstate_c(L), fR = fstate_c(R);
  double F5[5];
  const double unL = dot3(L.u, nV), cL = sqrt(L.gam * L.p / L.rho);
  const double unR = dot3(R.u, nV), cR = sqrt(R.gam * R.p / R.rho);
  const double cLR = fmax(cL, cR);
  if (haenel) {
    flux_haenel(F5, fL, fR, area, nV);
    const double mL = L.rho * hs_u_pm(unL, cLR, 1.0), mR = R.rho * hs_u_pm(unR, cLR, -1.0);
    for (int s = 0; s < NS; s++) F[5 + s] = (mL * L.sc[s] + mR * R.sc[s]) * area;
  } else {
    flux_ausmdv(F5, fL, fR, area, nV, fo);
    const double aL = ausm_alpha_L(L.p, L.rho, R.p, R.rho, fo);
    const double rh = L.rho * ausm_u_pm(aL, unL, cLR, 1.0) + R.rho * ausm_u_pm(2.0 - aL, unR, cLR, -1.0);
    const double dl = (fo & FO_EFIX) ? 0.125 * ausm_dlambda(unL, cL, unR, cR) : 0.0;
    for (int s = 0; s < NS; s++) {
      double fs = rh * (rh >= 0.0 ? L.sc[s] : R.sc[s]);
      if (dl != 0.0) fs -= dl * (R.rho * R.sc[s] - L.rho * L.sc[s]);
      F[5 + s] = fs * area;
    }
  }
  for (int i = 0; i < 5; i++) F[i] = F5[i];
}

template <int NS>
__device__ void matrices_ausm_c(double* AL, double* AR, const CState<NS>& L, const CState<NS>& R, double area,
                                const double* nV, bool only_p, bool haenel, int fo) {
  constexpr int B = 5 + NS, BB = B * B;
  if (only_p) {
    if (AL) {
      const double uLuL = dot3(L.u, L.u), g = L.gam, hL = L.h + 0.5 * uLuL + L.k;
      const double dpdrho = (1.0 - g) * (hL - uLuL) + g * L.p / L.rho;
      for (int e = 0; e < BB; e++) AL[e] = 0.0;
      for (int r = 0; r < 3; r++) {
        double* a = AL + B * (1 + r);
        a[0] = dpdrho * nV[r] * area;
        for (int c = 0; c < 3; c++) a[1 + c] = (1.0 - g) * L.u[c] * nV[r] * area;
        a[4] = (g - 1.0) * nV[r] * area;
      }
    }
    if (AR)
      for (int e = 0; e < BB; e++) AR[e] = 0.0;
  } else {
    const FState fL = fstate_c(L), fR = fstate_c(R);
    double A5L[25], A5R[25];
    if (haenel) matrices_haenel<double>(AL ? A5L : nullptr, AR ? A5R : nullptr, fL, fR, area, nV);
    else matrices_ausmdv<double>(AL ? A5L : nullptr, AR ? A5R : nullptr, fL, fR, area, nV, fo);
    const double unL = dot3(L.u, nV), cL = sqrt(L.gam * L.p / L.rho);
    const double unR = dot3(R.u, nV), cR = sqrt(R.gam * R.p / R.rho);
    const double cLR = fmax(cL, cR);
    double bp[5], bm[5], rh = 0.0, dl = 0.0, uLp = 0.0, uRm = 0.0;
    if (haenel) {
      uLp = hs_u_pm(unL, cLR, 1.0);
      uRm = hs_u_pm(unR, cLR, -1.0);
      hs_drhou_pm(bp, unL, cLR, nV, 1.0);
      hs_drhou_pm(bm, unR, cLR, nV, -1.0);
    } else {
      const double aL = ausm_alpha_L(L.p, L.rho, R.p, R.rho, fo);
      rh = L.rho * ausm_u_pm(aL, unL, cLR, 1.0) + R.rho * ausm_u_pm(2.0 - aL, unR, cLR, -1.0);
      if (fo & FO_EFIX) dl = ausm_dlambda(unL, cL, unR, cR);
      ausm_drhou_pm(bp, aL, unL, cLR, nV, 1.0);
      ausm_drhou_pm(bm, 2.0 - aL, unR, cLR, nV, -1.0);
    }
    for (int side = 0; side < 2; side++) {
      double* A = side ? AR : AL;
      if (!A) continue;
      const CState<NS>& S = side ? R : L;
      const CState<NS>& O = side ? L : R;
      const double* A5 = side ? A5R : A5L;
      const double* beta = side ? bm : bp;
      for (int e = 0; e < BB; e++) A[e] = 0.0;
      for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) A[B * i + j] = A5[5 * i + j];
      for (int q = 0; q < NS; q++) {
        double* a = A + B * (5 + q);
        if (haenel) {
          for (int j = 0; j < 5; j++) a[j] = beta[j] * S.sc[q] * area;
          a[5 + q] = S.rho * (side ? uRm : uLp) * area;
        } else {
          // the upwind side: d(rho u_1/2)/dQ phi plus rho u_1/2 on the diagonal; else the other side's phi
          const bool own = side ? (rh < 0.0) : (rh >= 0.0);
          const double ph = own ? S.sc[q] : O.sc[q];
          double v0 = beta[0] * ph, v[3], vd = own ? rh : 0.0;
          for (int j = 0; j < 3; j++) v[j] = beta[1 + j] * ph;
          if (dl != 0.0) {
            const double jump = L.rho * L.sc[q] - R.rho * R.sc[q], sg = side ? -1.0 : 1.0;
            const double un = side ? unR : unL;
            v0 += sg * 0.125 * (dl * S.sc[q] + un / S.rho * jump);
            for (int j = 0; j < 3; j++) v[j] += sg * (-0.125 * nV[j] / S.rho * jump);
            vd += sg * 0.125 * dl * S.rho;
          }
          a[0] = v0 * area;
          for (int j = 0; j < 3; j++) a[1 + j] = v[j] * area;
          a[5 + q] = vd * area;
        }
      }
    }
  }
  // dF/dQ times dQ/dU for the scalar columns
  for (int side = 0; side < 2; side++) {
    double* A = side ? AR : AL;
    if (!A) continue;
    const CState<NS>& S = side ? R : L;
    for (int j = 0; j < B; j++)
      for (int s = 0; s < NS; s++) {
        A[B * j] -= S.sc[s] / S.rho * A[B * j + 5 + s];
        A[B * j + 5 + s] /= S.rho;
      }
  }
}

// the coupled path's flux choice (calcFluxCoupled, JoeWithModels.cpp:4987-5057 and the boundary
// branches 5139-5799): FK 0 HLLC, FK 1 the AUSM family (haenel / fo as above)
template <int NS, int FK>
__device__ __forceinline__ void cflux(double* F, const CState<NS>& L, const CState<NS>& R, double area,
                                      const double* nV, bool only_p, bool haenel, int fo) {
  if (FK == 0) flux_hllc_c<NS>(F, L, R, area, nV, only_p);
  else flux_ausm_c<NS>(F, L, R, area, nV, only_p, haenel, fo);
}
template <int NS, int FK>
__device__ __forceinline__ void cmatrices(double* AL, double* AR, const CState<NS>& L, const CState<NS>& R,
                                          double area, const double* nV, bool only_p, bool haenel, int fo) {
  if (FK == 0) matrices_hllc_c<NS>(AL, AR, L, R, area, nV, only_p);
  else matrices_ausm_c<NS>(AL, AR, L, R, area, nV, only_p, haenel, fo);
}

// ---------------------------------------------------------------------------
// calcViscousFluxCoupled (UgpWithCvCompFlow.cpp:3040-3276) with the model's k
// ---------------------------------------------------------------------------
template <int NS>
struct VSideC {
  double rho, u[3], h, T, gam, sc[NS], k;
  const double* gu;      // [9]
  const double* gh;      // [3]
  const double* gs[NS];  // [3] scalar gradients (nullptr: zero)
};
template <int NS>
struct VFC {
  double tn[3], keff, muT, aas, dd[NS];
};

template <int NS>
__device__ void visc_flux_c(double* Fv, VFC<NS>& vf, const VSideC<NS>& a, const VSideC<NS>& b, double mul,
                            double mut, double lamOcp, double PrTurb, double kine_fa, const double* u_fa,
                            const double* diff, const double* diffTerm, double area, const double* nV, double smag,
                            const double* sV, double alpha) {
  double g[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) g[i][j] = 0.5 * (a.gu[3 * i + j] + b.gu[3 * i + j]);
  double fC[3] = {nV[0] - alpha * sV[0], nV[1] - alpha * sV[1], nV[2] - alpha * sV[2]};
  const double aos = alpha / smag;  // the normal-derivative weight, one division for all terms
  double muT = mul + mut;
  Fv[0] = 0.0;
  for (int i = 0; i < 3; i++)
    vf.tn[i] = muT * ((b.u[i] - a.u[i]) * aos + g[i][0] * fC[0] + g[0][i] * nV[0] + g[i][1] * fC[1] +
                      g[1][i] * nV[1] + g[i][2] * fC[2] + g[2][i] * nV[2]);
  double tmp = 2.0 / 3.0 * muT * (g[0][0] + g[1][1] + g[2][2]);
  tmp += 1.0 / 3.0 * (a.rho + b.rho) * kine_fa;
  for (int i = 0; i < 3; i++) vf.tn[i] -= tmp * nV[i];
  for (int i = 0; i < 3; i++) Fv[1 + i] = -area * vf.tn[i];
  vf.keff = lamOcp + mut / PrTurb;
  double enth = vf.keff * ((b.h - a.h) * aos + 0.5 * ((a.gh[0] + b.gh[0]) * fC[0] +
                                                             (a.gh[1] + b.gh[1]) * fC[1] +
                                                             (a.gh[2] + b.gh[2]) * fC[2]));
  double psi = muT * ((b.k - a.k) * aos);
  Fv[4] = -area * (enth + vf.tn[0] * u_fa[0] + vf.tn[1] * u_fa[1] + vf.tn[2] * u_fa[2] + psi);
  for (int s = 0; s < NS; s++) {
    double g0[3] = {0.0, 0.0, 0.0}, g1[3] = {0.0, 0.0, 0.0};
    if (a.gs[s])
      for (int i = 0; i < 3; i++) g0[i] = a.gs[s][i];
    if (b.gs[s])
      for (int i = 0; i < 3; i++) g1[i] = b.gs[s][i];
    Fv[5 + s] = -area * diffTerm[s] * diff[s] * ((b.sc[s] - a.sc[s]) * aos +
                                                 0.5 * ((g0[0] + g1[0]) * fC[0] + (g0[1] + g1[1]) * fC[1] +
                                                        (g0[2] + g1[2]) * fC[2]));
    vf.dd[s] = diffTerm[s] * diff[s];
  }
  vf.muT = muT;
  vf.aas = area * aos;
}

// acc += sgn * (A0 (side 0) or A1 (side 1)) of calcViscousFluxCoupled, from the state of that side
template <int NS>
__device__ void visc_jac_c_add(double* acc, double sgn, int side, const VFC<NS>& vf, const VSideC<NS>& v,
                               const double* u_fa, double R, double area) {
  constexpr int B = 5 + NS;
  double sg = side ? -1.0 : 1.0;
  double d11 = sg * vf.muT * vf.aas;
  double d41 = -area * vf.tn[0] * 0.5 + u_fa[0] * d11;
  double d42 = -area * vf.tn[1] * 0.5 + u_fa[1] * d11;
  double d43 = -area * vf.tn[2] * 0.5 + u_fa[2] * d11;
  double d44 = sg * vf.keff * vf.aas;
  double iR = 1.0 / v.rho;
  double q10 = -iR * v.u[0], q20 = -iR * v.u[1], q30 = -iR * v.u[2];
  double q40 = iR * v.gam * (-v.h - v.k + R * v.T + 0.5 * dot3(v.u, v.u));
  double q41 = -iR * v.u[0] * v.gam, q42 = -iR * v.u[1] * v.gam, q43 = -iR * v.u[2] * v.gam, q44 = iR * v.gam;
  acc[B + 0] += sgn * (d11 * q10);
  acc[B + 1] += sgn * (d11 * iR);
  acc[2 * B + 0] += sgn * (d11 * q20);
  acc[2 * B + 2] += sgn * (d11 * iR);
  acc[3 * B + 0] += sgn * (d11 * q30);
  acc[3 * B + 3] += sgn * (d11 * iR);
  acc[4 * B + 0] += sgn * (d41 * q10 + d42 * q20 + d43 * q30 + d44 * q40);
  acc[4 * B + 1] += sgn * (d41 * iR + d44 * q41);
  acc[4 * B + 2] += sgn * (d42 * iR + d44 * q42);
  acc[4 * B + 3] += sgn * (d43 * iR + d44 * q43);
  acc[4 * B + 4] += sgn * (d44 * q44);
  for (int s = 0; s < NS; s++) {
    double dss = sg * vf.dd[s] * vf.aas;
    acc[4 * B + 5 + s] += sgn * (d44 * (iR * iR * 0.0));
    acc[(5 + s) * B + 0] += sgn * (dss * (-iR * v.sc[s]));
    acc[(5 + s) * B + 5 + s] += sgn * (dss * iR);
  }
}

// ---------------------------------------------------------------------------
// states (scalars component-major: phi[q*N + c], phi_bfa[q*nfa_b + f])
// ---------------------------------------------------------------------------
template <int NS>
__device__ __forceinline__ CState<NS> cell_c(const Mesh& m, const Params& p, const State& st, const Turb& t, int c,
                                             bool sst) {
  CState<NS> s;
  s.rho = st.q[5 * c];
  for (int i = 0; i < 3; i++) s.u[i] = st.prim[8 * c + i];
  s.p = st.prim[8 * c + 3];
  s.T = st.prim[8 * c + 4];
  s.h = st.prim[8 * c + 5];
  s.gam = p.gamma;
  for (int q = 0; q < NS; q++) s.sc[q] = t.phi[(size_t)q * m.ncv + c];
  s.k = sst ? s.sc[0] : 0.0;
  return s;
}
template <int NS>
__device__ __forceinline__ CState<NS> bfa_c(const Mesh& m, const Params& p, const State& st, const Turb& t, int f) {
  const double* b = &st.bfa[8 * f];
  CState<NS> s;
  s.rho = b[0];
  s.u[0] = b[1]; s.u[1] = b[2]; s.u[2] = b[3];
  s.p = b[4];
  s.T = b[5];
  s.h = b[6];
  s.gam = p.gamma;
  for (int q = 0; q < NS; q++) s.sc[q] = t.phi_bfa[(size_t)q * m.nfa_b + f];
  s.k = 0.0;
  return s;
}
// reconstruction with the scalars and first-order fallback (JoeWithModels.cpp:4837-4921),
// then calcThermoProp_p (UgpWithCvCompFlow.h:1765-1771); k = the face kine (SST)
template <int NS>
__device__ __forceinline__ CState<NS> recon_c(const Mesh& m, const Params& p, const State& st, const Turb& t, int c,
                                              int f, bool sst) {
  CState<NS> s = cell_c<NS>(m, p, st, t, c, sst);
  if (!p.second_order) return s;
  double r0[3];
  for (int i = 0; i < 3; i++) r0[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
  double rr = s.rho + dot3(r0, &st.grho[3 * c]);
  double pp = s.p + dot3(r0, &st.gp[3 * c]);
  if ((pp <= 0.0) || (rr <= 0.0)) {
    pp = s.p;
    rr = s.rho;
  } else {
    for (int i = 0; i < 3; i++) s.u[i] += dot3(r0, &st.gu[9 * c + 3 * i]);
    for (int q = 0; q < NS; q++) s.sc[q] += dot3(r0, &t.grad_phi[((size_t)q * m.ncv + c) * 3]);
  }
  s.rho = rr;
  s.p = pp;
  s.T = pp / (rr * p.R);
  s.h = p.cp * s.T;
  s.k = sst ? s.sc[0] : 0.0;
  return s;
}
template <int NS>
__device__ __forceinline__ VSideC<NS> vcell_c(const Mesh& m, const State& st, const Turb& t, const Params& p, int c,
                                              bool sst) {
  VSideC<NS> v;
  v.rho = st.q[5 * c];
  for (int i = 0; i < 3; i++) v.u[i] = st.prim[8 * c + i];
  v.h = st.prim[8 * c + 5];
  v.T = st.prim[8 * c + 4];
  v.gam = p.gamma;
  for (int q = 0; q < NS; q++) {
    v.sc[q] = t.phi[(size_t)q * m.ncv + c];
    v.gs[q] = &t.grad_phi[((size_t)q * m.ncv + c) * 3];
  }
  v.k = sst ? v.sc[0] : 0.0;
  v.gu = &st.gu[9 * c];
  v.gh = &st.gh[3 * c];
  return v;
}
// boundary-face state for the viscous flux; scalars and their gradients set by the caller
template <int NS>
__device__ __forceinline__ VSideC<NS> vbfa_c(const State& st, const Params& p, int f, int c) {
  const double* b = &st.bfa[8 * f];
  VSideC<NS> v;
  v.rho = b[0];
  v.u[0] = b[1]; v.u[1] = b[2]; v.u[2] = b[3];
  v.h = b[6];
  v.T = b[5];
  v.gam = p.gamma;
  for (int q = 0; q < NS; q++) {
    v.sc[q] = 0.0;
    v.gs[q] = nullptr;
  }
  v.k = 0.0;
  v.gu = &st.gu[9 * c];
  v.gh = &st.gh[3 * c];
  return v;
}

template <int BB>
__device__ __forceinline__ size_t ell_c(const Mesh& m, int c, int col, int e) {
  int slice = c / SLICE, lane = c % SLICE;
  return ((size_t)(m.ell_off[slice] + col) * BB + e) * SLICE + lane;
}

// n x n LU without pivoting + inverse (ludeco / luinv, UgpWithCv.cpp:2489-2577)
template <int n>
__device__ void block_inverse_n(double* A, double* Ai) {
  for (int jc = 1; jc < n; jc++) A[jc] /= A[0];
  for (int jrjc = 1;; jrjc++) {
    for (int jr = jrjc; jr < n; jr++) {
      double sum = A[n * jr + jrjc];
      for (int jm = 0; jm < jrjc; jm++) sum -= A[n * jr + jm] * A[n * jm + jrjc];
      A[n * jr + jrjc] = sum;
    }
    if (jrjc == n - 1) break;
    for (int jc = jrjc + 1; jc < n; jc++) {
      double sum = A[n * jrjc + jc];
      for (int jm = 0; jm < jrjc; jm++) sum -= A[n * jrjc + jm] * A[n * jm + jc];
      A[n * jrjc + jc] = sum / A[n * jrjc + jrjc];
    }
  }
  for (int col = 0; col < n; col++) {
    double cv[n];
    for (int i = 0; i < n; i++) cv[i] = (i == col) ? 1.0 : 0.0;
    cv[0] = cv[0] / A[0];
    for (int jr = 1; jr < n; jr++) {
      double sum = cv[jr];
      for (int jm = 0; jm < jr; jm++) sum -= A[n * jr + jm] * cv[jm];
      cv[jr] = sum / A[n * jr + jr];
    }
    for (int jr = n - 2; jr >= 0; jr--) {
      double sum = cv[jr];
      for (int jm = jr + 1; jm < n; jm++) sum -= A[n * jr + jm] * cv[jm];
      cv[jr] = sum;
    }
    for (int i = 0; i < n; i++) Ai[n * i + col] = cv[i];
  }
}

// ---------------------------------------------------------------------------
// face loop: calcRhsCoupled (fluxes, boundary zones, model sources) + the
// implicit-step epilogue (vol/dt, under-relaxed rhs, D^-1)
// ---------------------------------------------------------------------------
template <typename BT, int MODEL, int FK>
__global__ void __launch_bounds__(128) k_flux_c(Mesh m, Params p, State st, Turb t, int implicit, int for_step) {
  constexpr int NS = TM<MODEL>::NS, B = TM<MODEL>::B, BB = TM<MODEL>::BB;
  constexpr bool SST = MODEL == JG_TURB_SST;
  extern __shared__ double sD[];  // [BB][blockDim.x]
  const int tid = threadIdx.x, bd = blockDim.x;
  const int c = blockIdx.x * bd + tid;
  if (c >= m.ncv || !st.case_active[m.case_of[c]]) return;  // a frozen case keeps its arrays
  const int N = m.ncv, nf = m.nfa;
  const bool only_p = p.symm_bc == JG_SYMM_ANALYTICAL;
  double rhs[B];
  for (int i = 0; i < B; i++) rhs[i] = 0.0;
  for (int e = 0; e < BB; e++) sD[e * bd + tid] = 0.0;
  BT* O = (BT*)st.O;
  double F[B];
  double one[NS], dfa[NS], dterm[NS];
  for (int q = 0; q < NS; q++) one[q] = 1.0;
  // boundary faces: AUSMDV without the shock fix (JoeWithModels.cpp:5177-5182)
  const bool ausmdv = FK && p.flux == JG_FLUX_AUSMDV, hz_b = FK && p.flux == JG_FLUX_HAENEL;
  const int fob = ausmdv ? bnd_opts<4>(p) : 0;
  for (int k = m.slot_i[c]; k < m.slot_i[c + 1]; k++) {
    const Slot s = m.slots[k];
    const int f = s.f;
    double nV[3], area;
    unit_normal_c(m, f, nV, area);
    for (int q = 0; q < NS; q++) dfa[q] = t.diff[(size_t)q * nf + f];
    if (s.nb >= 0) {
      const int c0 = s.side == 0 ? c : s.nb;
      const int c1 = s.side == 0 ? s.nb : c;
      const double sg = s.side == 0 ? -1.0 : 1.0;
      // the face's shock fix (JoeWithModels.cpp:4956-4982)
      const int fo = ausmdv ? face_opts<4>(p, st, c0, c1) : 0;
      const bool hz = hz_b || (fo & FO_HAENEL);
      {
        CState<NS> L = recon_c<NS>(m, p, st, t, c0, f, SST), R = recon_c<NS>(m, p, st, t, c1, f, SST);
        cflux<NS, FK>(F, L, R, area, nV, false, hz, fo);
        for (int i = 0; i < B; i++) rhs[i] += sg * F[i];
      }
      double Ob[BB];
      if (implicit) {
        CState<NS> L0 = cell_c<NS>(m, p, st, t, c0, SST), R0 = cell_c<NS>(m, p, st, t, c1, SST);
        double Apl[BB], Ami[BB];
        cmatrices<NS, FK>(Apl, Ami, L0, R0, area, nV, false, hz, fo);
        // row of c0: D += Apl, O = Ami ; row of c1: D -= Ami, O = -Apl
        if (s.side == 0) {
          for (int e = 0; e < BB; e++) { sD[e * bd + tid] += Apl[e]; Ob[e] = Ami[e]; }
        } else {
          for (int e = 0; e < BB; e++) { sD[e * bd + tid] -= Ami[e]; Ob[e] = -Apl[e]; }
        }
      }
      {
        VSideC<NS> v0 = vcell_c<NS>(m, st, t, p, c0, SST), v1 = vcell_c<NS>(m, st, t, p, c1, SST);
        double sV[3], smag;
        cell_to_cell(m, f, sV, smag);
        double alpha = dot3(nV, sV);
        double ufa[3] = {0.5 * (v0.u[0] + v1.u[0]), 0.5 * (v0.u[1] + v1.u[1]), 0.5 * (v0.u[2] + v1.u[2])};
        double kine_fa = 0.0;
        if (SST) {
          double d0[3], d1[3];
          for (int i = 0; i < 3; i++) {
            d0[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c0 + i];
            d1[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c1 + i];
          }
          double w0 = sqrt(dot3(d0, d0)), w1 = sqrt(dot3(d1, d1));
          kine_fa = (w1 * v0.k + w0 * v1.k) / (w0 + w1);
        }
        VFC<NS> vf;
        visc_flux_c<NS>(F, vf, v0, v1, st.mul_fa[f], st.mut_fa[f], st.lam_fa[f], p.PrTurb, kine_fa, ufa, dfa, one,
                        area, nV, smag, sV, alpha);
        for (int i = 0; i < B; i++) rhs[i] += sg * F[i];
        if (implicit) {
          // row of c0: D += A0, O += A1 ; row of c1: D -= A1, O -= A0  (JoeWithModels.cpp:5110-5127)
          double Dv[BB];
          for (int e = 0; e < BB; e++) Dv[e] = 0.0;
          if (s.side == 0) {
            visc_jac_c_add<NS>(Dv, 1.0, 0, vf, v0, ufa, p.R, area);
            visc_jac_c_add<NS>(Ob, 1.0, 1, vf, v1, ufa, p.R, area);
          } else {
            visc_jac_c_add<NS>(Dv, -1.0, 1, vf, v1, ufa, p.R, area);
            visc_jac_c_add<NS>(Ob, -1.0, 0, vf, v0, ufa, p.R, area);
          }
          for (int e = B; e < BB; e++) sD[e * bd + tid] += Dv[e];
        }
      }
      if (implicit)
        for (int e = 0; e < BB; e++) O[ell_c<BB>(m, c, s.col, e)] = (BT)Ob[e];
    } else {
      // boundary face; the cell is cvofa[f][0] (JoeWithModels.cpp:5139-5799)
      const DevZone z = m.zones[m.bzone[f]];
      for (int q = 0; q < NS; q++) dterm[q] = (z.scal_bc & ((1 << q) | (1 << (4 + q)))) ? 1.0 : 0.0;
      CState<NS> Bs = bfa_c<NS>(m, p, st, t, f);
      double Dv[BB];
      if (z.kind == JG_BC_SYMMETRY || z.kind == JG_BC_NEUMANN) {
        if (SST) Bs.k = Bs.sc[0];
        const bool op = (z.kind == JG_BC_SYMMETRY) && only_p;
        cflux<NS, FK>(F, Bs, Bs, area, nV, op, hz_b, fob);
        for (int i = 0; i < B; i++) rhs[i] -= F[i];
        if (implicit) {
          if (z.kind == JG_BC_NEUMANN || p.symm_bc == JG_SYMM_NEW_NUMERIC) {
            double Apl[BB], Ami[BB];
            cmatrices<NS, FK>(Apl, Ami, Bs, Bs, area, nV, false, hz_b, fob);
            for (int e = 0; e < BB; e++)
              sD[e * bd + tid] += (p.symm_bc == JG_SYMM_NEW_NUMERIC) ? Apl[e] + Ami[e] : Apl[e];
          } else {
            cmatrices<NS, FK>(Dv, nullptr, Bs, Bs, area, nV, only_p, hz_b, fob);
            for (int e = 0; e < BB; e++) sD[e * bd + tid] += Dv[e];
          }
        }
        if (z.kind == JG_BC_SYMMETRY) {
          const double* g = &st.gu[9 * c];
          double tmp = 2.0 / 3.0 * ((st.mul_fa[f] + st.mut_fa[f]) * (g[0] + g[4] + g[8]) + Bs.rho * Bs.k);
          for (int i = 0; i < 3; i++) rhs[1 + i] -= area * tmp * nV[i];
        } else {
          VSideC<NS> vb = vbfa_c<NS>(st, p, f, c);
          for (int q = 0; q < NS; q++) vb.sc[q] = Bs.sc[q];
          vb.k = Bs.k;
          double sV[3];
          for (int i = 0; i < 3; i++) sV[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
          double smag = fabs(dot3(sV, nV));
          VFC<NS> vf;
          visc_flux_c<NS>(F, vf, vb, vb, st.mul_fa[f], st.mut_fa[f], st.lam_fa[f], p.PrTurb, Bs.k, vb.u, dfa, one,
                          area, nV, smag, nV, 1.0);
          for (int i = 0; i < B; i++) rhs[i] -= F[i];
          if (implicit) {
            for (int e = 0; e < BB; e++) Dv[e] = 0.0;
            visc_jac_c_add<NS>(Dv, 1.0, 0, vf, vb, vb.u, p.R, area);
            for (int e = B; e < BB; e++) sD[e * bd + tid] += Dv[e];
          }
        }
      } else if (z.kind == JG_BC_WALL) {
        // the wall keeps the face kinetic energy at 0 (JoeWithModels.cpp:5448-5452)
        cflux<NS, FK>(F, Bs, Bs, area, nV, only_p, hz_b, fob);
        for (int i = 0; i < B; i++) rhs[i] -= F[i];
        if (implicit) {
          if (p.symm_bc == JG_SYMM_NEW_NUMERIC) {
            double Apl[BB], Ami[BB];
            cmatrices<NS, FK>(Apl, Ami, Bs, Bs, area, nV, false, hz_b, fob);
            for (int e = 0; e < BB; e++) sD[e * bd + tid] += Apl[e] + Ami[e];
          } else {
            cmatrices<NS, FK>(Dv, nullptr, Bs, Bs, area, nV, only_p, hz_b, fob);
            for (int e = 0; e < BB; e++) sD[e * bd + tid] += Dv[e];
          }
        }
        VSideC<NS> v0 = vcell_c<NS>(m, st, t, p, c, SST);
        VSideC<NS> vb = vbfa_c<NS>(st, p, f, c);
        for (int q = 0; q < NS; q++) {
          vb.sc[q] = Bs.sc[q];
          vb.gs[q] = v0.gs[q];
        }
        double sV[3];
        for (int i = 0; i < 3; i++) sV[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
        double smag = fabs(dot3(sV, nV));
        VFC<NS> vf;
        visc_flux_c<NS>(F, vf, v0, vb, st.mul_fa[f], 0.0, st.lam_fa[f], p.PrTurb, 0.0, vb.u, dfa, dterm, area, nV,
                        smag, nV, 1.0);
        for (int i = 0; i < B; i++) rhs[i] -= F[i];
        if (implicit) {
          for (int e = 0; e < BB; e++) Dv[e] = 0.0;
          visc_jac_c_add<NS>(Dv, 1.0, 0, vf, v0, vb.u, p.R, area);
          for (int e = B; e < BB; e++) sD[e * bd + tid] += Dv[e];
        }
      } else {
        // CBC, CBC_SUBSONIC_INLET/OUTLET, FARFIELD (JoeWithModels.cpp:5624-5788)
        CState<NS> L = recon_c<NS>(m, p, st, t, c, f, SST);
        if (SST) Bs.k = Bs.sc[0];
        cflux<NS, FK>(F, L, Bs, area, nV, false, hz_b, fob);
        for (int i = 0; i < B; i++) rhs[i] -= F[i];
        if (implicit) {
          CState<NS> L0 = cell_c<NS>(m, p, st, t, c, SST);
          cmatrices<NS, FK>(Dv, nullptr, L0, Bs, area, nV, false, hz_b, fob);
          for (int e = 0; e < BB; e++) sD[e * bd + tid] += Dv[e];
        }
        VSideC<NS> v0 = vcell_c<NS>(m, st, t, p, c, SST);
        // the outer state carries the reconstructed face scalars, as the reference passes them
        VSideC<NS> vb = vbfa_c<NS>(st, p, f, c);
        for (int q = 0; q < NS; q++) {
          vb.sc[q] = L.sc[q];
          vb.gs[q] = v0.gs[q];
        }
        vb.k = Bs.k;
        double sV[3];
        for (int i = 0; i < 3; i++) sV[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
        double smag = sqrt(dot3(sV, sV));
        for (int i = 0; i < 3; i++) sV[i] /= smag;
        double alpha = dot3(nV, sV);
        VFC<NS> vf;
        visc_flux_c<NS>(F, vf, v0, vb, st.mul_fa[f], st.mut_fa[f], st.lam_fa[f], p.PrTurb, Bs.k, vb.u, dfa, dterm,
                        area, nV, smag, sV, alpha);
        for (int i = 0; i < B; i++) rhs[i] -= F[i];
        if (implicit) {
          for (int e = 0; e < BB; e++) Dv[e] = 0.0;
          visc_jac_c_add<NS>(Dv, 1.0, 0, vf, v0, vb.u, p.R, area);
          for (int e = B; e < BB; e++) sD[e * bd + tid] += Dv[e];
        }
      }
    }
  }
  gravity_rhs(p, m, st, c, rhs);  // sourceHookCoupled
  // model sources: sourceHookRansTurbCoupled (TurbModel_SA.h:359-434; TurbModel_KOMSST.h:306-340)
  double dsrc[NS];
  {
    const double rho = st.q[5 * c], vol = m.vol[c];
    if constexpr (!SST) {
      double mue = face_avg_c(m, st.mul_fa, c);
      double Om = fmax(t.vortMag[c], 1.e-8);
      double Strainrate = fmax(t.strMag[c], 1.e-8);
      double d = t.wd[c];
      double nu = t.phi[c];
      double chi = nu * rho / mue;
      double chi_3 = pow(chi, 3.0);
      double inv_K2d2 = 1.0 / (SA_K2 * d * d);
      double fv1 = chi_3 / (chi_3 + SA_CV1_3);
      double fv2 = 1.0 - chi / (1.0 + chi * fv1);
      double S = fmax(Om + fmin(0.0, Strainrate - Om) * 0.0, 0.0);
      double Shat = S + nu * fv2 * inv_K2d2;
      double inv_Shat = 1.0 / fmax(Shat, 1.0e-8);
      double r = fmin(nu * inv_Shat * inv_K2d2, 10.0);
      double g = r + SA_CW2 * (pow(r, 6.0) - r);
      double g_6 = pow(g, 6.0);
      double fw = g * pow((1.0 + SA_CW3_6) / (g_6 + SA_CW3_6), 1.0 / 6.0);
      double H1 = SA_CB1 * Shat * nu;
      double H2 = -SA_CW1 * fw * nu * nu / sq(d);
      double H3 = SA_CB2 / SA_SIGMA * dot3(&t.grad_phi[3 * c], &t.grad_phi[3 * c]);
      rhs[5] += rho * vol * (H1 + H2 + H3);
      double d_H2 = -2.0 * SA_CW1 * fw * nu / sq(d);
      dsrc[0] = (0.0 + d_H2) * vol;
    } else {
      double k = t.phi[c], om = t.phi[N + c];
      double F1 = t.F1[c];
      double alfa_1 = SST_B1 / SST_BS - SST_SO1 * sq(0.41) / sqrt(SST_BS);
      double alfa_2 = SST_B2 / SST_BS - SST_SO2 * sq(0.41) / sqrt(SST_BS);
      double alfa = F1 * alfa_1 + (1.0 - F1) * alfa_2;
      double beta = F1 * SST_B1 + (1.0 - F1) * SST_B2;
      double zeta = fmin(1.0 / om, SST_A1 / (t.vortMag[c] * t.F2[c]));
      double mut = fmin(fmax(rho * k * zeta, 1.0e-8), 1.0e5);
      double str = t.strMag[c], div = t.diverg[c];
      double Pk = fmax(mut * str * str - 2. / 3. * rho * k * div, 0.0);
      Pk = fmin(Pk, 20.0 * SST_BS * rho * k * om);
      rhs[5] += (Pk - SST_BS * rho * om * k) * vol;
      zeta = fmax(om, t.vortMag[c] * t.F2[c] / SST_A1);
      Pk = fmax(str * str - 2. / 3. * zeta * div, 0.0);
      rhs[6] += (alfa * rho * Pk + (1.0 - F1) * t.crossDiff[c] - beta * rho * om * om) * vol;
      dsrc[0] = -SST_BS * om * vol;
      dsrc[1] = -2.0 * beta * om * vol;
    }
  }
  for (int i = 0; i < B; i++) st.rhs[(size_t)B * c + i] = rhs[i];
  if (implicit) {
    double Dm[BB];
    for (int e = 0; e < BB; e++) Dm[e] = sD[e * bd + tid];
    gravity_diag<B>(p, m, c, Dm);
    for (int q = 0; q < NS; q++) Dm[(B + 1) * (5 + q)] -= dsrc[q];
    if (for_step) {
      double tmp = m.vol[c] / st.local_dt[c];
      for (int i = 0; i < B; i++) Dm[(B + 1) * i] += tmp;
      for (int i = 0; i < B; i++) st.b[(size_t)B * c + i] = p.under_relax * rhs[i];
    }
    BT* Dg = (BT*)st.D;
    for (int e = 0; e < BB; e++) Dg[(size_t)e * m.ncv + c] = (BT)Dm[e];
    if (for_step) {
      double Di[BB];
      block_inverse_n<B>(Dm, Di);
      BT* Dig = (BT*)st.Dinv;
      for (int e = 0; e < BB; e++) Dig[(size_t)e * m.ncv + c] = (BT)Di[e];
    }
  }
}

// ---------------------------------------------------------------------------
// block relaxation of the B x B system: one warp per block row of a 32-cell
// slice (B*32 threads), as the 5x5 sweeps
// ---------------------------------------------------------------------------
template <typename BT, int B>
__global__ void __launch_bounds__(B * 32) k_jacobi_c(Mesh m, State st, const BT* __restrict__ xin,
                                                      BT* __restrict__ xout, int first) {
  __shared__ BT sacc[B][SLICE];
  const int row = threadIdx.x / SLICE, lane = threadIdx.x % SLICE;
  const int slice = blockIdx.x;
  const int c = slice * SLICE + lane;
  const bool active = c < m.ncv && st.case_active[m.case_of[c]];
  const int N = m.ncv;
  BT acc = active ? (BT)st.b[(size_t)B * c + row] : (BT)0;
  if (!first && active) {
    const BT* O = (const BT*)st.O;
    for (int j = m.ell_off[slice]; j < m.ell_off[slice + 1]; j++) {
      int nb = m.ell_nb[(size_t)j * SLICE + lane];
      const BT* Ob = O + ((size_t)j * B * B + B * row) * SLICE + lane;
      BT s = 0;
      for (int k = 0; k < B; k++) s += Ob[k * SLICE] * xin[(size_t)k * N + nb];
      acc -= s;
    }
  }
  sacc[row][lane] = acc;
  __syncthreads();
  if (active) {
    const BT* Di = (const BT*)st.Dinv;
    BT s = 0;
    for (int k = 0; k < B; k++) s += Di[(size_t)(B * row + k) * N + c] * sacc[k][lane];
    xout[(size_t)row * N + c] = s;
  }
}

template <typename BT, int B>
__global__ void __launch_bounds__(B * 32) k_gs_c(Mesh m, State st, BT* __restrict__ x, int color,
                                                 const int* __restrict__ slices) {
  __shared__ BT sacc[B][SLICE];
  const int row = threadIdx.x / SLICE, lane = threadIdx.x % SLICE;
  const int slice = slices ? slices[blockIdx.x] : blockIdx.x;  // slices: those holding this colour
  const int c = slice * SLICE + lane;
  const bool active = c < m.ncv && m.color[c] == color && st.case_active[m.case_of[c]];
  const int N = m.ncv;
  BT acc = 0;
  if (active) {
    acc = (BT)st.b[(size_t)B * c + row];
    const BT* O = (const BT*)st.O;
    for (int j = m.ell_off[slice]; j < m.ell_off[slice + 1]; j++) {
      int nb = m.ell_nb[(size_t)j * SLICE + lane];
      const BT* Ob = O + ((size_t)j * B * B + B * row) * SLICE + lane;
      BT s = 0;
      for (int k = 0; k < B; k++) s += Ob[k * SLICE] * x[(size_t)k * N + nb];
      acc -= s;
    }
  }
  sacc[row][lane] = acc;
  __syncthreads();
  if (active) {
    const BT* Di = (const BT*)st.Dinv;
    BT s = 0;
    for (int k = 0; k < B; k++) s += Di[(size_t)(B * row + k) * N + c] * sacc[k][lane];
    x[(size_t)row * N + c] = s;
  }
}

// runBackwardEulerCoupled update (JoeWithModels.cpp:4497-4517): Q += dq, then
// phi_s = clip((phi_s * (rho_new - dq0) + dq_{5+s}) / rho_new); dq kept in st.dq
template <typename BT, int NS>
__global__ void k_update_c(Mesh m, State st, Turb t, const BT* __restrict__ x, double lo0, double hi0, double lo1,
                           double hi1) {
  constexpr int B = 5 + NS;
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  if (!st.case_active[m.case_of[c]]) return;  // a frozen (retired) case of a batch keeps its state
  const int N = m.ncv;
  double dq[B];
  for (int i = 0; i < B; i++) {
    dq[i] = (double)x[(size_t)i * N + c];
    st.dq[(size_t)B * c + i] = dq[i];
  }
  double rho = st.q[5 * c] + dq[0];
  st.q[5 * c] = rho;
  for (int i = 1; i < 5; i++) st.q[5 * c + i] += dq[i];
  for (int q = 0; q < NS; q++) {
    double& ph = t.phi[(size_t)q * N + c];
    ph = fmin(fmax((ph * (rho - dq[0]) + dq[5 + q]) / rho, q ? lo1 : lo0), q ? hi1 : hi0);
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
constexpr int TBC = 128;

void launch_wall_distance(const Mesh& m, Turb& t, int c0, int c1, int w0, int w1, cudaStream_t s) {
  if (c1 > c0) k_wall_dist<<<grid_for(c1 - c0, 256), 256, 0, s>>>(m, t, c0, c1, w0, w1);
}
void launch_scalar_bc(const Mesh& m, const Params& p, State& st, Turb& t, cudaStream_t s) {
  if (m.nfa_b) k_scalar_bc<<<grid_for(m.nfa_b, TBC), TBC, 0, s>>>(m, p, st, t);
}
void launch_grad_coupled(const Mesh& m, const Params& p, State& st, cudaStream_t s);  // jg_kernels.cu
void launch_turb_props(const Mesh& m, const Params& p, State& st, Turb& t, cudaStream_t s) {
  launch_grad_coupled(m, p, st, s);
  k_grad_phi<<<grid_for(m.ncv, TBC), TBC, 0, s>>>(m, p, t);
  k_turb_cell<<<grid_for(m.ncv, TBC), TBC, 0, s>>>(m, st, t);
  k_turb_face<<<grid_for(m.nfa, TBC), TBC, 0, s>>>(m, st, t);
}
template <typename BT>
static void launch_flux_c_t(const Mesh& m, const Params& p, State& st, Turb& t, int implicit, int for_step,
                            cudaStream_t s) {
  // 64-cell blocks keep the 7x7 accumulators (49 x 64 doubles) within 48 KB
  const bool ausm = p.flux == JG_FLUX_AUSMDV || p.flux == JG_FLUX_HAENEL;
  if (t.model == JG_TURB_SST) {
    if (ausm)
      k_flux_c<BT, JG_TURB_SST, 1><<<grid_for(m.ncv, 64), 64, 49 * 64 * sizeof(double), s>>>(m, p, st, t, implicit,
                                                                                             for_step);
    else
      k_flux_c<BT, JG_TURB_SST, 0><<<grid_for(m.ncv, 64), 64, 49 * 64 * sizeof(double), s>>>(m, p, st, t, implicit,
                                                                                             for_step);
  } else {
    if (ausm)
      k_flux_c<BT, JG_TURB_SA, 1><<<grid_for(m.ncv, TBC), TBC, 36 * TBC * sizeof(double), s>>>(m, p, st, t,
                                                                                              implicit, for_step);
    else
      k_flux_c<BT, JG_TURB_SA, 0><<<grid_for(m.ncv, TBC), TBC, 36 * TBC * sizeof(double), s>>>(m, p, st, t,
                                                                                              implicit, for_step);
  }
}
void launch_flux6(const Mesh& m, const Params& p, State& st, Turb& t, int implicit, int for_step, cudaStream_t s) {
  launch_face_sensors(m, p, st, s);  // AUSMDV's shock sensor
  if (p.fp32) launch_flux_c_t<float>(m, p, st, t, implicit, for_step, s);
  else launch_flux_c_t<double>(m, p, st, t, implicit, for_step, s);
}
template <typename BT, int B>
static void relax_c(const Mesh& m, State& st, int sgs, int sweeps, cudaStream_t s) {
  if (sgs) {
    cudaMemsetAsync(st.x0, 0, B * (size_t)m.ncv * sizeof(BT), s);
    for (int it = 0; it < sweeps; it++)
      for (int q = 0; q < m.ncolors; q++) {
        int col = (it % 2 == 0) ? q : m.ncolors - 1 - q;
        const bool lists = m.color_slices != nullptr;
        const int* sl = lists ? m.color_slices + m.color_slice_off[col] : nullptr;
        const int g = lists ? m.color_slice_off[col + 1] - m.color_slice_off[col] : m.nslices;
        if (g > 0) k_gs_c<BT, B><<<g, B * SLICE, 0, s>>>(m, st, (BT*)st.x0, col, sl);
      }
  } else {
    for (int it = 0; it < sweeps; it++) {
      void* xin = (it % 2 == 0) ? st.x1 : st.x0;
      void* xout = (it % 2 == 0) ? st.x0 : st.x1;
      k_jacobi_c<BT, B><<<m.nslices, B * SLICE, 0, s>>>(m, st, (const BT*)xin, (BT*)xout, it == 0);
    }
  }
}
void launch_relax6(const Mesh& m, const Params& p, State& st, int sgs, int sweeps, int bs, cudaStream_t s) {
  if (bs == 7) {
    if (p.fp32) relax_c<float, 7>(m, st, sgs, sweeps, s);
    else relax_c<double, 7>(m, st, sgs, sweeps, s);
  } else {
    if (p.fp32) relax_c<float, 6>(m, st, sgs, sweeps, s);
    else relax_c<double, 6>(m, st, sgs, sweeps, s);
  }
}
void launch_update6(const Mesh& m, const Params& p, State& st, Turb& t, const void* x, cudaStream_t s) {
  // ScalarTranspEq bounds: SA nuSA 1e-10..1 (TurbModel_SA.h:35-36); SST kine 1e-10..1e10,
  // omega 1e-4..1e15 (TurbModel_KOMSST.h:42-51)
  int g = grid_for(m.ncv, TBC);
  if (t.model == JG_TURB_SST) {
    if (p.fp32) k_update_c<float, 2><<<g, TBC, 0, s>>>(m, st, t, (const float*)x, 1.0e-10, 1.0e10, 1.0e-4, 1.0e15);
    else k_update_c<double, 2><<<g, TBC, 0, s>>>(m, st, t, (const double*)x, 1.0e-10, 1.0e10, 1.0e-4, 1.0e15);
  } else {
    if (p.fp32) k_update_c<float, 1><<<g, TBC, 0, s>>>(m, st, t, (const float*)x, 1.0e-10, 1.0, 0.0, 0.0);
    else k_update_c<double, 1><<<g, TBC, 0, s>>>(m, st, t, (const double*)x, 1.0e-10, 1.0, 0.0, 0.0);
  }
}

}  // namespace jg
