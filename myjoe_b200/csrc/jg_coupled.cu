// jg_coupled.cu -- the coupled (5+1)x(5+1) path with the Spalart-Allmaras
// model: runBackwardEulerCoupled / calcRhsCoupled / calcFluxCoupled
// (src/joe/JoeWithModels.cpp:4326-5826) with RansTurbSA
// (src/joe/turbModels/TurbModel_SA.h).
//
// Same structure as the 5x5 path: one thread per cell walks its faces in the
// reference's faocv order, evaluates every face in the face's own orientation
// (bit-identical on both sides), owns its residual, its diagonal block and
// its row of off-diagonal blocks (sliced ELL, 36 components).  Row/column 5
// of every block is rho*nuSA.  Gradients, strain/vorticity, turbulent
// viscosity and scalar diffusivity are computed once after each update from
// the new state (the reference recomputes them from the same state inside the
// next calcFluxCoupled; the values are identical).
#include <cuda_runtime.h>
#include <math.h>

#include "jg_flux.cuh"
#include "jg_internal.h"

namespace jg {

constexpr int B6 = 6, B6SQ = 36;
// RansTurbSA defaults (TurbModel_SA.h:21-28) and ScalarTranspEq bounds (:31-36)
constexpr double SA_CV1_3 = 357.911, SA_CW1 = 3.239067817, SA_CW2 = 0.3, SA_CW3_6 = 64.0;
constexpr double SA_SIGMA = 0.6666666, SA_CB1 = 0.1355, SA_CB2 = 0.622, SA_K2 = 0.1681;
constexpr double SA_LOWER = 1.0e-10, SA_UPPER = 1.0;

__device__ __forceinline__ void unit_normal6(const Mesh& m, int f, double nV[3], double& area) {
  double n[3] = {m.fa_n[3 * f], m.fa_n[3 * f + 1], m.fa_n[3 * f + 2]};
  area = sqrt(dot3(n, n));
  for (int i = 0; i < 3; i++) nV[i] = n[i] / area;
}
__device__ __forceinline__ double sq(double x) { return x * x; }  // pow(x, 2.0) of the reference, exactly

// ---------------------------------------------------------------------------
// calcWallDistance (UgpWithCvCompFlow.h:1395-1535): nearest WALL face centroid
// (first in zone order on ties), then the normal distance when the cell lies
// over that face.  Wall-face centroids are staged through shared memory.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_wall_dist(Mesh m, Turb t) {
  __shared__ double sx[256][3];
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double x[3] = {0.0, 0.0, 0.0};
  if (c < m.ncv)
    for (int i = 0; i < 3; i++) x[i] = m.x_cv[3 * c + i];
  double minD = 1.0e20;
  int save = 0;
  for (int k0 = 0; k0 < t.nwall; k0 += 256) {
    int k = k0 + threadIdx.x;
    if (k < t.nwall)
      for (int i = 0; i < 3; i++) sx[threadIdx.x][i] = m.x_fa[3 * t.wall_f[k] + i];
    __syncthreads();
    int n = min(256, t.nwall - k0);
    for (int j = 0; j < n; j++) {
      double d = sqrt(sq(x[0] - sx[j][0]) + sq(x[1] - sx[j][1]) + sq(x[2] - sx[j][2]));
      if (d < minD) {
        minD = d;
        save = k0 + j;
      }
    }
    __syncthreads();
  }
  if (c >= m.ncv || t.nwall == 0) return;
  int f = t.wall_f[save];
  double n[3], sh[3], nmag;
  unit_normal6(m, f, n, nmag);
  for (int i = 0; i < 3; i++) sh[i] = m.x_fa[3 * f + i] - x[i];
  double sMag2 = dot3(sh, sh);
  double dNorm2 = dot3(sh, n) * dot3(sh, n);
  double dTang2 = sMag2 - dNorm2;
  double specRadius2 = 0.5 * nmag;
  t.wd[c] = (dTang2 > specRadius2) ? minD : fabs(dot3(sh, n));
}

// setScalarBC (Scalars.cpp:289-360): Dirichlet value on inflow, else zero flux
__global__ void k_scalar_bc(Mesh m, State st, Turb t) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nfa_b) return;
  const DevZone z = m.zones[m.bzone[f]];
  int c0 = m.cvofa[2 * f];
  const double* vb = &st.bfa[8 * f + 1];
  if (z.scal_bc & 1) {
    double un = vb[0] * m.fa_n[3 * f] + vb[1] * m.fa_n[3 * f + 1] + vb[2] * m.fa_n[3 * f + 2];
    t.phi_bfa[f] = (un > 1.0e-8) ? t.phi[c0] : z.v[6];
  } else {
    t.phi_bfa[f] = t.phi[c0];
  }
}

// calcCvScalarGrad + limitCvScalarGradBJ (UgpWithCv.h:881-938, 1009-1056) of nuSA
__global__ void k_grad_phi(Mesh m, Params p, Turb t) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  const double pc = t.phi[c];
  double g[3];
  int k0 = m.nb_i[c], k1 = m.nb_i[c + 1];
  for (int j = 0; j < 3; j++) g[j] = m.lsq[3 * k0 + j] * pc;
  double pmax = pc, pmin = pc;
  for (int k = k0 + 1; k < k1; k++) {
    double pn = t.phi[m.nb_v[k]];
    for (int j = 0; j < 3; j++) g[j] += m.lsq[3 * k + j] * pn;
    pmax = fmax(pmax, pn);
    pmin = fmin(pmin, pn);
  }
  for (int k = m.bf_i[c]; k < m.bf_i[c + 1]; k++) {
    int f = m.bf_v[k];
    for (int j = 0; j < 3; j++) g[j] += m.blsq[3 * f + j] * t.phi_bfa[f];
  }
  if (p.limiter) {
    double alfa = 1.0;
    if ((pmax - pmin) > 1.0e-12) {
      double e2 = sq(fmax(p.eps * fabs(pc), 1.0e-8));
      for (int k = m.slot_i[c]; k < m.slot_i[c + 1]; k++) {
        Slot s = m.slots[k];
        if (s.nb < 0) continue;
        double r0[3];
        for (int j = 0; j < 3; j++) r0[j] = m.x_fa[3 * s.f + j] - m.x_cv[3 * c + j];
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
  for (int j = 0; j < 3; j++) t.grad_phi[3 * c + j] = g[j];
}

// calcStrainRate + calcVorticity (UgpWithCvCompFlow.h:1348-1393) from the limited grad_u
__global__ void k_sa_cell(Mesh m, State st, Turb t) {
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
}

// InterpolateAtCellCenterFromFaceValues (UgpWithCvCompFlow.h:1538-1552)
__device__ __forceinline__ double face_avg6(const Mesh& m, const double* phi, int c) {
  double v = 0.0;
  int k0 = m.slot_i[c], k1 = m.slot_i[c + 1];
  for (int k = k0; k < k1; k++) v += phi[m.slots[k].f];
  return v / (double)(k1 - k0);
}

// RansTurbSA::calcRansTurbViscMuet (TurbModel_SA.h:74-128) and
// diffusivityHookScalarRansTurb (:130-173), one thread per face
__global__ void k_sa_face(Mesh m, State st, Turb t) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nfa) return;
  const double invSigma = 1.0 / SA_SIGMA;
  const double mul = st.mul_fa[f];
  if (f >= m.nfa_b) {
    int c0 = m.cvofa[2 * f], c1 = m.cvofa[2 * f + 1];
    double d0[3], d1[3];
    for (int i = 0; i < 3; i++) {
      d0[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c0 + i];
      d1[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c1 + i];
    }
    double w0 = sqrt(dot3(d0, d0)), w1 = sqrt(dot3(d1, d1));
    double rho_fa = (w1 * st.q[5 * c0] + w0 * st.q[5 * c1]) / (w0 + w1);
    double nu_fa = (w1 * t.phi[c0] + w0 * t.phi[c1]) / (w0 + w1);
    double muSA = rho_fa * nu_fa;
    double chi_3 = pow(muSA / mul, 3.0);
    double fv1 = chi_3 / (chi_3 + SA_CV1_3);
    st.mut_fa[f] = fmax(muSA * fv1, 0.0);
    t.diff[f] = invSigma * (mul + rho_fa * nu_fa);
  } else {
    const DevZone z = m.zones[m.bzone[f]];
    if (z.kind == JG_BC_WALL) {
      st.mut_fa[f] = 0.0;
      t.diff[f] = invSigma * mul;
    } else {
      int c0 = m.cvofa[2 * f];
      double muSA = st.q[5 * c0] * t.phi[c0];
      double mul0 = face_avg6(m, st.mul_fa, c0);
      double chi_3 = pow(muSA / mul0, 3.0);
      double fv1 = chi_3 / (chi_3 + SA_CV1_3);
      st.mut_fa[f] = fmax(muSA * fv1, 0.0);
      t.diff[f] = invSigma * (mul + st.bfa[8 * f] * t.phi_bfa[f]);
    }
  }
}

// ---------------------------------------------------------------------------
// coupled HLLC flux and matrices (UgpWithCvCompFlow.cpp:1808-2289, nScal = 1,
// no kinetic energy, dp/dscal = 0, ConvTerm = 1)
// ---------------------------------------------------------------------------
struct CState {
  double rho, u[3], p, T, h, gam, sc;
};

__device__ void flux_hllc6(double F[B6], const CState& L, const CState& R, double area, const double* nV,
                           bool only_p) {
  if (only_p) {
    F[0] = 0.0;
    for (int i = 1; i < 4; i++) F[i] = L.p * nV[i - 1];
    F[4] = 0.0;
    F[5] = 0.0;
  } else {
    double unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u), cL = sqrt(L.gam * L.p / L.rho);
    double rhoeL = (L.h + 0.5 * uLuL + 0.0) * L.rho - L.p;
    double unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u), cR = sqrt(R.gam * R.p / R.rho);
    double rhoeR = (R.h + 0.5 * uRuR + 0.0) * R.rho - R.p;
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
    if (sM >= 0.0) {
      if (sL > 0.0) {
        F[0] = L.rho * unL;
        for (int i = 0; i < 3; i++) F[1 + i] = L.rho * L.u[i] * unL + L.p * nV[i];
        F[4] = (rhoeL + L.p) * unL;
      } else {
        double inv = 1.0 / (sL - sM), d = sL - unL;
        double rS = L.rho * d * inv;
        F[0] = rS * sM;
        for (int i = 0; i < 3; i++) F[1 + i] = ((L.rho * L.u[i] * d + (pS - L.p) * nV[i]) * inv) * sM + pS * nV[i];
        F[4] = ((d * rhoeL - L.p * unL + pS * sM) * inv + pS) * sM;
      }
      F[5] = 1.0 * F[0] * L.sc;
    } else {
      if (sR >= 0.0) {
        double inv = 1.0 / (sR - sM), d = sR - unR;
        double rS = R.rho * d * inv;
        F[0] = rS * sM;
        for (int i = 0; i < 3; i++) F[1 + i] = ((R.rho * R.u[i] * d + (pS - R.p) * nV[i]) * inv) * sM + pS * nV[i];
        F[4] = ((d * rhoeR - R.p * unR + pS * sM) * inv + pS) * sM;
      } else {
        F[0] = R.rho * unR;
        for (int i = 0; i < 3; i++) F[1 + i] = R.rho * R.u[i] * unR + R.p * nV[i];
        F[4] = (rhoeR + R.p) * unR;
      }
      F[5] = 1.0 * F[0] * R.sc;
    }
  }
  for (int i = 0; i < B6; i++) F[i] *= area;
}

// calcJacobianCoupled_HLLC (UgpWithCvCompFlow.cpp:2180-2244); nA = n * area
__device__ void jac6(double* A, const double* vel, double pp, double rrho, double hh, double sc, const double* nA,
                     double gamma) {
  double kapm1 = gamma - 1.0;
  double nVel[3] = {vel[0] * nA[0], vel[1] * nA[1], vel[2] * nA[2]};
  double U_k = nVel[0] + nVel[1] + nVel[2];
  double vSquHlf = 0.5 * dot3(vel, vel);
  A[0] = 0.0; A[1] = nA[0]; A[2] = nA[1]; A[3] = nA[2]; A[4] = 0.0; A[5] = 0.0;
  for (int r = 0; r < 3; r++) {
    double* a = A + B6 * (1 + r);
    a[0] = -vel[r] * U_k + nA[r] * (kapm1 * vSquHlf + gamma * pp / rrho - kapm1 * hh);
    for (int c = 0; c < 3; c++)
      a[1 + c] = (r == c) ? (2.0 - gamma) * nVel[r] + U_k : vel[r] * nA[c] - kapm1 * vel[c] * nA[r];
    a[4] = kapm1 * nA[r];
    a[5] = 0.0 * nA[r];
  }
  double* a4 = A + 4 * B6;
  a4[0] = U_k * ((gamma - 2.0) * vSquHlf - gamma * (hh - pp / rrho));
  for (int c = 0; c < 3; c++) a4[1 + c] = (hh + vSquHlf) * nA[c] - kapm1 * vel[c] * U_k;
  a4[4] = gamma * U_k;
  a4[5] = 0.0 * U_k;
  double* a5 = A + 5 * B6;
  a5[0] = 0.0;
  for (int c = 0; c < 3; c++) a5[1 + c] = sc * nA[c];
  a5[4] = 0.0;
  a5[5] = rrho * U_k;
}

// calcdSMdU_HLLC (:2247-2266)
__device__ void dsmdu6(double* d, const double* vel, double pp, double rrho, double hh, const double* nV, double gamma,
                       double SM, double S, double invertrho, double Factor) {
  double kapm1 = gamma - 1.0;
  double U_k = vel[0] * nV[0] + vel[1] * nV[1] + vel[2] * nV[2];
  double vSquHlf = 0.5 * dot3(vel, vel);
  d[0] = Factor * invertrho * (-U_k * U_k + kapm1 * vSquHlf + gamma * pp / rrho - kapm1 * hh + SM * S);
  for (int i = 0; i < 3; i++) d[1 + i] = Factor * invertrho * ((2 * U_k - S - SM) * nV[i] - kapm1 * vel[i]);
  d[4] = Factor * invertrho * kapm1;
  d[5] = Factor * invertrho * 0.0;
}

// calcSubSonicJacobianCoupled_HLLC (:2270-2289)
__device__ void subsonic6(double* A, const double* d, double rhoS, const double* rhouS, double rhoeS, double sc, double pS,
                          double Om, double sM, double rhoSmq, const double* nV, double area) {
  double OmSM = Om * sM, OmSMp1 = OmSM + 1.0;
  double rr[B6] = {rhoS, rhouS[0] + rhoSmq * nV[0], rhouS[1] + rhoSmq * nV[1], rhouS[2] + rhoSmq * nV[2],
                   rhoeS + pS + rhoSmq * sM, rhoS * sc};
  for (int i = 0; i < B6; i++)
    for (int r = 0; r < B6; r++) A[B6 * r + i] = -OmSM * A[B6 * r + i] + area * OmSMp1 * d[i] * rr[r];
}

// calcEulerFluxMatricesCoupled_HLLC (:1934-2176), then dU/dQ of the scalar column
__device__ void matrices_hllc6(double* AL, double* AR, const CState& L, const CState& R, double area,
                               const double* nV, bool only_p) {
  if (!only_p) {
    double dd[B6];
    double unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u), cL = sqrt(L.gam * L.p / L.rho);
    double hL = L.h + 0.0, rhoeL = (hL + 0.5 * uLuL) * L.rho - L.p;
    double unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u), cR = sqrt(R.gam * R.p / R.rho);
    double hR = R.h + 0.0, rhoeR = (hR + 0.5 * uRuR) * R.rho - R.p;
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
        if (AL) jac6(AL, L.u, L.p, L.rho, hL, L.sc, nA, L.gam);
        if (AR)
          for (int e = 0; e < B6SQ; e++) AR[e] = 0.0;
      } else {
        double Om = 1.0 / (sL - sM), d = sL - unL;
        double rhoS = L.rho * d * Om, rhouS[3];
        for (int i = 0; i < 3; i++) rhouS[i] = (L.rho * L.u[i] * d + (pS - L.p) * nV[i]) * Om;
        double rhoeS = (d * rhoeL - L.p * unL + pS * sM) * Om;
        if (AL) {
          dsmdu6(dd, L.u, L.p, L.rho, hL, nV, L.gam, sM, sL, invrhotld, 1.0);
          jac6(AL, L.u, L.p, L.rho, hL, L.sc, nA, L.gam);
          subsonic6(AL, dd, rhoS, rhouS, rhoeS, L.sc, pS, Om, sM, R.rho * (sR - unR), nV, area);
          for (int i = 0; i < 5; i++) AL[7 * i] += area * Om * sM * sL;
          AL[30] += area * Om * sM * sL * L.sc;
          AL[35] += area * Om * sM * sL * L.rho;
        }
        if (AR) {
          dsmdu6(dd, R.u, R.p, R.rho, hR, nV, R.gam, sM, sR, invrhotld, -1.0);
          for (int e = 0; e < B6SQ; e++) AR[e] = 0.0;
          subsonic6(AR, dd, rhoS, rhouS, rhoeS, L.sc, pS, Om, sM, L.rho * (sL - unL), nV, area);
        }
      }
    } else {
      if (sR >= 0.0) {
        double Om = 1.0 / (sR - sM), d = sR - unR;
        double rhoS = R.rho * d * Om, rhouS[3];
        for (int i = 0; i < 3; i++) rhouS[i] = (R.rho * R.u[i] * d + (pS - R.p) * nV[i]) * Om;
        double rhoeS = (d * rhoeR - R.p * unR + pS * sM) * Om;
        if (AR) {
          dsmdu6(dd, R.u, R.p, R.rho, hR, nV, R.gam, sM, sR, invrhotld, -1.0);
          jac6(AR, R.u, R.p, R.rho, hR, R.sc, nA, R.gam);
          subsonic6(AR, dd, rhoS, rhouS, rhoeS, R.sc, pS, Om, sM, L.rho * (sL - unL), nV, area);
          for (int i = 0; i < 5; i++) AR[7 * i] += area * Om * sM * sR;
          AR[30] += area * Om * sM * sR * R.sc;
          AR[35] += area * Om * sM * sR * R.rho;
        }
        if (AL) {
          dsmdu6(dd, L.u, L.p, L.rho, hL, nV, L.gam, sM, sL, invrhotld, 1.0);
          for (int e = 0; e < B6SQ; e++) AL[e] = 0.0;
          subsonic6(AL, dd, rhoS, rhouS, rhoeS, R.sc, pS, Om, sM, R.rho * (sR - unR), nV, area);
        }
      } else {
        if (AR) jac6(AR, R.u, R.p, R.rho, hR, R.sc, nA, R.gam);
        if (AL)
          for (int e = 0; e < B6SQ; e++) AL[e] = 0.0;
      }
    }
  } else {
    if (AL) {
      double uLuL = dot3(L.u, L.u), hL = L.h + 0.0, g = L.gam;
      for (int j = 0; j < B6; j++) AL[j] = 0.0;
      double dpdrho = 0.5 * (g - 1.0) * uLuL - (g - 1.0) * hL + g * L.p / L.rho;
      for (int r = 0; r < 3; r++) {
        double* a = AL + B6 * (1 + r);
        a[0] = dpdrho * nV[r] * area;
        for (int c = 0; c < 3; c++) a[1 + c] = -(g - 1.0) * L.u[c] * nV[r] * area;
        a[4] = (g - 1.0) * nV[r] * area;
        a[5] = 0.0 * nV[r] * area;
      }
      for (int e = 4 * B6; e < B6SQ; e++) AL[e] = 0.0;
    }
    if (AR)
      for (int e = 0; e < B6SQ; e++) AR[e] = 0.0;
  }
  if (AL)
    for (int j = 0; j < B6; j++) {
      AL[B6 * j] -= L.sc / L.rho * AL[B6 * j + 5];
      AL[B6 * j + 5] /= L.rho;
    }
  if (AR)
    for (int j = 0; j < B6; j++) {
      AR[B6 * j] -= R.sc / R.rho * AR[B6 * j + 5];
      AR[B6 * j + 5] /= R.rho;
    }
}

// ---------------------------------------------------------------------------
// calcViscousFluxCoupled (UgpWithCvCompFlow.cpp:3040-3276), nScal = 1, k = 0
// ---------------------------------------------------------------------------
struct VSide6 {
  double rho, u[3], h, T, gam, sc;
  const double* gu;  // [9]
  const double* gh;  // [3]
  const double* gs;  // [3] scalar gradient (nullptr: zero)
};
struct VF6 {
  double tn[3], keff, muT, aas, dd;
};

__device__ void visc_flux6(double Fv[B6], VF6& vf, const VSide6& a, const VSide6& b, double mul, double mut,
                           double lamOcp, double PrTurb, const double* u_fa, double diff, double diffTerm,
                           double area, const double* nV, double smag, const double* sV, double alpha) {
  double g[3][3];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) g[i][j] = 0.5 * (a.gu[3 * i + j] + b.gu[3 * i + j]);
  double fC[3] = {nV[0] - alpha * sV[0], nV[1] - alpha * sV[1], nV[2] - alpha * sV[2]};
  double muT = mul + mut;
  Fv[0] = 0.0;
  for (int i = 0; i < 3; i++)
    vf.tn[i] = muT * (alpha * (b.u[i] - a.u[i]) / smag + g[i][0] * fC[0] + g[0][i] * nV[0] + g[i][1] * fC[1] +
                      g[1][i] * nV[1] + g[i][2] * fC[2] + g[2][i] * nV[2]);
  double tmp = 2.0 / 3.0 * muT * (g[0][0] + g[1][1] + g[2][2]);
  tmp += 1.0 / 3.0 * (a.rho + b.rho) * 0.0;
  for (int i = 0; i < 3; i++) vf.tn[i] -= tmp * nV[i];
  for (int i = 0; i < 3; i++) Fv[1 + i] = -area * vf.tn[i];
  vf.keff = lamOcp + mut / PrTurb;
  double enth = vf.keff * (alpha * (b.h - a.h) / smag + 0.5 * ((a.gh[0] + b.gh[0]) * fC[0] +
                                                             (a.gh[1] + b.gh[1]) * fC[1] +
                                                             (a.gh[2] + b.gh[2]) * fC[2]));
  double psi = muT * (alpha * (0.0 - 0.0) / smag);
  Fv[4] = -area * (enth + vf.tn[0] * u_fa[0] + vf.tn[1] * u_fa[1] + vf.tn[2] * u_fa[2] + psi);
  double gs0[3] = {0.0, 0.0, 0.0}, gs1[3] = {0.0, 0.0, 0.0};
  if (a.gs)
    for (int i = 0; i < 3; i++) gs0[i] = a.gs[i];
  if (b.gs)
    for (int i = 0; i < 3; i++) gs1[i] = b.gs[i];
  Fv[5] = -area * diffTerm * diff * (alpha * (b.sc - a.sc) / smag + 0.5 * ((gs0[0] + gs1[0]) * fC[0] +
                                                                        (gs0[1] + gs1[1]) * fC[1] +
                                                                        (gs0[2] + gs1[2]) * fC[2]));
  vf.muT = muT;
  vf.aas = area * alpha / smag;
  vf.dd = diffTerm * diff;
}

// acc += sgn * (A0 (side 0) or A1 (side 1)) of calcViscousFluxCoupled, from the state of that side
__device__ void visc_jac6_add(double* acc, double sgn, int side, const VF6& vf, const VSide6& v, const double* u_fa,
                              double R, double area) {
  double sg = side ? -1.0 : 1.0;
  double d11 = sg * vf.muT * vf.aas;
  double d41 = -area * vf.tn[0] * 0.5 + u_fa[0] * d11;
  double d42 = -area * vf.tn[1] * 0.5 + u_fa[1] * d11;
  double d43 = -area * vf.tn[2] * 0.5 + u_fa[2] * d11;
  double d44 = sg * vf.keff * vf.aas;
  double dss = sg * vf.dd * vf.aas;
  double iR = 1.0 / v.rho;
  double q10 = -iR * v.u[0], q20 = -iR * v.u[1], q30 = -iR * v.u[2];
  double q40 = iR * v.gam * (-v.h - 0.0 + R * v.T + 0.5 * dot3(v.u, v.u));
  double q41 = -iR * v.u[0] * v.gam, q42 = -iR * v.u[1] * v.gam, q43 = -iR * v.u[2] * v.gam, q44 = iR * v.gam;
  double q4s = iR * iR * 0.0, qs0 = -iR * v.sc;
  acc[6] += sgn * (d11 * q10);
  acc[7] += sgn * (d11 * iR);
  acc[12] += sgn * (d11 * q20);
  acc[14] += sgn * (d11 * iR);
  acc[18] += sgn * (d11 * q30);
  acc[21] += sgn * (d11 * iR);
  acc[24] += sgn * (d41 * q10 + d42 * q20 + d43 * q30 + d44 * q40);
  acc[25] += sgn * (d41 * iR + d44 * q41);
  acc[26] += sgn * (d42 * iR + d44 * q42);
  acc[27] += sgn * (d43 * iR + d44 * q43);
  acc[28] += sgn * (d44 * q44);
  acc[29] += sgn * (d44 * q4s);
  acc[30] += sgn * (dss * qs0);
  acc[35] += sgn * (dss * iR);
}

// ---------------------------------------------------------------------------
// states
// ---------------------------------------------------------------------------
__device__ __forceinline__ CState cell6(const Params& p, const State& st, const Turb& t, int c) {
  CState s;
  s.rho = st.q[5 * c];
  for (int i = 0; i < 3; i++) s.u[i] = st.prim[8 * c + i];
  s.p = st.prim[8 * c + 3];
  s.T = st.prim[8 * c + 4];
  s.h = st.prim[8 * c + 5];
  s.gam = p.gamma;
  s.sc = t.phi[c];
  return s;
}
__device__ __forceinline__ CState bfa6(const Params& p, const State& st, const Turb& t, int f) {
  const double* b = &st.bfa[8 * f];
  CState s;
  s.rho = b[0];
  s.u[0] = b[1]; s.u[1] = b[2]; s.u[2] = b[3];
  s.p = b[4];
  s.T = b[5];
  s.h = b[6];
  s.gam = p.gamma;
  s.sc = t.phi_bfa[f];
  return s;
}
// reconstruction with the scalar and first-order fallback (JoeWithModels.cpp:4837-4921),
// then calcThermoProp_p (UgpWithCvCompFlow.h:1765-1771)
__device__ __forceinline__ CState recon6(const Mesh& m, const Params& p, const State& st, const Turb& t, int c, int f) {
  CState s = cell6(p, st, t, c);
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
    s.sc += dot3(r0, &t.grad_phi[3 * c]);
  }
  s.rho = rr;
  s.p = pp;
  s.T = pp / (rr * p.R);
  s.h = p.gamma * p.R / (p.gamma - 1.0) * s.T;
  return s;
}
__device__ __forceinline__ VSide6 vcell6(const State& st, const Turb& t, const Params& p, int c) {
  VSide6 v;
  v.rho = st.q[5 * c];
  for (int i = 0; i < 3; i++) v.u[i] = st.prim[8 * c + i];
  v.h = st.prim[8 * c + 5];
  v.T = st.prim[8 * c + 4];
  v.gam = p.gamma;
  v.sc = t.phi[c];
  v.gu = &st.gu[9 * c];
  v.gh = &st.gh[3 * c];
  v.gs = &t.grad_phi[3 * c];
  return v;
}
__device__ __forceinline__ VSide6 vbfa6(const State& st, const Turb& t, const Params& p, int f, int c, double sc,
                                        const double* gs) {
  const double* b = &st.bfa[8 * f];
  VSide6 v;
  v.rho = b[0];
  v.u[0] = b[1]; v.u[1] = b[2]; v.u[2] = b[3];
  v.h = b[6];
  v.T = b[5];
  v.gam = p.gamma;
  v.sc = sc;
  v.gu = &st.gu[9 * c];
  v.gh = &st.gh[3 * c];
  v.gs = gs;
  return v;
}

template <typename BT>
__device__ __forceinline__ size_t ell6(const Mesh& m, int c, int col, int e) {
  int slice = c / SLICE, lane = c % SLICE;
  return ((size_t)(m.ell_off[slice] + col) * B6SQ + e) * SLICE + lane;
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
// face loop: calcRhsCoupled (fluxes, boundary zones, SA source) + the
// implicit-step epilogue (vol/dt, under-relaxed rhs, D^-1)
// ---------------------------------------------------------------------------
template <typename BT>
__global__ void __launch_bounds__(128) k_flux6(Mesh m, Params p, State st, Turb t, int implicit, int for_step) {
  extern __shared__ double sD[];  // [36][blockDim.x]
  const int tid = threadIdx.x, bd = blockDim.x;
  const int c = blockIdx.x * bd + tid;
  if (c >= m.ncv) return;
  const bool only_p = p.symm_bc == JG_SYMM_ANALYTICAL;
  double rhs[B6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int e = 0; e < B6SQ; e++) sD[e * bd + tid] = 0.0;
  BT* O = (BT*)st.O;
  double F[B6];
  for (int k = m.slot_i[c]; k < m.slot_i[c + 1]; k++) {
    const Slot s = m.slots[k];
    const int f = s.f;
    double nV[3], area;
    unit_normal6(m, f, nV, area);
    if (s.nb >= 0) {
      const int c0 = s.side == 0 ? c : s.nb;
      const int c1 = s.side == 0 ? s.nb : c;
      const double sg = s.side == 0 ? -1.0 : 1.0;
      {
        CState L = recon6(m, p, st, t, c0, f), R = recon6(m, p, st, t, c1, f);
        flux_hllc6(F, L, R, area, nV, false);
        for (int i = 0; i < B6; i++) rhs[i] += sg * F[i];
      }
      double Ob[B6SQ];
      if (implicit) {
        CState L0 = cell6(p, st, t, c0), R0 = cell6(p, st, t, c1);
        double Apl[B6SQ], Ami[B6SQ];
        matrices_hllc6(Apl, Ami, L0, R0, area, nV, false);
        // row of c0: D += Apl, O = Ami ; row of c1: D -= Ami, O = -Apl
        if (s.side == 0) {
          for (int e = 0; e < B6SQ; e++) { sD[e * bd + tid] += Apl[e]; Ob[e] = Ami[e]; }
        } else {
          for (int e = 0; e < B6SQ; e++) { sD[e * bd + tid] -= Ami[e]; Ob[e] = -Apl[e]; }
        }
      }
      {
        VSide6 v0 = vcell6(st, t, p, c0), v1 = vcell6(st, t, p, c1);
        double sV[3];
        for (int i = 0; i < 3; i++) sV[i] = m.x_cv[3 * c1 + i] - m.x_cv[3 * c0 + i];
        double smag = sqrt(dot3(sV, sV));
        for (int i = 0; i < 3; i++) sV[i] /= smag;
        double alpha = dot3(nV, sV);
        double ufa[3] = {0.5 * (v0.u[0] + v1.u[0]), 0.5 * (v0.u[1] + v1.u[1]), 0.5 * (v0.u[2] + v1.u[2])};
        VF6 vf;
        visc_flux6(F, vf, v0, v1, st.mul_fa[f], st.mut_fa[f], st.lam_fa[f], p.PrTurb, ufa, t.diff[f], 1.0, area, nV,
                   smag, sV, alpha);
        for (int i = 0; i < B6; i++) rhs[i] += sg * F[i];
        if (implicit) {
          // row of c0: D += A0, O += A1 ; row of c1: D -= A1, O -= A0  (JoeWithModels.cpp:5110-5127)
          double Dv[B6SQ];
          for (int e = 0; e < B6SQ; e++) Dv[e] = 0.0;
          if (s.side == 0) {
            visc_jac6_add(Dv, 1.0, 0, vf, v0, ufa, p.R, area);
            visc_jac6_add(Ob, 1.0, 1, vf, v1, ufa, p.R, area);
          } else {
            visc_jac6_add(Dv, -1.0, 1, vf, v1, ufa, p.R, area);
            visc_jac6_add(Ob, -1.0, 0, vf, v0, ufa, p.R, area);
          }
          for (int e = 6; e < B6SQ; e++) sD[e * bd + tid] += Dv[e];
        }
      }
      if (implicit)
        for (int e = 0; e < B6SQ; e++) O[ell6<BT>(m, c, s.col, e)] = (BT)Ob[e];
    } else {
      // boundary face; the cell is cvofa[f][0] (JoeWithModels.cpp:5139-5799)
      const DevZone z = m.zones[m.bzone[f]];
      const double diffTerm = (z.scal_bc & 1) ? 1.0 : 0.0;
      CState Bs = bfa6(p, st, t, f);
      double Dv[B6SQ];
      if (z.kind == JG_BC_SYMMETRY || z.kind == JG_BC_WALL) {
        flux_hllc6(F, Bs, Bs, area, nV, only_p);
        for (int i = 0; i < B6; i++) rhs[i] -= F[i];
        if (implicit) {
          if (p.symm_bc == JG_SYMM_NEW_NUMERIC) {
            double Apl[B6SQ], Ami[B6SQ];
            matrices_hllc6(Apl, Ami, Bs, Bs, area, nV, false);
            for (int e = 0; e < B6SQ; e++) sD[e * bd + tid] += Apl[e] + Ami[e];
          } else {
            matrices_hllc6(Dv, nullptr, Bs, Bs, area, nV, only_p);
            for (int e = 0; e < B6SQ; e++) sD[e * bd + tid] += Dv[e];
          }
        }
        if (z.kind == JG_BC_SYMMETRY) {
          const double* g = &st.gu[9 * c];
          double tmp = 2.0 / 3.0 * ((st.mul_fa[f] + st.mut_fa[f]) * (g[0] + g[4] + g[8]) + Bs.rho * 0.0);
          for (int i = 0; i < 3; i++) rhs[1 + i] -= area * tmp * nV[i];
        } else {
          VSide6 v0 = vcell6(st, t, p, c);
          VSide6 v1 = vbfa6(st, t, p, f, c, t.phi_bfa[f], &t.grad_phi[3 * c]);
          double sV[3];
          for (int i = 0; i < 3; i++) sV[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
          double smag = fabs(dot3(sV, nV));
          VF6 vf;
          visc_flux6(F, vf, v0, v1, st.mul_fa[f], 0.0, st.lam_fa[f], p.PrTurb, v1.u, t.diff[f], diffTerm, area, nV,
                     smag, nV, 1.0);
          for (int i = 0; i < B6; i++) rhs[i] -= F[i];
          if (implicit) {
            for (int e = 0; e < B6SQ; e++) Dv[e] = 0.0;
            visc_jac6_add(Dv, 1.0, 0, vf, v0, v1.u, p.R, area);
            for (int e = 6; e < B6SQ; e++) sD[e * bd + tid] += Dv[e];
          }
        }
      } else if (z.kind == JG_BC_NEUMANN) {
        flux_hllc6(F, Bs, Bs, area, nV, false);
        for (int i = 0; i < B6; i++) rhs[i] -= F[i];
        if (implicit) {
          double Apl[B6SQ], Ami[B6SQ];
          matrices_hllc6(Apl, Ami, Bs, Bs, area, nV, false);
          for (int e = 0; e < B6SQ; e++)
            sD[e * bd + tid] += (p.symm_bc == JG_SYMM_NEW_NUMERIC) ? Apl[e] + Ami[e] : Apl[e];
        }
        VSide6 vb = vbfa6(st, t, p, f, c, t.phi_bfa[f], nullptr);
        double sV[3];
        for (int i = 0; i < 3; i++) sV[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
        double smag = fabs(dot3(sV, nV));
        VF6 vf;
        visc_flux6(F, vf, vb, vb, st.mul_fa[f], st.mut_fa[f], st.lam_fa[f], p.PrTurb, vb.u, t.diff[f], 1.0, area, nV,
                   smag, nV, 1.0);
        for (int i = 0; i < B6; i++) rhs[i] -= F[i];
        if (implicit) {
          for (int e = 0; e < B6SQ; e++) Dv[e] = 0.0;
          visc_jac6_add(Dv, 1.0, 0, vf, vb, vb.u, p.R, area);
          for (int e = 6; e < B6SQ; e++) sD[e * bd + tid] += Dv[e];
        }
      } else {
        // CBC, CBC_SUBSONIC_INLET/OUTLET, FARFIELD (JoeWithModels.cpp:5624-5788)
        CState L = recon6(m, p, st, t, c, f);
        flux_hllc6(F, L, Bs, area, nV, false);
        for (int i = 0; i < B6; i++) rhs[i] -= F[i];
        if (implicit) {
          CState L0 = cell6(p, st, t, c);
          matrices_hllc6(Dv, nullptr, L0, Bs, area, nV, false);
          for (int e = 0; e < B6SQ; e++) sD[e * bd + tid] += Dv[e];
        }
        VSide6 v0 = vcell6(st, t, p, c);
        // the outer state carries the reconstructed face scalar, as the reference passes it
        VSide6 v1 = vbfa6(st, t, p, f, c, L.sc, &t.grad_phi[3 * c]);
        double sV[3];
        for (int i = 0; i < 3; i++) sV[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
        double smag = sqrt(dot3(sV, sV));
        for (int i = 0; i < 3; i++) sV[i] /= smag;
        double alpha = dot3(nV, sV);
        VF6 vf;
        visc_flux6(F, vf, v0, v1, st.mul_fa[f], st.mut_fa[f], st.lam_fa[f], p.PrTurb, v1.u, t.diff[f], diffTerm, area,
                   nV, smag, sV, alpha);
        for (int i = 0; i < B6; i++) rhs[i] -= F[i];
        if (implicit) {
          for (int e = 0; e < B6SQ; e++) Dv[e] = 0.0;
          visc_jac6_add(Dv, 1.0, 0, vf, v0, v1.u, p.R, area);
          for (int e = 6; e < B6SQ; e++) sD[e * bd + tid] += Dv[e];
        }
      }
    }
  }
  // RansTurbSA::sourceHookRansTurbCoupled (TurbModel_SA.h:359-434)
  double dH2v = 0.0;
  {
    double rho = st.q[5 * c];
    double mue = face_avg6(m, st.mul_fa, c);
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
    rhs[5] += rho * m.vol[c] * (H1 + H2 + H3);
    double d_H2 = -2.0 * SA_CW1 * fw * nu / sq(d);
    dH2v = (0.0 + d_H2) * m.vol[c];
  }
  for (int i = 0; i < B6; i++) st.rhs[B6 * c + i] = rhs[i];
  if (implicit) {
    double Dm[B6SQ];
    for (int e = 0; e < B6SQ; e++) Dm[e] = sD[e * bd + tid];
    Dm[35] -= dH2v;
    if (for_step) {
      double tmp = m.vol[c] / st.local_dt[c];
      for (int i = 0; i < B6; i++) Dm[7 * i] += tmp;
      for (int i = 0; i < B6; i++) st.b[B6 * c + i] = p.under_relax * rhs[i];
    }
    BT* Dg = (BT*)st.D;
    for (int e = 0; e < B6SQ; e++) Dg[(size_t)e * m.ncv + c] = (BT)Dm[e];
    if (for_step) {
      double Di[B6SQ];
      block_inverse_n<B6>(Dm, Di);
      BT* Dig = (BT*)st.Dinv;
      for (int e = 0; e < B6SQ; e++) Dig[(size_t)e * m.ncv + c] = (BT)Di[e];
    }
  }
}

// ---------------------------------------------------------------------------
// block relaxation of the 6x6 system: one warp per block row of a 32-cell
// slice (192 threads), as the 5x5 sweeps
// ---------------------------------------------------------------------------
template <typename BT>
__global__ void __launch_bounds__(192) k_jacobi6(Mesh m, State st, const BT* __restrict__ xin, BT* __restrict__ xout,
                                                 int first) {
  __shared__ BT sacc[B6][SLICE];
  const int row = threadIdx.x / SLICE, lane = threadIdx.x % SLICE;
  const int slice = blockIdx.x;
  const int c = slice * SLICE + lane;
  const bool active = c < m.ncv;
  const int N = m.ncv;
  BT acc = active ? (BT)st.b[B6 * c + row] : (BT)0;
  if (!first && active) {
    const BT* O = (const BT*)st.O;
    for (int j = m.ell_off[slice]; j < m.ell_off[slice + 1]; j++) {
      int nb = m.ell_nb[(size_t)j * SLICE + lane];
      const BT* Ob = O + ((size_t)j * B6SQ + B6 * row) * SLICE + lane;
      BT s = 0;
      for (int k = 0; k < B6; k++) s += Ob[k * SLICE] * xin[(size_t)k * N + nb];
      acc -= s;
    }
  }
  sacc[row][lane] = acc;
  __syncthreads();
  if (active) {
    const BT* Di = (const BT*)st.Dinv;
    BT s = 0;
    for (int k = 0; k < B6; k++) s += Di[(size_t)(B6 * row + k) * N + c] * sacc[k][lane];
    xout[(size_t)row * N + c] = s;
  }
}

template <typename BT>
__global__ void __launch_bounds__(192) k_gs6(Mesh m, State st, BT* __restrict__ x, int color) {
  __shared__ BT sacc[B6][SLICE];
  const int row = threadIdx.x / SLICE, lane = threadIdx.x % SLICE;
  const int slice = blockIdx.x;
  const int c = slice * SLICE + lane;
  const bool active = c < m.ncv && m.color[c] == color;
  const int N = m.ncv;
  BT acc = 0;
  if (active) {
    acc = (BT)st.b[B6 * c + row];
    const BT* O = (const BT*)st.O;
    for (int j = m.ell_off[slice]; j < m.ell_off[slice + 1]; j++) {
      int nb = m.ell_nb[(size_t)j * SLICE + lane];
      const BT* Ob = O + ((size_t)j * B6SQ + B6 * row) * SLICE + lane;
      BT s = 0;
      for (int k = 0; k < B6; k++) s += Ob[k * SLICE] * x[(size_t)k * N + nb];
      acc -= s;
    }
  }
  sacc[row][lane] = acc;
  __syncthreads();
  if (active) {
    const BT* Di = (const BT*)st.Dinv;
    BT s = 0;
    for (int k = 0; k < B6; k++) s += Di[(size_t)(B6 * row + k) * N + c] * sacc[k][lane];
    x[(size_t)row * N + c] = s;
  }
}

// runBackwardEulerCoupled update (JoeWithModels.cpp:4497-4517): Q += dq, then
// nuSA = clip((nuSA * (rho_new - dq0) + dq5) / rho_new); dq also kept in st.dq
template <typename BT>
__global__ void k_update6(Mesh m, State st, Turb t, const BT* __restrict__ x) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  const int N = m.ncv;
  double dq[B6];
  for (int i = 0; i < B6; i++) {
    dq[i] = (double)x[(size_t)i * N + c];
    st.dq[B6 * c + i] = dq[i];
  }
  double rho = st.q[5 * c] + dq[0];
  st.q[5 * c] = rho;
  for (int i = 1; i < 5; i++) st.q[5 * c + i] += dq[i];
  t.phi[c] = fmin(fmax((t.phi[c] * (rho - dq[0]) + dq[5]) / rho, SA_LOWER), SA_UPPER);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
constexpr int TB6 = 128;

void launch_wall_distance(const Mesh& m, Turb& t, cudaStream_t s) {
  k_wall_dist<<<grid_for(m.ncv, 256), 256, 0, s>>>(m, t);
}
void launch_scalar_bc(const Mesh& m, State& st, Turb& t, cudaStream_t s) {
  if (m.nfa_b) k_scalar_bc<<<grid_for(m.nfa_b, TB6), TB6, 0, s>>>(m, st, t);
}
void launch_grad_coupled(const Mesh& m, const Params& p, State& st, cudaStream_t s);  // jg_kernels.cu
void launch_turb_props(const Mesh& m, const Params& p, State& st, Turb& t, cudaStream_t s) {
  launch_grad_coupled(m, p, st, s);
  k_grad_phi<<<grid_for(m.ncv, TB6), TB6, 0, s>>>(m, p, t);
  k_sa_cell<<<grid_for(m.ncv, TB6), TB6, 0, s>>>(m, st, t);
  k_sa_face<<<grid_for(m.nfa, TB6), TB6, 0, s>>>(m, st, t);
}
void launch_flux6(const Mesh& m, const Params& p, State& st, Turb& t, int implicit, int for_step, cudaStream_t s) {
  size_t shm = B6SQ * TB6 * sizeof(double);
  if (p.fp32) k_flux6<float><<<grid_for(m.ncv, TB6), TB6, shm, s>>>(m, p, st, t, implicit, for_step);
  else k_flux6<double><<<grid_for(m.ncv, TB6), TB6, shm, s>>>(m, p, st, t, implicit, for_step);
}
void launch_relax6(const Mesh& m, const Params& p, State& st, int sgs, int sweeps, cudaStream_t s) {
  if (sgs) {
    cudaMemsetAsync(st.x0, 0, B6 * (size_t)m.ncv * (p.fp32 ? sizeof(float) : sizeof(double)), s);
    for (int it = 0; it < sweeps; it++)
      for (int q = 0; q < m.ncolors; q++) {
        int col = (it % 2 == 0) ? q : m.ncolors - 1 - q;
        if (p.fp32) k_gs6<float><<<m.nslices, B6 * SLICE, 0, s>>>(m, st, (float*)st.x0, col);
        else k_gs6<double><<<m.nslices, B6 * SLICE, 0, s>>>(m, st, (double*)st.x0, col);
      }
  } else {
    for (int it = 0; it < sweeps; it++) {
      void* xin = (it % 2 == 0) ? st.x1 : st.x0;
      void* xout = (it % 2 == 0) ? st.x0 : st.x1;
      if (p.fp32) k_jacobi6<float><<<m.nslices, B6 * SLICE, 0, s>>>(m, st, (const float*)xin, (float*)xout, it == 0);
      else k_jacobi6<double><<<m.nslices, B6 * SLICE, 0, s>>>(m, st, (const double*)xin, (double*)xout, it == 0);
    }
  }
}
void launch_update6(const Mesh& m, const Params& p, State& st, Turb& t, const void* x, cudaStream_t s) {
  if (p.fp32) k_update6<float><<<grid_for(m.ncv, TB6), TB6, 0, s>>>(m, st, t, (const float*)x);
  else k_update6<double><<<grid_for(m.ncv, TB6), TB6, 0, s>>>(m, st, t, (const double*)x);
}

}  // namespace jg
