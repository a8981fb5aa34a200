// jg_flux.cuh -- pointwise FP64 face physics for the B200 face loop.
//
// Each function restates one reference routine (paths inside the reference
// project); the arithmetic follows the reference term by term so that the
// per-face results agree with it to rounding (the GPU contracts a*b+c into
// FMA, the reference does not).
#pragma once
#include <cuda_runtime.h>

namespace jg {

// face state; the implicit matrices are templated on the arithmetic type (FP64
// for the plain form, FP32 for the preconditioner of the mixed form)
template <typename T>
struct FStateT {
  T rho, u[3], p, gam;
  T h;  // static enthalpy (the HAENEL flux reads it; the others derive what they need from p, rho)
};
using FState = FStateT<double>;

template <typename T>
__device__ __forceinline__ T dot3(const T* a, const T* b) {
  T d = T(0.0);
  d += a[0] * b[0];
  d += a[1] * b[1];
  d += a[2] * b[2];
  return d;
}
template <typename T>
__device__ __forceinline__ FStateT<T> fstate_as(const FState& s) {
  FStateT<T> o;
  o.rho = (T)s.rho;
  for (int i = 0; i < 3; i++) o.u[i] = (T)s.u[i];
  o.p = (T)s.p;
  o.gam = (T)s.gam;
  o.h = (T)s.h;
  return o;
}

// calcEulerFlux_HLLC, src/joe/UgpWithCvCompFlow.cpp:120-235 (k = 0, no scalars)
__device__ inline void flux_hllc(double F[5], const FState& L, const FState& R, double area, const double nV[3]) {
  double unL = dot3(L.u, nV);
  double uLuL = dot3(L.u, L.u);
  double cL = sqrt(L.gam * L.p / L.rho);
  double hL = L.gam / (L.gam - 1.0) * L.p / L.rho + 0.5 * uLuL;
  double eL = hL * L.rho - L.p;
  double unR = dot3(R.u, nV);
  double uRuR = dot3(R.u, R.u);
  double cR = sqrt(R.gam * R.p / R.rho);
  double hR = R.gam / (R.gam - 1.0) * R.p / R.rho + 0.5 * uRuR;
  double eR = hR * R.rho - R.p;
  double Rrho = sqrt(R.rho / L.rho);
  double tmp = 1.0 / (1.0 + Rrho);
  double vr[3] = {tmp * (L.u[0] + R.u[0] * Rrho), tmp * (L.u[1] + R.u[1] * Rrho), tmp * (L.u[2] + R.u[2] * Rrho)};
  double uRoe = dot3(vr, nV);
  double gpr = tmp * ((L.gam * L.p / L.rho + 0.5 * (L.gam - 1.0) * uLuL) +
                      (R.gam * R.p / R.rho + 0.5 * (R.gam - 1.0) * uRuR) * Rrho);
  double cRoe = sqrt(gpr - ((L.gam + R.gam) * 0.5 - 1.0) * 0.5 * dot3(vr, vr));
  double sL = fmin(uRoe - cRoe, unL - cL);
  double sR = fmax(uRoe + cRoe, unR + cR);
  double sM = (L.p - R.p - L.rho * unL * (sL - unL) + R.rho * unR * (sR - unR)) /
              (R.rho * (sR - unR) - L.rho * (sL - unL));
  double pStar = R.rho * (unR - sR) * (unR - sM) + R.p;
  if (sM >= 0.0) {
    if (sL > 0.0) {
      F[0] = L.rho * unL;
      for (int i = 0; i < 3; i++) F[1 + i] = L.rho * L.u[i] * unL + L.p * nV[i];
      F[4] = eL * unL + L.p * unL;
    } else {
      double inv = 1.0 / (sL - sM);
      double sLmuL = sL - unL;
      double rhoS = L.rho * sLmuL * inv;
      double eS = (sLmuL * eL - L.p * unL + pStar * sM) * inv;
      F[0] = rhoS * sM;
      for (int i = 0; i < 3; i++) F[1 + i] = ((L.rho * L.u[i] * sLmuL + (pStar - L.p) * nV[i]) * inv) * sM + pStar * nV[i];
      F[4] = (eS + pStar) * sM;
    }
  } else {
    if (sR >= 0.0) {
      double inv = 1.0 / (sR - sM);
      double sRmuR = sR - unR;
      double rhoS = R.rho * sRmuR * inv;
      double eS = (sRmuR * eR - R.p * unR + pStar * sM) * inv;
      F[0] = rhoS * sM;
      for (int i = 0; i < 3; i++) F[1 + i] = ((R.rho * R.u[i] * sRmuR + (pStar - R.p) * nV[i]) * inv) * sM + pStar * nV[i];
      F[4] = (eS + pStar) * sM;
    } else {
      F[0] = R.rho * unR;
      for (int i = 0; i < 3; i++) F[1 + i] = R.rho * R.u[i] * unR + R.p * nV[i];
      F[4] = eR * unR + R.p * unR;
    }
  }
  for (int i = 0; i < 5; i++) F[i] *= area;
}

// calcJacobianA, UgpWithCvCompFlow.cpp:666-709; nV carries the face area
template <typename T>
__device__ inline void jacobian_A(T* A, const T* vel, T pp, T rrho, const T* nV, T gamma) {
  T km1 = gamma - T(1.0);
  T nVel[3] = {vel[0] * nV[0], vel[1] * nV[1], vel[2] * nV[2]};
  T U_k = nVel[0] + nVel[1] + nVel[2];
  T vsh = T(0.5) * dot3(vel, vel);
  T c2 = gamma * pp / rrho;  // c*c with c = sqrt(gamma p / rho)
  T c = sqrt(c2);
  c2 = c * c;
  T ikm1 = T(1.0) / km1;
  A[0] = T(0.0); A[1] = nV[0]; A[2] = nV[1]; A[3] = nV[2]; A[4] = T(0.0);
  A[5] = -vel[0] * (nVel[1] + nVel[2]) + nV[0] * (km1 * vsh - vel[0] * vel[0]);
  A[6] = (T(2.) - gamma) * nVel[0] + U_k;
  A[7] = vel[0] * nV[1] - km1 * vel[1] * nV[0];
  A[8] = vel[0] * nV[2] - km1 * vel[2] * nV[0];
  A[9] = km1 * nV[0];
  A[10] = -vel[1] * (nVel[0] + nVel[2]) + nV[1] * (km1 * vsh - vel[1] * vel[1]);
  A[11] = -km1 * vel[0] * nV[1] + vel[1] * nV[0];
  A[12] = (T(2.) - gamma) * nVel[1] + U_k;
  A[13] = vel[1] * nV[2] - km1 * vel[2] * nV[1];
  A[14] = km1 * nV[1];
  A[15] = -vel[2] * (nVel[0] + nVel[1]) + nV[2] * (km1 * vsh - vel[2] * vel[2]);
  A[16] = -km1 * vel[0] * nV[2] + vel[2] * nV[0];
  A[17] = -km1 * vel[1] * nV[2] + vel[2] * nV[1];
  A[18] = (T(2.) - gamma) * nVel[2] + U_k;
  A[19] = km1 * nV[2];
  A[20] = U_k * ((gamma - T(2.)) * vsh - c2 * ikm1);
  A[21] = c2 * ikm1 * nV[0] - km1 * vel[0] * (nVel[1] + nVel[2]) - (km1 * vel[0] * vel[0] - vsh) * nV[0];
  A[22] = c2 * ikm1 * nV[1] - km1 * vel[1] * (nVel[0] + nVel[2]) - (km1 * vel[1] * vel[1] - vsh) * nV[1];
  A[23] = c2 * ikm1 * nV[2] - km1 * vel[2] * (nVel[0] + nVel[1]) - (km1 * vel[2] * vel[2] - vsh) * nV[2];
  A[24] = gamma * U_k;
}

// calcSubSonicJacobeanHLLC, UgpWithCvCompFlow.cpp:605-659.  "S" is the side
// whose star state is used (L when sM >= 0); "O" the other side.  AS/AO may be null.
template <typename T>
__device__ inline void subsonic_jac(T* AS, T* AO, T rhoS, const T* uS, T pS_, T eS_,
                                    T qS, T psiS, T SS, T rhoSt, const T* rhouSt, T eSt,
                                    const T* dSMdS, const T* dSMdO, const T* dpsdS, const T* dpsdO,
                                    T SM, T pStar, T gamma, const T* nV) {
  T gm1 = gamma - T(1.0);
  T om = T(1.0) / (SS - SM);
  if (AS) {
    AS[0] = SS + rhoSt * dSMdS[0];
    AS[1] = -nV[0] + rhoSt * dSMdS[1];
    AS[2] = -nV[1] + rhoSt * dSMdS[2];
    AS[3] = -nV[2] + rhoSt * dSMdS[3];
    AS[4] = +rhoSt * dSMdS[4];
    for (int r = 0; r < 3; r++) {
      T* row = AS + 5 * (r + 1);
      row[0] = qS * uS[r] - nV[r] * psiS * gm1 / T(2.0) + nV[r] * dpsdS[0] + rhouSt[r] * dSMdS[0];
      for (int k = 0; k < 3; k++) {
        T base = (k == r) ? (SS - qS + nV[r] * (gamma - T(2.0)) * uS[r]) : (-uS[r] * nV[k] + nV[r] * gm1 * uS[k]);
        row[1 + k] = base + nV[r] * dpsdS[1 + k] + rhouSt[r] * dSMdS[1 + k];
      }
      row[4] = -gm1 * nV[r] + nV[r] * dpsdS[4] + rhouSt[r] * dSMdS[4];
    }
    AS[20] = qS * (eS_ + pS_) / rhoS - qS * psiS * (gamma - T(1.0)) / T(2.0) + SM * dpsdS[0] + (pStar + eSt) * dSMdS[0];
    for (int k = 0; k < 3; k++)
      AS[21 + k] = -nV[k] * (eS_ + pS_) / rhoS + gm1 * uS[k] * qS + SM * dpsdS[1 + k] + (pStar + eSt) * dSMdS[1 + k];
    AS[24] = SS - qS * gamma + SM * dpsdS[4] + (pStar + eSt) * dSMdS[4];
    for (int i = 0; i < 25; i++) AS[i] *= om;
  }
  if (AO) {
    for (int i = 0; i < 5; i++) AO[i] = om * rhoSt * dSMdO[i];
    for (int r = 0; r < 3; r++)
      for (int i = 0; i < 5; i++) AO[5 * (r + 1) + i] = om * (nV[r] * dpsdO[i] + rhouSt[r] * dSMdO[i]);
    for (int i = 0; i < 5; i++) AO[20 + i] = om * (dpsdO[i] * SM + (pStar + eSt) * dSMdO[i]);
  }
}

// calcEulerFluxMatrices_HLLC, UgpWithCvCompFlow.cpp:242-595 (no scalars); AL/AR may be null
template <typename T>
__device__ inline void matrices_hllc(T* AL, T* AR, const FStateT<T>& L, const FStateT<T>& R, T area,
                                     const T nV[3]) {
  T unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u);
  T cL = sqrt(L.gam * L.p / L.rho);
  T eL = (L.gam / (L.gam - T(1.0)) * L.p / L.rho + T(0.5) * uLuL) * L.rho - L.p;
  T unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u);
  T cR = sqrt(R.gam * R.p / R.rho);
  T eR = (R.gam / (R.gam - T(1.0)) * R.p / R.rho + T(0.5) * uRuR) * R.rho - R.p;
  T Rrho = sqrt(R.rho / L.rho);
  T tmp = T(1.0) / (T(1.0) + Rrho);
  T vr[3] = {tmp * (L.u[0] + R.u[0] * Rrho), tmp * (L.u[1] + R.u[1] * Rrho), tmp * (L.u[2] + R.u[2] * Rrho)};
  T uRoe = dot3(vr, nV);
  T gpr = tmp * ((L.gam * L.p / L.rho + T(0.5) * (L.gam - T(1.0)) * uLuL) +
                      (R.gam * R.p / R.rho + T(0.5) * (R.gam - T(1.0)) * uRuR) * Rrho);
  T cRoe = sqrt(gpr - ((L.gam + R.gam) * T(0.5) - T(1.0)) * T(0.5) * dot3(vr, vr));
  T sL = fmin(uRoe - cRoe, unL - cL);
  T sR = fmax(uRoe + cRoe, unR + cR);
  T sM = (L.p - R.p - L.rho * unL * (sL - unL) + R.rho * unR * (sR - unR)) /
              (R.rho * (sR - unR) - L.rho * (sL - unL));
  T pStar = R.rho * (unR - sR) * (unR - sM) + R.p;
  T gmean = T(0.5) * (L.gam + R.gam);
  if ((sM >= T(0.0) && sL > T(0.0)) || (sM < T(0.0) && sR < T(0.0))) {
    // supersonic: the flux depends on one side only
    bool left = sM >= T(0.0);
    T* Aj = left ? AL : AR;
    T* Az = left ? AR : AL;
    const FStateT<T>& S = left ? L : R;
    if (Aj) {
      T nA[3] = {nV[0] * area, nV[1] * area, nV[2] * area};
      jacobian_A(Aj, S.u, S.p, S.rho, nA, gmean);
    }
    if (Az)
      for (int i = 0; i < 25; i++) Az[i] = T(0.0);
    return;
  }
  bool left = sM >= T(0.0);  // star state of the left (sM >= 0) or right wave
  const FStateT<T>& S = left ? L : R;
  T unS = left ? unL : unR, eS = left ? eL : eR, sS = left ? sL : sR;
  T inv = T(1.0) / (sS - sM);
  T sSmu = sS - unS;
  T rhoSt = S.rho * sSmu * inv;
  T rhouSt[3];
  for (int i = 0; i < 3; i++) rhouSt[i] = (S.rho * S.u[i] * sSmu + (pStar - S.p) * nV[i]) * inv;
  T eSt = (sSmu * eS - S.p * unS + pStar * sM) * inv;
  T invrhotld = T(1.0) / (R.rho * (sR - unR) - L.rho * (sL - unL));
  T dSMdUL[5] = {0, 0, 0, 0, 0}, dSMdUR[5] = {0, 0, 0, 0, 0};
  T dpsdUL[5] = {0, 0, 0, 0, 0}, dpsdUR[5] = {0, 0, 0, 0, 0};
  if (AL) {
    T g1 = L.gam - T(1.0);
    dSMdUL[0] = -unL * unL + uLuL * g1 / T(2.0) + sM * sL;
    for (int i = 0; i < 3; i++) dSMdUL[1 + i] = nV[i] * (T(2.0) * unL - sL - sM) - g1 * L.u[i];
    dSMdUL[4] = g1;
    for (int i = 0; i < 5; i++) {
      dSMdUL[i] *= invrhotld;
      dpsdUL[i] = R.rho * (sR - unR) * dSMdUL[i];
    }
  }
  if (AR) {
    T g1 = R.gam - T(1.0);
    dSMdUR[0] = unR * unR - uRuR * g1 / T(2.0) - sM * sR;
    for (int i = 0; i < 3; i++) dSMdUR[1 + i] = -nV[i] * (T(2.0) * unR - sR - sM) + g1 * R.u[i];
    dSMdUR[4] = -g1;
    for (int i = 0; i < 5; i++) {
      dSMdUR[i] *= invrhotld;
      dpsdUR[i] = L.rho * (sL - unL) * dSMdUR[i];
    }
  }
  if (left)
    subsonic_jac(AL, AR, L.rho, L.u, L.p, eL, unL, uLuL, sL, rhoSt, rhouSt, eSt, dSMdUL, dSMdUR, dpsdUL, dpsdUR, sM,
                 pStar, gmean, nV);
  else
    subsonic_jac(AR, AL, R.rho, R.u, R.p, eR, unR, uRuR, sR, rhoSt, rhouSt, eSt, dSMdUR, dSMdUL, dpsdUR, dpsdUL, sM,
                 pStar, gmean, nV);
  for (int side = 0; side < 2; side++) {
    T* A = side == 0 ? AL : AR;
    if (!A) continue;
    const T* dSM = side == 0 ? dSMdUL : dSMdUR;
    const T* dps = side == 0 ? dpsdUL : dpsdUR;
    for (int i = 0; i < 5; i++) A[i] = A[i] * sM + dSM[i] * rhoSt;
    for (int r = 0; r < 3; r++)
      for (int i = 0; i < 5; i++) A[5 * (r + 1) + i] = A[5 * (r + 1) + i] * sM + dSM[i] * rhouSt[r] + dps[i] * nV[r];
    for (int i = 0; i < 5; i++) A[20 + i] = (A[20 + i] + dps[i]) * sM + (eSt + pStar) * dSM[i];
    for (int i = 0; i < 25; i++) A[i] *= area;
  }
}

// calcEulerFlux_Roe, UgpWithCvCompFlow.cpp:3281-3380 (no entropy fix; a Roe-averaged
// c^2 < 1e-12 leaves only the central part, as in the reference's early return)
__device__ inline void flux_roe(double F[5], const FState& L, const FState& R, double area, const double nV[3]) {
  double gamma = 0.5 * (L.gam + R.gam);
  double gm1 = gamma - 1.0, igm1 = 1.0 / gm1;
  double run0 = L.rho * dot3(L.u, nV), run1 = R.rho * dot3(R.u, nV);
  double rE0 = L.p * igm1 + 0.5 * L.rho * dot3(L.u, L.u);
  double rE1 = R.p * igm1 + 0.5 * R.rho * dot3(R.u, R.u);
  double H0 = (rE0 + L.p) / L.rho, H1 = (rE1 + R.p) / R.rho;
  double ha = 0.5 * area;
  F[0] = ha * (run0 + run1);
  for (int i = 0; i < 3; i++) F[1 + i] = ha * (run0 * L.u[i] + run1 * R.u[i] + (L.p + R.p) * nV[i]);
  F[4] = ha * (run0 * H0 + run1 * H1);
  double s0 = sqrt(L.rho), s1 = sqrt(R.rho);
  double t = 1.0 / (s0 + s1);
  double ua = t * (L.u[0] * s0 + R.u[0] * s1), va = t * (L.u[1] * s0 + R.u[1] * s1), wa = t * (L.u[2] * s0 + R.u[2] * s1);
  double hA = t * (H0 * s0 + H1 * s1);
  double alA = 0.5 * (ua * ua + va * va + wa * wa);
  double a2 = gm1 * (hA - alA);
  if (a2 < 1.0e-12) return;
  double aA = sqrt(a2), iaA = 1.0 / aA;
  double unA = ua * nV[0] + va * nV[1] + wa * nV[2];
  double dr = R.rho - L.rho;
  double dru = R.rho * R.u[0] - L.rho * L.u[0];
  double drv = R.rho * R.u[1] - L.rho * L.u[1];
  double drw = R.rho * R.u[2] - L.rho * L.u[2];
  double drE = rE1 - rE0;
  double l1 = fabs(unA), l2 = fabs(unA + aA), l3 = fabs(unA - aA);
  double a1 = 0.5 * (l2 + l3), ab2 = 0.5 * (l2 - l3), ab3 = a1 - l1;
  double ab4 = gm1 * (alA * dr - ua * dru - va * drv - wa * drw + drE);
  double ab5 = unA * dr - nV[0] * dru - nV[1] * drv - nV[2] * drw;
  double ab6 = ab3 * ab4 * (iaA * iaA) - ab2 * ab5 * iaA;
  double ab7 = ab3 * ab5 - ab2 * ab4 * iaA;
  F[0] -= ha * (l1 * dr + ab6);
  F[1] -= ha * (l1 * dru + ua * ab6 - nV[0] * ab7);
  F[2] -= ha * (l1 * drv + va * ab6 - nV[1] * ab7);
  F[3] -= ha * (l1 * drw + wa * ab6 - nV[2] * ab7);
  F[4] -= ha * (l1 * drE + hA * ab6 - unA * ab7);
}

// calcEulerFluxMatrices_Roe with calcPMatrix / calcInvPMatrix,
// UgpWithCvCompFlow.cpp:3382-3559; AL/AR may be null.  The dissipation matrix
// P |Lambda| P^-1 is formed row by row (P row i generated on the fly) to keep
// the live register set small; each entry is the same k-ordered sum.
template <typename T>
__device__ __forceinline__ void roe_p_row(T Pr[5], int i, const T* v, T rr, T rhooc, T rhoxc,
                                          T km1, T vS, T vn, const T* nV) {
  switch (i) {
    case 0: Pr[0] = nV[0]; Pr[1] = nV[1]; Pr[2] = nV[2]; Pr[3] = T(0.5) * rhooc; Pr[4] = T(0.5) * rhooc; break;
    case 1:
      Pr[0] = v[0] * nV[0]; Pr[1] = v[0] * nV[1] - rr * nV[2]; Pr[2] = v[0] * nV[2] + rr * nV[1];
      Pr[3] = T(0.5) * (v[0] * rhooc + rr * nV[0]); Pr[4] = T(0.5) * (v[0] * rhooc - rr * nV[0]); break;
    case 2:
      Pr[0] = v[1] * nV[0] + rr * nV[2]; Pr[1] = v[1] * nV[1]; Pr[2] = v[1] * nV[2] - rr * nV[0];
      Pr[3] = T(0.5) * (v[1] * rhooc + rr * nV[1]); Pr[4] = T(0.5) * (v[1] * rhooc - rr * nV[1]); break;
    case 3:
      Pr[0] = v[2] * nV[0] - rr * nV[1]; Pr[1] = v[2] * nV[1] + rr * nV[0]; Pr[2] = v[2] * nV[2];
      Pr[3] = T(0.5) * (v[2] * rhooc + rr * nV[2]); Pr[4] = T(0.5) * (v[2] * rhooc - rr * nV[2]); break;
    default:
      Pr[0] = T(0.5) * vS * nV[0] + rr * v[1] * nV[2] - rr * v[2] * nV[1];
      Pr[1] = T(0.5) * vS * nV[1] - rr * v[0] * nV[2] + rr * v[2] * nV[0];
      Pr[2] = T(0.5) * vS * nV[2] + rr * v[0] * nV[1] - rr * v[1] * nV[0];
      Pr[3] = T(0.5) * (T(0.5) * vS * rhooc + rr * vn + rhoxc / km1);
      Pr[4] = T(0.5) * (T(0.5) * vS * rhooc - rr * vn + rhoxc / km1);
      break;
  }
}

template <typename T>
__device__ inline void matrices_roe(T* AL, T* AR, const FStateT<T>& L, const FStateT<T>& R, T area,
                                    const T nV[3]) {
  T uLuL = dot3(L.u, L.u), uRuR = dot3(R.u, R.u);
  T Rrho = sqrt(R.rho / L.rho);
  T rr = Rrho * L.rho;
  T tmp = T(1.0) / (T(1.0) + Rrho);
  T v[3] = {tmp * (L.u[0] + R.u[0] * Rrho), tmp * (L.u[1] + R.u[1] * Rrho), tmp * (L.u[2] + R.u[2] * Rrho)};
  T uRoe = dot3(v, nV);
  T gpr = tmp * ((L.gam * L.p / L.rho + T(0.5) * (L.gam - T(1.0)) * uLuL) +
                      (R.gam * R.p / R.rho + T(0.5) * (R.gam - T(1.0)) * uRuR) * Rrho);
  T c = sqrt(gpr - ((L.gam + R.gam) * T(0.5) - T(1.0)) * T(0.5) * dot3(v, v));
  T gamma = T(0.5) * (L.gam + R.gam);
  T km1 = gamma - T(1.0);
  T rhooc = rr / c, rhoxc = rr * c, c2 = c * c;
  T vS = dot3(v, v);
  T vn = v[0] * nV[0] + v[1] * nV[1] + v[2] * nV[2];
  // P^-1 (calcInvPMatrix): the reference divides by rho, c^2 and rho*c entry by
  // entry; one reciprocal of each replaces ~30 FP64 divides (<= 1 ulp per term)
  const T ir = T(1.0) / rr, ic2 = T(1.0) / c2, irc = T(1.0) / rhoxc;
  const T kc = km1 * ic2, kr = km1 * irc;
  T Q[25];
  Q[0] = nV[0] - nV[2] * v[1] * ir + nV[1] * v[2] * ir - nV[0] * T(0.5) * vS * kc;
  Q[1] = nV[0] * v[0] * kc;
  Q[2] = nV[2] * ir + nV[0] * v[1] * kc;
  Q[3] = -nV[1] * ir + nV[0] * v[2] * kc;
  Q[4] = -nV[0] * kc;
  Q[5] = nV[1] + nV[2] * v[0] * ir - nV[0] * v[2] * ir - nV[1] * T(0.5) * vS * kc;
  Q[6] = -nV[2] * ir + nV[1] * v[0] * kc;
  Q[7] = nV[1] * v[1] * kc;
  Q[8] = nV[0] * ir + nV[1] * v[2] * kc;
  Q[9] = -nV[1] * kc;
  Q[10] = nV[2] - nV[1] * v[0] * ir + nV[0] * v[1] * ir - nV[2] * T(0.5) * vS * kc;
  Q[11] = nV[1] * ir + nV[2] * v[0] * kc;
  Q[12] = -nV[0] * ir + nV[2] * v[1] * kc;
  Q[13] = nV[2] * v[2] * kc;
  Q[14] = -nV[2] * kc;
  Q[15] = -vn * ir + T(0.5) * vS * kr;
  Q[16] = nV[0] * ir - v[0] * kr;
  Q[17] = nV[1] * ir - v[1] * kr;
  Q[18] = nV[2] * ir - v[2] * kr;
  Q[19] = kr;
  Q[20] = vn * ir + T(0.5) * vS * kr;
  Q[21] = -nV[0] * ir - v[0] * kr;
  Q[22] = -nV[1] * ir - v[1] * kr;
  Q[23] = -nV[2] * ir - v[2] * kr;
  Q[24] = kr;
  T lam[5] = {fabs(uRoe), fabs(uRoe), fabs(uRoe), fabs(uRoe + c), fabs(uRoe - c)};
  T nA[3] = {nV[0] * area, nV[1] * area, nV[2] * area};
  if (AL) jacobian_A(AL, L.u, L.p, L.rho, nA, gamma);
  if (AR) jacobian_A(AR, R.u, R.p, R.rho, nA, gamma);
#pragma unroll
  for (int i = 0; i < 5; i++) {
    T Pr[5];
    roe_p_row(Pr, i, v, rr, rhooc, rhoxc, km1, vS, vn, nV);
#pragma unroll
    for (int j = 0; j < 5; j++) {
      T pm = T(0.0);
#pragma unroll
      for (int k = 0; k < 5; k++) pm += Pr[k] * lam[k] * Q[5 * k + j];
      if (AL) AL[5 * i + j] = T(0.5) * AL[5 * i + j] + T(0.5) * pm * area;
      if (AR) AR[5 * i + j] = T(0.5) * AR[5 * i + j] - T(0.5) * pm * area;
    }
  }
}

// calcEulerFlux_AUSM, UgpWithCvCompFlow.cpp:3566-3641
__device__ inline void flux_ausm(double F[5], const FState& L, const FState& R, double area, const double nV[3]) {
  double unL = dot3(L.u, nV), cL = sqrt(L.gam * L.p / L.rho);
  double hL = (L.gam / (L.gam - 1.0)) * (L.p / L.rho) + 0.5 * dot3(L.u, L.u);
  double mL = unL / cL;
  double unR = dot3(R.u, nV), cR = sqrt(R.gam * R.p / R.rho);
  double hR = (R.gam / (R.gam - 1.0)) * (R.p / R.rho) + 0.5 * dot3(R.u, R.u);
  double mR = unR / cR;
  double mLP = (fabs(mL) <= 1.0) ? 0.25 * (mL + 1.0) * (mL + 1.0) : 0.5 * (mL + fabs(mL));
  double mRM = (fabs(mR) <= 1.0) ? -0.25 * (mR - 1.0) * (mR - 1.0) : 0.5 * (mR - fabs(mR));
  double mF = mLP + mRM;
  double pLP = (fabs(mL) <= 1.0) ? 0.25 * L.p * (mL + 1.0) * (mL + 1.0) * (2.0 - mL) : 0.5 * L.p * (mL + fabs(mL)) / mL;
  double pRM = (fabs(mR) <= 1.0) ? 0.25 * R.p * (mR - 1.0) * (mR - 1.0) * (2.0 + mR) : 0.5 * R.p * (mR - fabs(mR)) / mR;
  double pF = pLP + pRM;
  double Phi = fabs(mF);
  double mL_ = L.rho * cL, mR_ = R.rho * cR;
  F[0] = 0.5 * (mF * (mL_ + mR_) - Phi * (mR_ - mL_));
  for (int i = 0; i < 3; i++)
    F[1 + i] = 0.5 * (mF * ((L.rho * cL * L.u[i]) + (R.rho * cR * R.u[i])) - Phi * ((R.rho * cR * R.u[i]) - (L.rho * cL * L.u[i]))) + nV[i] * pF;
  F[4] = 0.5 * (mF * ((L.rho * cL * hL) + (R.rho * cR * hR)) - Phi * ((R.rho * cR * hR) - (L.rho * cL * hL)));
  for (int i = 0; i < 5; i++) F[i] *= area;
}

// ---------------------------------------------------------------------------
// Haenel & Schwane (AUSM family with a common speed of sound), calcEulerFlux_HAENEL
// and calcEulerFluxMatrices_HAENEL, UgpWithCvCompFlow.cpp:1329-1505, with the split
// Mach-number polynomials p_plusminus / u_plusminus and their derivatives (753-877)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T hs_p_pm(T p, T un, T c, T sign) {
  T M = sign * un / c;
  if (T(1.0) <= M) return p;
  if (T(-1.0) <= M) return T(0.25) * p * (M + T(1.0)) * (M + T(1.0)) * (T(2.0) - M);
  return T(0.0);
}

template <typename T>
__device__ __forceinline__ T hs_u_pm(T un, T c, T sign) {  // alpha = 1
  T M = sign * un / c;
  if (T(1.0) <= M) return un;
  if (T(0.0) <= M) return sign * T(1.0) * c * T(0.25) * (M + T(1.0)) * (M + T(1.0)) + (T(1.0) - T(1.0)) * un;
  if (T(-1.0) <= M) return sign * T(1.0) * c * T(0.25) * (M + T(1.0)) * (M + T(1.0));
  return T(0.0);
}

// d(rho u^+-)/dQ, alpha = 1 (entry 5, the scalar's, is not needed here)
template <typename T>
__device__ __forceinline__ void hs_drhou_pm(T b[5], T un, T c, const T* n, T sign) {
  T M = sign * un / c;
  if (T(1.0) <= M) {
    b[0] = T(0.0);
    for (int i = 0; i < 3; i++) b[1 + i] = n[i];
  } else if (T(0.0) <= M) {
    b[0] = sign * T(0.25) * T(1.0) * c * (T(1.0) - M * M);
    for (int i = 0; i < 3; i++) b[1 + i] = n[i] * (T(0.5) * T(1.0) * (M + T(1.0)) + (T(1.0) - T(1.0)));
  } else if (T(-1.0) <= M) {
    b[0] = sign * T(0.25) * T(1.0) * c * (T(1.0) - M * M);
    for (int i = 0; i < 3; i++) b[1 + i] = n[i] * (T(0.5) * T(1.0) * (M + T(1.0)));
  } else {
    b[0] = T(0.0);
    for (int i = 0; i < 3; i++) b[1 + i] = T(0.0);
  }
  b[4] = T(0.0);
}

// dp^+-/dQ
template <typename T>
__device__ __forceinline__ void hs_dp_pm(T d[5], const T* u, T rho, T p, T un, T uu, T ht, T c, T gam, const T* n,
                                         T sign) {
  T M = sign * un / c;
  T dpdrho = gam * p / rho + (T(1.0) - gam) * (ht - uu);
  if (T(1.0) <= M) {
    d[0] = dpdrho;
    for (int i = 0; i < 3; i++) d[1 + i] = (T(1.0) - gam) * u[i];
    d[4] = gam - T(1.0);
  } else if (T(-1.0) <= M) {
    T w = T(0.25) * (M + T(1.0)) * (M + T(1.0)) * (T(2.0) - M);
    d[0] = w * dpdrho - T(0.75) * p / rho * (T(1.0) + M) * (T(1.0) - M) * M;
    for (int i = 0; i < 3; i++)
      d[1 + i] = w * (T(1.0) - gam) * u[i] + T(0.75) * p / (rho * c) * (T(1.0) + M) * (T(1.0) - M) * sign * n[i];
    d[4] = w * (gam - T(1.0));
  } else {
    for (int i = 0; i < 5; i++) d[i] = T(0.0);
  }
}

__device__ inline void flux_haenel(double F[5], const FState& L, const FState& R, double area, const double nV[3]) {
  double unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u), cL = sqrt(L.gam * L.p / L.rho), hL = L.h + 0.5 * uLuL + 0.0;
  double unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u), cR = sqrt(R.gam * R.p / R.rho), hR = R.h + 0.5 * uRuR + 0.0;
  double cLR = fmax(cL, cR);
  double p_half = hs_p_pm(L.p, unL, cLR, 1.0) + hs_p_pm(R.p, unR, cLR, -1.0);
  double uLp = hs_u_pm(unL, cLR, 1.0), uRm = hs_u_pm(unR, cLR, -1.0);
  F[0] = L.rho * uLp + R.rho * uRm;
  for (int i = 0; i < 3; i++) F[1 + i] = L.rho * uLp * L.u[i] + R.rho * uRm * R.u[i] + p_half * nV[i];
  F[4] = L.rho * uLp * hL + R.rho * uRm * hR;
  for (int i = 0; i < 5; i++) F[i] *= area;
}

// one side's matrix: the side's u^+- (upm), its derivative blocks (beta, delta)
template <typename T>
__device__ __forceinline__ void haenel_side(T* A, const FStateT<T>& S, T un, T uu, T hS, T upm, const T beta[5],
                                            const T delta[5], T area, const T nV[3]) {
  for (int j = 0; j < 5; j++) {
    A[j] = beta[j];
    for (int i = 0; i < 3; i++) A[5 * (1 + i) + j] = beta[j] * S.u[i] + delta[j] * nV[i];
    A[20 + j] = beta[j] * hS;
  }
  for (int i = 0; i < 3; i++) {
    A[5 * (1 + i)] += -upm * S.u[i];
    A[5 * (1 + i) + 1 + i] += upm;
  }
  A[20] += upm * ((S.gam - T(1.0)) * uu - S.gam * hS + S.gam * S.p / S.rho);
  for (int j = 0; j < 3; j++) A[21 + j] += upm * (T(1.0) - S.gam) * S.u[j];
  A[24] += upm * S.gam;
  for (int e = 0; e < 25; e++) A[e] *= area;
}

template <typename T>
__device__ inline void matrices_haenel(T* AL, T* AR, const FStateT<T>& L, const FStateT<T>& R, T area, const T nV[3]) {
  T unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u), cL = sqrt(L.gam * L.p / L.rho), hL = L.h + T(0.5) * uLuL + T(0.0);
  T unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u), cR = sqrt(R.gam * R.p / R.rho), hR = R.h + T(0.5) * uRuR + T(0.0);
  T cLR = fmax(cL, cR);
  T uLp = hs_u_pm(unL, cLR, T(1.0)), uRm = hs_u_pm(unR, cLR, T(-1.0));
  T bp[5], bm[5], dp[5], dm[5];
  hs_drhou_pm(bp, unL, cLR, nV, T(1.0));
  hs_drhou_pm(bm, unR, cLR, nV, T(-1.0));
  hs_dp_pm(dp, L.u, L.rho, L.p, unL, uLuL, hL, cLR, L.gam, nV, T(1.0));
  hs_dp_pm(dm, R.u, R.rho, R.p, unR, uRuR, hR, cLR, R.gam, nV, T(-1.0));
  if (AL) haenel_side(AL, L, unL, uLuL, hL, uLp, bp, dp, area, nV);
  if (AR) haenel_side(AR, R, unR, uRuR, hR, uRm, bm, dm, area, nV);
}

// ---------------------------------------------------------------------------
// AUSMDV (Wada & Liou), calcEulerFlux_AUSMDV and calcEulerFluxMatrices_AUSMDV,
// UgpWithCvCompFlow.cpp:879-1322, with the split polynomials of a general alpha
// (u_plusminus, drhou_plusminus_dQ, 753-877).  The face options `fo`:
// bits 0-1 the blend (FO_DV 0: AUSMDV, 1: AUSMV, 2: AUSMD), bit 2 the entropy fix
// for single expansion waves, bit 3 alpha from the densities alone (the ALPHA_LR
// shock fix), bit 4 the Haenel & Schwane flux instead (the HAENEL shock fix).
// ---------------------------------------------------------------------------
enum { FO_TYPE = 3, FO_EFIX = 4, FO_ALPHA_LR = 8, FO_HAENEL = 16 };

template <typename T>
__device__ __forceinline__ T ausm_u_pm(T alpha, T un, T c, T sign) {
  T M = sign * un / c;
  if (T(1.0) <= M) return un;
  if (T(0.0) <= M) return sign * alpha * c * T(0.25) * (M + T(1.0)) * (M + T(1.0)) + (T(1.0) - alpha) * un;
  if (T(-1.0) <= M) return sign * alpha * c * T(0.25) * (M + T(1.0)) * (M + T(1.0));
  return T(0.0);
}

template <typename T>
__device__ __forceinline__ void ausm_drhou_pm(T b[5], T alpha, T un, T c, const T* n, T sign) {
  T M = sign * un / c;
  if (T(1.0) <= M) {
    b[0] = T(0.0);
    for (int i = 0; i < 3; i++) b[1 + i] = n[i];
  } else if (T(0.0) <= M) {
    b[0] = sign * T(0.25) * alpha * c * (T(1.0) - M * M);
    for (int i = 0; i < 3; i++) b[1 + i] = n[i] * (T(0.5) * alpha * (M + T(1.0)) + (T(1.0) - alpha));
  } else if (T(-1.0) <= M) {
    b[0] = sign * T(0.25) * alpha * c * (T(1.0) - M * M);
    for (int i = 0; i < 3; i++) b[1 + i] = n[i] * (T(0.5) * alpha * (M + T(1.0)));
  } else {
    b[0] = T(0.0);
    for (int i = 0; i < 3; i++) b[1 + i] = T(0.0);
  }
  b[4] = T(0.0);
}

// alpha_LR_L (753-759)
template <typename T>
__device__ __forceinline__ T ausm_alpha_L(T pL, T rhoL, T pR, T rhoR, int fo) {
  if (fo & FO_ALPHA_LR) return T(2.0) * (T(1.0) / rhoL) / ((T(1.0) / rhoL) + (T(1.0) / rhoR));
  return T(2.0) * (pL / rhoL) / ((pL / rhoL) + (pR / rhoR));
}

// the AUSMD / AUSMV blend weight s
template <typename T>
__device__ __forceinline__ T ausm_s(T pL, T pR, int fo) {
  const int type = fo & FO_TYPE;
  if (type == 0) return T(0.5) * fmin(T(1.0), (T(10.0) * fabs(pR - pL)) / fmin(pL, pR));
  return type == 1 ? T(0.5) : T(-0.5);
}

// the entropy fix's wave-speed jump (cases A and B of Wada & Liou); 0 where it does not apply
template <typename T>
__device__ __forceinline__ T ausm_dlambda(T unL, T cL, T unR, T cR) {
  if ((unL <= -cL) && (unR >= cR)) return T(0.0);
  if (((unL - cL) < T(0.0)) && ((unR - cR) > T(0.0))) return (unR - cR) - (unL - cL);
  if (((unL + cL) < T(0.0)) && ((unR + cR) > T(0.0))) return (unR + cR) - (unL + cL);
  return T(0.0);
}

__device__ inline void flux_ausmdv(double F[5], const FState& L, const FState& R, double area, const double nV[3],
                                   int fo) {
  const double unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u), cL = sqrt(L.gam * L.p / L.rho);
  const double hL = L.h + 0.5 * uLuL + 0.0;
  const double alphaL = ausm_alpha_L(L.p, L.rho, R.p, R.rho, fo);
  const double unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u), cR = sqrt(R.gam * R.p / R.rho);
  const double hR = R.h + 0.5 * uRuR + 0.0;
  const double alphaR = 2.0 - alphaL;
  const double cLR = fmax(cL, cR);
  const double p_half = hs_p_pm(L.p, unL, cLR, 1.0) + hs_p_pm(R.p, unR, cLR, -1.0);
  const double uLp = ausm_u_pm(alphaL, unL, cLR, 1.0), uRm = ausm_u_pm(alphaR, unR, cLR, -1.0);
  const double rhou_half = L.rho * uLp + R.rho * uRm;
  const double s = ausm_s(L.p, R.p, fo);
  const double pn = (0.5 + s) * (L.rho * unL * uLp + R.rho * unR * uRm);
  F[0] = rhou_half;
  if (rhou_half >= 0.0) {
    for (int i = 0; i < 3; i++)
      F[1 + i] = rhou_half * (L.u[i] - unL * nV[i]) + nV[i] * (p_half + pn + (0.5 - s) * rhou_half * unL);
    F[4] = rhou_half * hL;
  } else {
    for (int i = 0; i < 3; i++)
      F[1 + i] = rhou_half * (R.u[i] - unR * nV[i]) + nV[i] * (p_half + pn + (0.5 - s) * rhou_half * unR);
    F[4] = rhou_half * hR;
  }
  if (fo & FO_EFIX) {
    const double dl = 0.125 * ausm_dlambda(unL, cL, unR, cR);
    if (dl != 0.0) {
      F[0] -= dl * (R.rho - L.rho);
      for (int i = 0; i < 3; i++) F[1 + i] -= dl * (R.rho * R.u[i] - L.rho * L.u[i]);
      F[4] -= dl * (R.rho * hR - L.rho * hL);
    }
  }
  for (int i = 0; i < 5; i++) F[i] *= area;
}

// one side's convective part of the AUSMDV matrix: d(rho u_half)/dQ times the upwind side's
// (tangential velocity, total enthalpy), plus rho u_half times their derivatives when this side is
// the upwind one (`own`); ut / hu: the upwind side's tangential velocity and total enthalpy
template <typename T>
__device__ __forceinline__ void ausmdv_side(T* A, const FStateT<T>& S, bool own, T uu, T hS, T rhou_half,
                                            const T beta[5], const T* ut, T hu, const T nV[3]) {
  for (int e = 0; e < 25; e++) A[e] = T(0.0);
  A[0] += beta[0];
  for (int j = 0; j < 3; j++) A[1 + j] += beta[1 + j];
  if (own) {
    const T eS = hS - S.p / S.rho;
    for (int i = 0; i < 3; i++) {
      A[5 * (1 + i)] += beta[0] * ut[i] - rhou_half * ut[i] / S.rho;
      for (int j = 0; j < 3; j++) A[5 * (1 + i) + 1 + j] += beta[1 + j] * ut[i] - rhou_half * nV[i] * nV[j] / S.rho;
      A[5 * (1 + i) + 1 + i] += rhou_half / S.rho;
    }
    A[20] += beta[0] * hS + rhou_half * ((S.gam - T(1.0)) * uu - S.gam * eS) / S.rho;
    for (int j = 0; j < 3; j++) A[21 + j] += beta[1 + j] * hS - rhou_half * (S.gam - T(1.0)) * S.u[j] / S.rho;
    A[24] += rhou_half * S.gam / S.rho;
  } else {
    for (int i = 0; i < 3; i++) {
      A[5 * (1 + i)] += beta[0] * ut[i];
      for (int j = 0; j < 3; j++) A[5 * (1 + i) + 1 + j] += beta[1 + j] * ut[i];
    }
    A[20] += beta[0] * hu;
    for (int j = 0; j < 3; j++) A[21 + j] += beta[1 + j] * hu;
  }
}

template <typename T>
__device__ inline void matrices_ausmdv(T* AL, T* AR, const FStateT<T>& L, const FStateT<T>& R, T area, const T nV[3],
                                       int fo) {
  const T unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u), cL = sqrt(L.gam * L.p / L.rho);
  const T hL = L.h + T(0.5) * uLuL + T(0.0);
  const T alphaL = ausm_alpha_L(L.p, L.rho, R.p, R.rho, fo);
  T utL[3], utR[3];
  for (int i = 0; i < 3; i++) utL[i] = L.u[i] - unL * nV[i];
  const T unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u), cR = sqrt(R.gam * R.p / R.rho);
  const T hR = R.h + T(0.5) * uRuR + T(0.0);
  const T alphaR = T(2.0) - alphaL;
  for (int i = 0; i < 3; i++) utR[i] = R.u[i] - unR * nV[i];
  const T cLR = fmax(cL, cR);
  const T uLp = ausm_u_pm(alphaL, unL, cLR, T(1.0)), uRm = ausm_u_pm(alphaR, unR, cLR, T(-1.0));
  const T rhou_half = L.rho * uLp + R.rho * uRm;
  const T s = ausm_s(L.p, R.p, fo);
  T bp[5], bm[5], dp[5], dm[5];
  ausm_drhou_pm(bp, alphaL, unL, cLR, nV, T(1.0));
  ausm_drhou_pm(bm, alphaR, unR, cLR, nV, T(-1.0));
  hs_dp_pm(dp, L.u, L.rho, L.p, unL, uLuL, hL, cLR, L.gam, nV, T(1.0));
  hs_dp_pm(dm, R.u, R.rho, R.p, unR, uRuR, hR, cLR, R.gam, nV, T(-1.0));
  T dl = T(0.0);
  if (fo & FO_EFIX) dl = ausm_dlambda(unL, cL, unR, cR);
  for (int side = 0; side < 2; side++) {
    T* A = side == 0 ? AL : AR;
    if (!A) continue;
    const FStateT<T>& S = side == 0 ? L : R;
    const T un = side == 0 ? unL : unR, uu = side == 0 ? uLuL : uRuR, hS = side == 0 ? hL : hR;
    const T upm = side == 0 ? uLp : uRm;
    const T* beta = side == 0 ? bp : bm;
    const T* delta = side == 0 ? dp : dm;
    const bool own = side == 0 ? (rhou_half >= T(0.0)) : (rhou_half < T(0.0));
    ausmdv_side<T>(A, S, own, uu, hS, rhou_half, beta, side == 0 ? (own ? utL : utR) : (own ? utR : utL),
                   side == 0 ? hR : hL, nV);
    // P_half: u* is the upwind side's normal velocity, its derivative this side's when upwind
    const T unstar = own ? un : (side == 0 ? unR : unL);
    T dun[4] = {T(0.0), T(0.0), T(0.0), T(0.0)};
    if (own) {
      dun[0] = -un / S.rho;
      for (int j = 0; j < 3; j++) dun[1 + j] = nV[j] / S.rho;
    }
    for (int i = 0; i < 3; i++) {
      for (int j = 0; j < 4; j++)
        A[5 * (1 + i) + j] +=
            nV[i] * (beta[j] * ((T(0.5) + s) * un + (T(0.5) - s) * unstar) + (T(0.5) - s) * rhou_half * dun[j]);
      A[5 * (1 + i)] += -nV[i] * (T(0.5) + s) * upm * un;
      for (int j = 0; j < 3; j++) A[5 * (1 + i) + 1 + j] += nV[i] * (T(0.5) + s) * upm * nV[j];
      for (int j = 0; j < 5; j++) A[5 * (1 + i) + j] += nV[i] * delta[j];
    }
  }
  if (dl != T(0.0)) {
    for (int side = 0; side < 2; side++) {
      T* A = side == 0 ? AL : AR;
      if (!A) continue;
      const FStateT<T>& S = side == 0 ? L : R;
      const T sg = side == 0 ? T(1.0) : T(-1.0);
      const T un = side == 0 ? unL : unR, uu = side == 0 ? uLuL : uRuR, hS = side == 0 ? hL : hR;
      // A_L += 0.125 (...), A_R -= 0.125 (...) with the side's own state
      T a[25];
      for (int e = 0; e < 25; e++) a[e] = T(0.0);
      a[0] = T(0.125) * (dl + un / S.rho * (L.rho - R.rho));
      for (int i = 0; i < 3; i++) a[5 * (1 + i)] = T(0.125) * un / S.rho * (L.rho * L.u[i] - R.rho * R.u[i]);
      a[20] = T(0.125) * (dl * ((T(1.0) - S.gam) * (hS - uu) + S.gam * S.p / S.rho) +
                          un / S.rho * (L.rho * hL - R.rho * hR));
      for (int j = 0; j < 3; j++) {
        a[1 + j] = -T(0.125) * nV[j] / S.rho * (L.rho - R.rho);
        a[5 * (1 + j) + 1 + j] += T(0.125) * dl;
        for (int i = 0; i < 3; i++) a[5 * (1 + i) + 1 + j] += -T(0.125) * nV[j] / S.rho * (L.rho * L.u[i] - R.rho * R.u[i]);
        a[21 + j] = T(0.125) * (dl * (T(1.0) - S.gam) * S.u[j] - nV[j] / S.rho * (L.rho * hL - R.rho * hR));
      }
      a[24] = T(0.125) * dl * S.gam;
      for (int e = 0; e < 25; e++) A[e] += sg * a[e];
    }
  }
  if (AL)
    for (int e = 0; e < 25; e++) AL[e] *= area;
  if (AR)
    for (int e = 0; e < 25; e++) AR[e] *= area;
}

// ---------------------------------------------------------------------------
// JST, calcEulerFlux_JST (UgpWithCvCompFlow.cpp:4050-4160): the central flux of
// the arithmetic-mean state plus the blended second / fourth difference
// dissipation; JL / JR = {pressure sensor, spectral radius, internal faces,
// undivided Laplacian[5]} of the two cells (the boundary cell's on both sides
// at a boundary face)
// ---------------------------------------------------------------------------
__device__ inline void flux_jst(double F[5], const FState& L, const FState& R, double area, const double nV[3],
                                const double* JL, const double* JR) {
  const double unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u), cL = sqrt(L.gam * L.p / L.rho);
  const double hL = L.gam / (L.gam - 1.0) * L.p / L.rho + 0.5 * uLuL + 0.0;
  const double unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u), cR = sqrt(R.gam * R.p / R.rho);
  const double hR = R.gam / (R.gam - 1.0) * R.p / R.rho + 0.5 * uRuR + 0.0;
  const double md = 0.5 * (L.rho + R.rho), mp = 0.5 * (L.p + R.p), mh = 0.5 * (hL + hR);
  double mv[3];
  for (int i = 0; i < 3; i++) mv[i] = 0.5 * (L.u[i] + R.u[i]);
  const double mun = md * dot3(mv, nV);  // the mean mass flux through the face
  F[0] = mun;
  for (int i = 0; i < 3; i++) F[1 + i] = mun * mv[i] + mp * nV[i];
  F[4] = mun * mh;
  for (int i = 0; i < 5; i++) F[i] *= area;
  double dU[5];
  dU[0] = L.rho - R.rho;
  for (int i = 0; i < 3; i++) dU[1 + i] = L.rho * L.u[i] - R.rho * R.u[i];
  dU[4] = L.rho * hL - R.rho * hR;
  const double mlam = 0.5 * ((fabs(unL) + cL) * area + (fabs(unR) + cR) * area);
  const double phiL = pow(JL[1] / (4.0 * mlam), 0.3), phiR = pow(JR[1] / (4.0 * mlam), 0.3);
  const double stretch = 4.0 * phiL * phiR / (phiL + phiR);
  const double nL = JL[2], nR = JR[2];
  const double sc2 = 3.0 * (nL + nR) / (nL * nR), sc4 = sc2 * sc2 / 4.0;
  const double e2 = 0.5 * 0.5 * (JL[0] + JR[0]) * sc2;
  const double e4 = fmax(0.0, 0.02 - e2) * sc4;
  for (int i = 0; i < 5; i++) F[i] += (e2 * dU[i] - e4 * (JL[3 + i] - JR[3 + i])) * stretch * mlam;
}

template <int KIND>
__device__ __forceinline__ void euler_flux_t(double F[5], const FState& L, const FState& R, double area,
                                             const double nV[3], int fo = 0, const double* JL = nullptr,
                                             const double* JR = nullptr) {
  if (KIND == 5) flux_jst(F, L, R, area, nV, JL, JR);
  else if (KIND == 1) flux_roe(F, L, R, area, nV);
  else if (KIND == 2) flux_ausm(F, L, R, area, nV);
  else if (KIND == 3) flux_haenel(F, L, R, area, nV);
  else if (KIND == 4) {
    if (fo & FO_HAENEL) flux_haenel(F, L, R, area, nV);
    else flux_ausmdv(F, L, R, area, nV, fo);
  } else flux_hllc(F, L, R, area, nV);
}

template <int KIND, typename T>
__device__ __forceinline__ void euler_matrices_t(T* AL, T* AR, const FStateT<T>& L, const FStateT<T>& R, T area,
                                                 const T nV[3], int fo = 0) {
  if (KIND == 1) matrices_roe<T>(AL, AR, L, R, area, nV);
  else if (KIND == 3) matrices_haenel<T>(AL, AR, L, R, area, nV);
  else if (KIND == 4) {
    if (fo & FO_HAENEL) matrices_haenel<T>(AL, AR, L, R, area, nV);
    else matrices_ausmdv<T>(AL, AR, L, R, area, nV, fo);
  } else matrices_hllc<T>(AL, AR, L, R, area, nV);
}

// per-face entry (jg_euler_flux_faces): kind 4 is AUSMDV with the entropy fix and no shock fix
__device__ __forceinline__ void euler_flux(int kind, double F[5], const FState& L, const FState& R, double area,
                                           const double nV[3]) {
  if (kind == 1) flux_roe(F, L, R, area, nV);
  else if (kind == 2) flux_ausm(F, L, R, area, nV);
  else if (kind == 3) flux_haenel(F, L, R, area, nV);
  else if (kind == 4) flux_ausmdv(F, L, R, area, nV, FO_EFIX);
  else flux_hllc(F, L, R, area, nV);
}

// implicit side: AUSM uses the HLLC matrices (src/joe/JoeWithModels.cpp:3057-3061), HAENEL and AUSMDV their own
__device__ __forceinline__ void euler_matrices(int kind, double* AL, double* AR, const FState& L, const FState& R,
                                               double area, const double nV[3]) {
  if (kind == 1) matrices_roe<double>(AL, AR, L, R, area, nV);
  else if (kind == 3) matrices_haenel<double>(AL, AR, L, R, area, nV);
  else if (kind == 4) matrices_ausmdv<double>(AL, AR, L, R, area, nV, FO_EFIX);
  else matrices_hllc<double>(AL, AR, L, R, area, nV);
}

// One side of the viscous flux state (addViscFlux arguments).
struct VSide {
  double rho, u[3], h, T, R, gam;
  const double* gu;  // grad_u [3][3] (row i = d u_i / d x_j)
  const double* gh;  // grad_h [3]
};

// addViscFlux, UgpWithCvCompFlow.cpp:1521-1763 (laminar + mut, no k, no Reynolds
// stresses), split into the flux and the implicit matrices.  The flux returns
// the "left hand side" momentum/energy fluxes and the face stress tau.
struct VFace {
  double alpha, smag, area, mul, mut, keff;
  double aos;  // alpha / smag
  double tau[3];
};

__device__ inline void visc_flux(double Fu[3], double& FE, VFace& vf, const VSide& s0, const VSide& s1, double mul,
                                 double mut, double lamOcp, double PrTurb, const double* u_fa, double area,
                                 const double nV[3], double smag, const double sV[3]) {
  double alpha = dot3(nV, sV);
  const double aos = alpha / smag;  // the normal-derivative weight, one division for all terms
  double g[9];
  for (int i = 0; i < 9; i++) g[i] = 0.5 * (s0.gu[i] + s1.gu[i]);
  double fC[3] = {nV[0] - alpha * sV[0], nV[1] - alpha * sV[1], nV[2] - alpha * sV[2]};
  double div = g[0] + g[4] + g[8];
  double tau[3];
  for (int i = 0; i < 3; i++) {
    double b = (s1.u[i] - s0.u[i]) * aos + g[3 * i + 0] * fC[0] + g[0 + i] * nV[0] + g[3 * i + 1] * fC[1] +
               g[3 + i] * nV[1] + g[3 * i + 2] * fC[2] + g[6 + i] * nV[2];
    double tl = mul * b - (2.0 / 3.0 * mul * div) * nV[i];
    double tt = mut * b - (2.0 / 3.0 * mut * div) * nV[i];
    tau[i] = tl + tt;
  }
  for (int i = 0; i < 3; i++) Fu[i] = -area * tau[i];
  double keff = lamOcp + mut / PrTurb;
  double enth = keff * ((s1.h - s0.h) * aos +
                        0.5 * ((s0.gh[0] + s1.gh[0]) * fC[0] + (s0.gh[1] + s1.gh[1]) * fC[1] + (s0.gh[2] + s1.gh[2]) * fC[2]));
  FE = -area * (enth + tau[0] * u_fa[0] + tau[1] * u_fa[1] + tau[2] * u_fa[2]);
  vf.alpha = alpha; vf.smag = smag; vf.area = area; vf.mul = mul; vf.mut = mut; vf.keff = keff; vf.aos = aos;
  for (int i = 0; i < 3; i++) vf.tau[i] = tau[i];
}

// dF/dU x dU/dQ of the viscous flux (UgpWithCvCompFlow.cpp:717-745, 1692-1760) for
// side 0 (A0) or side 1 (A1), scaled by sgn and added into the 5x5 row-major
// accumulator acc (rows 1..4; the other entries are zero).
// a 5x5 block seen through a stride (one thread's column of a [25][n] array)
template <typename T>
struct StridedBlock {
  T* p;
  int stride;
  __device__ T& operator[](int e) const { return p[e * stride]; }
};

// acc: a T* (a block in registers) or a StridedBlock<T> (accumulated in place)
template <typename T, typename Acc>
__device__ inline void visc_jac_add(Acc acc, T sgn, int side, const VFace& vf, const VSide& s,
                                    const double* u_fa) {
  // inputs rounded to T once, the arithmetic in T (FP64: the reference's expressions term by term)
  const T mm = (T)(vf.mul + vf.mut), aos = (T)vf.aos, area = (T)vf.area, keff = (T)vf.keff;
  const T tau[3] = {(T)vf.tau[0], (T)vf.tau[1], (T)vf.tau[2]};
  const T uf[3] = {(T)u_fa[0], (T)u_fa[1], (T)u_fa[2]};
  const T rho = (T)s.rho, hh = (T)s.h, RR = (T)s.R, TT = (T)s.T, gam = (T)s.gam;
  const T u[3] = {(T)s.u[0], (T)s.u[1], (T)s.u[2]};
  T d = (side == 0) ? -mm * aos * area : mm * aos * area;
  T f44 = (side == 0) ? -area * keff * aos : area * keff * aos;
  T f4[3] = {area * tau[0] * T(0.5) + uf[0] * d, area * tau[1] * T(0.5) + uf[1] * d,
             area * tau[2] * T(0.5) + uf[2] * d};
  T ir = T(1.0) / rho;
  T uq0[3] = {-u[0] * ir, -u[1] * ir, -u[2] * ir};
  T uq40 = gam * ir * (-hh + RR * TT + T(0.5) * dot3(u, u));
  for (int r = 0; r < 3; r++) {
    acc[5 * (r + 1) + 0] += sgn * (d * uq0[r]);
    acc[5 * (r + 1) + 1 + r] += sgn * (d * ir);
  }
  acc[20] += sgn * (f4[0] * uq0[0] + f4[1] * uq0[1] + f4[2] * uq0[2] + f44 * uq40);
  for (int k = 0; k < 3; k++) acc[21 + k] += sgn * (f4[k] * ir + f44 * (-gam * u[k] * ir));
  acc[24] += sgn * (f44 * (gam * ir));
}

}  // namespace jg
