// jg_rows.cuh -- the implicit flux matrices of a face delivered one row at a time.
//
// The Jacobian-assembly kernel consumes each row of the two face matrices as
// soon as it exists (into the cell's diagonal block and its off-diagonal
// block of the sliced-ELL row), so that no thread holds both 5x5 matrices and
// their factors at once.  Every entry is the same arithmetic, in the same
// order, as the whole-matrix routines of jg_flux.cuh (calcJacobianA,
// calcEulerFluxMatrices_Roe / _HLLC / calcSubSonicJacobeanHLLC,
// UgpWithCvCompFlow.cpp:242-709, 3382-3559); only the moment each row is formed
// changes.  emit(i, aL, aR) receives row i of A_L (d flux / d left state) and
// of A_R (d flux / d right state).
#pragma once
#include <cuda_runtime.h>

#include "jg_flux.cuh"

namespace jg {

// row i of calcJacobianA (UgpWithCvCompFlow.cpp:666-709), nV carrying the face area
template <typename T>
__device__ __forceinline__ void jacobian_A_row(T* A, int i, const T* vel, T c2, T ikm1, const T* nV, T gamma) {
  const T km1 = gamma - T(1.0);
  const T nVel[3] = {vel[0] * nV[0], vel[1] * nV[1], vel[2] * nV[2]};
  const T U_k = nVel[0] + nVel[1] + nVel[2];
  const T vsh = T(0.5) * dot3(vel, vel);
  switch (i) {
    case 0:
      A[0] = T(0.0); A[1] = nV[0]; A[2] = nV[1]; A[3] = nV[2]; A[4] = T(0.0);
      break;
    case 1:
      A[0] = -vel[0] * (nVel[1] + nVel[2]) + nV[0] * (km1 * vsh - vel[0] * vel[0]);
      A[1] = (T(2.) - gamma) * nVel[0] + U_k;
      A[2] = vel[0] * nV[1] - km1 * vel[1] * nV[0];
      A[3] = vel[0] * nV[2] - km1 * vel[2] * nV[0];
      A[4] = km1 * nV[0];
      break;
    case 2:
      A[0] = -vel[1] * (nVel[0] + nVel[2]) + nV[1] * (km1 * vsh - vel[1] * vel[1]);
      A[1] = -km1 * vel[0] * nV[1] + vel[1] * nV[0];
      A[2] = (T(2.) - gamma) * nVel[1] + U_k;
      A[3] = vel[1] * nV[2] - km1 * vel[2] * nV[1];
      A[4] = km1 * nV[1];
      break;
    case 3:
      A[0] = -vel[2] * (nVel[0] + nVel[1]) + nV[2] * (km1 * vsh - vel[2] * vel[2]);
      A[1] = -km1 * vel[0] * nV[2] + vel[2] * nV[0];
      A[2] = -km1 * vel[1] * nV[2] + vel[2] * nV[1];
      A[3] = (T(2.) - gamma) * nVel[2] + U_k;
      A[4] = km1 * nV[2];
      break;
    default: {
      // c2: the square of c = sqrt(gamma p / rho) (the reference squares the root), ikm1 = 1 / (gamma - 1)
      A[0] = U_k * ((gamma - T(2.)) * vsh - c2 * ikm1);
      A[1] = c2 * ikm1 * nV[0] - km1 * vel[0] * (nVel[1] + nVel[2]) - (km1 * vel[0] * vel[0] - vsh) * nV[0];
      A[2] = c2 * ikm1 * nV[1] - km1 * vel[1] * (nVel[0] + nVel[2]) - (km1 * vel[1] * vel[1] - vsh) * nV[1];
      A[3] = c2 * ikm1 * nV[2] - km1 * vel[2] * (nVel[0] + nVel[1]) - (km1 * vel[2] * vel[2] - vsh) * nV[2];
      A[4] = gamma * U_k;
    } break;
  }
}

// calcEulerFluxMatrices_Roe (UgpWithCvCompFlow.cpp:3382-3559), row by row.  The reference
// forms the dissipation matrix as the product P |Lambda| P^-1 (calcPMatrix, calcInvPMatrix);
// here it is the same matrix written as the rank-two update of |lambda_1| I that the
// reference's own Roe flux applies to the state jump (calcEulerFlux_Roe,
// UgpWithCvCompFlow.cpp:3339-3378): |A| = l1 I + r (a3 (g-1)/c^2 g - a2/c m)^T + s (a2 (g-1)/c g - a3 m)^T
// with r = (1, v, H), s = (0, n, v.n), g = (|v|^2/2, -v, 1), m = (v.n, -n, 0), H = c^2/(g-1) + |v|^2/2,
// a2 = (|vn+c| - |vn-c|)/2, a3 = (|vn+c| + |vn-c|)/2 - |vn|, for the Roe state (v, c) of the
// reference's matrices.  Equal to the reference's product to rounding, without its 25-entry
// P^-1 and 125-term product (and closer to the exact matrix: the product loses digits to
// cancellation near sonic faces).
template <typename T, typename Emit>
__device__ __forceinline__ void roe_rows(const FStateT<T>& L, const FStateT<T>& R, T area, const T nV[3],
                                         Emit&& emit) {
  const T uLuL = dot3(L.u, L.u), uRuR = dot3(R.u, R.u);
  const T Rrho = sqrt(R.rho / L.rho);
  const T tmp = T(1.0) / (T(1.0) + Rrho);
  const T v[3] = {tmp * (L.u[0] + R.u[0] * Rrho), tmp * (L.u[1] + R.u[1] * Rrho), tmp * (L.u[2] + R.u[2] * Rrho)};
  const T uRoe = dot3(v, nV);
  // gamma p / rho of each side: in the Roe sound speed and (rooted and squared) in calcJacobianA
  const T gpL = L.gam * L.p / L.rho, gpR = R.gam * R.p / R.rho;
  const T gpr = tmp * ((gpL + T(0.5) * (L.gam - T(1.0)) * uLuL) + (gpR + T(0.5) * (R.gam - T(1.0)) * uRuR) * Rrho);
  const T c = sqrt(gpr - ((L.gam + R.gam) * T(0.5) - T(1.0)) * T(0.5) * dot3(v, v));
  const T gamma = T(0.5) * (L.gam + R.gam);
  const T km1 = gamma - T(1.0), ikm1 = T(1.0) / km1;
  const T cL = sqrt(gpL), cR = sqrt(gpR), c2L = cL * cL, c2R = cR * cR;
  const T c2 = c * c, vS = dot3(v, v), ic = T(1.0) / c;
  const T l1 = fabs(uRoe), l4 = fabs(uRoe + c), l5 = fabs(uRoe - c);
  const T a2 = T(0.5) * (l4 - l5), a3 = T(0.5) * (l4 + l5) - l1;
  const T hA = c2 * ikm1 + T(0.5) * vS;
  const T cgr = a3 * km1 * ic * ic, cmr = -a2 * ic, cgs = a2 * km1 * ic, cms = -a3;
  const T g[5] = {T(0.5) * vS, -v[0], -v[1], -v[2], T(1.0)};
  const T mv[5] = {uRoe, -nV[0], -nV[1], -nV[2], T(0.0)};
  T wr[5], ws[5];
  for (int j = 0; j < 5; j++) {
    wr[j] = cgr * g[j] + cmr * mv[j];
    ws[j] = cgs * g[j] + cms * mv[j];
  }
  const T rv[5] = {T(1.0), v[0], v[1], v[2], hA};
  const T sv[5] = {T(0.0), nV[0], nV[1], nV[2], uRoe};
  const T nA[3] = {nV[0] * area, nV[1] * area, nV[2] * area};
#pragma unroll
  for (int i = 0; i < 5; i++) {
    T aL[5], aR[5];
    jacobian_A_row(aL, i, L.u, c2L, ikm1, nA, gamma);
    jacobian_A_row(aR, i, R.u, c2R, ikm1, nA, gamma);
#pragma unroll
    for (int j = 0; j < 5; j++) {
      const T pm = rv[i] * wr[j] + sv[i] * ws[j] + (i == j ? l1 : T(0.0));
      aL[j] = T(0.5) * aL[j] + T(0.5) * pm * area;
      aR[j] = T(0.5) * aR[j] - T(0.5) * pm * area;
    }
    emit(i, aL, aR);
  }
}

// calcEulerFluxMatrices_HLLC + calcSubSonicJacobeanHLLC (UgpWithCvCompFlow.cpp:242-659), row by row:
// row i of the star-side block (subsonic_jac's AS) and of the other side's (AO), then the
// product-rule terms of matrices_hllc's final loop, times the area
template <typename T, typename Emit>
__device__ __forceinline__ void hllc_rows(const FStateT<T>& L, const FStateT<T>& R, T area, const T nV[3],
                                          Emit&& emit) {
  const T unL = dot3(L.u, nV), uLuL = dot3(L.u, L.u);
  const T cL = sqrt(L.gam * L.p / L.rho);
  const T eL = (L.gam / (L.gam - T(1.0)) * L.p / L.rho + T(0.5) * uLuL) * L.rho - L.p;
  const T unR = dot3(R.u, nV), uRuR = dot3(R.u, R.u);
  const T cR = sqrt(R.gam * R.p / R.rho);
  const T eR = (R.gam / (R.gam - T(1.0)) * R.p / R.rho + T(0.5) * uRuR) * R.rho - R.p;
  const T Rrho = sqrt(R.rho / L.rho);
  const T tmp = T(1.0) / (T(1.0) + Rrho);
  const T vr[3] = {tmp * (L.u[0] + R.u[0] * Rrho), tmp * (L.u[1] + R.u[1] * Rrho), tmp * (L.u[2] + R.u[2] * Rrho)};
  const T uRoe = dot3(vr, nV);
  const T gpr = tmp * ((L.gam * L.p / L.rho + T(0.5) * (L.gam - T(1.0)) * uLuL) +
                       (R.gam * R.p / R.rho + T(0.5) * (R.gam - T(1.0)) * uRuR) * Rrho);
  const T cRoe = sqrt(gpr - ((L.gam + R.gam) * T(0.5) - T(1.0)) * T(0.5) * dot3(vr, vr));
  const T sL = fmin(uRoe - cRoe, unL - cL);
  const T sR = fmax(uRoe + cRoe, unR + cR);
  const T sM = (L.p - R.p - L.rho * unL * (sL - unL) + R.rho * unR * (sR - unR)) /
               (R.rho * (sR - unR) - L.rho * (sL - unL));
  const T pStar = R.rho * (unR - sR) * (unR - sM) + R.p;
  const T gmean = T(0.5) * (L.gam + R.gam);
  if ((sM >= T(0.0) && sL > T(0.0)) || (sM < T(0.0) && sR < T(0.0))) {
    // supersonic: the flux depends on one side only
    const bool left = sM >= T(0.0);
    const T Su[3] = {left ? L.u[0] : R.u[0], left ? L.u[1] : R.u[1], left ? L.u[2] : R.u[2]};
    const T Sp = left ? L.p : R.p, Srho = left ? L.rho : R.rho;
    const T nA[3] = {nV[0] * area, nV[1] * area, nV[2] * area};
#pragma unroll
    for (int i = 0; i < 5; i++) {
      T aj[5], az[5] = {T(0.0), T(0.0), T(0.0), T(0.0), T(0.0)};
      const T cS = sqrt(gmean * Sp / Srho);
      jacobian_A_row(aj, i, Su, cS * cS, T(1.0) / (gmean - T(1.0)), nA, gmean);
      if (left) emit(i, aj, az);
      else emit(i, az, aj);
    }
    return;
  }
  const bool left = sM >= T(0.0);  // star state of the left (sM >= 0) or right wave
  // the star side's values as scalars (no reference to one of two structs: they stay in registers)
  const T uS[3] = {left ? L.u[0] : R.u[0], left ? L.u[1] : R.u[1], left ? L.u[2] : R.u[2]};
  const T pS_ = left ? L.p : R.p, rhoS = left ? L.rho : R.rho;
  const T unS = left ? unL : unR, eS = left ? eL : eR, sS = left ? sL : sR;
  const T qS = unS, psiS = left ? uLuL : uRuR;
  const T inv = T(1.0) / (sS - sM);
  const T sSmu = sS - unS;
  const T rhoSt = rhoS * sSmu * inv;
  T rhouSt[3];
  for (int i = 0; i < 3; i++) rhouSt[i] = (rhoS * uS[i] * sSmu + (pStar - pS_) * nV[i]) * inv;
  const T eSt = (sSmu * eS - pS_ * unS + pStar * sM) * inv;
  const T invrhotld = T(1.0) / (R.rho * (sR - unR) - L.rho * (sL - unL));
  T dSMdUL[5], dSMdUR[5], dpsdUL[5], dpsdUR[5];
  {
    const T g1 = L.gam - T(1.0);
    dSMdUL[0] = -unL * unL + uLuL * g1 / T(2.0) + sM * sL;
    for (int i = 0; i < 3; i++) dSMdUL[1 + i] = nV[i] * (T(2.0) * unL - sL - sM) - g1 * L.u[i];
    dSMdUL[4] = g1;
    for (int i = 0; i < 5; i++) {
      dSMdUL[i] *= invrhotld;
      dpsdUL[i] = R.rho * (sR - unR) * dSMdUL[i];
    }
  }
  {
    const T g1 = R.gam - T(1.0);
    dSMdUR[0] = unR * unR - uRuR * g1 / T(2.0) - sM * sR;
    for (int i = 0; i < 3; i++) dSMdUR[1 + i] = -nV[i] * (T(2.0) * unR - sR - sM) + g1 * R.u[i];
    dSMdUR[4] = -g1;
    for (int i = 0; i < 5; i++) {
      dSMdUR[i] *= invrhotld;
      dpsdUR[i] = L.rho * (sL - unL) * dSMdUR[i];
    }
  }
  // the star side's and the other side's derivatives, selected value by value
  T dSMdS[5], dSMdO[5], dpsdS[5], dpsdO[5];
  for (int j = 0; j < 5; j++) {
    dSMdS[j] = left ? dSMdUL[j] : dSMdUR[j];
    dSMdO[j] = left ? dSMdUR[j] : dSMdUL[j];
    dpsdS[j] = left ? dpsdUL[j] : dpsdUR[j];
    dpsdO[j] = left ? dpsdUR[j] : dpsdUL[j];
  }
  const T gamma = gmean, gm1 = gamma - T(1.0);
  const T om = T(1.0) / (sS - sM);
  const T SS = sS, SM = sM;
#pragma unroll
  for (int i = 0; i < 5; i++) {
    T as[5], ao[5];
    // row i of subsonic_jac's AS (star side) and AO (other side)
    if (i == 0) {
      as[0] = SS + rhoSt * dSMdS[0];
      as[1] = -nV[0] + rhoSt * dSMdS[1];
      as[2] = -nV[1] + rhoSt * dSMdS[2];
      as[3] = -nV[2] + rhoSt * dSMdS[3];
      as[4] = +rhoSt * dSMdS[4];
      for (int j = 0; j < 5; j++) ao[j] = om * rhoSt * dSMdO[j];
    } else if (i < 4) {
      const int r = i - 1;
      as[0] = qS * uS[r] - nV[r] * psiS * gm1 / T(2.0) + nV[r] * dpsdS[0] + rhouSt[r] * dSMdS[0];
      for (int k = 0; k < 3; k++) {
        T base = (k == r) ? (SS - qS + nV[r] * (gamma - T(2.0)) * uS[r]) : (-uS[r] * nV[k] + nV[r] * gm1 * uS[k]);
        as[1 + k] = base + nV[r] * dpsdS[1 + k] + rhouSt[r] * dSMdS[1 + k];
      }
      as[4] = -gm1 * nV[r] + nV[r] * dpsdS[4] + rhouSt[r] * dSMdS[4];
      for (int j = 0; j < 5; j++) ao[j] = om * (nV[r] * dpsdO[j] + rhouSt[r] * dSMdO[j]);
    } else {
      as[0] = qS * (eS + pS_) / rhoS - qS * psiS * (gamma - T(1.0)) / T(2.0) + SM * dpsdS[0] +
              (pStar + eSt) * dSMdS[0];
      for (int k = 0; k < 3; k++)
        as[1 + k] = -nV[k] * (eS + pS_) / rhoS + gm1 * uS[k] * qS + SM * dpsdS[1 + k] + (pStar + eSt) * dSMdS[1 + k];
      as[4] = SS - qS * gamma + SM * dpsdS[4] + (pStar + eSt) * dSMdS[4];
      for (int j = 0; j < 5; j++) ao[j] = om * (dpsdO[j] * SM + (pStar + eSt) * dSMdO[j]);
    }
    for (int j = 0; j < 5; j++) as[j] *= om;
    // matrices_hllc's final loop on both sides: side 0 is A_L (its own dSMdUL / dpsdUL)
    T aL[5], aR[5];
    for (int j = 0; j < 5; j++) {
      const T AL = left ? as[j] : ao[j], AR = left ? ao[j] : as[j];
      if (i == 0) {
        aL[j] = AL * sM + dSMdUL[j] * rhoSt;
        aR[j] = AR * sM + dSMdUR[j] * rhoSt;
      } else if (i < 4) {
        aL[j] = AL * sM + dSMdUL[j] * rhouSt[i - 1] + dpsdUL[j] * nV[i - 1];
        aR[j] = AR * sM + dSMdUR[j] * rhouSt[i - 1] + dpsdUR[j] * nV[i - 1];
      } else {
        aL[j] = (AL + dpsdUL[j]) * sM + (eSt + pStar) * dSMdUL[j];
        aR[j] = (AR + dpsdUR[j]) * sM + (eSt + pStar) * dSMdUR[j];
      }
      aL[j] *= area;
      aR[j] *= area;
    }
    emit(i, aL, aR);
  }
}

// the face matrices of KIND row by row; HAENEL and AUSMDV form both matrices whole first
template <int KIND, typename T, typename Emit>
__device__ __forceinline__ void euler_rows_t(const FStateT<T>& L, const FStateT<T>& R, T area, const T nV[3], int fo,
                                             Emit&& emit) {
  if (KIND == 1) {
    roe_rows<T>(L, R, area, nV, emit);
  } else if (KIND == 3 || KIND == 4) {
    T AL[25], AR[25];
    euler_matrices_t<KIND, T>(AL, AR, L, R, area, nV, fo);
#pragma unroll
    for (int i = 0; i < 5; i++) emit(i, AL + 5 * i, AR + 5 * i);
  } else {
    hllc_rows<T>(L, R, area, nV, emit);  // HLLC; AUSM and JST take the HLLC matrices
  }
}

// The viscous matrices of one side of a face (visc_jac_add), reduced to the
// terms each row adds: rows 1-3 get a[r] in column 0 and b on the diagonal,
// row 4 gets w4[0..4].  Same expressions as visc_jac_add.
template <typename T>
struct VJacRows {
  T a[3], b, w4[5];
};

template <typename T>
__device__ __forceinline__ VJacRows<T> vjac_rows(int side, const VFace& vf, const VSide& s, const double* u_fa) {
  const T mm = (T)(vf.mul + vf.mut), aos = (T)vf.aos, area = (T)vf.area, keff = (T)vf.keff;
  const T tau[3] = {(T)vf.tau[0], (T)vf.tau[1], (T)vf.tau[2]};
  const T uf[3] = {(T)u_fa[0], (T)u_fa[1], (T)u_fa[2]};
  const T rho = (T)s.rho, hh = (T)s.h, RR = (T)s.R, TT = (T)s.T, gam = (T)s.gam;
  const T u[3] = {(T)s.u[0], (T)s.u[1], (T)s.u[2]};
  const T d = (side == 0) ? -mm * aos * area : mm * aos * area;
  const T f44 = (side == 0) ? -area * keff * aos : area * keff * aos;
  const T f4[3] = {area * tau[0] * T(0.5) + uf[0] * d, area * tau[1] * T(0.5) + uf[1] * d,
                   area * tau[2] * T(0.5) + uf[2] * d};
  const T ir = T(1.0) / rho;
  const T uq0[3] = {-u[0] * ir, -u[1] * ir, -u[2] * ir};
  const T uq40 = gam * ir * (-hh + RR * TT + T(0.5) * dot3(u, u));
  VJacRows<T> o;
  for (int r = 0; r < 3; r++) o.a[r] = d * uq0[r];
  o.b = d * ir;
  o.w4[0] = f4[0] * uq0[0] + f4[1] * uq0[1] + f4[2] * uq0[2] + f44 * uq40;
  for (int k = 0; k < 3; k++) o.w4[1 + k] = f4[k] * ir + f44 * (-gam * u[k] * ir);
  o.w4[4] = f44 * (gam * ir);
  return o;
}

// acc (row i of a block: a T* or a StridedBlock<T>) += sgn x row i of the side's viscous matrix
template <typename T, typename Acc>
__device__ __forceinline__ void vjac_row_add(Acc acc, int i, T sgn, const VJacRows<T>& v) {
  if (i >= 1 && i <= 3) {
    acc[0] += sgn * v.a[i - 1];
    acc[i] += sgn * v.b;
  } else if (i == 4) {
    for (int k = 0; k < 5; k++) acc[k] += sgn * v.w4[k];
  }
}

}  // namespace jg
