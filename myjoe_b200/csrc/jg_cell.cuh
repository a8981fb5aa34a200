// jg_cell.cuh -- per-cell and per-face helpers shared by the face-loop kernels:
// face normals, cell-centre states, second-order reconstruction, the viscous
// side state, the sliced-ELL index of an off-diagonal block entry, the 5x5
// block inverse and the AUSMDV face options.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "jg_flux.cuh"
#include "jg_internal.h"

namespace jg {

// an L1 prefetch of the cache line holding p (a hint: no registers held, no wait)
__device__ __forceinline__ void prefetch_l1(const void* p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

// the face loop's reads of a neighbour cell c, prefetched a face ahead: its state, primitives,
// centre, gradients (and the viscous gradients)
__device__ __forceinline__ void prefetch_cell(const State& st, const Mesh& m, int c, bool visc) {
  prefetch_l1(&st.q[5 * c]);
  prefetch_l1(&st.prim[8 * c]);
  prefetch_l1(&m.x_cv[3 * c]);
  prefetch_l1(&st.grho[3 * c]);
  prefetch_l1(&st.gp[3 * c]);
  prefetch_l1(&st.gu[9 * c]);
  if (visc) {
    prefetch_l1(&st.guv[9 * c]);
    prefetch_l1(&st.gh[3 * c]);
  }
}

// the Jacobian kernel's reads of a neighbour cell c: its state and primitives (and the viscous
// gradient the viscous matrices' stress needs)
__device__ __forceinline__ void prefetch_cell_jac(const State& st, int c, bool visc) {
  prefetch_l1(&st.q[5 * c]);
  prefetch_l1(&st.prim[8 * c]);
  if (visc) prefetch_l1(&st.guv[9 * c]);
}

// sourceHook / sourceHookCoupled (JoeWithModels.h:111-152): gravity in cell c's momentum and
// energy rows of the residual (after the fluxes) ...
__device__ __forceinline__ void gravity_rhs(const Params& p, const Mesh& m, const State& st, int c, double* rhs) {
  if (!p.has_gravity) return;
  const double vol = m.vol[c], rho = st.q[5 * c];
  const double* ru = &st.q[5 * c + 1];
  for (int i = 0; i < 3; i++) rhs[1 + i] += vol * rho * p.gravity[i];
  rhs[4] += vol * (p.gravity[0] * ru[0] + p.gravity[1] * ru[1] + p.gravity[2] * ru[2]);
}
// ... and in its diagonal block (B x B row-major, after the flux matrices)
template <int B>
__device__ __forceinline__ void gravity_diag(const Params& p, const Mesh& m, int c, double* Dm) {
  if (!p.has_gravity) return;
  const double vol = m.vol[c];
  for (int i = 0; i < 3; i++) {
    Dm[B * (1 + i)] -= vol * p.gravity[i];
    Dm[B * 4 + 1 + i] -= vol * p.gravity[i];
  }
}

// the unit normal and area of face f (normVec3d of fa_normal, formed once per mesh by k_face_geo)
__device__ __forceinline__ void unit_normal(const Mesh& m, int f, double nV[3], double& area) {
  const double* u = &m.fa_u[4 * f];
  for (int i = 0; i < 3; i++) nV[i] = u[i];
  area = u[3];
}

// the unit vector from an internal face's cvofa[f][0] centre to its cvofa[f][1] centre and its
// length (the viscous flux's sVec and smag, JoeWithModels.cpp:3626-3629)
__device__ __forceinline__ void cell_to_cell(const Mesh& m, int f, double sV[3], double& smag) {
  const double* s = &m.fa_s[4 * (f - m.nfa_b)];
  for (int i = 0; i < 3; i++) sV[i] = s[i];
  smag = s[3];
}

__device__ __forceinline__ FState cell_fstate(const Params& p, const State& st, int c) {
  FState s;
  s.rho = st.q[5 * c];
  for (int i = 0; i < 3; i++) s.u[i] = st.prim[8 * c + i];
  s.p = st.prim[8 * c + 3];
  s.gam = p.gamma;
  s.h = st.prim[8 * c + 5];
  return s;
}

// second-order reconstruction at x_fa with the first-order fallback, JoeWithModels.cpp:2832-2921;
// every input is loaded before the fallback test, so the gathers are in flight together
__device__ __forceinline__ FState recon(const Mesh& m, const Params& p, const State& st, int c, int f) {
  FState s = cell_fstate(p, st, c);
  if (!p.second_order) return s;
  double r0[3], gr[3], gp[3], gu[9];
  for (int i = 0; i < 3; i++) {
    r0[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
    gr[i] = st.grho[3 * c + i];
    gp[i] = st.gp[3 * c + i];
  }
  for (int i = 0; i < 9; i++) gu[i] = st.gu[9 * c + i];
  double rr = s.rho + dot3(r0, gr);
  double pp = s.p + dot3(r0, gp);
  if ((pp <= 0.0) || (rr <= 0.0)) return s;  // first order: the cell's own h is calcThermoProp_p of (p, rho)
  s.rho = rr;
  s.p = pp;
  for (int i = 0; i < 3; i++) s.u[i] += dot3(r0, &gu[3 * i]);
  const double T = pp / (rr * p.R);  // calcThermoProp_p at the face
  s.h = p.cp * T;
  return s;
}

__device__ __forceinline__ VSide cell_vside(const Params& p, const State& st, int c) {
  VSide v;
  v.rho = st.q[5 * c];
  for (int i = 0; i < 3; i++) v.u[i] = st.prim[8 * c + i];
  v.h = st.prim[8 * c + 5];
  v.T = st.prim[8 * c + 4];
  v.R = p.R;
  v.gam = p.gamma;
  v.gu = &st.guv[9 * c];
  v.gh = &st.gh[3 * c];
  return v;
}

template <typename BT>
__device__ __forceinline__ size_t ell_index(const Mesh& m, int c, int col, int e) {
  int slice = c / SLICE, lane = c % SLICE;
  return ((size_t)(m.ell_off[slice] + col) * 25 + e) * SLICE + lane;
}

// 5x5 LU without pivoting + inverse, ludeco / luinv (UgpWithCv.cpp:2489-2577); the loops have
// constant bounds so that they unroll and both blocks stay in registers
__device__ __forceinline__ void block_inverse(double* A, double* Ai) {
#pragma unroll
  for (int jc = 1; jc < 5; jc++) A[jc] /= A[0];
#pragma unroll
  for (int jrjc = 1; jrjc < 5; jrjc++) {
#pragma unroll
    for (int jr = jrjc; jr < 5; jr++) {
      double sum = A[5 * jr + jrjc];
#pragma unroll
      for (int jm = 0; jm < jrjc; jm++) sum -= A[5 * jr + jm] * A[5 * jm + jrjc];
      A[5 * jr + jrjc] = sum;
    }
    if (jrjc < 4) {
#pragma unroll
      for (int jc = jrjc + 1; jc < 5; jc++) {
        double sum = A[5 * jrjc + jc];
#pragma unroll
        for (int jm = 0; jm < jrjc; jm++) sum -= A[5 * jrjc + jm] * A[5 * jm + jc];
        A[5 * jrjc + jc] = sum / A[5 * jrjc + jrjc];
      }
    }
  }
#pragma unroll
  for (int col = 0; col < 5; col++) {
    double cv[5];
#pragma unroll
    for (int i = 0; i < 5; i++) cv[i] = (i == col) ? 1.0 : 0.0;
    cv[0] = cv[0] / A[0];
#pragma unroll
    for (int jr = 1; jr < 5; jr++) {
      double sum = cv[jr];
#pragma unroll
      for (int jm = 0; jm < jr; jm++) sum -= A[5 * jr + jm] * cv[jm];
      cv[jr] = sum / A[5 * jr + jr];
    }
#pragma unroll
    for (int jr = 3; jr >= 0; jr--) {
      double sum = cv[jr];
#pragma unroll
      for (int jm = jr + 1; jm < 5; jm++) sum -= A[5 * jr + jm] * cv[jm];
      cv[jr] = sum;
    }
#pragma unroll
    for (int i = 0; i < 5; i++) Ai[5 * i + col] = cv[i];
  }
}

// the AUSMDV options of an internal face (JoeWithModels.cpp:2933-2957): the shock fix where the
// cells' flags add up past the threshold, sonic faces included (SHOCKFIX_ACROSS_SHOCK is defined,
// JoeWithModels.cpp:4)
template <int KIND>
__device__ __forceinline__ int face_opts(const Params& p, const State& st, int c0, int c1) {
  if (KIND != 4) return 0;
  int fo = p.ausm_type | (p.entropy_fix ? FO_EFIX : 0);
  if (p.shock_fix != JG_SHOCK_FIX_NONE && double(st.shock_flag[c0]) + double(st.shock_flag[c1]) > p.shock_flag_sum)
    fo |= p.shock_fix == JG_SHOCK_FIX_HAENEL ? FO_HAENEL : FO_ALPHA_LR;
  return fo;
}

// boundary faces: AUSMDV without the shock fix (JoeWithModels.cpp:3149-3153)
template <int KIND>
__device__ __forceinline__ int bnd_opts(const Params& p) {
  return KIND == 4 ? (p.ausm_type | (p.entropy_fix ? FO_EFIX : 0)) : 0;
}

}  // namespace jg
