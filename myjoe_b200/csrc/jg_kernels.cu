// jg_kernels.cu -- sm_100a kernels of the implicit finite-volume iteration.
//
// One thread per cell for every cell pass.  The face loop is cell-centric:
// each cell walks its faces, evaluates every face flux in the face's own
// orientation (cvofa[f][0] -> cvofa[f][1]) so that the two cells of a face
// obtain bit-identical fluxes, and owns its residual, its diagonal block and
// its row of off-diagonal blocks.  No atomics, no colouring, deterministic.
#include <cuda_runtime.h>
#include <math.h>

#include "jg_cell.cuh"
#include "jg_flux.cuh"
#include "jg_internal.h"

namespace jg {

int grid_for(long n, int block) { return (int)((n + block - 1) / block); }

// ---------------------------------------------------------------------------
// thermodynamics helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double mu_law(const Params& p, double T) {
  // calcMuLam / calcMaterialProperties, src/joe/UgpWithCvCompFlow.h:1601-1621, 1701-1753
  if (p.mu_mode == JG_MU_SUTHERLAND) {
    const double t = T / p.SL_T;  // pow(t, 1.5) as t sqrt(t)
    return p.mu_ref * (t * sqrt(t)) * (p.SL_T + p.SL_S) / (T + p.SL_S);
  }
  return p.mu_ref * pow(T / p.T_ref, p.mu_pow);
}

// calcStateVariables, UgpWithCvCompFlow.h:1662-1694: a non-positive pressure keeps the old one
__device__ __forceinline__ void state_from_q(const Params& p, const double* q, double* prim, int* err,
                                             double kinecv = 0.0) {
  double r = q[0];
  double ru[3] = {q[1], q[2], q[3]};
  double u[3] = {ru[0] / r, ru[1] / r, ru[2] / r};
  double pr = (p.gamma - 1.0) * (q[4] - 0.5 * dot3(ru, ru) / r - r * kinecv);
  double pp = prim[3];
  if (pr > 0.0) pp = pr;
  if (!(r > 0.0) || !(pp > 0.0)) atomicOr(err, 1);
  double T = pp / (r * p.R);
  prim[0] = u[0];
  prim[1] = u[1];
  prim[2] = u[2];
  prim[3] = pp;
  prim[4] = T;
  prim[5] = p.cp * T;
  prim[6] = sqrt(p.gamma * pp / r);
}

// state errors are recorded per case (a batch keeps going); a frozen case keeps its primitives
__global__ void k_state(Mesh m, Params p, State st) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  const int k = m.case_of[c];
  if (!st.case_active[k]) return;
  double q[5], prim[8];
  for (int i = 0; i < 5; i++) q[i] = st.q[5 * c + i];
  for (int i = 0; i < 8; i++) prim[i] = st.prim[8 * c + i];
  state_from_q(p, q, prim, st.case_err + k, st.kine ? st.kine[c] : 0.0);
  for (int i = 0; i < 8; i++) st.prim[8 * c + i] = prim[i];
}

// Q += dq (runBackwardEuler, JoeWithModels.cpp:1028-1035), then the new state.
// Cells of a frozen (retired) case keep their state; state errors are
// recorded per case.
__global__ void k_update_state(Mesh m, Params p, State st) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  int k = m.case_of[c];
  if (!st.case_active[k]) return;
  double q[5], prim[8];
  for (int i = 0; i < 5; i++) q[i] = st.q[5 * c + i] + st.dq[5 * c + i];
  for (int i = 0; i < 5; i++) st.q[5 * c + i] = q[i];
  for (int i = 0; i < 8; i++) prim[i] = st.prim[8 * c + i];
  state_from_q(p, q, prim, st.case_err + k);
  for (int i = 0; i < 8; i++) st.prim[8 * c + i] = prim[i];
}

// the same with the relaxation's result x ([5][N], matrix precision) in place of dq = (double) x
template <typename BT>
__global__ void k_update_state_x(Mesh m, Params p, State st, const BT* __restrict__ x) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  int k = m.case_of[c];
  if (!st.case_active[k]) return;
  double q[5], prim[8];
  for (int i = 0; i < 5; i++) q[i] = st.q[5 * c + i] + (double)x[(size_t)i * m.ncv + c];
  for (int i = 0; i < 5; i++) st.q[5 * c + i] = q[i];
  for (int i = 0; i < 8; i++) prim[i] = st.prim[8 * c + i];
  state_from_q(p, q, prim, st.case_err + k);
  for (int i = 0; i < 8; i++) st.prim[8 * c + i] = prim[i];
}

// calcMaterialProperties on internal faces: distance-weighted face temperature
__device__ __forceinline__ void face_props(const Mesh& m, const Params& p, State& st, int f) {
  int c0 = m.cvofa[2 * f], c1 = m.cvofa[2 * f + 1];
  double d0[3], d1[3];
  for (int i = 0; i < 3; i++) {
    d0[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c0 + i];
    d1[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c1 + i];
  }
  double w0 = sqrt(dot3(d0, d0)), w1 = sqrt(dot3(d1, d1));
  double T = (w1 * st.prim[8 * c0 + 4] + w0 * st.prim[8 * c1 + 4]) / (w0 + w1);
  double mu = mu_law(p, T);
  st.mul_fa[f] = mu;
  st.lam_fa[f] = mu / p.Pr;
}
__global__ void k_face_props(Mesh m, Params p, State st) {
  int f = m.nfa_b + blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nfa) return;
  face_props(m, p, st, f);
}

// setBC + ComputeBCProperties_T/H + the EOS density, JoeWithModels.cpp:3857-4300,
// UgpWithCvCompFlow.h:1783-1839, for boundary face f.
__device__ __forceinline__ void bc_face(const Mesh& m, const Params& p, State& st, int f) {
  const DevZone z = m.zones[m.bzone[f]];
  int c0 = m.cvofa[2 * f];
  const double* pc = &st.prim[8 * c0];
  const double* qc = &st.q[5 * c0];
  double nV[3], area;
  unit_normal(m, f, nV, area);
  double T = 0.0, v[3] = {0.0, 0.0, 0.0}, pb = 0.0, h;
  double rho_ff = 0.0;
  double cp = p.cp;
  switch (z.kind) {
    case JG_BC_CBC: {
      if (dot3(z.v, nV) > 0.0) {
        double un = dot3(pc, nV);
        double mach = fabs(un) / pc[6];
        T = pc[4];
        for (int i = 0; i < 3; i++) v[i] = pc[i];
        pb = (mach >= 1.0) ? pc[3] : z.v[4];
      } else {
        T = z.v[3];
        for (int i = 0; i < 3; i++) v[i] = z.v[i];
        pb = z.v[4];
      }
    } break;
    case JG_BC_CBC_SUBSONIC_INLET: {
      double r = qc[0];
      double u[3] = {qc[1] / r, qc[2] / r, qc[3] / r};
      double vm = sqrt(dot3(u, u));
      for (int i = 0; i < 3; i++) v[i] = z.v[i] * vm;
      double Ttot = z.v[3], ptot = z.v[4];
      double htot = cp * Ttot;               // ComputeBCProperties_T with T = Ttot
      double hs = htot - 0.5 * dot3(v, v);   // static enthalpy
      T = hs * (p.gamma - 1.0) / (p.gamma * p.R);  // ComputeBCProperties_H
      pb = ptot * pow(T / Ttot, p.gamma / (p.gamma - 1.0));
      h = hs;
    } break;
    case JG_BC_CBC_SUBSONIC_OUTLET: {
      pb = z.v[0];
      for (int i = 0; i < 3; i++) v[i] = qc[1 + i] / qc[0];
      T = pc[4];
    } break;
    case JG_BC_SYMMETRY: {
      double un = dot3(nV, pc);
      for (int i = 0; i < 3; i++) v[i] = pc[i] - 1.0 * un * nV[i];
      T = pc[4];
      pb = pc[3];
    } break;
    case JG_BC_NEUMANN: {
      for (int i = 0; i < 3; i++) v[i] = qc[1 + i] / qc[0];
      T = pc[4];
      pb = pc[3];
    } break;
    case JG_BC_WALL: {
      T = (z.v[0] > 0.0) ? z.v[0] : pc[4];
      pb = pc[3];
    } break;
    case JG_BC_FARFIELD: {
      double gb = z.v[5], pbc = z.v[3], rbc = z.v[4];
      double gm1 = gb - 1.0, ovgm1 = 1.0 / gm1;
      double c_bc = sqrt(gb * pbc / rbc);
      double s_bc = pow(rbc, gb) / pbc;
      double qn_bc = dot3(nV, z.v);
      double vn_bc = qn_bc;
      double qne = dot3(nV, pc);
      double r0 = qc[0];
      double ce = sqrt(p.gamma * pc[3] / r0);
      double ac1 = (vn_bc > -c_bc) ? qne + 2.0 * ovgm1 * ce : qn_bc + 2.0 * ovgm1 * c_bc;
      double ac2 = (vn_bc > c_bc) ? qne - 2.0 * ovgm1 * ce : qn_bc - 2.0 * ovgm1 * c_bc;
      double qnf = 0.5 * (ac1 + ac2);
      double cf = 0.25 * (ac1 - ac2) * gm1;
      double sf;
      if (vn_bc > 0) {
        for (int i = 0; i < 3; i++) v[i] = pc[i] + (qnf - qne) * nV[i];
        sf = pow(r0, p.gamma) / pc[3];
      } else {
        for (int i = 0; i < 3; i++) v[i] = z.v[i] + (qnf - qn_bc) * nV[i];
        sf = s_bc;
      }
      rho_ff = pow((sf * cf * cf / p.gamma), ovgm1);
      pb = rho_ff * cf * cf / p.gamma;
      T = pb / (p.R * rho_ff);
    } break;
    default:
      atomicOr(st.err, 2);
      break;
  }
  if (z.kind != JG_BC_CBC_SUBSONIC_INLET) h = cp * T;
  double* b = &st.bfa[8 * f];
  b[0] = pb / (p.R * T);  // EOS, JoeWithModels.cpp:4291-4293
  b[1] = v[0];
  b[2] = v[1];
  b[3] = v[2];
  b[4] = pb;
  b[5] = T;
  b[6] = h;
  if (p.viscous) {
    double mu = mu_law(p, T);
    st.mul_fa[f] = mu;
    st.lam_fa[f] = mu / p.Pr;
  }
}
// one thread per boundary face
__global__ void k_bc(Mesh m, Params p, State st) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nfa_b) return;
  bc_face(m, p, st, f);
}
// both passes that follow a state update in one launch: boundary faces take setBC, internal
// faces (viscous cases) the face properties; the faces are independent
__global__ void k_faces_after_update(Mesh m, Params p, State st) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f < m.nfa_b) bc_face(m, p, st, f);
  else if (p.viscous && f < m.nfa) face_props(m, p, st, f);
}

// CFL ramp of runBackwardEuler (JoeWithModels.cpp:977-978), on the device so a
// captured step graph can be replayed: ctrl[0] = cfl, ctrl[1] = step
__global__ void k_ctrl_step(Params p, State st) {
  double step = st.ctrl[1] + 1.0;
  st.ctrl[1] = step;
  long s = (long)step;
  if ((s >= p.cfl_after) && (s % p.cfl_interval == 0) && (st.ctrl[0] < p.cfl_max)) st.ctrl[0] *= p.cfl_factor;
}

// calcDt, UgpWithCvCompFlow.cpp:5-110 (per-block minimum in st.blk)
__global__ void k_dt(Mesh m, Params p, State st, int use_ctrl, double cfl_arg) {
  __shared__ double smin[256];
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double dtc = 1.0e20;
  double cfl = use_ctrl ? st.ctrl[0] : cfl_arg;
  if (c < m.ncv && st.case_active[m.case_of[c]]) {
    if (p.ts_mode == JG_TS_DT) {
      dtc = p.dt_fixed;
    } else {
      const double* q = &st.q[5 * c];
      double r = q[0];
      double pr = st.prim[8 * c + 3];
      double cs = sqrt(p.gamma * pr / r);
      double ru[3] = {q[1], q[2], q[3]};
      double vol = m.vol[c];
      if (p.ts_method == JG_DT_MAX_BASED) {
        double lmax = 0.0;
        for (int k = m.slot_i[c]; k < m.slot_i[c + 1]; k++) {
          int f = m.slots[k].f;
          double nV[3], area;
          unit_normal(m, f, nV, area);
          double Uk = dot3(ru, nV) / r;
          double lam = (fabs(Uk) + cs) * area;
          double mut = st.mut_fa ? st.mut_fa[f] : 0.0;
          double ld = p.viscous ? 4.0 * (st.mul_fa[f] + mut) / r * area * area / vol : 0.0;
          lam = fmax(lam, ld);
          lmax = fmax(lmax, lam);
        }
        dtc = cfl * vol / lmax;
      } else {
        double lc = 0.0, ld = 0.0;
        for (int k = m.slot_i[c]; k < m.slot_i[c + 1]; k++) {
          Slot s = m.slots[k];
          double nV[3], area;
          unit_normal(m, s.f, nV, area);
          double Uk = dot3(ru, nV) / r;
          double v2 = (s.nb >= 0) ? 0.5 * (m.vol[c] + m.vol[s.nb]) : 0.5 * vol;
          if (s.nb >= 0 && s.side == 1) v2 = 0.5 * (m.vol[s.nb] + m.vol[c]);
          lc += (fabs(Uk) + cs) * area;
          double mut = st.mut_fa ? st.mut_fa[s.f] : 0.0;
          if (p.viscous) ld += area * area * ((4.0 / 3.0) * (st.mul_fa[s.f] + mut) / r) / v2;
        }
        double dconv = cfl * vol / lc;
        double dvisc = p.viscous ? 0.25 * cfl * vol / ld : 1.0e20;
        dtc = fmin(dconv, dvisc);
      }
    }
    st.local_dt[c] = dtc;
  }
  smin[threadIdx.x] = dtc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) st.blk[blockIdx.x] = smin[0];
}

__global__ void k_dt_final(Mesh m, Params p, State st, int nblk) {
  __shared__ double smin[256];
  double v = 1.0e20;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) v = fmin(v, st.blk[i]);
  smin[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) smin[threadIdx.x] = fmin(smin[threadIdx.x], smin[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) st.ctrl[2] = smin[0];
}

__global__ void k_dt_min_all(Mesh m, State st) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < m.ncv) st.local_dt[c] = st.ctrl[2];
}

// ---------------------------------------------------------------------------
// LSQ gradients + smooth Barth-Jespersen limiter, UgpWithCv.h:803-1083.
// Fields: velocity (ref = speed of sound), density, pressure, enthalpy.
// ---------------------------------------------------------------------------
// the limiter ratio of one face as a (numerator, denominator) pair: the denominator is positive
// (dp^2 + dm dp + 2 dm^2 >= 0 for every dm, dp), so the smallest ratio over a cell's faces is
// tracked by cross-multiplication and divided out once per cell (bj_min)
struct BjRatio {
  double n = 1.0, d = 1.0;
};
__device__ __forceinline__ void bj_min(BjRatio& r, double phi_c, double phifa, double pmax, double pmin, double eps2) {
  double dm = phifa - phi_c;
  double dp = ((phifa - phi_c) >= 0.0) ? pmax - phi_c : pmin - phi_c;
  const double n = dp * dp + 2.0 * dm * dp + eps2, d = dp * dp + 2 * dm * dm + dm * dp + eps2;
  if (n * r.d < r.n * d) {
    r.n = n;
    r.d = d;
  }
}

// calcCvScalarGradSDWLS / calcCvVectorGradSDWLS (UgpWithCv.h:1418-1800) for one cell.  Each quantity
// weighs its neighbours and boundary faces by 1 / (|dx|^2 (|dphi| + e)) (van Leer weight, geomWeighting
// |dx|^2, UgpWithCv.h:16-23; the velocity by |du|), so each has its own moment matrix: a first pass
// sums the four matrices, a second applies their adjugates.  e = max(EPS ref, 1e-8) for rho, p, h
// (ref = the quantity itself), EPS c for the velocity.
struct Sdwls {
  double sw[6];  // xx yy zz xy xz yz
  __device__ void add(double w, const double* dx) {
    sw[0] += w * dx[0] * dx[0];
    sw[1] += w * dx[1] * dx[1];
    sw[2] += w * dx[2] * dx[2];
    sw[3] += w * dx[0] * dx[1];
    sw[4] += w * dx[0] * dx[2];
    sw[5] += w * dx[1] * dx[2];
  }
  __device__ double denom() const {
    return 2.0 * sw[3] * sw[4] * sw[5] + sw[0] * sw[1] * sw[2] - sw[0] * sw[5] * sw[5] - sw[1] * sw[4] * sw[4] -
           sw[2] * sw[3] * sw[3];
  }
  // adjugate row j . dx
  __device__ double row(int j, const double* dx) const {
    if (j == 0)
      return (sw[1] * sw[2] - sw[5] * sw[5]) * dx[0] + (sw[4] * sw[5] - sw[3] * sw[2]) * dx[1] +
             (sw[3] * sw[5] - sw[4] * sw[1]) * dx[2];
    if (j == 1)
      return (sw[4] * sw[5] - sw[3] * sw[2]) * dx[0] + (sw[0] * sw[2] - sw[4] * sw[4]) * dx[1] +
             (sw[3] * sw[4] - sw[5] * sw[0]) * dx[2];
    return (sw[3] * sw[5] - sw[4] * sw[1]) * dx[0] + (sw[3] * sw[4] - sw[5] * sw[0]) * dx[1] +
           (sw[0] * sw[1] - sw[3] * sw[3]) * dx[2];
  }
};

// one neighbour (or boundary face) at offset dx with values (u, rho, p, h) = v: pass 0 adds to the
// moments, pass 1 to the gradients
__device__ __forceinline__ void sdwls_visit(int pass, const double* dx, const double* vc, const double* v,
                                            const double* e, Sdwls* M, const double* den, double* gu, double* gr,
                                            double* gpr, double* gh) {
  const double dist2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
  double du[3], du2 = 0.0;
  for (int i = 0; i < 3; i++) {
    du[i] = v[i] - vc[i];
    du2 += du[i] * du[i];
  }
  const double d[3] = {v[3] - vc[3], v[4] - vc[4], v[5] - vc[5]};  // rho, p, h
  const double wu = 1.0 / (dist2 * (sqrt(du2) + e[0]));
  double ws[3];
  for (int q = 0; q < 3; q++) ws[q] = 1.0 / (dist2 * (fabs(d[q]) + e[1 + q]));
  if (pass == 0) {
    M[0].add(wu, dx);
    for (int q = 0; q < 3; q++) M[1 + q].add(ws[q], dx);
    return;
  }
  for (int j = 0; j < 3; j++) {
    const double t = wu * M[0].row(j, dx) / den[0];
    for (int i = 0; i < 3; i++) gu[3 * i + j] += du[i] * t;
  }
  double* gs[3] = {gr, gpr, gh};
  for (int q = 0; q < 3; q++)
    for (int j = 0; j < 3; j++) gs[q][j] += d[q] * ws[q] * M[1 + q].row(j, dx) / den[1 + q];
}

__device__ void grad_sdwls(const Mesh& m, const Params& p, const State& st, int c, double* gu, double* gr,
                           double* gpr, double* gh) {
  const double* pc = &st.prim[8 * c];
  const double vc[6] = {pc[0], pc[1], pc[2], st.q[5 * c], pc[3], pc[5]};
  const double e[4] = {p.eps * pc[6], fmax(p.eps * vc[3], 1.0e-8), fmax(p.eps * vc[4], 1.0e-8),
                       fmax(p.eps * vc[5], 1.0e-8)};
  Sdwls M[4];
  for (int q = 0; q < 4; q++)
    for (int k = 0; k < 6; k++) M[q].sw[k] = 0.0;
  double den[4] = {0.0, 0.0, 0.0, 0.0};
  for (int j = 0; j < 9; j++) gu[j] = 0.0;
  for (int j = 0; j < 3; j++) gr[j] = gpr[j] = gh[j] = 0.0;
  for (int pass = 0; pass < 2; pass++) {
    if (pass == 1)
      for (int q = 0; q < 4; q++) den[q] = M[q].denom();
    for (int k = m.nb_i[c] + 1; k < m.nb_i[c + 1]; k++) {
      const int nb = m.nb_v[k];
      const double* pn = &st.prim[8 * nb];
      const double v[6] = {pn[0], pn[1], pn[2], st.q[5 * nb], pn[3], pn[5]};
      double dx[3];
      for (int i = 0; i < 3; i++) dx[i] = m.x_cv[3 * nb + i] - m.x_cv[3 * c + i];
      sdwls_visit(pass, dx, vc, v, e, M, den, gu, gr, gpr, gh);
    }
    for (int k = m.bf_i[c]; k < m.bf_i[c + 1]; k++) {
      const int f = m.bf_v[k];
      const double* b = &st.bfa[8 * f];
      const double v[6] = {b[1], b[2], b[3], b[0], b[4], b[6]};
      double dx[3];
      for (int i = 0; i < 3; i++) dx[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
      sdwls_visit(pass, dx, vc, v, e, M, den, gu, gr, gpr, gh);
    }
  }
}

// SCHEME: the gradient scheme (JG_GRAD_*) as a template parameter, so that each
// scheme's kernel holds only its own registers
template <int SCHEME>
__global__ void k_grad(Mesh m, Params p, State st, int do_euler, int do_visc, int visc_lim_u, int visc_lim_h,
                       int separate_guv) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv || !st.case_active[m.case_of[c]]) return;  // a frozen case keeps its arrays
  const double* pc = &st.prim[8 * c];
  double rc = st.q[5 * c];
  // raw LSQ sums: diagonal, neighbours (nbocv order), then boundary faces
  double gu[9], gr[3], gpr[3], gh[3];
  int k0 = m.nb_i[c], k1 = m.nb_i[c + 1];
  {
    double w[3] = {m.lsq[3 * k0], m.lsq[3 * k0 + 1], m.lsq[3 * k0 + 2]};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) gu[3 * i + j] = w[j] * pc[i];
    for (int j = 0; j < 3; j++) {
      gr[j] = w[j] * rc;
      gpr[j] = w[j] * pc[3];
      gh[j] = w[j] * pc[5];
    }
  }
  double umax[3], umin[3], rmax = rc, rmin = rc, pmax = pc[3], pmin = pc[3], hmax = pc[5], hmin = pc[5];
  for (int i = 0; i < 3; i++) umax[i] = umin[i] = pc[i];
  for (int k = k0 + 1; k < k1; k++) {
    int nb = m.nb_v[k];
    double w[3] = {m.lsq[3 * k], m.lsq[3 * k + 1], m.lsq[3 * k + 2]};
    const double* pn = &st.prim[8 * nb];
    double rn = st.q[5 * nb];
    for (int i = 0; i < 3; i++) {
      for (int j = 0; j < 3; j++) gu[3 * i + j] += w[j] * pn[i];
      umax[i] = fmax(umax[i], pn[i]);
      umin[i] = fmin(umin[i], pn[i]);
    }
    for (int j = 0; j < 3; j++) {
      gr[j] += w[j] * rn;
      gpr[j] += w[j] * pn[3];
      gh[j] += w[j] * pn[5];
    }
    rmax = fmax(rmax, rn); rmin = fmin(rmin, rn);
    pmax = fmax(pmax, pn[3]); pmin = fmin(pmin, pn[3]);
    hmax = fmax(hmax, pn[5]); hmin = fmin(hmin, pn[5]);
  }
  for (int k = m.bf_i[c]; k < m.bf_i[c + 1]; k++) {
    int f = m.bf_v[k];
    double w[3] = {m.blsq[3 * f], m.blsq[3 * f + 1], m.blsq[3 * f + 2]};
    const double* b = &st.bfa[8 * f];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) gu[3 * i + j] += w[j] * b[1 + i];
    for (int j = 0; j < 3; j++) {
      gr[j] += w[j] * b[0];
      gpr[j] += w[j] * b[4];
      gh[j] += w[j] * b[6];
    }
  }
  if (SCHEME == JG_GRAD_GREENGAUSS) {
    // calcCv{Scalar,Vector}GradGreenGauss (UgpWithCv.h:1091-1184, GG_WITH_DIST): the cell's internal
    // faces in face order with the distance-weighted face value, then its boundary faces, over V
    for (int j = 0; j < 9; j++) gu[j] = 0.0;
    for (int j = 0; j < 3; j++) gr[j] = gpr[j] = gh[j] = 0.0;
    for (int k = m.slot_i[c]; k < m.slot_i[c + 1]; k++) {
      const Slot s = m.slots[k];
      if (s.nb < 0) continue;
      const int f = s.f, c0 = m.cvofa[2 * f], c1 = m.cvofa[2 * f + 1];
      double d0[3], d1[3];
      for (int j = 0; j < 3; j++) {
        d0[j] = m.x_fa[3 * f + j] - m.x_cv[3 * c0 + j];
        d1[j] = m.x_fa[3 * f + j] - m.x_cv[3 * c1 + j];
      }
      const double w0 = sqrt(dot3(d0, d0)), w1 = sqrt(dot3(d1, d1));
      const double* p0 = &st.prim[8 * c0];
      const double* p1 = &st.prim[8 * c1];
      const double n[3] = {m.fa_n[3 * f], m.fa_n[3 * f + 1], m.fa_n[3 * f + 2]};
      const double fr = (w1 * st.q[5 * c0] + w0 * st.q[5 * c1]) / (w0 + w1);
      const double fp = (w1 * p0[3] + w0 * p1[3]) / (w0 + w1);
      const double fh = (w1 * p0[5] + w0 * p1[5]) / (w0 + w1);
      if (s.side == 0) {
        for (int i = 0; i < 3; i++) {
          const double fu = (w1 * p0[i] + w0 * p1[i]) / (w0 + w1);
          for (int j = 0; j < 3; j++) gu[3 * i + j] += fu * n[j];
        }
        for (int j = 0; j < 3; j++) {
          gr[j] += fr * n[j];
          gpr[j] += fp * n[j];
          gh[j] += fh * n[j];
        }
      } else {
        for (int i = 0; i < 3; i++) {
          const double fu = (w1 * p0[i] + w0 * p1[i]) / (w0 + w1);
          for (int j = 0; j < 3; j++) gu[3 * i + j] -= fu * n[j];
        }
        for (int j = 0; j < 3; j++) {
          gr[j] -= fr * n[j];
          gpr[j] -= fp * n[j];
          gh[j] -= fh * n[j];
        }
      }
    }
    for (int k = m.bf_i[c]; k < m.bf_i[c + 1]; k++) {
      const int f = m.bf_v[k];
      const double* b = &st.bfa[8 * f];
      const double n[3] = {m.fa_n[3 * f], m.fa_n[3 * f + 1], m.fa_n[3 * f + 2]};
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) gu[3 * i + j] += b[1 + i] * n[j];
      for (int j = 0; j < 3; j++) {
        gr[j] += b[0] * n[j];
        gpr[j] += b[4] * n[j];
        gh[j] += b[6] * n[j];
      }
    }
    const double V = m.vol[c];
    for (int j = 0; j < 9; j++) gu[j] /= V;
    for (int j = 0; j < 3; j++) {
      gr[j] /= V;
      gpr[j] /= V;
      gh[j] /= V;
    }
  }
  if (SCHEME == JG_GRAD_SDWLS) grad_sdwls(m, p, st, c, gu, gr, gpr, gh);
  // limiter factors over the internal faces of the cell
  double au[3] = {1.0, 1.0, 1.0}, ar = 1.0, ap = 1.0, ah = 1.0;
  const double eps = p.eps;
  // pow(x, 2.0) of the reference, as x * x
  const double vu = eps * pc[6], vr = fmax(eps * fabs(rc), 1.0e-8), vp = fmax(eps * fabs(pc[3]), 1.0e-8),
               vh = fmax(eps * fabs(pc[5]), 1.0e-8);
  const double e2u = vu * vu, e2r = vr * vr, e2p = vp * vp, e2h = vh * vh;
  bool lu[3], lr = (rmax - rmin) > 1.0e-12, lp = (pmax - pmin) > 1.0e-12, lh = (hmax - hmin) > 1.0e-12;
  for (int i = 0; i < 3; i++) lu[i] = (umax[i] - umin[i]) > 1.0e-8;
  if (p.limiter) {
    BjRatio bu[3], br, bp, bh;
    for (int k = m.slot_i[c]; k < m.slot_i[c + 1]; k++) {
      Slot s = m.slots[k];
      if (s.nb < 0) continue;
      double r0[3];
      for (int j = 0; j < 3; j++) r0[j] = m.x_fa[3 * s.f + j] - m.x_cv[3 * c + j];
      for (int i = 0; i < 3; i++)
        if (lu[i]) bj_min(bu[i], pc[i], pc[i] + dot3(r0, &gu[3 * i]), umax[i], umin[i], e2u);
      if (lr) bj_min(br, rc, rc + dot3(r0, gr), rmax, rmin, e2r);
      if (lp) bj_min(bp, pc[3], pc[3] + dot3(r0, gpr), pmax, pmin, e2p);
      if (lh && do_visc) bj_min(bh, pc[5], pc[5] + dot3(r0, gh), hmax, hmin, e2h);
    }
    for (int i = 0; i < 3; i++) au[i] = bu[i].n / bu[i].d;
    ar = br.n / br.d;
    ap = bp.n / bp.d;
    ah = bh.n / bh.d;
    for (int i = 0; i < 3; i++)
      if (!lu[i]) au[i] = 0.0;
    if (!lr) ar = 0.0;
    if (!lp) ap = 0.0;
    if (!lh) ah = 0.0;
  }
  if (do_euler) {
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) st.gu[9 * c + 3 * i + j] = p.limiter ? gu[3 * i + j] * au[i] : gu[3 * i + j];
    for (int j = 0; j < 3; j++) {
      st.grho[3 * c + j] = p.limiter ? gr[j] * ar : gr[j];
      st.gp[3 * c + j] = p.limiter ? gpr[j] * ap : gpr[j];
    }
  }
  if (do_visc) {
    if (separate_guv || !do_euler) {
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) st.guv[9 * c + 3 * i + j] = visc_lim_u ? gu[3 * i + j] * au[i] : gu[3 * i + j];
    }
    for (int j = 0; j < 3; j++) st.gh[3 * c + j] = visc_lim_h ? gh[j] * ah : gh[j];
  }
}

// ---------------------------------------------------------------------------
// face loop (calcEulerFlux + calcViscousFluxNS, JoeWithModels.cpp:2621-3855)
// ---------------------------------------------------------------------------
// AUSMDV shock sensor (JoeWithModels.cpp:2753-2781): is internal face f sonic between its
// cells' centre states, a compression through u_n - c or u_n + c
__device__ __forceinline__ bool face_sonic(const Mesh& m, const Params& p, const State& st, int f) {
  const int c0 = m.cvofa[2 * f], c1 = m.cvofa[2 * f + 1];
  double nV[3], area;
  unit_normal(m, f, nV, area);
  const double* p0 = &st.prim[8 * c0];
  const double* p1 = &st.prim[8 * c1];
  const double unL = dot3(p0, nV), unR = dot3(p1, nV);
  const double cL = sqrt(p.gamma * p0[3] / st.q[5 * c0]), cR = sqrt(p.gamma * p1[3] / st.q[5 * c1]);
  return (((unL - cL) > 0.0) && ((unR - cR) < 0.0)) || (((unL + cL) > 0.0) && ((unR + cR) < 0.0));
}

// the cells beside a sonic internal face; cell-centric, so no two threads write one flag
__global__ void k_shock_flag(Mesh m, Params p, State st) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  unsigned char flag = 0;
  for (int k = m.slot_i[c]; k < m.slot_i[c + 1] && !flag; k++) {
    const Slot s = m.slots[k];
    if (s.nb >= 0 && face_sonic(m, p, st, s.f)) flag = 1;
  }
  st.shock_flag[c] = flag;
}

// JST coefficients of the current state, calcJSTCoeff_Var (JoeWithModels.cpp:13435-13492), per
// cell over its internal faces (each face in its own orientation, as the reference's face loop
// sees it): the spectral radius sum, the pressure sensor |sum dp| / sum (p0 + p1) and the
// undivided Laplacian of (rho, rhou, rhoE + p), a face counting for a cell unless the cell is
// interior-flagged and the other one not (the reference's BoundaryCV rule)
__global__ void k_jst(Mesh m, Params p, State st) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  double lam = 0.0, p1 = 0.0, p2 = 0.0, lap[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  int nint = 0;
  for (int k = m.slot_i[c]; k < m.slot_i[c + 1]; k++) {
    const Slot s = m.slots[k];
    if (s.nb < 0) continue;
    nint++;
    const int f = s.f, c0 = m.cvofa[2 * f], c1 = m.cvofa[2 * f + 1];
    double nV[3], area;
    unit_normal(m, f, nV, area);
    const double r0 = st.q[5 * c0], r1 = st.q[5 * c1];
    const double P0 = st.prim[8 * c0 + 3], P1 = st.prim[8 * c1 + 3];
    double u0[3], u1[3];
    for (int i = 0; i < 3; i++) {
      u0[i] = st.q[5 * c0 + 1 + i] / r0;
      u1[i] = st.q[5 * c1 + 1 + i] / r1;
    }
    const double l0 = 0.5 * (fabs(dot3(u0, nV)) + sqrt(p.gamma * P0 / r0)) * area;
    const double l1 = 0.5 * (fabs(dot3(u1, nV)) + sqrt(p.gamma * P1 / r1)) * area;
    lam += l0;
    lam += l1;
    const bool first = c == c0;
    p1 += first ? (P1 - P0) : (P0 - P1);
    p2 += (P0 + P1);
    const bool b0 = st.jst_bcv[c0] != 0, b1 = st.jst_bcv[c1] != 0;
    const bool take = first ? !(b0 && !b1) : !(!b0 && b1);
    if (take) {
      double d[5];
      d[0] = r0 - r1;
      for (int i = 0; i < 3; i++) d[1 + i] = st.q[5 * c0 + 1 + i] - st.q[5 * c1 + 1 + i];
      d[4] = (st.q[5 * c0 + 4] + P0) - (st.q[5 * c1 + 4] + P1);
      for (int i = 0; i < 5; i++) lap[i] += first ? -d[i] : d[i];
    }
  }
  double* J = &st.jst[8 * c];
  J[0] = fabs(p1) / p2;
  J[1] = lam;
  J[2] = (double)nint;
  for (int i = 0; i < 5; i++) J[3 + i] = lap[i];
}

// Block point relaxation, one warp per block row: a 160-thread block handles
// one 32-cell slice; warp i computes row i of (b - O x) for the 32 cells
// (coalesced ELL reads), the 5 rows meet in shared memory for the Dinv product.
template <typename BT>
__global__ void __launch_bounds__(160) k_jacobi2(Mesh m, State st, const BT* __restrict__ xin,
                                                 BT* __restrict__ xout, int first) {
  __shared__ BT sacc[5][SLICE];
  const int row = threadIdx.x / SLICE, lane = threadIdx.x % SLICE;
  const int slice = blockIdx.x;
  const int c = slice * SLICE + lane;
  const bool active = c < m.ncv && st.case_active[m.case_of[c]];
  const int N = m.ncv;
  BT acc = active ? (BT)st.b[5 * c + row] : (BT)0;
  if (!first && active) {
    const BT* O = (const BT*)st.O;
    int j0 = m.ell_off[slice], j1 = m.ell_off[slice + 1];
    for (int j = j0; j < j1; j++) {
      int nb = m.ell_nb[(size_t)j * SLICE + lane];
      const BT* Ob = O + ((size_t)j * 25 + 5 * row) * SLICE + lane;
      BT s = 0;
      for (int k = 0; k < 5; k++) s += Ob[k * SLICE] * xin[(size_t)k * N + nb];
      acc -= s;
    }
  }
  sacc[row][lane] = acc;
  __syncthreads();
  if (active) {
    const BT* Di = (const BT*)st.Dinv;
    BT s = 0;
    for (int k = 0; k < 5; k++) s += Di[(size_t)(5 * row + k) * N + c] * sacc[k][lane];
    xout[(size_t)row * N + c] = s;
  }
}

// residual history entry: sum of the per-block partials in block order
__global__ void k_resid_final(State st, int nblk, int hist_from_ctrl) {
  __shared__ double s[5][256];
  int t = threadIdx.x;
  double v[5] = {0, 0, 0, 0, 0};
  for (int b = t; b < nblk; b += blockDim.x)
    for (int i = 0; i < 5; i++) v[i] += st.blk[5 * b + i];
  for (int i = 0; i < 5; i++) s[i][t] = v[i];
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (t < w)
      for (int i = 0; i < 5; i++) s[i][t] += s[i][t + w];
    __syncthreads();
  }
  if (t == 0) {
    long idx = hist_from_ctrl ? (long)st.ctrl[1] - (long)st.ctrl[4] - 1 : 0;
    idx = ((idx % st.hist_cap) + st.hist_cap) % st.hist_cap;  // ring buffer
    for (int i = 0; i < 5; i++) st.resid[5 * idx + i] = s[i][0];
    if (!(s[4][0] == s[4][0])) atomicOr(st.err, 4);  // NaN energy residual (doneSolver)
  }
}

// Per-case L1 residual: block k sums |RHS| over the cells of case k in a fixed
// order that depends only on that case, so a case's residual history is the
// same alone and inside a batch.  out[(idx*ncases + k)*5 + i].
template <int B>
__global__ void __launch_bounds__(64 * B) k_resid_chunks(State st, const int* __restrict__ case_off,
                                                         const int* __restrict__ rblk_off,
                                                         const int* __restrict__ rblk_case) {
  constexpr int T = 64 * B;
  __shared__ double s[T];
  const int b = blockIdx.x, t = threadIdx.x;
  const int k = rblk_case[b];
  const long c0 = case_off[k] + (long)(b - rblk_off[k]) * RCHUNK;
  const long c1 = min((long)case_off[k + 1], c0 + RCHUNK);
  const double* r = st.rhs + B * c0;
  const long n = B * (c1 - c0);
  double v = 0.0;  // stride 64 x B: thread t always sums component t % B
  for (long e = t; e < n; e += T) v += fabs(r[e]);
  s[t] = v;
  __syncthreads();
  for (int w = 32; w > 0; w >>= 1) {  // fixed-order tree over the 64 threads of each component
    if (t / B < w) s[t] += s[t + B * w];
    __syncthreads();
  }
  if (t < B) st.rpart[B * b + t] = s[t];
}
template <int B>
__global__ void k_resid_cases(State st, const int* __restrict__ rblk_off, int ncases, int hist_from_ctrl) {
  const int k = blockIdx.x, lane = threadIdx.x;
  double v[B];
  for (int i = 0; i < B; i++) v[i] = 0.0;
  for (int b = rblk_off[k] + lane; b < rblk_off[k + 1]; b += 32)
    for (int i = 0; i < B; i++) v[i] += st.rpart[B * b + i];
  for (int o = 16; o > 0; o >>= 1)
    for (int i = 0; i < B; i++) v[i] += __shfl_down_sync(0xffffffffu, v[i], o);
  if (lane == 0) {
    long idx = hist_from_ctrl ? (long)st.ctrl[1] - (long)st.ctrl[4] - 1 : 0;
    idx = ((idx % st.hist_cap) + st.hist_cap) % st.hist_cap;  // ring buffer
    for (int i = 0; i < B; i++) st.resid[(idx * ncases + k) * B + i] = v[i];
    if (!(v[4] == v[4]) && st.case_active[k]) atomicOr(st.case_err + k, 4);  // NaN energy residual (doneSolver)
    // a lagged Jacobian formed at this step is next due jac_lag steps later (the face loop, which
    // read the schedule, ran before this kernel)
    const long long step = (long long)st.ctrl[1];
    if (hist_from_ctrl && st.jac_next && step >= st.jac_next[k]) st.jac_next[k] = step + st.jac_lag;
  }
}
void launch_resid_cases(State& st, const int* case_off, const int* rblk_off, const int* rblk_case, int nrblk,
                        int ncases, int hist_from_ctrl, cudaStream_t s) {
  if (st.bs == 7) {
    k_resid_chunks<7><<<nrblk, 64 * 7, 0, s>>>(st, case_off, rblk_off, rblk_case);
    k_resid_cases<7><<<ncases, 32, 0, s>>>(st, rblk_off, ncases, hist_from_ctrl);
  } else if (st.bs == 6) {
    k_resid_chunks<6><<<nrblk, 64 * 6, 0, s>>>(st, case_off, rblk_off, rblk_case);
    k_resid_cases<6><<<ncases, 32, 0, s>>>(st, rblk_off, ncases, hist_from_ctrl);
  } else {
    k_resid_chunks<5><<<nrblk, 64 * 5, 0, s>>>(st, case_off, rblk_off, rblk_case);
    k_resid_cases<5><<<ncases, 32, 0, s>>>(st, rblk_off, ncases, hist_from_ctrl);
  }
}

// ---------------------------------------------------------------------------
// block point relaxation: x_out = Dinv (b - O x_in); x in [5][N]
// ---------------------------------------------------------------------------
template <typename BT>
__global__ void __launch_bounds__(128) k_jacobi(Mesh m, State st, const BT* __restrict__ xin, BT* __restrict__ xout,
                                                int first) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv || !st.case_active[m.case_of[c]]) return;
  const int N = m.ncv;
  BT acc[5];
  for (int i = 0; i < 5; i++) acc[i] = (BT)st.b[5 * c + i];
  if (!first) {
    const BT* O = (const BT*)st.O;
    int slice = c / SLICE, lane = c % SLICE;
    int j0 = m.ell_off[slice], j1 = m.ell_off[slice + 1];
    for (int j = j0; j < j1; j++) {
      int nb = m.ell_nb[(size_t)j * SLICE + lane];
      BT xn[5];
      for (int k = 0; k < 5; k++) xn[k] = xin[(size_t)k * N + nb];
      const BT* Ob = O + (size_t)j * 25 * SLICE + lane;
      for (int i = 0; i < 5; i++) {
        BT s = 0;
        for (int k = 0; k < 5; k++) s += Ob[(5 * i + k) * SLICE] * xn[k];
        acc[i] -= s;
      }
    }
  }
  const BT* Di = (const BT*)st.Dinv;
  for (int i = 0; i < 5; i++) {
    BT s = 0;
    for (int k = 0; k < 5; k++) s += Di[(size_t)(5 * i + k) * N + c] * acc[k];
    xout[(size_t)i * N + c] = s;
  }
}

// Multicolour block Gauss-Seidel pass over one colour, in place: the cells of
// a colour have no neighbours of the same colour, so each reads the latest
// values of the others.  Same row-parallel layout as k_jacobi2.
// slices (may be null: every slice): the slices that hold a cell of this colour
template <typename BT>
__global__ void __launch_bounds__(160) k_gs2(Mesh m, State st, BT* __restrict__ x, int color,
                                             const int* __restrict__ slices) {
  __shared__ BT sacc[5][SLICE];
  const int row = threadIdx.x / SLICE, lane = threadIdx.x % SLICE;
  const int slice = slices ? slices[blockIdx.x] : blockIdx.x;
  const int c = slice * SLICE + lane;
  const bool active = c < m.ncv && m.color[c] == color && st.case_active[m.case_of[c]];
  const int N = m.ncv;
  BT acc = 0;
  if (active) {
    acc = (BT)st.b[5 * c + row];
    const BT* O = (const BT*)st.O;
    int j0 = m.ell_off[slice], j1 = m.ell_off[slice + 1];
    for (int j = j0; j < j1; j++) {
      int nb = m.ell_nb[(size_t)j * SLICE + lane];
      const BT* Ob = O + ((size_t)j * 25 + 5 * row) * SLICE + lane;
      BT s = 0;
      for (int k = 0; k < 5; k++) s += Ob[k * SLICE] * x[(size_t)k * N + nb];
      acc -= s;
    }
  }
  sacc[row][lane] = acc;
  __syncthreads();
  if (active) {
    const BT* Di = (const BT*)st.Dinv;
    BT s = 0;
    for (int k = 0; k < 5; k++) s += Di[(size_t)(5 * row + k) * N + c] * sacc[k][lane];
    x[(size_t)row * N + c] = s;
  }
}

template <typename BT>
__global__ void k_dq_from_x(Mesh m, State st, const BT* x) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  for (int i = 0; i < 5; i++) st.dq[5 * c + i] = (double)x[(size_t)i * m.ncv + c];
}

// Dinv from D (for linear systems handed in from the host)
template <typename BT>
__global__ void k_dinv(Mesh m, State st) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  double A[25], Ai[25];
  const BT* D = (const BT*)st.D;
  for (int e = 0; e < 25; e++) A[e] = (double)D[(size_t)e * m.ncv + c];
  block_inverse(A, Ai);
  BT* Dg = (BT*)st.Dinv;
  for (int e = 0; e < 25; e++) Dg[(size_t)e * m.ncv + c] = (BT)Ai[e];
}

// solveCvVectorR5Lusgs, UgpWithCv.cpp:3172-3239 (phi = 0 on entry):
//   x* = D^-1 b ;  x1 = D^-1 (D x* - U x*)
__global__ void k_lusgs2(Mesh m, State st, const double* xs, double* x1) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  const int N = m.ncv;
  const double* D = (const double*)st.D;
  const double* Di = (const double*)st.Dinv;
  const double* O = (const double*)st.O;
  double aux[5];
  for (int i = 0; i < 5; i++) {
    double s = 0.0;
    for (int k = 0; k < 5; k++) s += D[(size_t)(5 * i + k) * N + c] * xs[(size_t)k * N + c];
    aux[i] = s;
  }
  int slice = c / SLICE, lane = c % SLICE;
  for (int j = m.ell_off[slice]; j < m.ell_off[slice + 1]; j++) {
    size_t e = (size_t)j * SLICE + lane;
    if (m.ell_lower[e] != 2) continue;  // 2 = upper neighbour
    int nb = m.ell_nb[e];
    const double* Ob = O + (size_t)j * 25 * SLICE + lane;
    for (int i = 0; i < 5; i++) {
      double s = 0.0;
      for (int k = 0; k < 5; k++) s += Ob[(5 * i + k) * SLICE] * xs[(size_t)k * N + nb];
      aux[i] -= s;
    }
  }
  for (int i = 0; i < 5; i++) {
    double s = 0.0;
    for (int k = 0; k < 5; k++) s += Di[(size_t)(5 * i + k) * N + c] * aux[k];
    x1[(size_t)i * N + c] = s;
  }
}

// ---------------------------------------------------------------------------
// BiCGSTAB building blocks (solveCvVectorR5Bcgstab, UgpWithCv.cpp:2660-2876), FP64, [5][N]
// ---------------------------------------------------------------------------
__global__ void k_spmv(Mesh m, State st, const double* x, double* y) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  const int N = m.ncv;
  const double* D = (const double*)st.D;
  const double* O = (const double*)st.O;
  double acc[5];
  for (int i = 0; i < 5; i++) {
    double s = 0.0;
    for (int k = 0; k < 5; k++) s += D[(size_t)(5 * i + k) * N + c] * x[(size_t)k * N + c];
    acc[i] = s;
  }
  int slice = c / SLICE, lane = c % SLICE;
  for (int j = m.ell_off[slice]; j < m.ell_off[slice + 1]; j++) {
    int nb = m.ell_nb[(size_t)j * SLICE + lane];
    const double* Ob = O + (size_t)j * 25 * SLICE + lane;
    for (int i = 0; i < 5; i++) {
      double s = 0.0;
      for (int k = 0; k < 5; k++) s += Ob[(5 * i + k) * SLICE] * x[(size_t)k * N + nb];
      acc[i] += s;
    }
  }
  for (int i = 0; i < 5; i++) y[(size_t)i * N + c] = acc[i];
}

__global__ void k_precond(Mesh m, State st, const double* x, double* y) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.ncv) return;
  const int N = m.ncv;
  const double* Di = (const double*)st.Dinv;
  double xv[5];
  for (int k = 0; k < 5; k++) xv[k] = x[(size_t)k * N + c];
  for (int i = 0; i < 5; i++) {
    double s = 0.0;
    for (int k = 0; k < 5; k++) s += Di[(size_t)(5 * i + k) * N + c] * xv[k];
    y[(size_t)i * N + c] = s;
  }
}

__global__ void k_dot_partial(int n, const double* a, const double* b, double* partial) {
  __shared__ double s[256];
  double v = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v += a[i] * b[i];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void k_sum_final(int nblk, const double* partial, double* out, int is_max) {
  __shared__ double s[256];
  double v = 0.0;
  for (int i = threadIdx.x; i < nblk; i += blockDim.x) v = is_max ? fmax(v, partial[i]) : v + partial[i];
  s[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] = is_max ? fmax(s[threadIdx.x], s[threadIdx.x + w]) : s[threadIdx.x] + s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

// max over cells of |D^-1 r| (the reference's preconditioned residual norm)
__global__ void k_resmax_partial(Mesh m, State st, const double* r, double* partial) {
  __shared__ double s[256];
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (c < m.ncv) {
    const int N = m.ncv;
    const double* Di = (const double*)st.Dinv;
    double rv[5];
    for (int k = 0; k < 5; k++) rv[k] = r[(size_t)k * N + c];
    for (int i = 0; i < 5; i++) {
      double t = 0.0;
      for (int k = 0; k < 5; k++) t += Di[(size_t)(5 * i + k) * N + c] * rv[k];
      v = fmax(v, fabs(t));
    }
  }
  s[threadIdx.x] = v;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) s[threadIdx.x] = fmax(s[threadIdx.x], s[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

// out = a*x + b*y + c*z (z may be null); out may alias x, y or z
__global__ void k_lin3(long n, double* out, double a, const double* x, double b, const double* y, double c,
                       const double* z) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = a * x[i] + b * y[i];
  if (z) v += c * z[i];
  out[i] = v;
}

// batched face fluxes (per-face parity entry point)
__global__ void k_flux_faces(int kind, int n, const double* L, const double* R, const double* area, const double* nvec,
                             double* F, double* AL, double* AR) {
  int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  FState sl, sr;
  sl.rho = L[6 * f]; sl.u[0] = L[6 * f + 1]; sl.u[1] = L[6 * f + 2]; sl.u[2] = L[6 * f + 3]; sl.p = L[6 * f + 4]; sl.gam = L[6 * f + 5];
  sr.rho = R[6 * f]; sr.u[0] = R[6 * f + 1]; sr.u[1] = R[6 * f + 2]; sr.u[2] = R[6 * f + 3]; sr.p = R[6 * f + 4]; sr.gam = R[6 * f + 5];
  // ideal-gas enthalpy from the state (HAENEL)
  sl.h = sl.gam * sl.p / ((sl.gam - 1.0) * sl.rho);
  sr.h = sr.gam * sr.p / ((sr.gam - 1.0) * sr.rho);
  double nV[3] = {nvec[3 * f], nvec[3 * f + 1], nvec[3 * f + 2]};
  double Fl[5];
  euler_flux(kind, Fl, sl, sr, area[f], nV);
  for (int i = 0; i < 5; i++) F[5 * f + i] = Fl[i];
  if (AL || AR) {
    double a[25], b[25];
    euler_matrices(kind, AL ? a : nullptr, AR ? b : nullptr, sl, sr, area[f], nV);
    if (AL)
      for (int e = 0; e < 25; e++) AL[25 * f + e] = a[e];
    if (AR)
      for (int e = 0; e < 25; e++) AR[25 * f + e] = b[e];
  }
}

// state staging: io = [rho(N) | rhou(N*3) | rhoE(N)] in the reference's layouts
__global__ void k_pack_state(int n, const double* io, double* q, const int* perm) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  int r = perm ? perm[c] : c;
  q[5 * c] = io[r];
  for (int i = 0; i < 3; i++) q[5 * c + 1 + i] = io[n + 3 * r + i];
  q[5 * c + 4] = io[4 * n + r];
}

__global__ void k_unpack_state(int n, const double* q, double* io, const int* perm) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  int r = perm ? perm[c] : c;
  io[r] = q[5 * c];
  for (int i = 0; i < 3; i++) io[n + 3 * r + i] = q[5 * c + 1 + i];
  io[4 * n + r] = q[5 * c + 4];
}

__global__ void k_aos_to_soa5(int n, const double* aos, double* soa) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  for (int i = 0; i < 5; i++) soa[(size_t)i * n + c] = aos[5 * (size_t)c + i];
}

// A host-resident state stepped in place (jg_step_host, one case, 5x5): the upload's pack fused
// with calcStateVariables (the state preamble's memset of the primitives kept as prim[3] = 0,
// the only entry state_from_q reads), the history base of the call and the lag schedule's reset
// rho, rhou, rhoE: the staged copy of the caller's arrays in device memory
__global__ void k_state_in(Mesh m, Params p, State st, const double* rho, const double* rhou, const double* rhoE,
                           const int* perm) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c == 0) {
    st.ctrl[4] = st.ctrl[1];
    if (st.jac_next) st.jac_next[0] = 0;
  }
  if (c >= m.ncv) return;
  const int r = perm ? perm[c] : c;
  double q[5], prim[8];
  q[0] = rho[r];
  for (int i = 0; i < 3; i++) q[1 + i] = rhou[3 * r + i];
  q[4] = rhoE[r];
  for (int i = 0; i < 5; i++) st.q[5 * c + i] = q[i];
  for (int i = 0; i < 8; i++) prim[i] = 0.0;
  state_from_q(p, q, prim, st.case_err + m.case_of[c]);
  for (int i = 0; i < 8; i++) st.prim[8 * c + i] = prim[i];
}
// ... and the download's unpack with the call's error flags and residual history gathered into
// out[0..2+nres) (err, case_err[0], resid), the flags cleared for the next call
__global__ void k_state_out(Mesh m, State st, double* rho, double* rhou, double* rhoE, const int* perm, double* out,
                            int nres) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c == 0) {
    out[0] = (double)*st.err;
    out[1] = (double)st.case_err[0];
    *st.err = 0;
    st.case_err[0] = 0;
  }
  if (c < nres) out[2 + c] = st.resid[c];
  if (c >= m.ncv) return;
  const int r = perm ? perm[c] : c;
  rho[r] = st.q[5 * c];
  for (int i = 0; i < 3; i++) rhou[3 * r + i] = st.q[5 * c + 1 + i];
  rhoE[r] = st.q[5 * c + 4];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_state_in(const Mesh& m, const Params& p, State& st, const double* rho, const double* rhou,
                     const double* rhoE, const int* perm, cudaStream_t s) {
  k_state_in<<<grid_for(m.ncv, 256), 256, 0, s>>>(m, p, st, rho, rhou, rhoE, perm);
}
void launch_state_out(const Mesh& m, State& st, double* rho, double* rhou, double* rhoE, const int* perm, double* out,
                      int nres, cudaStream_t s) {
  k_state_out<<<grid_for(m.ncv > nres ? m.ncv : nres, 256), 256, 0, s>>>(m, st, rho, rhou, rhoE, perm, out, nres);
}
void launch_aos_to_soa5(int n, const double* aos, double* soa, cudaStream_t s) {
  k_aos_to_soa5<<<grid_for(n, 256), 256, 0, s>>>(n, aos, soa);
}
void launch_pack_state(int n, const double* io, double* q, const int* perm, cudaStream_t s) {
  k_pack_state<<<grid_for(n, 256), 256, 0, s>>>(n, io, q, perm);
}
void launch_unpack_state(int n, const double* q, double* io, const int* perm, cudaStream_t s) {
  k_unpack_state<<<grid_for(n, 256), 256, 0, s>>>(n, q, io, perm);
}
constexpr int TB = 128;

// static face geometry, once per mesh: the unit normal and area of every face; for internal
// faces the unit vector between the cell centres and its length
__global__ void k_face_geo(Mesh m, double* fa_u, double* fa_s) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nfa) return;
  const double n[3] = {m.fa_n[3 * f], m.fa_n[3 * f + 1], m.fa_n[3 * f + 2]};
  const double area = sqrt(dot3(n, n));
  for (int i = 0; i < 3; i++) fa_u[4 * f + i] = n[i] / area;
  fa_u[4 * f + 3] = area;
  if (f >= m.nfa_b) {
    const int c0 = m.cvofa[2 * f], c1 = m.cvofa[2 * f + 1];
    double sV[3];
    for (int i = 0; i < 3; i++) sV[i] = m.x_cv[3 * c1 + i] - m.x_cv[3 * c0 + i];
    const double smag = sqrt(dot3(sV, sV));
    double* o = &fa_s[4 * (f - m.nfa_b)];
    for (int i = 0; i < 3; i++) o[i] = sV[i] / smag;
    o[3] = smag;
  }
}
void launch_face_geo(const Mesh& m, double* fa_u, double* fa_s, cudaStream_t s) {
  if (m.nfa > 0) k_face_geo<<<grid_for(m.nfa, TB), TB, 0, s>>>(m, fa_u, fa_s);
}

void launch_state(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  k_state<<<grid_for(m.ncv, TB), TB, 0, s>>>(m, p, st);
}
void launch_update_state(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  k_update_state<<<grid_for(m.ncv, TB), TB, 0, s>>>(m, p, st);
}
void launch_update_state_x(const Mesh& m, const Params& p, State& st, const void* x, int x_fp32, cudaStream_t s) {
  if (x_fp32) k_update_state_x<float><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, p, st, (const float*)x);
  else k_update_state_x<double><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, p, st, (const double*)x);
}
void launch_faces_after_update(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  const int n = p.viscous ? m.nfa : m.nfa_b;
  if (n > 0) k_faces_after_update<<<grid_for(n, TB), TB, 0, s>>>(m, p, st);
}
void launch_face_props(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  if (!p.viscous || m.nfa == m.nfa_b) return;
  k_face_props<<<grid_for(m.nfa - m.nfa_b, TB), TB, 0, s>>>(m, p, st);
}
void launch_bc(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  if (m.nfa_b == 0) return;
  k_bc<<<grid_for(m.nfa_b, TB), TB, 0, s>>>(m, p, st);
}
void launch_ctrl_step(const Params& p, State& st, cudaStream_t s) { k_ctrl_step<<<1, 1, 0, s>>>(p, st); }
// the residual history of the steps that follow starts at entry 0: ctrl[4] = the step count now
__global__ void k_hist_base(State st) { st.ctrl[4] = st.ctrl[1]; }
void launch_hist_base(State& st, cudaStream_t s) { k_hist_base<<<1, 1, 0, s>>>(st); }
void launch_dt(const Mesh& m, const Params& p, State& st, int use_ctrl, double cfl, cudaStream_t s) {
  int nb = grid_for(m.ncv, 256);
  k_dt<<<nb, 256, 0, s>>>(m, p, st, use_ctrl, cfl);
  // the minimum over the cells: asked for by jg_calc_dt and by CFL_MIN; a step needs it only then
  if (!use_ctrl || p.ts_mode == JG_TS_CFL_MIN) k_dt_final<<<1, 256, 0, s>>>(m, p, st, nb);
  if (p.ts_mode == JG_TS_CFL_MIN) k_dt_min_all<<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st);
}
static void launch_grad_k(const Mesh& m, const Params& p, State& st, int do_euler, int do_visc, int lim_u, int lim_h,
                          int separate, cudaStream_t s) {
  const int g = grid_for(m.ncv, TB);
  if (p.grad_scheme == JG_GRAD_GREENGAUSS)
    k_grad<JG_GRAD_GREENGAUSS><<<g, TB, 0, s>>>(m, p, st, do_euler, do_visc, lim_u, lim_h, separate);
  else if (p.grad_scheme == JG_GRAD_SDWLS)
    k_grad<JG_GRAD_SDWLS><<<g, TB, 0, s>>>(m, p, st, do_euler, do_visc, lim_u, lim_h, separate);
  else
    k_grad<JG_GRAD_LSQ><<<g, TB, 0, s>>>(m, p, st, do_euler, do_visc, lim_u, lim_h, separate);
}
void launch_grad(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  int do_euler = p.second_order;
  int do_visc = p.viscous;
  if (!do_euler && !do_visc) return;
  // viscous velocity gradient: limited like the Euler one when VISC_LIMITER=YES
  int visc_lim = p.visc_limiter && p.limiter;
  int separate = do_visc && do_euler && !p.visc_limiter && p.limiter;
  launch_grad_k(m, p, st, do_euler, do_visc, visc_lim, visc_lim, separate, s);
}
// per-cell sensors the face loop of some flux kinds reads: the AUSMDV shock-fix flags, the JST
// coefficients (both before the face loop, cell-centric)
void launch_face_sensors(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  if (p.flux == JG_FLUX_AUSMDV && p.shock_fix != JG_SHOCK_FIX_NONE)
    k_shock_flag<<<grid_for(m.ncv, TB), TB, 0, s>>>(m, p, st);
  if (p.flux == JG_FLUX_JST) k_jst<<<grid_for(m.ncv, TB), TB, 0, s>>>(m, p, st);
}
// calcFluxCoupled (JoeWithModels.cpp:4683-4702): grad_u (second order or viscous), grad_rho,
// grad_p (second order) and grad_enthalpy (viscous), all with the flow limiter; one grad_u
void launch_grad_coupled(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  launch_grad_k(m, p, st, p.second_order, 1, p.limiter, p.limiter, 0, s);
}
// both sweep kernels do the same arithmetic in the same order (bit-identical results)
void launch_jacobi(const Mesh& m, const Params& p, State& st, int sweeps, cudaStream_t s) {
  for (int it = 0; it < sweeps; it++) {
    void* xin = (it % 2 == 0) ? st.x1 : st.x0;
    void* xout = (it % 2 == 0) ? st.x0 : st.x1;
    if (p.relax_variant == 1) {
      if (p.fp32)
        k_jacobi<float><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st, (const float*)xin, (float*)xout, it == 0);
      else
        k_jacobi<double><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st, (const double*)xin, (double*)xout, it == 0);
    } else if (p.fp32) {
      k_jacobi2<float><<<m.nslices, 5 * SLICE, 0, s>>>(m, st, (const float*)xin, (float*)xout, it == 0);
    } else {
      k_jacobi2<double><<<m.nslices, 5 * SLICE, 0, s>>>(m, st, (const double*)xin, (double*)xout, it == 0);
    }
  }
}
void launch_sgs(const Mesh& m, const Params& p, State& st, int sweeps, cudaStream_t s) {
  size_t bytes = 5 * (size_t)m.ncv * (p.fp32 ? sizeof(float) : sizeof(double));
  cudaMemsetAsync(st.x0, 0, bytes, s);
  for (int it = 0; it < sweeps; it++)
    for (int q = 0; q < m.ncolors; q++) {
      int col = (it % 2 == 0) ? q : m.ncolors - 1 - q;  // forward, then backward colour order
      const bool lists = m.color_slices != nullptr;
      const int* sl = lists ? m.color_slices + m.color_slice_off[col] : nullptr;
      const int g = lists ? m.color_slice_off[col + 1] - m.color_slice_off[col] : m.nslices;
      if (g == 0) continue;
      if (p.fp32) k_gs2<float><<<g, 5 * SLICE, 0, s>>>(m, st, (float*)st.x0, col, sl);
      else k_gs2<double><<<g, 5 * SLICE, 0, s>>>(m, st, (double*)st.x0, col, sl);
    }
}
void launch_dq_from_x(const Mesh& m, const Params& p, State& st, const void* x, cudaStream_t s) {
  if (p.fp32)
    k_dq_from_x<float><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st, (const float*)x);
  else
    k_dq_from_x<double><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st, (const double*)x);
}
void launch_dinv(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  if (p.fp32)
    k_dinv<float><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st);
  else
    k_dinv<double><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st);
}
void launch_lusgs(const Mesh& m, const Params& p, State& st, cudaStream_t s) {
  // x* = Dinv b into x0 (one Jacobi sweep from zero), then the upper correction into x1
  k_jacobi<double><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st, (const double*)st.x1, (double*)st.x0, 1);
  k_lusgs2<<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st, (const double*)st.x0, (double*)st.x1);
}
void launch_spmv(const Mesh& m, const State& st, const double* x, double* y, cudaStream_t s) {
  k_spmv<<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st, x, y);
}
void launch_precond(const Mesh& m, const State& st, const double* x, double* y, cudaStream_t s) {
  k_precond<<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st, x, y);
}
void launch_dot(int n, const double* a, const double* b, double* partial, double* out, cudaStream_t s) {
  int nb = grid_for(n, 256);
  if (nb > 1024) nb = 1024;
  k_dot_partial<<<nb, 256, 0, s>>>(n, a, b, partial);
  k_sum_final<<<1, 256, 0, s>>>(nb, partial, out, 0);
}
void launch_resmax(const Mesh& m, const State& st, const double* r, double* partial, double* out, cudaStream_t s) {
  int nb = grid_for(m.ncv, 256);
  k_resmax_partial<<<nb, 256, 0, s>>>(m, st, r, partial);
  k_sum_final<<<1, 256, 0, s>>>(nb, partial, out, 1);
}
void launch_lin3(long n, double* out, double a, const double* x, double b, const double* y, double c, const double* z,
                 cudaStream_t s) {
  k_lin3<<<grid_for(n, 256), 256, 0, s>>>(n, out, a, x, b, y, c, z);
}
void launch_flux_faces(int kind, int n, const double* L, const double* R, const double* area, const double* nvec,
                       double* F, double* AL, double* AR, cudaStream_t s) {
  k_flux_faces<<<grid_for(n, 64), 64, 0, s>>>(kind, n, L, R, area, nvec, F, AL, AR);
}

// addViscFlux per face (jg_visc_flux_faces): the face-loop's visc_flux and visc_jac_add on given
// side states; A0 / A1 are the blocks calcViscousFluxNS subtracts from the first cell's row
// (JoeWithModels.cpp:3678-3696)
__global__ void k_visc_faces(int n, const double* S0, const double* S1, const double* gu0, const double* gu1,
                             const double* gh0, const double* gh1, const double* mul, const double* lam,
                             const double* ufa, const double* area, const double* nvec, const double* svec,
                             const double* smag, double* F, double* A0, double* A1) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= n) return;
  VSide v[2];
  const double* S[2] = {S0 + 8 * (size_t)f, S1 + 8 * (size_t)f};
  const double* gu[2] = {gu0 + 9 * (size_t)f, gu1 + 9 * (size_t)f};
  const double* gh[2] = {gh0 + 3 * (size_t)f, gh1 + 3 * (size_t)f};
  for (int k = 0; k < 2; k++) {
    v[k].rho = S[k][0];
    for (int i = 0; i < 3; i++) v[k].u[i] = S[k][1 + i];
    v[k].h = S[k][4];
    v[k].T = S[k][5];
    v[k].R = S[k][6];
    v[k].gam = S[k][7];
    v[k].gu = gu[k];
    v[k].gh = gh[k];
  }
  const double nV[3] = {nvec[3 * f], nvec[3 * f + 1], nvec[3 * f + 2]};
  const double sV[3] = {svec[3 * f], svec[3 * f + 1], svec[3 * f + 2]};
  const double u_fa[3] = {ufa[3 * f], ufa[3 * f + 1], ufa[3 * f + 2]};
  double Fu[3], FE;
  VFace vf;
  visc_flux(Fu, FE, vf, v[0], v[1], mul[f], 0.0, lam[f], 0.9, u_fa, area[f], nV, smag[f], sV);
  for (int i = 0; i < 3; i++) F[4 * (size_t)f + i] = Fu[i];
  F[4 * (size_t)f + 3] = FE;
  if (A0) {
    double a[25];
    for (int e = 0; e < 25; e++) a[e] = 0.0;
    visc_jac_add<double>(a, 1.0, 0, vf, v[0], u_fa);
    for (int e = 0; e < 25; e++) A0[25 * (size_t)f + e] = a[e];
  }
  if (A1) {
    double a[25];
    for (int e = 0; e < 25; e++) a[e] = 0.0;
    visc_jac_add<double>(a, 1.0, 1, vf, v[1], u_fa);
    for (int e = 0; e < 25; e++) A1[25 * (size_t)f + e] = a[e];
  }
}
void launch_visc_faces(int n, const double* const* in, double* F, double* A0, double* A1, cudaStream_t s) {
  k_visc_faces<<<grid_for(n, 64), 64, 0, s>>>(n, in[0], in[1], in[2], in[3], in[4], in[5], in[6], in[7], in[8],
                                               in[9], in[10], in[11], in[12], F, A0, A1);
}

}  // namespace jg
