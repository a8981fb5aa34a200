// jg_faceloop.cu -- the face loop (calcEulerFlux + calcViscousFluxNS,
// JoeWithModels.cpp:2621-3855) as two kernels on two streams:
//
//  * k_res: the residual.  Second-order reconstruction at the face, the
//    Riemann flux, the viscous flux; FL lanes per cell (lane l takes the cell's
//    face slots l, l+FL, ...), the lanes' sums combined by a butterfly in a
//    fixed order.  No Jacobian live set, so ~120 registers and many warps.
//  * k_jac: the Jacobian blocks, which the reference forms at the cell-centre
//    states (JoeWithModels.cpp:3032-3102).  One thread per cell walks the
//    cell's faces; each face's two matrices come one row at a time
//    (jg_rows.cuh) and go straight into the cell's diagonal block (shared
//    memory) and its off-diagonal block of the sliced-ELL row (one coalesced
//    store per entry across the 32 cells of a slice).  The epilogue adds
//    vol/dt, stores D and its inverse (ludeco / luinv).
//
// Both kernels are cell-centric: each face is evaluated from both of its
// cells, in the face's own orientation, so the two cells obtain bit-identical
// face fluxes and every row has a single writer (no atomics, deterministic).
//
// Lagged Jacobian (State::jac_lag > 1): k_jac runs only on the steps a case's
// blocks are due; it keeps the face part of the diagonal in D0.  On the other
// steps k_diag adds that step's vol/dt to D0 and inverts.  The residual and
// the state update stay FP64 and exact every step, so the converged field is
// unchanged (defect correction); only the preconditioner ages.
#include <cuda_runtime.h>
#include <math.h>

#include "jg_cell.cuh"
#include "jg_flux.cuh"
#include "jg_internal.h"
#include "jg_rows.cuh"

namespace jg {

namespace {
constexpr int TB = 128;

// are case k's Jacobian blocks formed at this step (the step counter ctrl[1] is already advanced)
__device__ __forceinline__ bool jac_due(const State& st, int k) {
  return st.jac_next == nullptr || (long long)st.ctrl[1] >= st.jac_next[k];
}
}  // namespace

// ---------------------------------------------------------------------------
// residual
// ---------------------------------------------------------------------------
template <int FL>
__device__ __forceinline__ double lanes_sum(double v) {
#pragma unroll
  for (int o = FL / 2; o >= 1; o /= 2) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <int KIND, int VISC, int FL>
__global__ void __launch_bounds__(TB) k_res(Mesh m, Params p, State st, int for_step) {
  const int t = threadIdx.x, lane = t % FL;
  const int c = blockIdx.x * (TB / FL) + t / FL;
  const bool active = c < m.ncv && st.case_active[m.case_of[c]];  // a frozen case keeps its arrays
  double rhs[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  const int k0 = active ? m.slot_i[c] : 0, k1 = active ? m.slot_i[c + 1] : 0;
  if (k0 + lane < k1) {
    const int nb = m.slots[k0 + lane].nb;
    if (nb >= 0) prefetch_cell(st, m, nb, VISC);
  }
  for (int k = k0 + lane; k < k1; k += FL) {
    const Slot s = m.slots[k];
    const int f = s.f;
    if (k + FL < k1) {  // the next face's neighbour, a face ahead
      const int nb = m.slots[k + FL].nb;
      if (nb >= 0) prefetch_cell(st, m, nb, VISC);
    }
    double nV[3], area;
    unit_normal(m, f, nV, area);
    if (s.nb >= 0) {
      const int c0 = s.side == 0 ? c : s.nb;
      const int c1 = s.side == 0 ? s.nb : c;
      const double sg = s.side == 0 ? -1.0 : 1.0;  // residual sign of this cell
      {
        FState L = recon(m, p, st, c0, f), R = recon(m, p, st, c1, f);
        double F[5];
        euler_flux_t<KIND>(F, L, R, area, nV, face_opts<KIND>(p, st, c0, c1), KIND == 5 ? &st.jst[8 * c0] : nullptr,
                           KIND == 5 ? &st.jst[8 * c1] : nullptr);
        for (int i = 0; i < 5; i++) rhs[i] += sg * F[i];
      }
      if (VISC) {
        VSide v0 = cell_vside(p, st, c0), v1 = cell_vside(p, st, c1);
        double sV[3], smag;
        cell_to_cell(m, f, sV, smag);
        double ufa[3] = {0.5 * (v0.u[0] + v1.u[0]), 0.5 * (v0.u[1] + v1.u[1]), 0.5 * (v0.u[2] + v1.u[2])};
        double Fu[3], FE;
        VFace vf;
        visc_flux(Fu, FE, vf, v0, v1, st.mul_fa[f], 0.0, st.lam_fa[f], p.PrTurb, ufa, area, nV, smag, sV);
        for (int i = 0; i < 3; i++) rhs[1 + i] += sg * Fu[i];
        rhs[4] += sg * FE;
      }
    } else {
      // boundary face (the cell is cvofa[f][0])
      const DevZone z = m.zones[m.bzone[f]];
      const double* bb = &st.bfa[8 * f];
      FState B;
      B.rho = bb[0]; B.u[0] = bb[1]; B.u[1] = bb[2]; B.u[2] = bb[3]; B.p = bb[4]; B.gam = p.gamma; B.h = bb[6];
      double F[5];
      const int fob = bnd_opts<KIND>(p);
      const double* jb = KIND == 5 ? &st.jst[8 * c] : nullptr;
      if (z.kind == JG_BC_SYMMETRY || z.kind == JG_BC_WALL) {
        euler_flux_t<KIND>(F, B, B, area, nV, fob, jb, jb);
        if (z.kind == JG_BC_SYMMETRY && p.symm_bc == JG_SYMM_ANALYTICAL) {
          for (int i = 0; i < 3; i++) rhs[1 + i] -= bb[4] * nV[i] * area;
        } else {
          for (int i = 0; i < 5; i++) rhs[i] -= F[i];
        }
      } else {
        FState L = recon(m, p, st, c, f);
        euler_flux_t<KIND>(F, L, B, area, nV, fob, jb, jb);
        for (int i = 0; i < 5; i++) rhs[i] -= F[i];
      }
      if (VISC && z.kind != JG_BC_SYMMETRY) {
        VSide v0 = cell_vside(p, st, c);
        VSide v1;
        v1.rho = bb[0]; v1.u[0] = bb[1]; v1.u[1] = bb[2]; v1.u[2] = bb[3];
        v1.h = bb[6]; v1.T = bb[5]; v1.R = p.R; v1.gam = p.gamma;
        v1.gu = v0.gu; v1.gh = v0.gh;
        double sV[3], smag;
        for (int i = 0; i < 3; i++) sV[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
        if (z.kind == JG_BC_WALL) {
          smag = fabs(dot3(sV, nV));  // projected on the wall normal; nVec is used as sVec
          for (int i = 0; i < 3; i++) sV[i] = nV[i];
        } else {
          smag = sqrt(dot3(sV, sV));
          for (int i = 0; i < 3; i++) sV[i] /= smag;
        }
        double Fu[3], FE;
        VFace vf;
        visc_flux(Fu, FE, vf, v0, v1, st.mul_fa[f], 0.0, st.lam_fa[f], p.PrTurb, v1.u, area, nV, smag, sV);
        for (int i = 0; i < 3; i++) rhs[1 + i] -= Fu[i];
        rhs[4] -= FE;
      }
    }
  }
  // the lanes of a cell share its activity, so every lane of the warp reaches the shuffles
  if (FL > 1)
    for (int i = 0; i < 5; i++) rhs[i] = lanes_sum<FL>(rhs[i]);
  if (active && lane == 0) {
    gravity_rhs(p, m, st, c, rhs);
    for (int i = 0; i < 5; i++) st.rhs[5 * c + i] = rhs[i];
    if (for_step)
      for (int i = 0; i < 5; i++) st.b[5 * c + i] = p.under_relax * rhs[i];
  }
}

// ---------------------------------------------------------------------------
// Jacobian blocks
// ---------------------------------------------------------------------------
// Resident blocks per SM the register allocation must allow: 3 for FP64 (168 registers, a few
// hundred bytes of L1-cached spills on the Roe and HLLC paths), 4 for FP32 (128 registers); the
// AUSMDV matrices are formed whole and keep the full register file
template <typename BT, int KIND>
constexpr int jac_min_blocks() {
  return KIND == 4 ? 1 : (sizeof(BT) == 8 ? 3 : 4);
}

// sched: 1 inside a step (the lag schedule decides, and D0 is kept), 0 always form the blocks
template <typename BT, int KIND, int VISC>
__global__ void __launch_bounds__(TB, jac_min_blocks<BT, KIND>()) k_jac(Mesh m, Params p, State st, int for_step,
                                                                      int sched) {
  using JT = BT;  // FP64 for the plain form, FP32 for the mixed form's preconditioner
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int t = threadIdx.x;
  const int c = blockIdx.x * TB + t;
  if (c >= m.ncv || !st.case_active[m.case_of[c]]) return;
  if (sched && !jac_due(st, m.case_of[c])) return;
  JT* sd = reinterpret_cast<JT*>(smem_raw) + t;  // this cell's diagonal block: entry e at sd[e * TB]
  for (int e = 0; e < 25; e++) sd[e * TB] = JT(0);
  BT* O = (BT*)st.O;
  const int slice = c / SLICE, lane = c % SLICE;
  const int k0 = m.slot_i[c], k1 = m.slot_i[c + 1];
  if (k0 < k1 && m.slots[k0].nb >= 0) prefetch_cell_jac(st, m.slots[k0].nb, VISC);
  for (int k = k0; k < k1; k++) {
    const Slot s = m.slots[k];
    const int f = s.f;
    if (k + 1 < k1 && m.slots[k + 1].nb >= 0) prefetch_cell_jac(st, m.slots[k + 1].nb, VISC);  // a face ahead
    double nV[3], area;
    unit_normal(m, f, nV, area);
    const JT nVt[3] = {(JT)nV[0], (JT)nV[1], (JT)nV[2]};
    if (s.nb >= 0) {
      // ---------------- internal face ----------------
      const int c0 = s.side == 0 ? c : s.nb;
      const int c1 = s.side == 0 ? s.nb : c;
      const int fo = face_opts<KIND>(p, st, c0, c1);
      // viscous rows (calcViscousFluxNS 3678-3696): row of c0: D -= A0, O -= A1; row of c1: D += A1, O += A0
      VJacRows<JT> vd, vo;
      JT vsg = JT(0);
      if (VISC) {
        VSide v0 = cell_vside(p, st, c0), v1 = cell_vside(p, st, c1);
        double sV[3], smag;
        cell_to_cell(m, f, sV, smag);
        double ufa[3] = {0.5 * (v0.u[0] + v1.u[0]), 0.5 * (v0.u[1] + v1.u[1]), 0.5 * (v0.u[2] + v1.u[2])};
        double Fu[3], FE;
        VFace vf;
        visc_flux(Fu, FE, vf, v0, v1, st.mul_fa[f], 0.0, st.lam_fa[f], p.PrTurb, ufa, area, nV, smag, sV);
        if (s.side == 0) {
          vd = vjac_rows<JT>(0, vf, v0, ufa);
          vo = vjac_rows<JT>(1, vf, v1, ufa);
          vsg = JT(-1.0);
        } else {
          vd = vjac_rows<JT>(1, vf, v1, ufa);
          vo = vjac_rows<JT>(0, vf, v0, ufa);
          vsg = JT(1.0);
        }
      }
      const FStateT<JT> L0 = fstate_as<JT>(cell_fstate(p, st, c0)), R0 = fstate_as<JT>(cell_fstate(p, st, c1));
      BT* ob = O + (size_t)(m.ell_off[slice] + s.col) * 25 * SLICE + lane;
      const bool first = s.side == 0;
      // row of c0: D += A_L, O(c0,c1) = A_R ; row of c1: D -= A_R, O(c1,c0) = -A_L
      euler_rows_t<KIND, JT>(L0, R0, (JT)area, nVt, fo, [&](int i, const JT* aL, const JT* aR) {
        JT orow[5];
        const StridedBlock<JT> drow{sd + 5 * i * TB, TB};
        for (int j = 0; j < 5; j++) {
          drow[j] += first ? aL[j] : -aR[j];
          orow[j] = first ? aR[j] : -aL[j];
        }
        if (VISC) {
          vjac_row_add(drow, i, vsg, vd);
          vjac_row_add(orow, i, vsg, vo);
        }
        for (int j = 0; j < 5; j++) ob[(5 * i + j) * SLICE] = (BT)orow[j];
      });
    } else {
      // ---------------- boundary face (the cell is cvofa[f][0]) ----------------
      const DevZone z = m.zones[m.bzone[f]];
      const double* bb = &st.bfa[8 * f];
      FState B;
      B.rho = bb[0]; B.u[0] = bb[1]; B.u[1] = bb[2]; B.u[2] = bb[3]; B.p = bb[4]; B.gam = p.gamma; B.h = bb[6];
      const FStateT<JT> Bt = fstate_as<JT>(B);
      const int fob = bnd_opts<KIND>(p);
      if (z.kind == JG_BC_SYMMETRY && p.symm_bc == JG_SYMM_ANALYTICAL) {
        // analytical pressure Jacobian, JoeWithModels.cpp:3231-3251
        double a2 = p.gamma - 1.0;
        double phi = 0.5 * a2 * (B.u[0] * B.u[0] + B.u[1] * B.u[1] + B.u[2] * B.u[2]);
        for (int i = 0; i < 3; i++) {
          sd[(5 * (i + 1) + 0) * TB] += (JT)(phi * nV[i] * area);
          for (int j = 0; j < 3; j++) sd[(5 * (i + 1) + 1 + j) * TB] += (JT)(-a2 * B.u[j] * nV[i] * area);
          sd[(5 * (i + 1) + 4) * TB] += (JT)(a2 * nV[i] * area);
        }
      } else if (z.kind == JG_BC_SYMMETRY && p.symm_bc == JG_SYMM_NEW_NUMERIC) {
        euler_rows_t<KIND, JT>(Bt, Bt, (JT)area, nVt, fob, [&](int i, const JT* aL, const JT* aR) {
          for (int j = 0; j < 5; j++) sd[(5 * i + j) * TB] += aL[j] + aR[j];
        });
      } else {
        // SYMMETRY (original numeric) and WALL: A_L at the boundary state; the others at the cell state
        const bool bstate = z.kind == JG_BC_SYMMETRY || z.kind == JG_BC_WALL;
        const FStateT<JT> L0 = bstate ? Bt : fstate_as<JT>(cell_fstate(p, st, c));
        euler_rows_t<KIND, JT>(L0, Bt, (JT)area, nVt, fob, [&](int i, const JT* aL, const JT*) {
          for (int j = 0; j < 5; j++) sd[(5 * i + j) * TB] += aL[j];
        });
      }
      if (VISC && z.kind != JG_BC_SYMMETRY) {
        VSide v0 = cell_vside(p, st, c);
        VSide v1;
        v1.rho = bb[0]; v1.u[0] = bb[1]; v1.u[1] = bb[2]; v1.u[2] = bb[3];
        v1.h = bb[6]; v1.T = bb[5]; v1.R = p.R; v1.gam = p.gamma;
        v1.gu = v0.gu; v1.gh = v0.gh;
        double sV[3], smag;
        for (int i = 0; i < 3; i++) sV[i] = m.x_fa[3 * f + i] - m.x_cv[3 * c + i];
        if (z.kind == JG_BC_WALL) {
          smag = fabs(dot3(sV, nV));
          for (int i = 0; i < 3; i++) sV[i] = nV[i];
        } else {
          smag = sqrt(dot3(sV, sV));
          for (int i = 0; i < 3; i++) sV[i] /= smag;
        }
        double Fu[3], FE;
        VFace vf;
        visc_flux(Fu, FE, vf, v0, v1, st.mul_fa[f], 0.0, st.lam_fa[f], p.PrTurb, v1.u, area, nV, smag, sV);
        const VJacRows<JT> vd = vjac_rows<JT>(0, vf, v0, v1.u);
        for (int i = 1; i < 5; i++) vjac_row_add(StridedBlock<JT>{sd + 5 * i * TB, TB}, i, JT(-1.0), vd);
      }
    }
  }
  // ---------------- epilogue: D (+ vol/dt), D0, Dinv ----------------
  const int N = m.ncv;
  double Dm[25];
  for (int e = 0; e < 25; e++) Dm[e] = (double)sd[e * TB];
  gravity_diag<5>(p, m, c, Dm);
  if (sched && st.D0) {
    BT* D0 = (BT*)st.D0;
    for (int e = 0; e < 25; e++) D0[(size_t)e * N + c] = (BT)Dm[e];
  }
  if (for_step) {
    const double tmp = m.vol[c] / st.local_dt[c];
    for (int i = 0; i < 5; i++) Dm[6 * i] += tmp;
  }
  BT* Dg = (BT*)st.D;
  for (int e = 0; e < 25; e++) Dg[(size_t)e * N + c] = (BT)Dm[e];
  if (for_step) {
    double Di[25];
    block_inverse(Dm, Di);
    BT* Dig = (BT*)st.Dinv;
    for (int e = 0; e < 25; e++) Dig[(size_t)e * N + c] = (BT)Di[e];
  }
}

// the steps between refreshes of a lagged Jacobian: D = D0 + vol/dt, Dinv
template <typename BT>
__global__ void __launch_bounds__(TB) k_diag(Mesh m, State st) {
  const int c = blockIdx.x * TB + threadIdx.x;
  if (c >= m.ncv || !st.case_active[m.case_of[c]]) return;
  if (jac_due(st, m.case_of[c])) return;  // k_jac formed this case's blocks at this step
  const int N = m.ncv;
  const BT* D0 = (const BT*)st.D0;
  double Dm[25], Di[25];
  for (int e = 0; e < 25; e++) Dm[e] = (double)D0[(size_t)e * N + c];
  const double tmp = m.vol[c] / st.local_dt[c];
  for (int i = 0; i < 5; i++) Dm[6 * i] += tmp;
  BT* Dg = (BT*)st.D;
  for (int e = 0; e < 25; e++) Dg[(size_t)e * N + c] = (BT)Dm[e];
  block_inverse(Dm, Di);
  BT* Dig = (BT*)st.Dinv;
  for (int e = 0; e < 25; e++) Dig[(size_t)e * N + c] = (BT)Di[e];
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <int KIND, int VISC>
static void launch_res_kv(const Mesh& m, const Params& p, State& st, int fl, int for_step, cudaStream_t s) {
  switch (fl) {
    case 1: k_res<KIND, VISC, 1><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, p, st, for_step); break;
    case 2: k_res<KIND, VISC, 2><<<grid_for(m.ncv, TB / 2), TB, 0, s>>>(m, p, st, for_step); break;
    case 4: k_res<KIND, VISC, 4><<<grid_for(m.ncv, TB / 4), TB, 0, s>>>(m, p, st, for_step); break;
    default: k_res<KIND, VISC, 8><<<grid_for(m.ncv, TB / 8), TB, 0, s>>>(m, p, st, for_step); break;
  }
}
template <int KIND>
static void launch_res_k(const Mesh& m, const Params& p, State& st, int fl, int for_step, cudaStream_t s) {
  if (p.viscous) launch_res_kv<KIND, 1>(m, p, st, fl, for_step, s);
  else launch_res_kv<KIND, 0>(m, p, st, fl, for_step, s);
}
static void launch_res(const Mesh& m, const Params& p, State& st, int fl, int for_step, cudaStream_t s) {
  switch (p.flux) {
    case JG_FLUX_ROE: launch_res_k<1>(m, p, st, fl, for_step, s); break;
    case JG_FLUX_AUSM: launch_res_k<2>(m, p, st, fl, for_step, s); break;
    case JG_FLUX_HAENEL: launch_res_k<3>(m, p, st, fl, for_step, s); break;
    case JG_FLUX_AUSMDV: launch_res_k<4>(m, p, st, fl, for_step, s); break;
    case JG_FLUX_JST: launch_res_k<5>(m, p, st, fl, for_step, s); break;
    default: launch_res_k<0>(m, p, st, fl, for_step, s); break;
  }
}

template <typename BT, int KIND>
static void launch_jac_k(const Mesh& m, const Params& p, State& st, int for_step, int sched, cudaStream_t s) {
  const size_t shm = 25 * TB * sizeof(BT);
  const int g = grid_for(m.ncv, TB);
  if (p.viscous) k_jac<BT, KIND, 1><<<g, TB, shm, s>>>(m, p, st, for_step, sched);
  else k_jac<BT, KIND, 0><<<g, TB, shm, s>>>(m, p, st, for_step, sched);
}
template <typename BT>
static void launch_jac_t(const Mesh& m, const Params& p, State& st, int for_step, int sched, cudaStream_t s) {
  switch (p.flux) {
    case JG_FLUX_ROE: launch_jac_k<BT, 1>(m, p, st, for_step, sched, s); break;
    case JG_FLUX_HAENEL: launch_jac_k<BT, 3>(m, p, st, for_step, sched, s); break;
    case JG_FLUX_AUSMDV: launch_jac_k<BT, 4>(m, p, st, for_step, sched, s); break;
    // HLLC; AUSM and JST take the HLLC matrices (JoeWithModels.cpp:3057-3061)
    default: launch_jac_k<BT, 0>(m, p, st, for_step, sched, s); break;
  }
}

// the implicit blocks (and, in a step under a lag schedule, the diagonal of the steps between)
static void launch_jacobian(const Mesh& m, const Params& p, State& st, int for_step, cudaStream_t s) {
  const int sched = for_step && st.jac_lag > 1 && st.D0 != nullptr;
  if (p.fp32) {
    launch_jac_t<float>(m, p, st, for_step, sched, s);
    if (sched) k_diag<float><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st);
  } else {
    launch_jac_t<double>(m, p, st, for_step, sched, s);
    if (sched) k_diag<double><<<grid_for(m.ncv, TB), TB, 0, s>>>(m, st);
  }
}

void launch_flux(const Mesh& m, const Params& p, State& st, int implicit, int for_step, cudaStream_t s) {
  launch_face_sensors(m, p, st, s);
  if (!implicit) {
    launch_res(m, p, st, flux_split(p, st) ? flux_split_lanes(p) : 8, for_step, s);
    return;
  }
  if (!flux_split(p, st)) {
    launch_flux_fused(m, p, st, for_step, s);
    return;
  }
  const int fl = flux_split_lanes(p);
  if (st.aux && st.ev_fork && st.ev_join) {
    // the two kernels are independent: the Jacobian on the second stream, joined before the caller's next work
    cudaEventRecord(st.ev_fork, s);
    cudaStreamWaitEvent(st.aux, st.ev_fork, 0);
    launch_jacobian(m, p, st, for_step, st.aux);
    launch_res(m, p, st, fl, for_step, s);
    cudaEventRecord(st.ev_join, st.aux);
    cudaStreamWaitEvent(s, st.ev_join, 0);
  } else {
    launch_jacobian(m, p, st, for_step, s);
    launch_res(m, p, st, fl, for_step, s);
  }
}

}  // namespace jg
