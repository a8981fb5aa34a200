// jg_fused.cu -- the face loop as one kernel: residual and Jacobian blocks in
// the same pass over each cell's faces (calcEulerFlux + calcViscousFluxNS,
// JoeWithModels.cpp:2621-3855).  Kept as launch shapes the autotuner can pick
// beside the split face loop of jg_faceloop.cu.
#include <cuda_runtime.h>
#include <math.h>

#include "jg_cell.cuh"
#include "jg_flux.cuh"
#include "jg_internal.h"

namespace jg {

namespace {
constexpr int TB = 128;
}

// CL lanes per cell (a launch shape chosen per handle, jg_autotune): lane l
// of a cell evaluates the cell's face slots l, l+CL, ...; each lane
// accumulates its own partial diagonal block (shared memory) and residual,
// summed over the lanes in a fixed order.  More lanes shorten each thread's
// dependent chain and give the scheduler more warps to spread over the SMs
// (a small mesh is otherwise a one-and-a-bit-wave grid at the
// register-limited occupancy); they cost repeated reads of the cell's data.
// Measured: the viscous Roe plate (49k cells) is 2% faster with two lanes,
// inviscid HLLC bumps (430k cells) 1.4x faster with one.
// MINB: resident blocks per SM the register allocation must allow (__launch_bounds__): 2 lets the
// compiler use all 255 registers; 3 caps it near 168 (some spills to L1-cached local memory) for
// 12 instead of 8 warps per SM, which hides more FP64 latency on some meshes (jg_autotune decides)
template <typename BT, int KIND, int VISC, int CL, int MINB>
__global__ void __launch_bounds__(128, MINB) k_flux(Mesh m, Params p, State st, int implicit, int for_step) {
  // the Jacobian blocks are formed in BT arithmetic: FP64 for the plain form,
  // FP32 for the mixed form's preconditioner (the residual is FP64 in both)
  using JT = BT;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  JT* sD = reinterpret_cast<JT*>(smem_raw);  // [25][blockDim.x] partial diagonal blocks, one per thread
  const int t = threadIdx.x, bd = blockDim.x;
  const int lane = t % CL;
  int c = blockIdx.x * (bd / CL) + t / CL;
  bool active = c < m.ncv && st.case_active[m.case_of[c]];
  double rhs[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (active) {
    for (int e = 0; e < 25; e++) sD[e * bd + t] = JT(0);
    BT* O = (BT*)st.O;
    for (int k = m.slot_i[c] + lane; k < m.slot_i[c + 1]; k += CL) {
      const Slot s = m.slots[k];
      const int f = s.f;
      double nV[3], area;
      unit_normal(m, f, nV, area);
      if (s.nb >= 0) {
        // ---------------- internal face ----------------
        const int c0 = s.side == 0 ? c : s.nb;
        const int c1 = s.side == 0 ? s.nb : c;
        const double sg = s.side == 0 ? -1.0 : 1.0;  // residual sign of this cell
        const int fo = face_opts<KIND>(p, st, c0, c1);
        {
          FState L = recon(m, p, st, c0, f), R = recon(m, p, st, c1, f);
          double F[5];
          euler_flux_t<KIND>(F, L, R, area, nV, fo, KIND == 5 ? &st.jst[8 * c0] : nullptr,
                             KIND == 5 ? &st.jst[8 * c1] : nullptr);
          for (int i = 0; i < 5; i++) rhs[i] += sg * F[i];
        }
        JT Ob[25];
        const JT nVt[3] = {(JT)nV[0], (JT)nV[1], (JT)nV[2]};
        if (implicit) {
          FStateT<JT> L0 = fstate_as<JT>(cell_fstate(p, st, c0)), R0 = fstate_as<JT>(cell_fstate(p, st, c1));
          JT Apl[25], Ami[25];
          euler_matrices_t<KIND, JT>(Apl, Ami, L0, R0, (JT)area, nVt, fo);
          // row of c0: D += Apl, O(c0,c1) = Ami ; row of c1: D -= Ami, O(c1,c0) = -Apl
          if (s.side == 0) {
            for (int e = 0; e < 25; e++) { sD[e * bd + t] += Apl[e]; Ob[e] = Ami[e]; }
          } else {
            for (int e = 0; e < 25; e++) { sD[e * bd + t] -= Ami[e]; Ob[e] = -Apl[e]; }
          }
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
          if (implicit) {
            // row of c0: D -= A0, O -= A1 ; row of c1: D += A1, O += A0  (calcViscousFluxNS 3678-3696);
            // the diagonal part goes straight into the cell's shared-memory block
            const StridedBlock<JT> Ds{sD + t, bd};
            if (s.side == 0) {
              visc_jac_add<JT>(Ds, JT(-1.0), 0, vf, v0, ufa);
              visc_jac_add<JT>(Ob, JT(-1.0), 1, vf, v1, ufa);
            } else {
              visc_jac_add<JT>(Ds, JT(1.0), 1, vf, v1, ufa);
              visc_jac_add<JT>(Ob, JT(1.0), 0, vf, v0, ufa);
            }
          }
        }
        if (implicit)
          for (int e = 0; e < 25; e++) O[ell_index<BT>(m, c, s.col, e)] = (BT)Ob[e];
      } else {
        // ---------------- boundary face (the cell is cvofa[f][0]) ----------------
        const DevZone z = m.zones[m.bzone[f]];
        const double* bb = &st.bfa[8 * f];
        FState B;
        B.rho = bb[0]; B.u[0] = bb[1]; B.u[1] = bb[2]; B.u[2] = bb[3]; B.p = bb[4]; B.gam = p.gamma; B.h = bb[6];
        const FStateT<JT> Bt = fstate_as<JT>(B);
        const JT nVt[3] = {(JT)nV[0], (JT)nV[1], (JT)nV[2]};
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
          if (implicit) {
            if (z.kind == JG_BC_SYMMETRY && p.symm_bc == JG_SYMM_ANALYTICAL) {
              // analytical pressure Jacobian, JoeWithModels.cpp:3231-3251
              double a2 = p.gamma - 1.0;
              double phi = 0.5 * a2 * (B.u[0] * B.u[0] + B.u[1] * B.u[1] + B.u[2] * B.u[2]);
              for (int i = 0; i < 3; i++) {
                sD[(5 * (i + 1) + 0) * bd + t] += (JT)(phi * nV[i] * area);
                for (int j = 0; j < 3; j++) sD[(5 * (i + 1) + 1 + j) * bd + t] += (JT)(-a2 * B.u[j] * nV[i] * area);
                sD[(5 * (i + 1) + 4) * bd + t] += (JT)(a2 * nV[i] * area);
              }
            } else if (z.kind == JG_BC_SYMMETRY && p.symm_bc == JG_SYMM_NEW_NUMERIC) {
              JT Apl[25], Ami[25];
              euler_matrices_t<KIND, JT>(Apl, Ami, Bt, Bt, (JT)area, nVt, fob);
              for (int e = 0; e < 25; e++) sD[e * bd + t] += Apl[e] + Ami[e];
            } else {
              JT Apl[25];
              euler_matrices_t<KIND, JT>(Apl, (JT*)nullptr, Bt, Bt, (JT)area, nVt, fob);
              for (int e = 0; e < 25; e++) sD[e * bd + t] += Apl[e];
            }
          }
        } else {
          FState L = recon(m, p, st, c, f);
          euler_flux_t<KIND>(F, L, B, area, nV, fob, jb, jb);
          for (int i = 0; i < 5; i++) rhs[i] -= F[i];
          if (implicit) {
            FStateT<JT> L0 = fstate_as<JT>(cell_fstate(p, st, c));
            JT Apl[25];
            euler_matrices_t<KIND, JT>(Apl, (JT*)nullptr, L0, Bt, (JT)area, nVt, fob);
            for (int e = 0; e < 25; e++) sD[e * bd + t] += Apl[e];
          }
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
          if (implicit) visc_jac_add<JT>(StridedBlock<JT>{sD + t, bd}, JT(-1.0), 0, vf, v0, v1.u);
        }
      }
    }
  }
  // ---------------- epilogue ----------------
  // the lanes' partial residuals and diagonal blocks, summed in lane order (lanes of a cell share
  // its activity, so the whole warp reaches the shuffles)
  if (CL > 1) {
    for (int i = 0; i < 5; i++) {
      double tot = 0.0;
      for (int l = 0; l < CL; l++) tot += __shfl_sync(0xffffffffu, rhs[i], (t & 31) - lane + l);
      rhs[i] = tot;
    }
    __syncwarp();
  }
  if (active && lane == 0) {
    gravity_rhs(p, m, st, c, rhs);
    for (int i = 0; i < 5; i++) st.rhs[5 * c + i] = rhs[i];
    if (implicit) {
      double Dm[25];
      for (int e = 0; e < 25; e++) {
        JT d = sD[e * bd + t];
        for (int l = 1; l < CL; l++) d += sD[e * bd + t + l];
        Dm[e] = (double)d;
      }
      gravity_diag<5>(p, m, c, Dm);
      if (for_step) {
        double tmp = m.vol[c] / st.local_dt[c];
        for (int i = 0; i < 5; i++) Dm[6 * i] += tmp;
        for (int i = 0; i < 5; i++) st.b[5 * c + i] = p.under_relax * rhs[i];
      }
      BT* Dg = (BT*)st.D;
      for (int e = 0; e < 25; e++) Dg[(size_t)e * m.ncv + c] = (BT)Dm[e];
      if (for_step) {
        double Di[25];
        block_inverse(Dm, Di);
        BT* Dig = (BT*)st.Dinv;
        for (int e = 0; e < 25; e++) Dig[(size_t)e * m.ncv + c] = (BT)Di[e];
      }
    }
  }
}


template <typename BT, int KIND, int CL, int MINB>
static void launch_fused_cl(const Mesh& m, const Params& p, State& st, int for_step, cudaStream_t s) {
  size_t shm = 25 * TB * sizeof(BT);
  const int g = grid_for(m.ncv, TB / CL);
  if (p.viscous) k_flux<BT, KIND, 1, CL, MINB><<<g, TB, shm, s>>>(m, p, st, 1, for_step);
  else k_flux<BT, KIND, 0, CL, MINB><<<g, TB, shm, s>>>(m, p, st, 1, for_step);
}
// p.flux_cl: lanes per cell 1, 2 or 4 (two 128-thread blocks per SM), or JG_FLUX_CL1_3BLK
// (one lane, three blocks per SM)
template <typename BT, int KIND>
static void launch_fused_k(const Mesh& m, const Params& p, State& st, int for_step, cudaStream_t s) {
  if (p.flux_cl == 1) launch_fused_cl<BT, KIND, 1, 2>(m, p, st, for_step, s);
  else if (p.flux_cl == JG_FLUX_CL1_3BLK) launch_fused_cl<BT, KIND, 1, 3>(m, p, st, for_step, s);
  else if (p.flux_cl == 4) launch_fused_cl<BT, KIND, 4, 2>(m, p, st, for_step, s);
  else launch_fused_cl<BT, KIND, 2, 2>(m, p, st, for_step, s);
}
template <typename BT>
static void launch_fused_t(const Mesh& m, const Params& p, State& st, int for_step, cudaStream_t s) {
  if (p.flux == JG_FLUX_ROE) launch_fused_k<BT, 1>(m, p, st, for_step, s);
  else if (p.flux == JG_FLUX_AUSM) launch_fused_k<BT, 2>(m, p, st, for_step, s);
  else if (p.flux == JG_FLUX_HAENEL) launch_fused_k<BT, 3>(m, p, st, for_step, s);
  else if (p.flux == JG_FLUX_AUSMDV) launch_fused_k<BT, 4>(m, p, st, for_step, s);
  else if (p.flux == JG_FLUX_JST) launch_fused_k<BT, 5>(m, p, st, for_step, s);
  else launch_fused_k<BT, 0>(m, p, st, for_step, s);
}
// residual + Jacobian in one kernel, one thread (or CL lanes) per cell, so that the 32 lanes of a
// warp walk the same face position of neighbouring cells (coherent branches)
void launch_flux_fused(const Mesh& m, const Params& p, State& st, int for_step, cudaStream_t s) {
  if (p.fp32) launch_fused_t<float>(m, p, st, for_step, s);
  else launch_fused_t<double>(m, p, st, for_step, s);
}

}  // namespace jg
