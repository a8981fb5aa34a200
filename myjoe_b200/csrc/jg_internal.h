// jg_internal.h -- device-side data layout of one case and the kernel launchers.
//
// Cells keep the caller's numbering unless the handle renumbers them
// (jg_renumber.cu).  Per-cell vectors are stored
// cell-major ([N][k], a warp reads them contiguously); the implicit matrix is
// stored per row in a sliced-ELL layout: 32-cell slices (one warp), each
// slice padded to its widest row, components innermost across the 32 cells,
// so that writing a row block (flux kernel) and reading it (relaxation) are
// 256-byte coalesced transactions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/joe_b200.h"

namespace jg {

constexpr int SLICE = 32;
constexpr int MAX_COLOR_LISTS = 16;

struct DevZone {
  int kind;
  int scal_bc;      // bit 0: the transported scalar is Dirichlet (value v[6]) on this zone
  double v[8];
};

// face slot of a cell: face index, neighbour (-1 on boundary faces), side (0:
// the cell is cvofa[f][0], 1: it is cvofa[f][1]), ELL column (-1 on boundary faces)
struct Slot {
  int f, nb, side, col;
};

struct Mesh {
  int ncv, nfa, nfa_b, nzones;
  int nslices;
  const double* x_cv;      // [N][3]
  const double* vol;       // [N]
  const double* x_fa;      // [nfa][3]
  const double* fa_n;      // [nfa][3] area-weighted normal
  // static face geometry, formed once per mesh (k_face_geo) with the expressions the face loop used
  // to evaluate per face: fa_u[nfa][4] the unit normal and the area; fa_s[nfa - nfa_b][4] the unit
  // vector from cvofa[f][0]'s centre to cvofa[f][1]'s and its length (sVec, smag) of internal faces
  const double* fa_u;
  const double* fa_s;
  const int* cvofa;        // [nfa][2]
  const int* slot_i;       // [N+1] cell -> face slots (reference faocv order)
  const Slot* slots;       // [faocv_s]
  const int* nb_i;         // [N+1] nbocv CSR (diagonal first)
  const int* nb_v;         // [nbocv_s]
  const double* lsq;       // [nbocv_s][3]
  const int* bf_i;         // [N+1] cell -> its boundary faces (increasing face index)
  const int* bf_v;
  const double* blsq;      // [nfa_b][3]
  const int* bzone;        // [nfa_b] zone of each boundary face
  const DevZone* zones;
  const int* ell_off;      // [nslices+1] first ELL column row of each slice
  const int* ell_nb;       // [ell_rows*32] neighbour per ELL entry (padding: the cell itself)
  const uint8_t* ell_lower;// [ell_rows*32] 1 when the neighbour precedes the cell (LU-SGS)
  int ell_rows;
  const uint8_t* color;    // [N] colour of the cell (no two neighbours share one)
  int ncolors;
  // per colour q (q < MAX_COLOR_LISTS): the slices holding a cell of that colour are
  // color_slices[color_slice_off[q] .. color_slice_off[q+1]) (host-side offsets; no lists when
  // ncolors > MAX_COLOR_LISTS: every colour pass covers every slice)
  const int* color_slices;
  int color_slice_off[17];
  const int* case_of;      // [N] case of each cell (batches)
};

// Per-case device state.  Primitive record: u,v,w,p,T,h,c,pad.  Boundary
// record: rho,u,v,w,p,T,h,pad.  Gradients: [N][9] u, [N][3] rho, p, h.
struct State {
  double* q;        // [N][5] conserved (rho, rhou, rhoE)
  double* prim;     // [N][8]
  double* bfa;      // [nfa_b][8]
  double* mul_fa;   // [nfa]
  double* lam_fa;   // [nfa] lambda/cp
  double* gu;       // [N][9] Euler (second order) gradient of velocity
  double* guv;      // [N][9] viscous gradient of velocity (may alias gu)
  double* grho;     // [N][3]
  double* gp;       // [N][3]
  double* gh;       // [N][3]
  double* local_dt; // [N]
  double* rhs;      // [N][5] RHS of calcRhs (rho, rhou, rhoE)
  unsigned char* shock_flag;  // [N] AUSMDV shock fix: the cell touches a sonic internal face
  double* jst;                // [N][8] JST: pressure sensor, spectral radius, internal faces, undivided Laplacian[5]
  const unsigned char* jst_bcv;  // [N] JST's BoundaryCV: the cell is the first cell of an internal face
  double* b;        // [N][5] under-relaxed rhs of the linear system
  void* D;          // [25][N] diagonal block (double or float), component-major
  void* Dinv;       // [25][N] its inverse
  void* O;          // ELL off-diagonal blocks
  void* x0;         // [5][N] relaxation vectors (double or float)
  void* x1;
  double* dq;       // [N][5]
  double* blk;      // per-block partial sums (residual, dt min)
  double* ctrl;     // device control: [0]=cfl [1]=step [2]=dt_min [3..]=flags
  double* resid;    // [hist_cap][ncases][5] residual history (ring buffer)
  double* rpart;    // [nrblk][5] per-chunk L1 residual partials (chunks never straddle cases)
  int hist_cap;
  int* err;         // error flags
  int* case_err;    // [ncases] per-case error flags (1: rho/p <= 0, 4: NaN residual)
  uint8_t* case_active;  // [ncases] 0: case frozen (retired), its state is not updated
  double* mut_fa;   // [nfa] turbulent viscosity (coupled path), nullptr without a model
  const double* kine;  // [N] turbulent kinetic energy in the pressure recovery (SST), nullptr otherwise
  int bs;           // block size of the system: 5, or 6 with SA (rhs, b, dq, x, D, O, resid use it)
  // lagged Jacobian (jac_lag > 1, 5x5 path): the flux blocks of case k are formed again at the
  // step jac_next[k] (0: at the next step) and kept in between; D0 holds the face part of the
  // diagonal block ([25][N], matrix precision) to which each step adds its own vol/dt
  int jac_lag;
  void* D0;
  long long* jac_next;   // [ncases]
  // the face loop's residual and Jacobian kernels run on two streams; a step's control and time
  // step run beside its gradients, its residual norms beside its relaxation (host-side only)
  cudaStream_t aux;
  cudaEvent_t ev_fork, ev_join, ev_pre, ev_dt, ev_res, ev_resid;
};

// Transported scalars and turbulence-model arrays (coupled path only).
// Scalars are stored component-major: phi[s*N + c], phi_bfa[s*nfa_b + f],
// grad_phi[(s*N + c)*3 + j], diff[s*nfa + f].  SA: s = 0 nuSA; SST: s = 0
// kine, s = 1 omega.
struct Turb {
  int model;         // JG_TURB_SA / JG_TURB_SST
  int ns;            // scalars
  double* phi;
  double* phi_bfa;
  double* grad_phi;  // limited like the flow gradients
  double* diff;      // scalar diffusivities at faces
  double* wd;        // [N] wall distance
  double* strMag;    // [N]
  double* vortMag;   // [N]
  double* diverg;    // [N] (SST)
  double* crossDiff; // [N] (SST)
  double* F1;        // [N] Menter blending functions (SST)
  double* F2;
  const int* wall_f; // [nwall] WALL faces in zone order
  int nwall;
};

struct Params {
  double gamma, R, Pr, PrTurb;
  double cp;        // gamma R / (gamma - 1), the enthalpy per kelvin (set with gamma and R)
  double gravity[3];  // GX, GY, GZ of sourceHook; has_gravity: any of them non-zero
  int has_gravity;
  int mu_mode, flux;
  double mu_ref, mu_pow, SL_T, SL_S, T_ref;
  int second_order, limiter;
  double eps;
  int visc_limiter, symm_bc;
  int ts_mode, ts_method;
  double dt_fixed;
  int cfl_after, cfl_interval;
  double cfl_factor, cfl_max;
  double under_relax;
  int viscous;      // mu_ref > 0
  int fp32;         // matrix + relaxation in FP32
  int turb;         // JG_TURB_*
  // launch shapes (jg_autotune / jg_set_launch_config): the 5x5 face loop (fused: 1, 2 or 4
  // lanes per cell or JG_FLUX_CL1_3BLK; split: JG_FLUX_SPLIT + lanes per cell of the residual
  // kernel), and the 5x5 Jacobi sweep's kernel (0: a block per 32-cell slice with a thread per
  // block row, 1: a thread per cell)
  int flux_cl;
  int relax_variant;
  int grad_scheme;  // JG_GRAD_*
  // AUSMDV: the blend (JG_AUSM_*), entropy fix, shock fix (JG_SHOCK_FIX_*) and the flag
  // sum a face's two cells must exceed for it (1.1: both flagged, 0.9: either)
  int ausm_type, entropy_fix, shock_fix;
  double shock_flag_sum;
};

// launchers (jg_kernels.cu); all enqueue on stream s
void launch_state(const Mesh& m, const Params& p, State& st, cudaStream_t s);
void launch_hist_base(State& st, cudaStream_t s);
// in[13]: S0, S1, gu0, gu1, gh0, gh1, mul, lamOcp, u_fa, area, nvec, svec, smag (device arrays)
void launch_visc_faces(int n, const double* const* in, double* F, double* A0, double* A1, cudaStream_t s);
void launch_update_state(const Mesh& m, const Params& p, State& st, cudaStream_t s);
// the update from the relaxation's result x ([5][N], FP32 when x_fp32) without the dq copy
void launch_update_state_x(const Mesh& m, const Params& p, State& st, const void* x, int x_fp32, cudaStream_t s);
// launch_bc and launch_face_props in one launch
void launch_faces_after_update(const Mesh& m, const Params& p, State& st, cudaStream_t s);
void launch_face_props(const Mesh& m, const Params& p, State& st, cudaStream_t s);
void launch_bc(const Mesh& m, const Params& p, State& st, cudaStream_t s);
void launch_ctrl_step(const Params& p, State& st, cudaStream_t s);
void launch_dt(const Mesh& m, const Params& p, State& st, int use_ctrl_cfl, double cfl, cudaStream_t s);
void launch_grad(const Mesh& m, const Params& p, State& st, cudaStream_t s);
// the face loop: residual (+ Jacobian blocks when implicit; for_step adds vol/dt, inverts the
// diagonal and writes the under-relaxed rhs) -- split into a residual and a Jacobian kernel
// (jg_faceloop.cu) or fused (jg_fused.cu), by p.flux_cl
void launch_flux(const Mesh& m, const Params& p, State& st, int implicit, int for_step, cudaStream_t s);
void launch_flux_fused(const Mesh& m, const Params& p, State& st, int for_step, cudaStream_t s);
void launch_face_sensors(const Mesh& m, const Params& p, State& st, cudaStream_t s);
void launch_face_geo(const Mesh& m, double* fa_u, double* fa_s, cudaStream_t s);
// jg_step_host's upload (pack + state + history base) and download (unpack + flags + residuals)
void launch_state_in(const Mesh& m, const Params& p, State& st, const double* rho, const double* rhou,
                     const double* rhoE, const int* perm, cudaStream_t s);
void launch_state_out(const Mesh& m, State& st, double* rho, double* rhou, double* rhoE, const int* perm, double* out,
                      int nres, cudaStream_t s);
// face-loop launch shapes: split (residual kernel with FL lanes per cell + Jacobian kernel)
// are JG_FLUX_SPLIT + FL; the others are the fused kernel's
inline bool flux_split(const Params& p, const State& st) { return p.flux_cl >= JG_FLUX_SPLIT || st.jac_lag > 1; }
inline int flux_split_lanes(const Params& p) { return p.flux_cl >= JG_FLUX_SPLIT ? p.flux_cl - JG_FLUX_SPLIT : 4; }
void launch_resid(const Mesh& m, State& st, int hist_index_from_ctrl, cudaStream_t s);
// per-case residual history, resid[(idx*ncases + case)*5 + i]
// per-case L1 residual: RCHUNK-cell chunks counted from each case's first cell
// (rblk_off[k]..rblk_off[k+1] are case k's chunks, rblk_case maps a chunk to
// its case), then one warp per case sums its chunks in order
constexpr int RCHUNK = 256;
void launch_resid_cases(State& st, const int* case_off, const int* rblk_off, const int* rblk_case, int nrblk,
                        int ncases, int hist_from_ctrl, cudaStream_t s);
void launch_jacobi(const Mesh& m, const Params& p, State& st, int sweeps, cudaStream_t s);
// multicolour Gauss-Seidel: result in st.x0
void launch_sgs(const Mesh& m, const Params& p, State& st, int sweeps, cudaStream_t s);
void launch_dq_from_x(const Mesh& m, const Params& p, State& st, const void* x, cudaStream_t s);
void launch_lusgs(const Mesh& m, const Params& p, State& st, cudaStream_t s);
void launch_dinv(const Mesh& m, const Params& p, State& st, cudaStream_t s);
// BiCGSTAB building blocks (FP64)
void launch_spmv(const Mesh& m, const State& st, const double* x, double* y, cudaStream_t s);
void launch_precond(const Mesh& m, const State& st, const double* x, double* y, cudaStream_t s);
void launch_dot(int n, const double* a, const double* b, double* partial, double* out, cudaStream_t s);
void launch_resmax(const Mesh& m, const State& st, const double* r, double* partial, double* out, cudaStream_t s);
void launch_lin3(long n, double* out, double a, const double* x, double b, const double* y, double c, const double* z,
                 cudaStream_t s);
void launch_flux_faces(int kind, int n, const double* L, const double* R, const double* area, const double* nvec,
                       double* F, double* AL, double* AR, cudaStream_t s);

// io ([5][n] planes rho, rhou, rhoE) <-> q ([n][5]); perm (or nullptr): the io row of each cell
void launch_pack_state(int n, const double* io, double* q, const int* perm, cudaStream_t s);
void launch_unpack_state(int n, const double* q, double* io, const int* perm, cudaStream_t s);

int grid_for(long n, int block);
int record_error(int code, const char* msg);  // sets the jg_last_error message

}  // namespace jg

namespace jg {
// coupled turbulence-model path (jg_coupled.cu), block size 5 + ns
// wall distance of cells [c0, c1) to the WALL faces t.wall_f[w0 .. w1)
void launch_wall_distance(const Mesh& m, Turb& t, int c0, int c1, int w0, int w1, cudaStream_t s);
void launch_scalar_bc(const Mesh& m, const Params& p, State& st, Turb& t, cudaStream_t s);
// gradients of the flow (limited, as calcFluxCoupled takes them) and of nuSA,
// strain/vorticity magnitudes, turbulent viscosity and scalar diffusivity
void launch_turb_props(const Mesh& m, const Params& p, State& st, Turb& t, cudaStream_t s);
// calcRhsCoupled + the implicit-step epilogue: rhs[N][6], D/O (6x6), b, Dinv
void launch_flux6(const Mesh& m, const Params& p, State& st, Turb& t, int implicit, int for_step, cudaStream_t s);
void launch_relax6(const Mesh& m, const Params& p, State& st, int sgs, int sweeps, int bs, cudaStream_t s);
// Q += dq (x: the relaxation result, [6][N]), nuSA = clip((nuSA (rho_new - dq0) + dq5) / rho_new)
void launch_update6(const Mesh& m, const Params& p, State& st, Turb& t, const void* x, cudaStream_t s);
// the flow gradients as calcFluxCoupled takes them (jg_kernels.cu)
void launch_grad_coupled(const Mesh& m, const Params& p, State& st, cudaStream_t s);
}  // namespace jg

namespace jg {
// Lines of the BCGSTAB_LINELET preconditioner (jg_linelet.cu): the lines of
// two or more cells, cells in line order; per line cell the inverse of its
// eliminated diagonal block, the multiplier A(c_i, c_{i-1}) inv_{i-1} and the
// upper block A(c_{i-1}, c_i) (row-major 5x5), and the forward-substitution
// vector.
struct Lines {
  int nlines;
  const int* off;  // [nlines+1]
  const int* cv;   // [off[nlines]]
  // per line position k > off[l]: the ELL row index of the block coupling cv[k] to cv[k-1] in
  // cv[k]'s row (jlo) and of the block coupling cv[k-1] to cv[k] in cv[k-1]'s row (jup); -1: no
  // coupling, -2: several faces between the two cells (their blocks are summed by a search)
  const int* jlo;
  const int* jup;
  // BCGSTAB_LINELET (5x5, FP64)
  double* inv;     // [off[nlines]][25]
  double* low;     // [off[nlines]][25] (position 0 of a line unused)
  double* up;      // [off[nlines]][25] (position 0 of a line unused)
  double* v;       // [off[nlines]][5]
  // LINE relaxation (B x B blocks in the matrix precision)
  const uint8_t* on_line;     // [N] 1 on the cells of the lines
  const uint8_t* ell_inline;  // [ell_rows*32] 1 where the ELL entry couples a cell to its line neighbour
  void* binv;      // [off[nlines]][B*B]
  void* blow;      // [off[nlines]][B*B]
  void* bup;       // [off[nlines]][B*B]
  void* bv;        // [off[nlines]][B]
};
// initializeLinelet on a mesh: wall_zones holds the faces of each WALL zone in zone order
// (relaxed: the LINE relaxation's rule, which also crosses prism/hexahedron interfaces)
int build_lines(const jg_mesh& m, const std::vector<std::vector<int>>& wall_zones, std::vector<int>& off,
                std::vector<int>& cv, bool relaxed);
void launch_line_factor(const Mesh& m, const State& st, const Lines& L, cudaStream_t s);
// y = the line-implicit preconditioner applied to x ([5][N] both)
void launch_line_precond(const Mesh& m, const State& st, const Lines& L, const double* x, double* y,
                         cudaStream_t s);
// [N][5] -> [5][N]
void launch_aos_to_soa5(int n, const double* aos, double* soa, cudaStream_t s);
// LINE relaxation of the assembled system (block size bs, matrix precision of p): the
// block-tridiagonal factors of every line, then `sweeps` line-Jacobi sweeps from x = 0;
// the result is in st.x0 (odd sweeps) or st.x1 (even)
void launch_line_relax(const Mesh& m, const Params& p, State& st, const Lines& L, int bs, int sweeps,
                       cudaStream_t s);

// A mesh in jg_mesh's layout whose arrays the struct owns (concatenated
// batches, renumbered cases); bind() points m at the vectors.
struct MeshOwned {
  std::vector<int> cvofa, faocv_i, faocv_v, nbocv_i, nbocv_v;
  std::vector<double> x_cv, x_fa, fa_normal, vol, lsq, blsq;
  std::vector<jg_zone> zones;
  jg_mesh m{};
  void bind();
};
// the caller's id of each cell, face and nbocv entry in a handle's own order (jg_renumber.cu)
struct Renumbering {
  std::vector<int> cell_old, face_old, nbs_old;
};
int rcm_order(const jg_mesh& m, std::vector<int>& cell_old);
int rcm_color_order(const jg_mesh& m, std::vector<int>& cell_old);
int rcm_lines_order(const jg_mesh& m, std::vector<int>& cell_old);
int cell_order(const jg_mesh& m, int method, std::vector<int>& cell_old);
int renumber_mesh(const jg_mesh& in, int method, MeshOwned& out, Renumbering& r);
}  // namespace jg

// per-case operations used by the serving engine (defined in jg_api.cu)
struct jg_case;
namespace jg {
int serve_case_create(const jg_mesh* mesh, const jg_params* params, jg_case** out);
int serve_case_start(jg_case* h, const double* rho, const double* rhou, const double* rhoE);
int serve_case_launch(jg_case* h, int nsteps, double* h_ring, int* h_err, cudaEvent_t ev);
int serve_case_ring(jg_case* h);
size_t serve_case_bytes(jg_case* h);
int serve_case_ncv(jg_case* h);
int serve_set_err(int code, const char* msg);
// what the restart bridge needs of a handle: caller cells, transported
// scalars, turbulence model, cases, the CFL the ramp starts from
int case_restart_info(jg_case* h, int* ncv, int* nscal, int* turb_model, int* ncases, double* cfl0);
}  // namespace jg
