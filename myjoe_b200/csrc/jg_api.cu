// jg_api.cu -- host side of libjoe_b200.so: the C ABI declared in
// include/joe_b200.h.  Builds the device layout of a case from the
// reference's arrays, runs the operators, captures the backward-Euler step in
// a CUDA graph, and converts between the reference's block-CSR matrix and the
// device's sliced-ELL rows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "jg_internal.h"

using namespace jg;

static thread_local std::string g_err;

static int set_err(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(x)                                                                                       \
  do {                                                                                              \
    cudaError_t e_ = (x);                                                                           \
    if (e_ != cudaSuccess)                                                                          \
      return set_err(e_ == cudaErrorMemoryAllocation ? JG_ERR_NOMEM : JG_ERR_CUDA, "%s: %s (%s:%d)", \
                     #x, cudaGetErrorString(e_), __FILE__, __LINE__);                              \
  } while (0)

#define CKL()                                                                                      \
  do {                                                                                             \
    cudaError_t e_ = cudaGetLastError();                                                           \
    if (e_ != cudaSuccess)                                                                         \
      return set_err(JG_ERR_CUDA, "launch: %s (%s:%d)", cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

struct jg_case {
  // host copies needed for conversions
  int ncv, nfa, nfa_b, nbs, nzones;
  std::vector<int> nbocv_i, nbocv_v;
  std::vector<int> cell_cols;     // [ncv+1] CSR over (cell, ELL column) -> neighbour
  std::vector<int> col_nb;
  std::vector<int> ell_off;
  jg_params hp;
  Params p;
  Mesh m;
  State st;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  size_t eltsz = 8;   // matrix element size
  size_t ell_elems = 0;
  int hist_cap = 0;
  double* d_tmp = nullptr;  // BiCGSTAB work vectors (9 x 5N) + partials
  double* d_red = nullptr;
  cudaGraphExec_t graph = nullptr;
  int graph_sweeps = -1;
  int primed = 0;           // state + BC computed since the last set_state
  int ncolors = 1;
  int ncases = 1;           // independent cases concatenated in this handle (jg_batch_create)
  std::vector<int> case_off;        // [ncases+1] first cell of each case
  std::vector<int> case_nfa_b_off;  // [ncases+1] first boundary face of each case
  int* d_case_off = nullptr;
  int nrblk = 0;                    // residual chunks (RCHUNK cells, case-local)
  int* d_rblk_off = nullptr;        // [ncases+1]
  int* d_rblk_case = nullptr;       // [nrblk]
  int profiling = 0;        // record events around the face loop and the relaxation in the graph
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t graph_kernels = 0;
  double* d_io = nullptr;   // [5][N] staging for direct host<->device state copies
  // pinned host staging for the error flags and a call's residual history: the reads of a call
  // are asynchronous copies that one synchronisation completes
  void* hpin = nullptr;
  size_t hpin_bytes = 0;
  double* d_out = nullptr;  // jg_step_host: the call's flags and residuals gathered on the device
  int d_out_cap = 0;
  long graph_gen = 0;       // counts the step graph's instantiations
  // jg_step_host on page-locked arrays, one step: the whole call (copies, state passes, the
  // step, copies back) captured as one graph, for the arrays, staging and step graph it was made with
  cudaGraphExec_t host_graph = nullptr;
  const void* host_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  long host_gen = -1;
  int host_nres = -1;
  int async_alloc = 0;      // stream-ordered allocation (serving): no device-wide sync on free
  size_t bytes = 0;         // device bytes held by this handle
  int bs = 5;               // block size: 5, or 6 on the coupled SA path
  Turb turb{};              // SA arrays (coupled path)
  Renumbering rn;           // caller's id of each internal cell / face / nbocv entry (empty: same order)
  Lines lines{};            // BCGSTAB_LINELET lines (nlines 0 otherwise)
  int* d_cell_old = nullptr;  // rn.cell_old on the device (state staging)
  // a renumbered batch: each case's caller-order id of its cells (case-local), host and device
  std::vector<int> case_cell_old;
  int* d_case_cell_old = nullptr;
};

// Rows between the handle's order and the caller's: an array of nblk blocks
// of n rows of w doubles; perm[r] is the caller's row of internal row r
// (empty: the same order).
static void rows_to_caller(const std::vector<int>& perm, const double* in, double* out, size_t n, size_t w,
                           size_t nblk = 1) {
  if (perm.empty()) {
    memcpy(out, in, n * w * nblk * sizeof(double));
    return;
  }
  for (size_t b = 0; b < nblk; b++)
    for (size_t r = 0; r < n; r++) memcpy(out + (b * n + perm[r]) * w, in + (b * n + r) * w, w * sizeof(double));
}

static void rows_from_caller(const std::vector<int>& perm, const double* in, double* out, size_t n, size_t w,
                             size_t nblk = 1) {
  if (perm.empty()) {
    memcpy(out, in, n * w * nblk * sizeof(double));
    return;
  }
  for (size_t b = 0; b < nblk; b++)
    for (size_t r = 0; r < n; r++) memcpy(out + (b * n + r) * w, in + (b * n + perm[r]) * w, w * sizeof(double));
}


// every device allocation of a handle goes through here; sizes are rounded to
// 256 bytes so that the footprint estimate (jg_case_footprint) can mirror them
static inline size_t alloc_round(size_t bytes) { return (std::max<size_t>(bytes, 8) + 255) & ~(size_t)255; }

static int dmalloc_bytes(jg_case* h, void** p, size_t bytes) {
  void* q = nullptr;
  bytes = alloc_round(bytes);
  if (h->async_alloc) {
    CK(cudaMallocAsync(&q, bytes, h->stream));
    h->allocs.push_back(q);
    CK(cudaMemsetAsync(q, 0, bytes, h->stream));
  } else {
    CK(cudaMalloc(&q, bytes));
    h->allocs.push_back(q);
    CK(cudaMemsetAsync(q, 0, bytes, h->stream));  // ordered before the handle's own kernels
  }
  h->bytes += bytes;
  *p = q;
  return JG_OK;
}

#define RC(x)                \
  do {                       \
    int rc_ = (x);           \
    if (rc_ != JG_OK) return rc_; \
  } while (0)

template <typename T>
static int dmalloc(jg_case* h, T** p, size_t count) {
  void* q = nullptr;
  RC(dmalloc_bytes(h, &q, std::max<size_t>(count, 1) * sizeof(T)));
  *p = (T*)q;
  return JG_OK;
}

template <typename T>
static int upload(jg_case* h, const T** dst, const T* src, size_t count) {
  T* d = nullptr;
  int rc = dmalloc(h, &d, count);
  if (rc) return rc;
  // pageable source: the call returns once the data is staged, so the caller's
  // (temporary) host array may go away at once
  if (count) CK(cudaMemcpyAsync(d, src, count * sizeof(T), cudaMemcpyHostToDevice, h->stream));
  *dst = d;
  return JG_OK;
}

// a device array of the handle -> the caller's host array, rows in the caller's order
static int download_rows(jg_case* h, const double* dev, double* host, const std::vector<int>& perm, size_t n,
                         size_t w, size_t nblk = 1) {
  const size_t len = n * w * nblk;
  if (perm.empty()) {
    if (len) CK(cudaMemcpyAsync(host, dev, len * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return JG_OK;
  }
  std::vector<double> tmp(len);
  if (len) CK(cudaMemcpyAsync(tmp.data(), dev, len * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  rows_to_caller(perm, tmp.data(), host, n, w, nblk);
  return JG_OK;
}

// the caller's host rows -> a device array of the handle (synchronous: the caller's array may go away)
static int upload_rows(jg_case* h, double* dev, const double* host, const std::vector<int>& perm, size_t n,
                       size_t w, size_t nblk = 1) {
  const size_t len = n * w * nblk;
  std::vector<double> tmp(len);
  rows_from_caller(perm, host, tmp.data(), n, w, nblk);
  if (len) CK(cudaMemcpyAsync(dev, tmp.data(), len * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return JG_OK;
}

// the faces of each WALL zone, zone by zone, each zone in the caller's face order
static std::vector<std::vector<int>> wall_zone_faces(const jg_mesh* mesh, const std::vector<int>& face_old) {
  std::vector<std::vector<int>> zs;
  for (int z = 0; z < mesh->nzones; z++)
    if (mesh->zones[z].kind == JG_BC_WALL) {
      std::vector<int> f;
      for (int i = mesh->zones[z].ifa_f; i <= mesh->zones[z].ifa_l; i++) f.push_back(i);
      if (!face_old.empty())
        std::sort(f.begin(), f.end(), [&](int a, int b) { return face_old[a] < face_old[b]; });
      zs.push_back(std::move(f));
    }
  return zs;
}

// the lines of two or more cells of initializeLinelet, longest first: the line kernels give a
// warp one line (factors) or four (substitutions), and lines of equal length side by side keep
// the warps of a block, and the lanes of a warp, busy to the same step (each line's elimination
// is independent of the others, so their order changes no result)
static void multi_cell_lines(const jg_mesh* mesh, const std::vector<int>& face_old, std::vector<int>& off,
                             std::vector<int>& cv, bool relaxed) {
  std::vector<int> o, c;
  build_lines(*mesh, wall_zone_faces(mesh, face_old), o, c, relaxed);
  std::vector<int> ls;
  for (size_t l = 0; l + 1 < o.size(); l++)
    if (o[l + 1] - o[l] >= 2) ls.push_back((int)l);
  std::stable_sort(ls.begin(), ls.end(), [&](int a, int b) { return o[a + 1] - o[a] > o[b + 1] - o[b]; });
  off.assign(1, 0);
  cv.clear();
  for (int l : ls) {
    cv.insert(cv.end(), c.begin() + o[l], c.begin() + o[l + 1]);
    off.push_back((int)cv.size());
  }
}

static Params make_params(const jg_params& q) {
  Params p;
  memset(&p, 0, sizeof(p));
  p.gamma = q.gamma;
  p.R = q.R_gas;
  p.cp = p.gamma * p.R / (p.gamma - 1.0);
  for (int i = 0; i < 3; i++) p.gravity[i] = q.gravity[i];
  p.has_gravity = q.gravity[0] != 0.0 || q.gravity[1] != 0.0 || q.gravity[2] != 0.0;
  p.Pr = q.Pr;
  p.PrTurb = q.PrTurb;
  p.mu_mode = q.mu_mode;
  p.flux = q.flux;
  p.mu_ref = q.mu_ref;
  p.mu_pow = q.mu_power_law;
  p.SL_T = q.SL_Tref;
  p.SL_S = q.SL_Sref;
  p.T_ref = q.T_ref;
  p.second_order = q.second_order;
  p.limiter = q.limiter;
  p.eps = q.eps;
  p.visc_limiter = q.visc_limiter;
  p.symm_bc = q.symm_bc;
  p.ts_mode = q.time_step_mode;
  p.ts_method = q.time_step;
  p.dt_fixed = q.dt;
  p.cfl_after = q.cfl_after;
  p.cfl_interval = q.cfl_interval > 0 ? q.cfl_interval : 1;
  p.cfl_factor = q.cfl_factor;
  p.cfl_max = q.cfl_max;
  p.under_relax = q.under_relax;
  p.viscous = q.mu_ref > 0.0;
  p.fp32 = q.precision == JG_PREC_MIXED;
  p.flux_cl = JG_FLUX_SPLIT + 4;  // the split face loop, 4 lanes per cell in the residual
  p.relax_variant = 0;
  p.grad_scheme = q.grad_scheme;
  p.ausm_type = q.ausm_type;
  p.entropy_fix = q.entropy_fix ? 1 : 0;
  p.shock_fix = q.flux == JG_FLUX_AUSMDV ? q.shock_fix : JG_SHOCK_FIX_NONE;
  p.shock_flag_sum = q.shock_flag == JG_SHOCK_FLAG_TET ? 0.9 : 1.1;
  return p;
}

static int check_params(const jg_params* q) {
  if (!q) return set_err(JG_ERR_ARG, "null params");
  if (q->flux < 0 || q->flux > 5) return set_err(JG_ERR_ARG, "unsupported flux %d", q->flux);
  if (q->flux == JG_FLUX_AUSMDV) {
    if (q->ausm_type < 0 || q->ausm_type > 2) return set_err(JG_ERR_ARG, "unsupported AUSM type %d", q->ausm_type);
    if (q->shock_fix < 0 || q->shock_fix > 2) return set_err(JG_ERR_ARG, "unsupported shock fix %d", q->shock_fix);
    if (q->shock_flag < 0 || q->shock_flag > 1) return set_err(JG_ERR_ARG, "unsupported shock flag %d", q->shock_flag);
  }
  if (q->symm_bc < 0 || q->symm_bc > 2) return set_err(JG_ERR_ARG, "unsupported SYMM_BC %d", q->symm_bc);
  if (q->lin_solver < 0 || q->lin_solver > 5) return set_err(JG_ERR_ARG, "unsupported linear solver %d", q->lin_solver);
  if (q->precision != JG_PREC_FP64 && q->precision != JG_PREC_MIXED)
    return set_err(JG_ERR_ARG, "unsupported precision %d", q->precision);
  if (q->precision == JG_PREC_MIXED && (q->lin_solver == JG_LS_BCGSTAB || q->lin_solver == JG_LS_LUSGS ||
                                        q->lin_solver == JG_LS_BCGSTAB_LINELET))
    return set_err(JG_ERR_ARG, "the mixed-precision form relaxes with JACOBI, SGS or LINE sweeps");
  if (q->turb_model == JG_TURB_SA || q->turb_model == JG_TURB_SST) {
    if (q->nscal != (q->turb_model == JG_TURB_SA ? 1 : 2))
      return set_err(JG_ERR_ARG, "SA transports one scalar (nscal = 1), SST two (nscal = 2)");
    if (!(q->mu_ref > 0.0)) return set_err(JG_ERR_ARG, "a turbulence model needs a viscous case (mu_ref > 0)");
    // calcFluxCoupled's flux choices (JoeWithModels.cpp:4987-5057)
    if (q->flux != JG_FLUX_HLLC && q->flux != JG_FLUX_AUSMDV && q->flux != JG_FLUX_HAENEL)
      return set_err(JG_ERR_ARG, "the coupled path takes the HLLC, AUSMDV (AUSMV, AUSMD) or HAENEL flux");
    if (q->lin_solver != JG_LS_JACOBI && q->lin_solver != JG_LS_SGS && q->lin_solver != JG_LS_LINE)
      return set_err(JG_ERR_ARG, "the coupled path relaxes with JACOBI, SGS or LINE sweeps");
  } else if (q->turb_model != JG_TURB_NONE) {
    return set_err(JG_ERR_ARG, "unsupported turbulence model %d", q->turb_model);
  } else if (q->nscal != 0) {
    return set_err(JG_ERR_ARG, "transported scalars need a turbulence model");
  }
  if (q->time_step_mode < 0 || q->time_step_mode > 2) return set_err(JG_ERR_ARG, "bad time step mode");
  if (q->grad_scheme != JG_GRAD_LSQ && q->grad_scheme != JG_GRAD_GREENGAUSS && q->grad_scheme != JG_GRAD_SDWLS)
    return set_err(JG_ERR_ARG, "unsupported gradient scheme %d", q->grad_scheme);
  if (q->grad_scheme != JG_GRAD_LSQ && q->turb_model != JG_TURB_NONE)
    return set_err(JG_ERR_ARG, "Green-Gauss and SDWLS gradients: cases without a turbulence model");
  if (q->grad_scheme == JG_GRAD_SDWLS && q->limiter)
    return set_err(JG_ERR_ARG, "SDWLS gradients take no limiter (limiter = 0)");
  if (q->renumber < JG_RENUMBER_NONE || q->renumber > JG_RENUMBER_RCM_LINES)
    return set_err(JG_ERR_ARG, "unsupported renumbering %d", q->renumber);
  if (!(q->gamma > 1.0) || !(q->R_gas > 0.0)) return set_err(JG_ERR_ARG, "bad gas constants");
  if (q->jac_lag < 0) return set_err(JG_ERR_ARG, "bad Jacobian lag %d", q->jac_lag);
  if (q->jac_lag > 1 && q->turb_model != JG_TURB_NONE)
    return set_err(JG_ERR_ARG, "a lagged Jacobian: cases without a turbulence model");
  if (q->jac_lag > 1 && (q->lin_solver == JG_LS_BCGSTAB || q->lin_solver == JG_LS_BCGSTAB_LINELET))
    return set_err(JG_ERR_ARG, "a lagged Jacobian: captured linear solvers (JACOBI, SGS, LINE, LUSGS)");
  return JG_OK;
}

namespace jg {
// lets the other translation units of the library set the jg_last_error message
int record_error(int code, const char* msg) { return set_err(code, "%s", msg); }
}  // namespace jg

extern "C" {

const char* jg_last_error(void) { return g_err.c_str(); }

int jg_version(void) { return 1; }

int jg_device_count(int* n) {
  int c = 0;
  cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) c = 0;
  if (n) *n = c;
  return c > 0 ? JG_OK : set_err(JG_ERR_NODEVICE, "no CUDA device: %s", cudaGetErrorString(e));
}

int jg_destroy(jg_case_t* h) {
  if (!h) return JG_OK;
  if (h->graph) cudaGraphExecDestroy(h->graph);
  if (h->host_graph) cudaGraphExecDestroy(h->host_graph);
  for (int i = 0; i < 4; i++)
    if (h->ev[i]) cudaEventDestroy(h->ev[i]);
  if (h->async_alloc) {
    for (void* p : h->allocs) cudaFreeAsync(p, h->stream);
  } else {
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (void* p : h->allocs) cudaFree(p);
  }
  if (h->st.aux) cudaStreamSynchronize(h->st.aux);
  if (h->stream) cudaStreamDestroy(h->stream);
  if (h->st.aux) cudaStreamDestroy(h->st.aux);
  if (h->st.ev_fork) cudaEventDestroy(h->st.ev_fork);
  if (h->st.ev_join) cudaEventDestroy(h->st.ev_join);
  if (h->hpin) cudaFreeHost(h->hpin);
  if (h->st.ev_pre) cudaEventDestroy(h->st.ev_pre);
  if (h->st.ev_dt) cudaEventDestroy(h->st.ev_dt);
  if (h->st.ev_res) cudaEventDestroy(h->st.ev_res);
  if (h->st.ev_resid) cudaEventDestroy(h->st.ev_resid);
  delete h;
  return JG_OK;
}

// Greedy colouring of the cell graph (neighbours through internal faces) in cell order: each cell
// takes the smallest colour none of its lower-numbered neighbours has.  With at most
// MAX_COLOR_LISTS colours, also the slices holding a cell of each colour, colour by colour
// (cslices[coff[q] .. coff[q+1])).  Returns the number of colours.
static int color_cells(const jg_mesh* mesh, std::vector<uint8_t>& color, std::vector<int>& cslices,
                       std::vector<int>& coff) {
  const int N = mesh->ncv;
  std::vector<int> adj_i(N + 1, 0), adj_v;
  for (int f = mesh->nfa_b; f < mesh->nfa; f++) {
    adj_i[mesh->cvofa[2 * f] + 1]++;
    adj_i[mesh->cvofa[2 * f + 1] + 1]++;
  }
  for (int c = 0; c < N; c++) adj_i[c + 1] += adj_i[c];
  adj_v.resize(adj_i[N]);
  {
    std::vector<int> fill(adj_i.begin(), adj_i.end() - 1);
    for (int f = mesh->nfa_b; f < mesh->nfa; f++) {
      const int a = mesh->cvofa[2 * f], b = mesh->cvofa[2 * f + 1];
      adj_v[fill[a]++] = b;
      adj_v[fill[b]++] = a;
    }
  }
  color.assign(N, 0);
  int ncolors = 1;
  std::vector<int> mark(256, -1);
  for (int c = 0; c < N; c++) {
    for (int k = adj_i[c]; k < adj_i[c + 1]; k++)
      if (adj_v[k] < c) mark[color[adj_v[k]]] = c;
    int k = 0;
    while (k < 255 && mark[k] == c) k++;
    color[c] = (uint8_t)k;
    ncolors = std::max(ncolors, k + 1);
  }
  cslices.clear();
  coff.assign(1, 0);
  if (ncolors <= MAX_COLOR_LISTS) {
    const int nslices = (N + SLICE - 1) / SLICE;
    std::vector<uint32_t> has(nslices, 0);  // bit q: the slice holds a cell of colour q
    for (int c = 0; c < N; c++) has[c / SLICE] |= 1u << color[c];
    for (int q = 0; q < ncolors; q++) {
      for (int sl = 0; sl < nslices; sl++)
        if (has[sl] & (1u << q)) cslices.push_back(sl);
      coff.push_back((int)cslices.size());
    }
  }
  return ncolors;
}

static int build(jg_case* h, const jg_mesh* mesh, const jg_params* q) {
  const int N = mesh->ncv, nfa = mesh->nfa, nfa_b = mesh->nfa_b;
  if (!h->stream) CK(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  if (q->turb_model == JG_TURB_NONE && !h->st.aux) {
    // the face loop's Jacobian kernel runs beside its residual kernel on a second stream; the
    // step control and time step beside the gradients, the residual norms beside the relaxation
    CK(cudaStreamCreateWithFlags(&h->st.aux, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&h->st.ev_fork, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->st.ev_join, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->st.ev_pre, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->st.ev_dt, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->st.ev_res, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&h->st.ev_resid, cudaEventDisableTiming));
  }
  h->ncv = N;
  h->nfa = nfa;
  h->nfa_b = nfa_b;
  h->nbs = mesh->nbocv_s;
  h->nzones = mesh->nzones;
  h->hp = *q;
  h->p = make_params(*q);
  h->eltsz = h->p.fp32 ? 4 : 8;
  h->bs = (q->turb_model == JG_TURB_NONE) ? 5 : 5 + q->nscal;
  const int bs = h->bs;
  h->nbocv_i.assign(mesh->nbocv_i, mesh->nbocv_i + N + 1);
  h->nbocv_v.assign(mesh->nbocv_v, mesh->nbocv_v + mesh->nbocv_s);
  // boundary-face zones
  std::vector<int> bzone(nfa_b, -1);
  std::vector<DevZone> zones(std::max(1, mesh->nzones));
  for (int z = 0; z < mesh->nzones; z++) {
    const jg_zone& zn = mesh->zones[z];
    if (zn.ifa_f < 0 || zn.ifa_l >= nfa_b || zn.ifa_f > zn.ifa_l + 1)
      return set_err(JG_ERR_ARG, "zone %d face range [%d,%d] outside the boundary faces", z, zn.ifa_f, zn.ifa_l);
    if (zn.kind < JG_BC_SYMMETRY || zn.kind > JG_BC_FARFIELD)
      return set_err(JG_ERR_ARG, "zone %d: unsupported boundary kind %d", z, zn.kind);
    zones[z].kind = zn.kind;
    zones[z].scal_bc = zn.scal_bc;
    for (int k = 0; k < 8; k++) zones[z].v[k] = zn.v[k];
    for (int f = zn.ifa_f; f <= zn.ifa_l; f++) bzone[f] = z;
  }
  for (int f = 0; f < nfa_b; f++)
    if (bzone[f] < 0) return set_err(JG_ERR_ARG, "boundary face %d has no zone (reference: no bc set)", f);
  // cell face slots
  const int* fi = mesh->faocv_i;
  const int* fv = mesh->faocv_v;
  std::vector<Slot> slots(fi[N]);
  std::vector<int> ncols(N, 0);
  std::vector<int> bf_i(N + 1, 0), bf_v;
  h->cell_cols.assign(N + 1, 0);
  h->col_nb.clear();
  for (int c = 0; c < N; c++) {
    for (int k = fi[c]; k < fi[c + 1]; k++) {
      int f = fv[k];
      if (f < 0 || f >= nfa) return set_err(JG_ERR_ARG, "faocv_v[%d] = %d out of range", k, f);
      Slot s;
      s.f = f;
      if (f < nfa_b) {
        if (mesh->cvofa[2 * f] != c) return set_err(JG_ERR_ARG, "boundary face %d is not owned by cell %d", f, c);
        s.nb = -1; s.side = 0; s.col = -1;
        bf_v.push_back(f);
      } else {
        int c0 = mesh->cvofa[2 * f], c1 = mesh->cvofa[2 * f + 1];
        if (c1 < 0 || c1 >= N || c0 < 0 || c0 >= N || (c0 != c && c1 != c))
          return set_err(JG_ERR_ARG, "internal face %d does not connect cell %d", f, c);
        s.side = (c0 == c) ? 0 : 1;
        s.nb = (c0 == c) ? c1 : c0;
        s.col = ncols[c]++;
        h->col_nb.push_back(s.nb);
      }
      slots[k] = s;
    }
    bf_i[c + 1] = (int)bf_v.size();
    h->cell_cols[c + 1] = (int)h->col_nb.size();
  }
  // sliced ELL
  int nslices = (N + SLICE - 1) / SLICE;
  h->ell_off.assign(nslices + 1, 0);
  for (int s = 0; s < nslices; s++) {
    int w = 0;
    for (int c = s * SLICE; c < std::min(N, (s + 1) * SLICE); c++) w = std::max(w, ncols[c]);
    h->ell_off[s + 1] = h->ell_off[s] + w;
  }
  int rows = h->ell_off[nslices];
  std::vector<int> ell_nb((size_t)rows * SLICE, 0);
  std::vector<uint8_t> ell_lower((size_t)rows * SLICE, 0);
  for (int c = 0; c < N; c++) {
    int s = c / SLICE, lane = c % SLICE;
    int w = h->ell_off[s + 1] - h->ell_off[s];
    for (int j = 0; j < w; j++) {
      size_t e = (size_t)(h->ell_off[s] + j) * SLICE + lane;
      if (j < ncols[c]) {
        int nb = h->col_nb[h->cell_cols[c] + j];
        ell_nb[e] = nb;
        ell_lower[e] = nb < c ? 1 : 2;
      } else {
        ell_nb[e] = c;  // padding: zero block times the cell's own value
      }
    }
  }
  h->ell_elems = (size_t)rows * bs * bs * SLICE;
  // greedy colouring of the cell graph (neighbours through internal faces), in cell order, and per
  // colour the slices that hold a cell of that colour (a colour pass launches over these only)
  std::vector<uint8_t> color;
  std::vector<int> cslices, coff;
  const int ncolors = color_cells(mesh, color, cslices, coff);
  h->ncolors = ncolors;
  // device mesh
  Mesh& m = h->m;
  memset(&m, 0, sizeof(m));
  if (ncolors <= MAX_COLOR_LISTS) {
    RC(upload(h, &m.color_slices, cslices.data(), cslices.size()));
    for (int c = 0; c <= ncolors; c++) m.color_slice_off[c] = coff[c];
  }
  m.ncv = N; m.nfa = nfa; m.nfa_b = nfa_b; m.nzones = mesh->nzones; m.nslices = nslices; m.ell_rows = rows;
  RC(upload(h, &m.x_cv, mesh->x_cv, 3 * (size_t)N));
  RC(upload(h, &m.vol, mesh->cv_volume, (size_t)N));
  RC(upload(h, &m.x_fa, mesh->x_fa, 3 * (size_t)nfa));
  RC(upload(h, &m.fa_n, mesh->fa_normal, 3 * (size_t)nfa));
  RC(upload(h, &m.cvofa, mesh->cvofa, 2 * (size_t)nfa));
  {
    double *fu = nullptr, *fs = nullptr;
    RC(dmalloc(h, &fu, 4 * (size_t)nfa));
    RC(dmalloc(h, &fs, 4 * (size_t)(nfa - nfa_b)));
    m.fa_u = fu;
    m.fa_s = fs;
  }
  RC(upload(h, &m.slot_i, fi, (size_t)N + 1));
  RC(upload(h, &m.slots, slots.data(), slots.size()));
  RC(upload(h, &m.nb_i, mesh->nbocv_i, (size_t)N + 1));
  RC(upload(h, &m.nb_v, mesh->nbocv_v, (size_t)mesh->nbocv_s));
  RC(upload(h, &m.lsq, mesh->nbocv_lsg_coeff, 3 * (size_t)mesh->nbocv_s));
  RC(upload(h, &m.bf_i, bf_i.data(), bf_i.size()));
  RC(upload(h, &m.bf_v, bf_v.data(), bf_v.size()));
  RC(upload(h, &m.blsq, mesh->boundary_fa_lsg_coeff, 3 * (size_t)nfa_b));
  RC(upload(h, &m.bzone, bzone.data(), bzone.size()));
  RC(upload(h, &m.zones, zones.data(), zones.size()));
  RC(upload(h, &m.ell_off, h->ell_off.data(), h->ell_off.size()));
  RC(upload(h, &m.ell_nb, ell_nb.data(), ell_nb.size()));
  RC(upload(h, &m.ell_lower, ell_lower.data(), ell_lower.size()));
  RC(upload(h, &m.color, color.data(), color.size()));
  m.ncolors = ncolors;
  launch_face_geo(m, (double*)m.fa_u, (double*)m.fa_s, h->stream);
  CKL();
  // device state
  State& st = h->st;
  memset(&st, 0, sizeof(st));
  RC(dmalloc(h, &st.q, 5 * (size_t)N));
  RC(dmalloc(h, &st.prim, 8 * (size_t)N));
  RC(dmalloc(h, &st.bfa, 8 * (size_t)nfa_b));
  RC(dmalloc(h, &st.mul_fa, (size_t)nfa));
  RC(dmalloc(h, &st.lam_fa, (size_t)nfa));
  RC(dmalloc(h, &st.gu, 9 * (size_t)N));
  int separate = h->p.viscous && h->p.second_order && !h->p.visc_limiter && h->p.limiter && bs == 5;
  if (separate) RC(dmalloc(h, &st.guv, 9 * (size_t)N));
  else st.guv = st.gu;
  RC(dmalloc(h, &st.grho, 3 * (size_t)N));
  RC(dmalloc(h, &st.gp, 3 * (size_t)N));
  RC(dmalloc(h, &st.gh, 3 * (size_t)N));
  RC(dmalloc(h, &st.local_dt, (size_t)N));
  RC(dmalloc(h, &st.rhs, bs * (size_t)N));
  st.shock_flag = nullptr;
  if (q->flux == JG_FLUX_AUSMDV && q->shock_fix != JG_SHOCK_FIX_NONE)
    RC(dmalloc(h, &st.shock_flag, (size_t)N));
  st.jst = nullptr;
  st.jst_bcv = nullptr;
  if (q->flux == JG_FLUX_JST) {
    // calcJSTCoeff_Const (JoeWithModels.cpp:13380-13395): BoundaryCV marks the first cell of every
    // internal face (the reference's rule, kept as it changes the dissipation)
    RC(dmalloc(h, &st.jst, 8 * (size_t)N));
    std::vector<unsigned char> bcv((size_t)N, 0);
    for (int f = nfa_b; f < nfa; f++) bcv[mesh->cvofa[2 * f]] = 1;
    RC(upload(h, &st.jst_bcv, bcv.data(), bcv.size()));
  }
  RC(dmalloc(h, &st.b, bs * (size_t)N));
  RC(dmalloc_bytes(h, &st.D, bs * bs * (size_t)N * h->eltsz));
  RC(dmalloc_bytes(h, &st.Dinv, bs * bs * (size_t)N * h->eltsz));
  RC(dmalloc_bytes(h, &st.O, h->ell_elems * h->eltsz));
  RC(dmalloc_bytes(h, &st.x0, bs * (size_t)N * h->eltsz));
  RC(dmalloc_bytes(h, &st.x1, bs * (size_t)N * h->eltsz));
  RC(dmalloc(h, &st.dq, bs * (size_t)N));
  st.bs = bs;
  st.jac_lag = bs == 5 ? std::max(q->jac_lag, 1) : 1;
  st.D0 = nullptr;
  st.jac_next = nullptr;
  // per-block partials: k_flux2 writes 5 per 16-cell block, k_dt 1 per 256-cell block
  RC(dmalloc(h, &st.blk, 5 * (size_t)grid_for(N, 16) + 5 * (size_t)grid_for(N, 256) + 16));
  RC(dmalloc(h, &st.ctrl, 16));
  RC(dmalloc(h, &st.err, 4));
  h->hist_cap = 64;
  st.hist_cap = h->hist_cap;
  if (h->case_off.empty()) {
    h->case_off = {0, N};
    h->case_nfa_b_off = {0, nfa_b};
  }
  h->ncases = (int)h->case_off.size() - 1;
  RC(dmalloc(h, &st.resid, bs * (size_t)h->hist_cap * h->ncases));
  {
    const int* d = nullptr;
    RC(upload(h, &d, h->case_off.data(), h->case_off.size()));
    h->d_case_off = (int*)d;
    std::vector<int> case_of(N);
    for (int k = 0; k < h->ncases; k++)
      for (int c = h->case_off[k]; c < h->case_off[k + 1]; c++) case_of[c] = k;
    RC(upload(h, &h->m.case_of, case_of.data(), case_of.size()));
    RC(dmalloc(h, &st.case_err, (size_t)h->ncases));
    std::vector<int> rblk_off(h->ncases + 1, 0), rblk_case;
    for (int k = 0; k < h->ncases; k++) {
      int nb = (h->case_off[k + 1] - h->case_off[k] + RCHUNK - 1) / RCHUNK;
      rblk_off[k + 1] = rblk_off[k] + nb;
      rblk_case.insert(rblk_case.end(), nb, k);
    }
    h->nrblk = rblk_off[h->ncases];
    RC(upload(h, &d, rblk_off.data(), rblk_off.size()));
    h->d_rblk_off = (int*)d;
    RC(upload(h, &d, rblk_case.data(), rblk_case.size()));
    h->d_rblk_case = (int*)d;
    RC(dmalloc(h, &st.rpart, bs * (size_t)h->nrblk));
    if (st.jac_lag > 1) {
      // the kept face part of the diagonal blocks and each case's next refresh step (0: the next step)
      RC(dmalloc_bytes(h, &st.D0, bs * bs * (size_t)N * h->eltsz));
      RC(dmalloc(h, &st.jac_next, (size_t)h->ncases));
    }
    std::vector<uint8_t> on(h->ncases, 1);
    const uint8_t* da = nullptr;
    RC(upload(h, &da, on.data(), on.size()));
    st.case_active = (uint8_t*)da;
  }
  if (bs > 5) {
    // model arrays, the WALL faces in zone order and the wall distance (initialHookScalarRansTurbModel)
    Turb& t = h->turb;
    t.model = q->turb_model;
    t.ns = q->nscal;
    const size_t ns = t.ns;
    RC(dmalloc(h, &t.phi, ns * N));
    RC(dmalloc(h, &t.phi_bfa, ns * nfa_b));
    RC(dmalloc(h, &t.grad_phi, 3 * ns * N));
    RC(dmalloc(h, &t.diff, ns * nfa));
    RC(dmalloc(h, &t.wd, (size_t)N));
    RC(dmalloc(h, &t.strMag, (size_t)N));
    RC(dmalloc(h, &t.vortMag, (size_t)N));
    if (t.model == JG_TURB_SST) {
      RC(dmalloc(h, &t.diverg, (size_t)N));
      RC(dmalloc(h, &t.crossDiff, (size_t)N));
      RC(dmalloc(h, &t.F1, (size_t)N));
      RC(dmalloc(h, &t.F2, (size_t)N));
      st.kine = t.phi;  // scalar 0: the pressure recovery subtracts rho k
    }
    RC(dmalloc(h, &st.mut_fa, (size_t)nfa));
    // WALL faces zone by zone in the caller's face order (the nearest-face search keeps the first of equals)
    std::vector<int> wall;
    for (int z = 0; z < mesh->nzones; z++)
      if (mesh->zones[z].kind == JG_BC_WALL) {
        size_t w0 = wall.size();
        for (int f = mesh->zones[z].ifa_f; f <= mesh->zones[z].ifa_l; f++) wall.push_back(f);
        if (!h->rn.face_old.empty())
          std::sort(wall.begin() + w0, wall.end(),
                    [&](int a, int b) { return h->rn.face_old[a] < h->rn.face_old[b]; });
      }
    // the cases of a batch are concatenated zone by zone: the WALL faces of case k are one segment
    std::vector<int> woff(h->ncases + 1, 0);
    for (int k = 0, w = 0; k < h->ncases; k++) {
      while (w < (int)wall.size() && wall[w] < h->case_nfa_b_off[k + 1]) w++;
      woff[k + 1] = w;
      if (woff[k + 1] == woff[k])
        return set_err(JG_ERR_ARG, "case %d: a turbulence model needs a WALL zone (wall distance)", k);
    }
    const int* dw = nullptr;
    RC(upload(h, &dw, wall.data(), wall.size()));
    t.wall_f = dw;
    t.nwall = (int)wall.size();
    for (int k = 0; k < h->ncases; k++)
      launch_wall_distance(h->m, t, h->case_off[k], h->case_off[k + 1], woff[k], woff[k + 1], h->stream);
    CKL();
  }
  if (q->lin_solver == JG_LS_BCGSTAB_LINELET || q->lin_solver == JG_LS_LINE) {
    std::vector<int> off, cv;
    multi_cell_lines(mesh, h->rn.face_old, off, cv, q->lin_solver == JG_LS_LINE);
    Lines& L = h->lines;
    L.nlines = (int)off.size() - 1;
    const size_t nc = std::max<size_t>(cv.size(), 1);
    RC(upload(h, &L.off, off.data(), off.size()));
    RC(upload(h, &L.cv, cv.data(), nc));
    {
      // the ELL row of each coupling along the lines, so that the factorisations read the blocks
      // directly instead of searching the rows
      std::vector<int> jlo(nc, -1), jup(nc, -1);
      auto ell_row = [&](int row, int nbc) {
        int found = -1, cnt = 0;
        for (int j = 0; j < ncols[row]; j++)
          if (h->col_nb[h->cell_cols[row] + j] == nbc) {
            if (!cnt) found = j;
            cnt++;
          }
        return cnt == 0 ? -1 : cnt > 1 ? -2 : h->ell_off[row / SLICE] + found;
      };
      for (int l = 0; l < L.nlines; l++)
        for (int k = off[l] + 1; k < off[l + 1]; k++) {
          jlo[k] = ell_row(cv[k], cv[k - 1]);
          jup[k] = ell_row(cv[k - 1], cv[k]);
        }
      RC(upload(h, &L.jlo, jlo.data(), nc));
      RC(upload(h, &L.jup, jup.data(), nc));
    }
    if (q->lin_solver == JG_LS_BCGSTAB_LINELET) {
      RC(dmalloc(h, &L.inv, 25 * nc));
      RC(dmalloc(h, &L.low, 25 * nc));
      RC(dmalloc(h, &L.up, 25 * nc));
      RC(dmalloc(h, &L.v, 5 * nc));
    } else {
      // the line cells and, per ELL entry, whether it couples a cell to its predecessor or successor on its line
      std::vector<uint8_t> on_line(N, 0), inl((size_t)rows * SLICE, 0);
      std::vector<int> prev(N, -1), next(N, -1);
      for (int l = 0; l < L.nlines; l++)
        for (int k = off[l]; k < off[l + 1]; k++) {
          on_line[cv[k]] = 1;
          if (k > off[l]) prev[cv[k]] = cv[k - 1];
          if (k + 1 < off[l + 1]) next[cv[k]] = cv[k + 1];
        }
      for (int c = 0; c < N; c++) {
        if (!on_line[c]) continue;
        const int sl = c / SLICE, lane = c % SLICE;
        for (int j = 0; j < ncols[c]; j++) {
          const size_t e = (size_t)(h->ell_off[sl] + j) * SLICE + lane;
          if (ell_nb[e] == prev[c] || ell_nb[e] == next[c]) inl[e] = 1;
        }
      }
      RC(upload(h, &L.on_line, on_line.data(), on_line.size()));
      RC(upload(h, &L.ell_inline, inl.data(), inl.size()));
      RC(dmalloc_bytes(h, &L.binv, (size_t)bs * bs * nc * h->eltsz));
      RC(dmalloc_bytes(h, &L.blow, (size_t)bs * bs * nc * h->eltsz));
      RC(dmalloc_bytes(h, &L.bup, (size_t)bs * bs * nc * h->eltsz));
      RC(dmalloc_bytes(h, &L.bv, (size_t)bs * nc * h->eltsz));
    }
  }
  double ctrl0[16] = {0};
  ctrl0[0] = q->cfl;
  CK(cudaMemcpyAsync(st.ctrl, ctrl0, sizeof(ctrl0), cudaMemcpyHostToDevice, h->stream));
  if (!h->async_alloc) CK(cudaStreamSynchronize(h->stream));
  return JG_OK;
}

// build() on the caller's mesh, or on its renumbered copy (with the device copy of the cell order)
static int build_case(jg_case* h, const jg_mesh* mesh, const jg_params* params) {
  if (params->renumber == JG_RENUMBER_NONE) return build(h, mesh, params);
  MeshOwned mo;
  RC(renumber_mesh(*mesh, params->renumber, mo, h->rn));
  RC(build(h, &mo.m, params));
  const int* d = nullptr;
  RC(upload(h, &d, h->rn.cell_old.data(), h->rn.cell_old.size()));
  h->d_cell_old = (int*)d;
  CK(cudaStreamSynchronize(h->stream));  // the renumbered host arrays go out of scope
  return JG_OK;
}

int jg_create(const jg_mesh* mesh, const jg_params* params, jg_case_t** out) {
  if (!mesh || !out) return set_err(JG_ERR_ARG, "null argument");
  *out = nullptr;
  RC(check_params(params));
  if (mesh->ncv <= 0 || mesh->nfa < mesh->nfa_b || mesh->nfa_b < 0 || mesh->nbocv_s < mesh->ncv)
    return set_err(JG_ERR_ARG, "inconsistent mesh sizes");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(JG_ERR_NODEVICE, "no CUDA device");
  jg_case* h = new jg_case();
  int rc = build_case(h, mesh, params);
  if (rc != JG_OK) {
    std::string keep = g_err;
    jg_destroy(h);
    g_err = keep;
    return rc;
  }
  *out = h;
  return JG_OK;
}

// Device bytes a handle made by jg_create holds once its state is set: the
// allocations of build() plus the state staging buffer, each rounded like
// dmalloc_bytes rounds it.  CUDA-graph and event storage is not included.
static size_t footprint(const jg_mesh* mesh, const jg_params* q, const std::vector<int>& face_old) {
  const size_t N = mesh->ncv, nfa = mesh->nfa, nfa_b = mesh->nfa_b, nbs = mesh->nbocv_s;
  const size_t e = q->precision == JG_PREC_MIXED ? 4 : 8;
  const size_t bs = q->turb_model == JG_TURB_NONE ? 5 : 5 + q->nscal, b2 = bs * bs;
  const int* fi = mesh->faocv_i;
  const int* fv = mesh->faocv_v;
  size_t nbslot = 0, rows = 0;
  const size_t nslices = (N + SLICE - 1) / SLICE;
  for (size_t sl = 0; sl < nslices; sl++) {
    size_t w = 0;
    for (size_t c = sl * SLICE; c < std::min(N, (sl + 1) * SLICE); c++) {
      size_t nc = 0;
      for (int k = fi[c]; k < fi[c + 1]; k++) (fv[k] < (int)nfa_b) ? nbslot++ : nc++;
      w = std::max(w, nc);
    }
    rows += w;
  }
  const size_t d = 8, i = 4;
  const size_t nz = std::max(1, mesh->nzones);
  const size_t a[] = {
      // mesh
      3 * N * d, N * d, 3 * nfa * d, 3 * nfa * d, 2 * nfa * i, 4 * nfa * d, std::max<size_t>(4 * (nfa - nfa_b), 1) * d,
      (N + 1) * i, (size_t)fi[N] * sizeof(Slot),
      (N + 1) * i, nbs * i, 3 * nbs * d, (N + 1) * i, std::max<size_t>(nbslot, 1) * i, 3 * nfa_b * d,
      nfa_b * i, nz * sizeof(DevZone), (nslices + 1) * i, rows * SLICE * i, rows * SLICE, N,
      // state
      5 * N * d, 8 * N * d, 8 * nfa_b * d, nfa * d, nfa * d, 9 * N * d,
      (q->mu_ref > 0.0 && q->second_order && !q->visc_limiter && q->limiter && bs == 5) ? 9 * N * d : 0,
      3 * N * d, 3 * N * d, 3 * N * d, N * d, bs * N * d, bs * N * d,
      b2 * N * e, b2 * N * e, rows * b2 * SLICE * e, bs * N * e, bs * N * e, bs * N * d,
      (5 * (size_t)grid_for((int)N, 16) + 5 * (size_t)grid_for((int)N, 256) + 16) * d, 16 * d, 4 * i,
      bs * 64 * d, 2 * i, N * i, 1 * i, 1,
      2 * i, ((N + RCHUNK - 1) / RCHUNK) * i, bs * ((N + RCHUNK - 1) / RCHUNK) * d,
      // state staging (jg_set_state / jg_get_state)
      5 * N * d};
  size_t b = 0;
  for (size_t x : a)
    if (x) b += alloc_round(x);
  {
    // the per-colour slice lists
    std::vector<uint8_t> color;
    std::vector<int> cslices, coff;
    if (color_cells(mesh, color, cslices, coff) <= MAX_COLOR_LISTS)
      b += alloc_round(std::max<size_t>(cslices.size(), 1) * i);
  }
  // AUSMDV shock flags; JST coefficients and BoundaryCV
  if (q->flux == JG_FLUX_AUSMDV && q->shock_fix != JG_SHOCK_FIX_NONE) b += alloc_round(N);
  if (q->flux == JG_FLUX_JST) b += alloc_round(8 * N * d) + alloc_round(N);
  // lagged Jacobian: the kept diagonal face part and the refresh step of the case
  if (bs == 5 && q->jac_lag > 1) b += alloc_round(b2 * N * e) + alloc_round(sizeof(long long));
  if (bs > 5) {
    // model arrays: phi, phi_bfa, grad_phi, diff (per scalar), wall distance, strain, vorticity
    // (+ divergence, cross-diffusion, F1, F2 for SST), mut_fa, the wall faces
    const size_t ns = bs - 5;
    size_t nwall = 0;
    for (int z = 0; z < mesh->nzones; z++)
      if (mesh->zones[z].kind == JG_BC_WALL) nwall += mesh->zones[z].ifa_l - mesh->zones[z].ifa_f + 1;
    const size_t t[] = {ns * N * d, ns * nfa_b * d, 3 * ns * N * d, ns * nfa * d, N * d, N * d, N * d,
                        nfa * d, nwall * i};
    for (size_t x : t) b += alloc_round(x);
    if (q->turb_model == JG_TURB_SST) b += 4 * alloc_round(N * d);
  }
  if (q->lin_solver == JG_LS_BCGSTAB_LINELET || q->lin_solver == JG_LS_LINE) {
    std::vector<int> off, cv;
    multi_cell_lines(mesh, face_old, off, cv, q->lin_solver == JG_LS_LINE);
    const size_t nc = std::max<size_t>(cv.size(), 1);
    b += alloc_round(off.size() * i) + 3 * alloc_round(nc * i);
    if (q->lin_solver == JG_LS_BCGSTAB_LINELET)
      b += 3 * alloc_round(25 * nc * d) + alloc_round(5 * nc * d);
    else
      b += alloc_round(N) + alloc_round(rows * SLICE) + 3 * alloc_round(b2 * nc * e) + alloc_round(bs * nc * e);
  }
  return b;
}

extern "C" int jg_case_footprint(const jg_mesh* mesh, const jg_params* params, double* bytes) {
  if (!mesh || !params || !bytes) return set_err(JG_ERR_ARG, "null argument");
  RC(check_params(params));
  if (mesh->ncv <= 0 || mesh->nfa < mesh->nfa_b || mesh->nfa_b < 0 || mesh->nbocv_s < mesh->ncv)
    return set_err(JG_ERR_ARG, "inconsistent mesh sizes");
  if (params->renumber != JG_RENUMBER_NONE) {
    // the sliced-ELL padding follows the renumbered order; plus the device copy of the cell order
    MeshOwned mo;
    Renumbering rn;
    RC(renumber_mesh(*mesh, params->renumber, mo, rn));
    *bytes = (double)(footprint(&mo.m, params, rn.face_old) + alloc_round((size_t)mesh->ncv * sizeof(int)));
    return JG_OK;
  }
  *bytes = (double)footprint(mesh, params, {});
  return JG_OK;
}

extern "C" int jg_case_device_bytes(jg_case_t* h, double* bytes) {
  if (!h || !bytes) return set_err(JG_ERR_ARG, "null argument");
  *bytes = (double)h->bytes;
  return JG_OK;
}

static int prime(jg_case* h);

// ---------------------------------------------------------------------------
// batches: many independent cases concatenated into one block-diagonal system
// ---------------------------------------------------------------------------
// Boundary faces of every case first (case by case), then the internal faces
// (case by case); cells case by case.  Per case, the relative order of cells,
// faces and CSR entries is the case's own, so every per-cell computation sees
// exactly what it sees when the case runs alone.
static int concat_meshes(int ncases, const jg_mesh* ms, MeshOwned& o, std::vector<int>& case_off,
                         std::vector<int>& bfa_off) {
  long N = 0, NF = 0, NB = 0, NBS = 0, NZ = 0;
  for (int k = 0; k < ncases; k++) {
    const jg_mesh& m = ms[k];
    if (m.ncv <= 0 || m.nfa < m.nfa_b || m.nfa_b < 0 || m.nbocv_s < m.ncv)
      return set_err(JG_ERR_ARG, "case %d: inconsistent mesh sizes", k);
    N += m.ncv; NF += m.nfa; NB += m.nfa_b; NBS += m.nbocv_s; NZ += m.nzones;
  }
  if (N > 2000000000L || NF > 2000000000L || NBS > 2000000000L) return set_err(JG_ERR_ARG, "batch too large");
  case_off.assign(ncases + 1, 0);
  bfa_off.assign(ncases + 1, 0);
  for (int k = 0; k < ncases; k++) {
    case_off[k + 1] = case_off[k] + ms[k].ncv;
    bfa_off[k + 1] = bfa_off[k] + ms[k].nfa_b;
  }
  std::vector<long> int_off(ncases + 1, 0);
  for (int k = 0; k < ncases; k++) int_off[k + 1] = int_off[k] + (ms[k].nfa - ms[k].nfa_b);
  o.cvofa.assign(2 * NF, -1);
  o.x_fa.assign(3 * NF, 0.0);
  o.fa_normal.assign(3 * NF, 0.0);
  o.blsq.assign(3 * NB, 0.0);
  o.faocv_i.assign(N + 1, 0);
  o.nbocv_i.assign(N + 1, 0);
  o.faocv_v.clear();
  o.nbocv_v.clear();
  o.x_cv.clear(); o.vol.clear(); o.lsq.clear(); o.zones.clear();
  for (int k = 0; k < ncases; k++) {
    const jg_mesh& m = ms[k];
    const int co = case_off[k];
    auto gf = [&](int f) -> long { return f < m.nfa_b ? bfa_off[k] + f : NB + int_off[k] + (f - m.nfa_b); };
    for (int f = 0; f < m.nfa; f++) {
      long g = gf(f);
      o.cvofa[2 * g] = m.cvofa[2 * f] + co;
      o.cvofa[2 * g + 1] = m.cvofa[2 * f + 1] >= 0 ? m.cvofa[2 * f + 1] + co : -1;
      for (int i = 0; i < 3; i++) {
        o.x_fa[3 * g + i] = m.x_fa[3 * f + i];
        o.fa_normal[3 * g + i] = m.fa_normal[3 * f + i];
      }
    }
    for (int f = 0; f < m.nfa_b; f++)
      for (int i = 0; i < 3; i++) o.blsq[3 * (bfa_off[k] + f) + i] = m.boundary_fa_lsg_coeff[3 * f + i];
    for (int c = 0; c < m.ncv; c++) {
      for (int q = m.faocv_i[c]; q < m.faocv_i[c + 1]; q++) o.faocv_v.push_back((int)gf(m.faocv_v[q]));
      o.faocv_i[co + c + 1] = (int)o.faocv_v.size();
      for (int q = m.nbocv_i[c]; q < m.nbocv_i[c + 1]; q++) {
        o.nbocv_v.push_back(m.nbocv_v[q] + co);
        for (int i = 0; i < 3; i++) o.lsq.push_back(m.nbocv_lsg_coeff[3 * q + i]);
      }
      o.nbocv_i[co + c + 1] = (int)o.nbocv_v.size();
      for (int i = 0; i < 3; i++) o.x_cv.push_back(m.x_cv[3 * c + i]);
      o.vol.push_back(m.cv_volume[c]);
    }
    for (int z = 0; z < m.nzones; z++) {
      jg_zone zz = m.zones[z];
      zz.ifa_f += bfa_off[k];
      zz.ifa_l += bfa_off[k];
      o.zones.push_back(zz);
    }
  }
  jg_mesh& m = o.m;
  m.ncv = (int)N; m.nfa = (int)NF; m.nfa_b = (int)NB; m.nbocv_s = (int)NBS; m.nzones = (int)o.zones.size();
  m.cvofa = o.cvofa.data(); m.faocv_i = o.faocv_i.data(); m.faocv_v = o.faocv_v.data();
  m.nbocv_i = o.nbocv_i.data(); m.nbocv_v = o.nbocv_v.data();
  m.x_cv = o.x_cv.data(); m.x_fa = o.x_fa.data(); m.fa_normal = o.fa_normal.data(); m.cv_volume = o.vol.data();
  m.nbocv_lsg_coeff = o.lsq.data(); m.boundary_fa_lsg_coeff = o.blsq.data(); m.zones = o.zones.data();
  return JG_OK;
}

int jg_batch_create(int ncases, const jg_mesh* meshes, const jg_params* params, jg_case_t** out) {
  if (ncases <= 0 || !meshes || !out) return set_err(JG_ERR_ARG, "bad argument");
  *out = nullptr;
  RC(check_params(params));
  if (params->lin_solver == JG_LS_BCGSTAB || params->lin_solver == JG_LS_BCGSTAB_LINELET)
    return set_err(JG_ERR_ARG, "a batch relaxes with JACOBI, SGS or LUSGS (BiCGSTAB's dot products would couple the cases)");
  if (params->time_step_mode == JG_TS_CFL_MIN)
    return set_err(JG_ERR_ARG, "CFL_MIN would couple the cases of a batch");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(JG_ERR_NODEVICE, "no CUDA device");
  MeshOwned cat;
  jg_case* h = new jg_case();
  int rc = JG_OK;
  if (params->renumber != JG_RENUMBER_NONE) {
    // each case renumbered on its own (cells never leave their case), then concatenated; the
    // case-local cell order of every case is kept for the per-case state and scalar calls
    std::vector<MeshOwned> mo(ncases);
    std::vector<jg_mesh> rm(ncases);
    std::vector<std::vector<int>> fold(ncases);
    for (int k = 0; k < ncases && rc == JG_OK; k++) {
      Renumbering r;
      rc = renumber_mesh(meshes[k], params->renumber, mo[k], r);
      if (rc == JG_OK) {
        mo[k].bind();
        rm[k] = mo[k].m;
        h->case_cell_old.insert(h->case_cell_old.end(), r.cell_old.begin(), r.cell_old.end());
        fold[k].swap(r.face_old);
      }
    }
    if (rc == JG_OK) rc = concat_meshes(ncases, rm.data(), cat, h->case_off, h->case_nfa_b_off);
    if (rc == JG_OK) {
      // each concatenated face's id in the concatenation of the caller's meshes, so that the WALL
      // faces are taken in each case's own face order (the order in which lines grow and wall
      // distances break ties, as the case alone takes them)
      const int NB = h->case_nfa_b_off[ncases];
      std::vector<int> int_off(ncases + 1, 0);
      for (int k = 0; k < ncases; k++) int_off[k + 1] = int_off[k] + (meshes[k].nfa - meshes[k].nfa_b);
      h->rn.face_old.assign((size_t)cat.m.nfa, 0);
      for (int k = 0; k < ncases; k++) {
        const int nb = meshes[k].nfa_b;
        auto gf = [&](int f) { return f < nb ? h->case_nfa_b_off[k] + f : NB + int_off[k] + (f - nb); };
        for (int f = 0; f < meshes[k].nfa; f++) h->rn.face_old[gf(f)] = gf(fold[k][f]);
      }
    }
    if (rc == JG_OK) rc = build(h, &cat.m, params);
    if (rc == JG_OK) {
      const int* d = nullptr;
      rc = upload(h, &d, h->case_cell_old.data(), h->case_cell_old.size());
      h->d_case_cell_old = (int*)d;
    }
    if (rc == JG_OK && cudaStreamSynchronize(h->stream) != cudaSuccess) rc = set_err(JG_ERR_CUDA, "batch upload");
  } else {
    rc = concat_meshes(ncases, meshes, cat, h->case_off, h->case_nfa_b_off);
    if (rc == JG_OK) rc = build(h, &cat.m, params);
  }
  if (rc != JG_OK) {
    std::string keep = g_err;
    jg_destroy(h);
    g_err = keep;
    return rc;
  }
  *out = h;
  return JG_OK;
}

int jg_batch_info(jg_case_t* h, int* ncases, int* cell_offsets) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  if (ncases) *ncases = h->ncases;
  if (cell_offsets)
    for (int k = 0; k <= h->ncases; k++) cell_offsets[k] = h->case_off[k];
  return JG_OK;
}

int jg_batch_set_state(jg_case_t* h, int k, const double* rho, const double* rhou, const double* rhoE) {
  if (!h || !rho || !rhou || !rhoE || k < 0 || k >= h->ncases) return set_err(JG_ERR_ARG, "bad argument");
  const size_t N = h->ncv, n = h->case_off[k + 1] - h->case_off[k], c0 = h->case_off[k];
  if (!h->d_io) RC(dmalloc(h, &h->d_io, 5 * N));
  CK(cudaMemcpyAsync(h->d_io, rho, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_io + n, rhou, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_io + 4 * n, rhoE, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_pack_state((int)n, h->d_io, h->st.q + 5 * c0, h->d_case_cell_old ? h->d_case_cell_old + c0 : nullptr,
                    h->stream);
  CK(cudaMemsetAsync(h->st.prim + 8 * c0, 0, 8 * n * sizeof(double), h->stream));
  CKL();
  // the state/BC preamble runs at the next operator call, once every case has its state
  h->primed = 0;
  return JG_OK;
}

int jg_batch_get_state(jg_case_t* h, int k, double* rho, double* rhou, double* rhoE) {
  if (!h || k < 0 || k >= h->ncases) return set_err(JG_ERR_ARG, "bad argument");
  const size_t N = h->ncv, n = h->case_off[k + 1] - h->case_off[k], c0 = h->case_off[k];
  if (!h->d_io) RC(dmalloc(h, &h->d_io, 5 * N));
  launch_unpack_state((int)n, h->st.q + 5 * c0, h->d_io, h->d_case_cell_old ? h->d_case_cell_old + c0 : nullptr,
                      h->stream);
  CKL();
  if (rho) CK(cudaMemcpyAsync(rho, h->d_io, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (rhou) CK(cudaMemcpyAsync(rhou, h->d_io + n, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (rhoE) CK(cudaMemcpyAsync(rhoE, h->d_io + 4 * n, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return JG_OK;
}

int jg_batch_set_scalars(jg_case_t* h, int k, const double* phi) {
  if (!h || !phi || k < 0 || k >= h->ncases) return set_err(JG_ERR_ARG, "bad argument");
  if (h->bs == 5) return set_err(JG_ERR_ARG, "the batch transports no scalar");
  const size_t N = h->ncv, ns = h->turb.ns, n = h->case_off[k + 1] - h->case_off[k], c0 = h->case_off[k];
  std::vector<double> cm(ns * n);  // [n][ns] -> [ns][n], in the batch's cell order
  const int* perm = h->case_cell_old.empty() ? nullptr : h->case_cell_old.data() + c0;
  for (size_t c = 0; c < n; c++)
    for (size_t q = 0; q < ns; q++) cm[q * n + c] = phi[ns * (perm ? (size_t)perm[c] : c) + q];
  for (size_t q = 0; q < ns; q++)
    CK(cudaMemcpyAsync(h->turb.phi + q * N + c0, cm.data() + q * n, n * sizeof(double), cudaMemcpyHostToDevice,
                       h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->primed = 0;
  return JG_OK;
}

int jg_batch_get_scalars(jg_case_t* h, int k, double* phi) {
  if (!h || !phi || k < 0 || k >= h->ncases) return set_err(JG_ERR_ARG, "bad argument");
  if (h->bs == 5) return set_err(JG_ERR_ARG, "the batch transports no scalar");
  const size_t N = h->ncv, ns = h->turb.ns, n = h->case_off[k + 1] - h->case_off[k], c0 = h->case_off[k];
  std::vector<double> cm(ns * n);
  for (size_t q = 0; q < ns; q++)
    CK(cudaMemcpyAsync(cm.data() + q * n, h->turb.phi + q * N + c0, n * sizeof(double), cudaMemcpyDeviceToHost,
                       h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const int* perm = h->case_cell_old.empty() ? nullptr : h->case_cell_old.data() + c0;
  for (size_t c = 0; c < n; c++)
    for (size_t q = 0; q < ns; q++) phi[ns * (perm ? (size_t)perm[c] : c) + q] = cm[q * n + c];
  return JG_OK;
}

int jg_get_stream(jg_case_t* h, void** stream) {
  if (!h || !stream) return set_err(JG_ERR_ARG, "null argument");
  *stream = (void*)h->stream;
  return JG_OK;
}

// The handle's error flags.  Per-case state errors count for a single case,
// and for every case of a batch with all_cases (the preamble: a bad input
// state); during batch steps they stay per case (jg_batch_status).
// the handle's pinned staging area, at least `bytes` long (grown on demand; every call that
// copies into it synchronises before it returns, so no copy into an old area is in flight)
static int pinned(jg_case* h, size_t bytes, void** out) {
  if (bytes > h->hpin_bytes) {
    if (h->hpin) CK(cudaFreeHost(h->hpin));
    h->hpin = nullptr;
    h->hpin_bytes = 0;
    const size_t b = std::max<size_t>(bytes, 4096);
    CK(cudaHostAlloc(&h->hpin, b, cudaHostAllocDefault));
    h->hpin_bytes = b;
  }
  *out = h->hpin;
  return JG_OK;
}

// Reads (and clears) the error flags; with nres > 0 also copies nres doubles from the device
// array dres to res_out, in the same synchronisation (the copy is made whatever the flags say).
static int check_err_flags(jg_case* h, bool all_cases = false, const double* dres = nullptr, size_t nres = 0,
                           double* res_out = nullptr) {
  const int nc = (h->ncases == 1 || all_cases) ? h->ncases : 0;
  const size_t off = (sizeof(int) * (1 + (size_t)nc) + 15) & ~(size_t)15;
  void* hp = nullptr;
  RC(pinned(h, off + nres * sizeof(double), &hp));
  int* hi = (int*)hp;
  double* hr = (double*)((char*)hp + off);
  CK(cudaMemcpyAsync(hi, h->st.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if (nc) CK(cudaMemcpyAsync(hi + 1, h->st.case_err, nc * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  if (nres) CK(cudaMemcpyAsync(hr, dres, nres * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (nres) memcpy(res_out, hr, nres * sizeof(double));
  int e = hi[0], ec = 0;
  for (int k = 0; k < nc; k++) ec |= hi[1 + k];
  if (ec) {
    CK(cudaMemsetAsync(h->st.case_err, 0, nc * sizeof(int), h->stream));
    e |= ec;
  }
  if (e) {
    CK(cudaMemsetAsync(h->st.err, 0, sizeof(int), h->stream));
    if (e & 2) return set_err(JG_ERR_ARG, "unrecognised boundary condition");
    return set_err(JG_ERR_STATE, "non-physical state (flags %d): negative density/pressure or NaN residual", e);
  }
  return JG_OK;
}

// calcStateVariables + calcMaterialProperties + setBC (+ mut = 0), the
// runBackwardEuler preamble (JoeWithModels.cpp:942-957)
static int prime_enqueue(jg_case* h) {
  // a new state: every case forms its Jacobian blocks at its next step
  if (h->st.jac_next) CK(cudaMemsetAsync(h->st.jac_next, 0, sizeof(long long) * h->ncases, h->stream));
  launch_state(h->m, h->p, h->st, h->stream);
  if (h->bs > 5) {
    launch_face_props(h->m, h->p, h->st, h->stream);
    launch_bc(h->m, h->p, h->st, h->stream);
    launch_scalar_bc(h->m, h->p, h->st, h->turb, h->stream);
    launch_turb_props(h->m, h->p, h->st, h->turb, h->stream);
  } else {
    launch_faces_after_update(h->m, h->p, h->st, h->stream);  // setBC and the face properties, one launch
  }
  CKL();
  h->primed = 1;
  return JG_OK;
}
static int prime(jg_case* h) {
  RC(prime_enqueue(h));
  return check_err_flags(h, true);
}

// the caller's state -> the handle (enqueued; pinned host memory makes the copies asynchronous DMA)
static int stage_state_in(jg_case* h, const double* rho, const double* rhou, const double* rhoE) {
  const size_t N = h->ncv;
  if (!h->d_io) RC(dmalloc(h, &h->d_io, 5 * N));
  CK(cudaMemcpyAsync(h->d_io, rho, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_io + N, rhou, 3 * N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_io + 4 * N, rhoE, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_pack_state((int)N, h->d_io, h->st.q, h->d_cell_old, h->stream);
  CK(cudaMemsetAsync(h->st.prim, 0, 8 * N * sizeof(double), h->stream));
  return JG_OK;
}
// the handle's state -> the caller's arrays (enqueued; any pointer may be NULL)
static int stage_state_out(jg_case* h, double* rho, double* rhou, double* rhoE) {
  const size_t N = h->ncv;
  if (!h->d_io) RC(dmalloc(h, &h->d_io, 5 * N));
  launch_unpack_state((int)N, h->st.q, h->d_io, h->d_cell_old, h->stream);
  CKL();
  if (rho) CK(cudaMemcpyAsync(rho, h->d_io, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (rhou) CK(cudaMemcpyAsync(rhou, h->d_io + N, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  if (rhoE) CK(cudaMemcpyAsync(rhoE, h->d_io + 4 * N, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return JG_OK;
}

int jg_set_state(jg_case_t* h, const double* rho, const double* rhou, const double* rhoE) {
  if (!h || !rho || !rhou || !rhoE) return set_err(JG_ERR_ARG, "null argument");
  RC(stage_state_in(h, rho, rhou, rhoE));
  return prime(h);
}

int jg_calc_state(jg_case_t* h) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  return prime(h);
}

int jg_get_state(jg_case_t* h, double* rho, double* rhou, double* rhoE) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  RC(stage_state_out(h, rho, rhou, rhoE));
  CK(cudaStreamSynchronize(h->stream));
  return JG_OK;
}

int jg_get_primitives(jg_case_t* h, double* vel, double* press, double* temp, double* enthalpy, double* sos) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  const int N = h->ncv;
  std::vector<double> pr(8 * (size_t)N);
  CK(cudaMemcpyAsync(pr.data(), h->st.prim, pr.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const std::vector<int>& perm = h->rn.cell_old;
  for (int r = 0; r < N; r++) {
    const int c = perm.empty() ? r : perm[r];
    if (vel)
      for (int i = 0; i < 3; i++) vel[3 * c + i] = pr[8 * r + i];
    if (press) press[c] = pr[8 * r + 3];
    if (temp) temp[c] = pr[8 * r + 4];
    if (enthalpy) enthalpy[c] = pr[8 * r + 5];
    if (sos) sos[c] = pr[8 * r + 6];
  }
  return JG_OK;
}

int jg_get_bfa(jg_case_t* h, double* rho_bfa, double* vel_bfa, double* p_bfa, double* T_bfa, double* h_bfa,
               double* mul_fa, double* lamOcp_fa) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  const int nb = h->nfa_b;
  std::vector<double> b(8 * (size_t)std::max(nb, 1));
  CK(cudaMemcpyAsync(b.data(), h->st.bfa, 8 * (size_t)nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const std::vector<int>& perm = h->rn.face_old;
  for (int r = 0; r < nb; r++) {
    const int f = perm.empty() ? r : perm[r];
    if (rho_bfa) rho_bfa[f] = b[8 * r];
    if (vel_bfa)
      for (int i = 0; i < 3; i++) vel_bfa[3 * f + i] = b[8 * r + 1 + i];
    if (p_bfa) p_bfa[f] = b[8 * r + 4];
    if (T_bfa) T_bfa[f] = b[8 * r + 5];
    if (h_bfa) h_bfa[f] = b[8 * r + 6];
  }
  if (mul_fa) RC(download_rows(h, h->st.mul_fa, mul_fa, perm, h->nfa, 1));
  if (lamOcp_fa) RC(download_rows(h, h->st.lam_fa, lamOcp_fa, perm, h->nfa, 1));
  return JG_OK;
}

int jg_calc_dt(jg_case_t* h, double cfl, double* dt_min, double* local_dt) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  if (!h->primed) RC(prime(h));
  launch_dt(h->m, h->p, h->st, 0, cfl, h->stream);
  CKL();
  double ctrl[3];
  CK(cudaMemcpyAsync(ctrl, h->st.ctrl, sizeof(ctrl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (local_dt) RC(download_rows(h, h->st.local_dt, local_dt, h->rn.cell_old, h->ncv, 1));
  if (dt_min) *dt_min = ctrl[2];
  return JG_OK;
}

// device D/O (sliced ELL) -> reference block CSR A[nbocv_s][5][5]
static int download_csr(jg_case* h, double* A) {
  const int N = h->ncv, bs = h->bs, b2 = bs * bs;
  size_t es = h->eltsz;
  std::vector<char> D(b2 * (size_t)N * es), O(h->ell_elems * es);
  CK(cudaMemcpyAsync(D.data(), h->st.D, D.size(), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(O.data(), h->st.O, O.size(), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  auto get = [&](const std::vector<char>& v, size_t i) -> double {
    return es == 8 ? ((const double*)v.data())[i] : (double)((const float*)v.data())[i];
  };
  memset(A, 0, sizeof(double) * b2 * (size_t)h->nbs);
  const std::vector<int>& so = h->rn.nbs_old;  // the caller's nbocv entry of each internal one
  auto slot = [&](int k) -> size_t { return so.empty() ? (size_t)k : (size_t)so[k]; };
  for (int c = 0; c < N; c++) {
    int kd = h->nbocv_i[c];
    for (int e = 0; e < b2; e++) A[b2 * slot(kd) + e] = get(D, (size_t)e * N + c);
    int s = c / SLICE, lane = c % SLICE;
    for (int j = 0; j < h->cell_cols[c + 1] - h->cell_cols[c]; j++) {
      int nb = h->col_nb[h->cell_cols[c] + j];
      int k = kd + 1;
      while (k < h->nbocv_i[c + 1] && h->nbocv_v[k] != nb) k++;
      if (k >= h->nbocv_i[c + 1]) return set_err(JG_ERR_ARG, "neighbour %d of cell %d missing from nbocv", nb, c);
      for (int e = 0; e < b2; e++)
        A[b2 * slot(k) + e] += get(O, ((size_t)(h->ell_off[s] + j) * b2 + e) * SLICE + lane);
    }
  }
  return JG_OK;
}

// reference block CSR -> device D/O (a pair of cells sharing several faces keeps the block once)
static int upload_csr(jg_case* h, const double* A) {
  const int N = h->ncv;
  size_t es = h->eltsz;
  std::vector<char> D(25 * (size_t)N * es), O(h->ell_elems * es, 0);
  auto put = [&](std::vector<char>& v, size_t i, double x) {
    if (es == 8) ((double*)v.data())[i] = x;
    else ((float*)v.data())[i] = (float)x;
  };
  std::vector<int> used;
  const std::vector<int>& so = h->rn.nbs_old;
  auto slot = [&](int k) -> size_t { return so.empty() ? (size_t)k : (size_t)so[k]; };
  for (int c = 0; c < N; c++) {
    int kd = h->nbocv_i[c];
    for (int e = 0; e < 25; e++) put(D, (size_t)e * N + c, A[25 * slot(kd) + e]);
    int s = c / SLICE, lane = c % SLICE;
    used.clear();
    for (int j = 0; j < h->cell_cols[c + 1] - h->cell_cols[c]; j++) {
      int nb = h->col_nb[h->cell_cols[c] + j];
      if (std::find(used.begin(), used.end(), nb) != used.end()) continue;
      used.push_back(nb);
      int k = kd + 1;
      while (k < h->nbocv_i[c + 1] && h->nbocv_v[k] != nb) k++;
      if (k >= h->nbocv_i[c + 1]) return set_err(JG_ERR_ARG, "neighbour %d of cell %d missing from nbocv", nb, c);
      for (int e = 0; e < 25; e++) put(O, ((size_t)(h->ell_off[s] + j) * 25 + e) * SLICE + lane, A[25 * slot(k) + e]);
    }
  }
  CK(cudaMemcpyAsync(h->st.D, D.data(), D.size(), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->st.O, O.data(), O.size(), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return JG_OK;
}

int jg_calc_rhs(jg_case_t* h, double* rhs_rho, double* rhs_rhou, double* rhs_rhoE, double* A, int flagImplicit) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  if (h->bs != 5) return set_err(JG_ERR_ARG, "a turbulence-model case assembles with jg_calc_rhs_coupled");
  if (!h->primed) RC(prime(h));
  int implicit = flagImplicit && A != nullptr;
  launch_grad(h->m, h->p, h->st, h->stream);
  launch_flux(h->m, h->p, h->st, implicit, 0, h->stream);
  CKL();
  const int N = h->ncv;
  std::vector<double> r(5 * (size_t)N);
  CK(cudaMemcpyAsync(r.data(), h->st.rhs, r.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const std::vector<int>& perm = h->rn.cell_old;
  for (int q = 0; q < N; q++) {
    const int c = perm.empty() ? q : perm[q];
    if (rhs_rho) rhs_rho[c] = r[5 * q];
    if (rhs_rhou)
      for (int i = 0; i < 3; i++) rhs_rhou[3 * c + i] = r[5 * q + 1 + i];
    if (rhs_rhoE) rhs_rhoE[c] = r[5 * q + 4];
  }
  if (implicit) RC(download_csr(h, A));
  return JG_OK;
}

int jg_get_gradients(jg_case_t* h, double* grad_u, double* grad_rho, double* grad_p, double* grad_h) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  const int N = h->ncv;
  // the reference's grad_u after calcRhs: the viscous pass overwrites it (unlimited when VISC_LIMITER=NO)
  const double* gu = h->p.viscous ? h->st.guv : h->st.gu;
  const std::vector<int>& perm = h->rn.cell_old;
  if (grad_u) RC(download_rows(h, gu, grad_u, perm, N, 9));
  if (grad_rho) RC(download_rows(h, h->st.grho, grad_rho, perm, N, 3));
  if (grad_p) RC(download_rows(h, h->st.gp, grad_p, perm, N, 3));
  if (grad_h) RC(download_rows(h, h->st.gh, grad_h, perm, N, 3));
  return JG_OK;
}

// partial-sum buffer of the BiCGSTAB reductions: launch_dot uses <= 1024
// blocks, launch_resmax one per 256 cells; the last 16 entries hold scalars
static size_t red_size(int N) { return (size_t)std::max(1024, grid_for(N, 256)) + 16; }

// BiCGSTAB with the block-diagonal preconditioner, solveCvVectorR5Bcgstab
// (UgpWithCv.cpp:2660-2876); operates on [5][N] vectors, phi in/out in d_tmp.
static int bcgstab(jg_case* h, double* phi, const double* rhs, double zeroAbs, double zeroRel, int maxiter, int* iters,
                   bool lines = false) {
  const int N = h->ncv;
  const long n5 = 5L * N;
  if (!h->d_tmp) {
    RC(dmalloc(h, &h->d_tmp, 8 * (size_t)n5));
    RC(dmalloc(h, &h->d_red, red_size(N)));
  }
  double *res = h->d_tmp, *res0 = res + n5, *p = res0 + n5, *v = p + n5, *t = v + n5, *s = t + n5, *phat = s + n5,
         *shat = phat + n5;
  double* part = h->d_red;
  double* scal = h->d_red + red_size(N) - 16;
  cudaStream_t S = h->stream;
  auto dot = [&](const double* a, const double* b, double& out) -> int {
    launch_dot((int)n5, a, b, part, scal, S);
    CKL();
    CK(cudaMemcpyAsync(&out, scal, sizeof(double), cudaMemcpyDeviceToHost, S));
    CK(cudaStreamSynchronize(S));
    return JG_OK;
  };
  auto resmax = [&](const double* r, double& out) -> int {
    launch_resmax(h->m, h->st, r, part, scal, S);
    CKL();
    CK(cudaMemcpyAsync(&out, scal, sizeof(double), cudaMemcpyDeviceToHost, S));
    CK(cudaStreamSynchronize(S));
    return JG_OK;
  };
  CK(cudaMemsetAsync(p, 0, n5 * sizeof(double), S));
  CK(cudaMemsetAsync(v, 0, n5 * sizeof(double), S));
  // the preconditioner: block diagonal, or line-implicit (the lines' elimination once per solve)
  if (lines) launch_line_factor(h->m, h->st, h->lines, S);
  auto precond = [&](const double* x, double* y) {
    if (lines) launch_line_precond(h->m, h->st, h->lines, x, y, S);
    else launch_precond(h->m, h->st, x, y, S);
  };
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  launch_spmv(h->m, h->st, phi, res, S);
  launch_lin3(n5, res, 1.0, rhs, -1.0, res, 0.0, nullptr, S);
  CK(cudaMemcpyAsync(res0, res, n5 * sizeof(double), cudaMemcpyDeviceToDevice, S));
  double res0_max = 0.0, res_max = 0.0;
  RC(resmax(res, res0_max));
  int iter = 0, done = 0;
  while (!done) {
    iter++;
    double rho_prime = -omega * rho;
    RC(dot(res, res0, rho));
    if (fabs(rho_prime) < 1.0E-20) rho_prime = 1.0E-20;
    double beta = alpha * rho / rho_prime;
    // p = res - beta*(p - omega*v)
    launch_lin3(n5, p, 1.0, res, -beta, p, beta * omega, v, S);
    precond(p, phat);
    launch_spmv(h->m, h->st, phat, v, S);
    double gamma;
    RC(dot(v, res0, gamma));
    if (fabs(gamma) < 1.0E-20) gamma = 1.0E-20;
    alpha = rho / gamma;
    launch_lin3(n5, s, 1.0, res, -alpha, v, 0.0, nullptr, S);
    precond(s, shat);
    launch_spmv(h->m, h->st, shat, t, S);
    double st_, tt_;
    RC(dot(s, t, st_));
    RC(dot(t, t, tt_));
    omega = st_ / (tt_ + 1.0E-20);
    launch_lin3(n5, phi, 1.0, phi, alpha, phat, omega, shat, S);
    launch_spmv(h->m, h->st, phi, res, S);
    launch_lin3(n5, res, 1.0, rhs, -1.0, res, 0.0, nullptr, S);
    RC(resmax(res, res_max));
    if ((res_max <= zeroAbs) || (res_max / (res0_max + 1.0E-12) <= zeroRel)) done = 1;
    else if (iter > maxiter) done = 2;
  }
  if (iters) *iters = iter;
  return JG_OK;
}

// the caller's [N][5] rows -> [5][N] planes in the handle's order
static void to_soa(const double* aos, std::vector<double>& soa, int N, const std::vector<int>& perm) {
  soa.resize(5 * (size_t)N);
  for (int c = 0; c < N; c++) {
    const int o = perm.empty() ? c : perm[c];
    for (int i = 0; i < 5; i++) soa[(size_t)i * N + c] = aos[5 * o + i];
  }
}

int jg_solve_lin_sys(jg_case_t* h, double* dq, const double* A, const double* rhs, double zeroAbs, double zeroRel,
                     int maxIter, int* iters) {
  if (!h || !dq || !A || !rhs) return set_err(JG_ERR_ARG, "null argument");
  if (h->bs != 5) return set_err(JG_ERR_ARG, "jg_solve_lin_sys takes the 5x5 system");
  const int N = h->ncv;
  RC(upload_csr(h, A));
  launch_dinv(h->m, h->p, h->st, h->stream);
  RC(upload_rows(h, h->st.b, rhs, h->rn.cell_old, N, 5));
  CKL();
  int it = 0;
  switch (h->hp.lin_solver) {
    case JG_LS_BCGSTAB:
    case JG_LS_BCGSTAB_LINELET: {
      if (!h->d_tmp) {
        RC(dmalloc(h, &h->d_tmp, 8 * 5 * (size_t)N));
        RC(dmalloc(h, &h->d_red, red_size(N)));
      }
      double* phi = (double*)h->st.x0;
      double* b = (double*)h->st.x1;
      std::vector<double> soa;
      to_soa(dq, soa, N, h->rn.cell_old);
      CK(cudaMemcpyAsync(phi, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
      to_soa(rhs, soa, N, h->rn.cell_old);
      CK(cudaMemcpyAsync(b, soa.data(), soa.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
      RC(bcgstab(h, phi, b, zeroAbs, zeroRel, maxIter, &it, h->hp.lin_solver == JG_LS_BCGSTAB_LINELET));
      launch_dq_from_x(h->m, h->p, h->st, phi, h->stream);
    } break;
    case JG_LS_LUSGS:
      launch_lusgs(h->m, h->p, h->st, h->stream);
      launch_dq_from_x(h->m, h->p, h->st, h->st.x1, h->stream);
      it = 1;
      break;
    case JG_LS_JACOBI: {
      int sweeps = std::max(1, maxIter);
      launch_jacobi(h->m, h->p, h->st, sweeps, h->stream);
      launch_dq_from_x(h->m, h->p, h->st, (sweeps % 2 == 1) ? h->st.x0 : h->st.x1, h->stream);
      it = sweeps;
    } break;
    case JG_LS_SGS: {
      int sweeps = std::max(1, maxIter);
      launch_sgs(h->m, h->p, h->st, sweeps, h->stream);
      launch_dq_from_x(h->m, h->p, h->st, h->st.x0, h->stream);
      it = sweeps;
    } break;
    case JG_LS_LINE: {
      int sweeps = std::max(1, maxIter);
      launch_line_relax(h->m, h->p, h->st, h->lines, 5, sweeps, h->stream);
      launch_dq_from_x(h->m, h->p, h->st, (sweeps % 2 == 1) ? h->st.x0 : h->st.x1, h->stream);
      it = sweeps;
    } break;
  }
  CKL();
  RC(download_rows(h, h->st.dq, dq, h->rn.cell_old, N, 5));
  if (iters) *iters = it;
  return JG_OK;
}

// one backward-Euler iteration on the device (runBackwardEuler loop body)
// one runBackwardEulerCoupled iteration (JoeWithModels.cpp:4416-4529) with the SA model
static int enqueue_step_coupled(jg_case* h) {
  cudaStream_t S = h->stream;
  launch_ctrl_step(h->p, h->st, S);
  launch_dt(h->m, h->p, h->st, 1, 0.0, S);
  if (h->profiling) CK(cudaEventRecordWithFlags(h->ev[0], S, cudaEventRecordExternal));
  launch_flux6(h->m, h->p, h->st, h->turb, 1, 1, S);
  if (h->profiling) CK(cudaEventRecordWithFlags(h->ev[1], S, cudaEventRecordExternal));
  launch_resid_cases(h->st, h->d_case_off, h->d_rblk_off, h->d_rblk_case, h->nrblk, h->ncases, 1, S);
  if (h->profiling) CK(cudaEventRecordWithFlags(h->ev[2], S, cudaEventRecordExternal));
  int sgs = h->hp.lin_solver == JG_LS_SGS;
  int sweeps = std::max(1, h->hp.ls_max_iter);
  if (h->hp.lin_solver == JG_LS_LINE) launch_line_relax(h->m, h->p, h->st, h->lines, h->bs, sweeps, S);
  else launch_relax6(h->m, h->p, h->st, sgs, sweeps, h->bs, S);
  if (h->profiling) CK(cudaEventRecordWithFlags(h->ev[3], S, cudaEventRecordExternal));
  launch_update6(h->m, h->p, h->st, h->turb, (sgs || sweeps % 2 == 1) ? h->st.x0 : h->st.x1, S);
  launch_state(h->m, h->p, h->st, S);
  launch_faces_after_update(h->m, h->p, h->st, S);
  launch_scalar_bc(h->m, h->p, h->st, h->turb, S);
  launch_turb_props(h->m, h->p, h->st, h->turb, S);
  CKL();
  return JG_OK;
}

static int enqueue_step(jg_case* h, int for_graph) {
  if (h->bs > 5) return enqueue_step_coupled(h);
  cudaStream_t S = h->stream;
  // Off the critical path on the second stream: the CFL ramp and calcDt beside the gradients
  // (neither reads what the other writes; the split face loop's Jacobian kernel follows them on
  // that stream and its join brings them back, the fused face loop waits for them here), and the
  // residual norms beside the relaxation (joined before the update).
  const int solver = h->hp.lin_solver;
  const bool aside = h->st.aux && h->st.ev_pre && h->st.ev_dt && h->st.ev_res && h->st.ev_resid;
  const bool resid_aside = aside && solver != JG_LS_BCGSTAB && solver != JG_LS_BCGSTAB_LINELET;
  if (aside) {
    CK(cudaEventRecord(h->st.ev_pre, S));
    CK(cudaStreamWaitEvent(h->st.aux, h->st.ev_pre, 0));
    launch_ctrl_step(h->p, h->st, h->st.aux);
    launch_dt(h->m, h->p, h->st, 1, 0.0, h->st.aux);
    CK(cudaEventRecord(h->st.ev_dt, h->st.aux));
  } else {
    launch_ctrl_step(h->p, h->st, S);
    launch_dt(h->m, h->p, h->st, 1, 0.0, S);
  }
  launch_grad(h->m, h->p, h->st, S);
  if (aside && !flux_split(h->p, h->st)) CK(cudaStreamWaitEvent(S, h->st.ev_dt, 0));
  if (h->profiling) CK(cudaEventRecordWithFlags(h->ev[0], S, cudaEventRecordExternal));
  launch_flux(h->m, h->p, h->st, 1, 1, S);
  if (h->profiling) CK(cudaEventRecordWithFlags(h->ev[1], S, cudaEventRecordExternal));
  if (resid_aside) {
    CK(cudaEventRecord(h->st.ev_res, S));
    CK(cudaStreamWaitEvent(h->st.aux, h->st.ev_res, 0));
    launch_resid_cases(h->st, h->d_case_off, h->d_rblk_off, h->d_rblk_case, h->nrblk, h->ncases, 1, h->st.aux);
    CK(cudaEventRecord(h->st.ev_resid, h->st.aux));
  } else {
    if (aside) CK(cudaStreamWaitEvent(S, h->st.ev_dt, 0));
    launch_resid_cases(h->st, h->d_case_off, h->d_rblk_off, h->d_rblk_case, h->nrblk, h->ncases, 1, S);
  }
  if (h->profiling) CK(cudaEventRecordWithFlags(h->ev[2], S, cudaEventRecordExternal));
  // the relaxation's result (x, [5][N]); the update reads it directly
  const void* x = nullptr;
  int x_fp32 = h->p.fp32;
  if (solver == JG_LS_LUSGS) {
    launch_lusgs(h->m, h->p, h->st, S);
    x = h->st.x1;
    x_fp32 = 0;  // LU-SGS is FP64
  } else if (solver == JG_LS_JACOBI) {
    int sweeps = std::max(1, h->hp.ls_max_iter);
    launch_jacobi(h->m, h->p, h->st, sweeps, S);
    x = (sweeps % 2 == 1) ? h->st.x0 : h->st.x1;
  } else if (solver == JG_LS_SGS) {
    launch_sgs(h->m, h->p, h->st, std::max(1, h->hp.ls_max_iter), S);
    x = h->st.x0;
  } else if (solver == JG_LS_LINE) {
    int sweeps = std::max(1, h->hp.ls_max_iter);
    launch_line_relax(h->m, h->p, h->st, h->lines, 5, sweeps, S);
    x = (sweeps % 2 == 1) ? h->st.x0 : h->st.x1;
  } else {
    if (for_graph) return set_err(JG_ERR_ARG, "BCGSTAB is not captured");
    // host-driven BiCGSTAB on the assembled system, zero initial guess; the rhs ([N][5] in st.b) as [5][N]
    const long n5 = 5L * h->ncv;
    double* phi = (double*)h->st.x0;
    double* b = (double*)h->st.x1;
    CK(cudaMemsetAsync(phi, 0, n5 * sizeof(double), S));
    launch_aos_to_soa5(h->ncv, h->st.b, b, S);
    int it;
    RC(bcgstab(h, phi, b, h->hp.ls_abs, h->hp.ls_rel, h->hp.ls_max_iter, &it, solver == JG_LS_BCGSTAB_LINELET));
    x = phi;
    x_fp32 = 0;  // BiCGSTAB is FP64
  }
  if (h->profiling) CK(cudaEventRecordWithFlags(h->ev[3], S, cudaEventRecordExternal));
  if (resid_aside) CK(cudaStreamWaitEvent(S, h->st.ev_resid, 0));
  launch_update_state_x(h->m, h->p, h->st, x, x_fp32, S);
  launch_faces_after_update(h->m, h->p, h->st, S);
  CKL();
  return JG_OK;
}

static int ensure_graph(jg_case* h) {
  int sweeps = std::max(1, h->hp.ls_max_iter);
  if (h->graph && h->graph_sweeps == sweeps) return JG_OK;
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
  int rc = enqueue_step(h, 1);
  cudaError_t e = cudaStreamEndCapture(h->stream, &g);
  if (rc != JG_OK) return rc;
  if (e != cudaSuccess) return set_err(JG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
  size_t nn = 0;
  CK(cudaGraphGetNodes(g, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  CK(cudaGraphGetNodes(g, nodes.data(), &nn));
  h->graph_kernels = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    CK(cudaGraphNodeGetType(nd, &t));
    if (t == cudaGraphNodeTypeKernel) h->graph_kernels++;
  }
  CK(cudaGraphInstantiate(&h->graph, g, 0));
  cudaGraphDestroy(g);
  h->graph_sweeps = sweeps;
  h->graph_gen++;
  return JG_OK;
}

// nsteps steps enqueued on the case stream (the host-driven BiCGSTAB synchronises inside);
// hist_set: the call's history base is already set on the device
static int enqueue_steps(jg_case* h, int nsteps, bool hist_set = false) {
  if (nsteps > h->hist_cap) {
    int cap = std::max(nsteps, 2 * h->hist_cap);
    double* r = nullptr;
    RC(dmalloc(h, &r, h->bs * (size_t)cap * h->ncases));
    h->st.resid = r;
    h->hist_cap = cap;
    h->st.hist_cap = cap;
    if (h->graph) {
      cudaGraphExecDestroy(h->graph);
      h->graph = nullptr;
    }
  }
  // history base: residual k of this call goes to resid[k] (set on the device, no round trip)
  if (!hist_set) launch_hist_base(h->st, h->stream);
  bool use_graph = h->hp.lin_solver != JG_LS_BCGSTAB && h->hp.lin_solver != JG_LS_BCGSTAB_LINELET;
  if (use_graph) RC(ensure_graph(h));
  for (int k = 0; k < nsteps; k++) {
    if (use_graph) CK(cudaGraphLaunch(h->graph, h->stream));
    else RC(enqueue_step(h, 0));
  }
  CKL();
  return JG_OK;
}

// the per-step residual history of the last call, summed over the cases of a batch
static int batch_resid_sum(jg_case* h, int nsteps, double* resid) {
  const int bs = h->bs;
  std::vector<double> all(bs * (size_t)nsteps * h->ncases);
  CK(cudaMemcpy(all.data(), h->st.resid, all.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int k = 0; k < nsteps; k++)
    for (int i = 0; i < bs; i++) {
      double v = 0.0;
      for (int c = 0; c < h->ncases; c++) v += all[((size_t)k * h->ncases + c) * bs + i];
      resid[(size_t)bs * k + i] = v;
    }
  return JG_OK;
}

int jg_step(jg_case_t* h, int nsteps, double* resid) {
  if (!h || nsteps < 0) return set_err(JG_ERR_ARG, "bad argument");
  if (!h->primed) RC(prime(h));
  RC(enqueue_steps(h, nsteps));
  // a single case's residual history rides on the error-flag read's synchronisation
  const bool direct = resid && nsteps > 0 && h->ncases == 1;
  RC(check_err_flags(h, false, direct ? h->st.resid : nullptr, direct ? h->bs * (size_t)nsteps : 0, resid));
  if (resid && nsteps > 0 && !direct) RC(batch_resid_sum(h, nsteps, resid));
  return JG_OK;
}

// jg_step_host's stream work on the 5x5 path: the copies up, one kernel (pack + state + history
// base), one (setBC + face properties), the steps (recorded in place when captured), one kernel
// (unpack + flags + residuals gathered), the copies down.  The kernels reading and writing
// page-locked caller memory in place over the bus measured slower than the copy engines (495
// against 381 us a step on a 49k-cell case), so the state is staged.
static int host_step_enqueue(jg_case* h, double* rho, double* rhou, double* rhoE, int nsteps, int nres, void* hp,
                             bool capture) {
  const size_t N = h->ncv;
  double* ir = h->d_io;
  double* iu = h->d_io + N;
  double* ie = h->d_io + 4 * N;
  CK(cudaMemcpyAsync(ir, rho, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(iu, rhou, 3 * N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(ie, rhoE, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_state_in(h->m, h->p, h->st, ir, iu, ie, h->d_cell_old, h->stream);
  launch_faces_after_update(h->m, h->p, h->st, h->stream);
  if (capture) {
    for (int k = 0; k < nsteps; k++) RC(enqueue_step(h, 1));
  } else {
    h->primed = 1;
    RC(enqueue_steps(h, nsteps, true));
  }
  launch_state_out(h->m, h->st, ir, iu, ie, h->d_cell_old, h->d_out, nres, h->stream);
  CKL();
  CK(cudaMemcpyAsync(rho, ir, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(rhou, iu, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(rhoE, ie, N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(hp, h->d_out, (2 + (size_t)nres) * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return JG_OK;
}

// set_state + step + get_state with one synchronisation: the state goes up, the preamble and the
// steps run, the new state comes back into the same arrays
int jg_step_host(jg_case_t* h, double* rho, double* rhou, double* rhoE, int nsteps, double* resid) {
  if (!h || !rho || !rhou || !rhoE || nsteps < 0) return set_err(JG_ERR_ARG, "bad argument");
  if (h->ncases != 1) return set_err(JG_ERR_ARG, "jg_step_host takes a single case (batches: jg_batch_*)");
  const size_t N = h->ncv;
  if (h->bs == 5) {
    // the 5x5 path in few stream operations: the copies up, one kernel (pack + state + history
    // base), one (setBC + face properties), the steps, one kernel (unpack + flags + residuals
    // gathered), the copies down and one synchronisation
    if (!h->d_io) RC(dmalloc(h, &h->d_io, 5 * N));
    const int nres = resid && nsteps > 0 ? h->bs * nsteps : 0;
    if (h->d_out_cap < 2 + nres) {
      double* o = nullptr;
      RC(dmalloc(h, &o, 2 + (size_t)nres));
      h->d_out = o;
      h->d_out_cap = 2 + nres;
    }
    void* hp = nullptr;
    RC(pinned(h, (2 + (size_t)nres) * sizeof(double), &hp));
    // one step on page-locked arrays: the whole call as one graph (made once for these arrays)
    bool locked = nsteps == 1 && h->hp.lin_solver != JG_LS_BCGSTAB && h->hp.lin_solver != JG_LS_BCGSTAB_LINELET;
    const double* arr[3] = {rho, rhou, rhoE};
    for (int i = 0; i < 3 && locked; i++) {
      cudaPointerAttributes a;
      if (cudaPointerGetAttributes(&a, arr[i]) != cudaSuccess) {
        cudaGetLastError();  // an unregistered pointer is not an error here
        locked = false;
      } else {
        locked = a.type == cudaMemoryTypeHost;
      }
    }
    if (locked) {
      RC(ensure_graph(h));  // (the history holds 64 steps from the start)
      const void* key[5] = {rho, rhou, rhoE, hp, h->d_out};
      if (!h->host_graph || h->host_gen != h->graph_gen || memcmp(key, h->host_key, sizeof(key)) != 0 ||
          h->host_nres != nres) {
        if (h->host_graph) cudaGraphExecDestroy(h->host_graph);
        h->host_graph = nullptr;
        cudaGraph_t g;
        CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        int rc = host_step_enqueue(h, rho, rhou, rhoE, 1, nres, hp, true);
        cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        if (rc != JG_OK) return rc;
        if (e != cudaSuccess) return set_err(JG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        CK(cudaGraphInstantiate(&h->host_graph, g, 0));
        cudaGraphDestroy(g);
        memcpy(h->host_key, key, sizeof(key));
        h->host_gen = h->graph_gen;
        h->host_nres = nres;
      }
      CK(cudaGraphLaunch(h->host_graph, h->stream));
      h->primed = 1;
    } else {
      RC(host_step_enqueue(h, rho, rhou, rhoE, nsteps, nres, hp, false));
    }
    CK(cudaStreamSynchronize(h->stream));
    const double* o = (const double*)hp;
    if (nres) memcpy(resid, o + 2, nres * sizeof(double));
    const int e = (int)o[0] | (int)o[1];
    if (e & 2) return set_err(JG_ERR_ARG, "unrecognised boundary condition");
    if (e) return set_err(JG_ERR_STATE, "non-physical state (flags %d): negative density/pressure or NaN residual", e);
    return JG_OK;
  }
  RC(stage_state_in(h, rho, rhou, rhoE));
  RC(prime_enqueue(h));
  RC(enqueue_steps(h, nsteps));
  RC(stage_state_out(h, rho, rhou, rhoE));
  const size_t nres = resid && nsteps > 0 ? h->bs * (size_t)nsteps : 0;
  return check_err_flags(h, true, nres ? h->st.resid : nullptr, nres, resid);
}

// per-case status of a batch: status[k] = error flags of case k since the last
// call (1: non-positive density or pressure, 4: NaN residual), then cleared
int jg_batch_status(jg_case_t* h, int* status) {
  if (!h || !status) return set_err(JG_ERR_ARG, "bad argument");
  CK(cudaMemcpyAsync(status, h->st.case_err, h->ncases * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemsetAsync(h->st.case_err, 0, h->ncases * sizeof(int), h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return JG_OK;
}

// freeze (active = 0) or resume a case of the batch; a frozen case's state is not updated
int jg_batch_set_active(jg_case_t* h, int k, int active) {
  if (!h || k < 0 || k >= h->ncases) return set_err(JG_ERR_ARG, "bad argument");
  uint8_t v = active ? 1 : 0;
  CK(cudaMemcpyAsync(h->st.case_active + k, &v, 1, cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return JG_OK;
}

// nsteps backward-Euler iterations of every case of the batch; resid[nsteps][ncases][5]
int jg_batch_step(jg_case_t* h, int nsteps, double* resid) {
  if (!h || nsteps < 0) return set_err(JG_ERR_ARG, "bad argument");
  RC(jg_step(h, nsteps, nullptr));
  if (resid && nsteps > 0) {
    // jg_step sized the ring buffer to hold nsteps entries starting at index 0
    CK(cudaMemcpy(resid, h->st.resid, (size_t)h->bs * nsteps * h->ncases * sizeof(double), cudaMemcpyDeviceToHost));
  }
  return JG_OK;
}

// enqueue nsteps without synchronising (device-resident throughput runs)
int jg_step_async(jg_case_t* h, int nsteps) {
  if (!h || nsteps < 0) return set_err(JG_ERR_ARG, "bad argument");
  if (h->hp.lin_solver == JG_LS_BCGSTAB || h->hp.lin_solver == JG_LS_BCGSTAB_LINELET)
    return set_err(JG_ERR_ARG, "jg_step_async needs a captured solver");
  if (!h->primed) RC(prime(h));
  RC(ensure_graph(h));
  for (int k = 0; k < nsteps; k++) CK(cudaGraphLaunch(h->graph, h->stream));
  return JG_OK;
}

int jg_get_cfl_step(jg_case_t* h, double* cfl, int* step) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  double ctrl[3];
  CK(cudaMemcpyAsync(ctrl, h->st.ctrl, sizeof(ctrl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (cfl) *cfl = ctrl[0];
  if (step) *step = (int)ctrl[1];
  return JG_OK;
}

int jg_set_cfl_step(jg_case_t* h, double cfl, int step) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  if (step < 0 || !(cfl >= 0.0)) return set_err(JG_ERR_ARG, "bad cfl or step");
  double ctrl[16];
  CK(cudaMemcpyAsync(ctrl, h->st.ctrl, sizeof(ctrl), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  ctrl[0] = cfl;
  ctrl[1] = (double)step;
  CK(cudaMemcpyAsync(h->st.ctrl, ctrl, sizeof(ctrl), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return JG_OK;
}

int jg_euler_flux_faces(int kind, int n, const double* L, const double* R, const double* area, const double* nvec,
                        double* F, double* AL, double* AR) {
  if (n < 0 || !L || !R || !area || !nvec || !F) return set_err(JG_ERR_ARG, "bad argument");
  if (kind < 0 || kind > 4) return set_err(JG_ERR_ARG, "unsupported flux %d", kind);
  if (n == 0) return JG_OK;
  double *dL, *dR, *dA, *dN, *dF, *dAL = nullptr, *dAR = nullptr;
  size_t b6 = 6 * (size_t)n * 8, b3 = 3 * (size_t)n * 8;
  CK(cudaMalloc(&dL, b6));
  CK(cudaMalloc(&dR, b6));
  CK(cudaMalloc(&dA, (size_t)n * 8));
  CK(cudaMalloc(&dN, b3));
  CK(cudaMalloc(&dF, 5 * (size_t)n * 8));
  if (AL) CK(cudaMalloc(&dAL, 25 * (size_t)n * 8));
  if (AR) CK(cudaMalloc(&dAR, 25 * (size_t)n * 8));
  CK(cudaMemcpy(dL, L, b6, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dR, R, b6, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dA, area, (size_t)n * 8, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(dN, nvec, b3, cudaMemcpyHostToDevice));
  launch_flux_faces(kind, n, dL, dR, dA, dN, dF, dAL, dAR, 0);
  CKL();
  CK(cudaMemcpy(F, dF, 5 * (size_t)n * 8, cudaMemcpyDeviceToHost));
  if (AL) CK(cudaMemcpy(AL, dAL, 25 * (size_t)n * 8, cudaMemcpyDeviceToHost));
  if (AR) CK(cudaMemcpy(AR, dAR, 25 * (size_t)n * 8, cudaMemcpyDeviceToHost));
  cudaFree(dL); cudaFree(dR); cudaFree(dA); cudaFree(dN); cudaFree(dF);
  if (dAL) cudaFree(dAL);
  if (dAR) cudaFree(dAR);
  return JG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// coupled path (turbulence model): scalars, calcRhsCoupled, model arrays
// ---------------------------------------------------------------------------
extern "C" int jg_set_scalars(jg_case_t* h, const double* phi) {
  if (!h || !phi) return set_err(JG_ERR_ARG, "null argument");
  if (h->bs == 5) return set_err(JG_ERR_ARG, "the case transports no scalar");
  const size_t N = h->ncv, ns = h->turb.ns;
  std::vector<double> cm(ns * N);  // [ncv][ns] -> [ns][ncv]
  const std::vector<int>& perm = h->rn.cell_old;
  for (size_t c = 0; c < N; c++) {
    const size_t o = perm.empty() ? c : (size_t)perm[c];
    for (size_t q = 0; q < ns; q++) cm[q * N + c] = phi[ns * o + q];
  }
  CK(cudaMemcpyAsync(h->turb.phi, cm.data(), cm.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->primed = 0;  // the state, scalar boundary values and turbulent viscosity follow at the next call
  return JG_OK;
}

extern "C" int jg_get_scalars(jg_case_t* h, double* phi) {
  if (!h || !phi) return set_err(JG_ERR_ARG, "null argument");
  if (h->bs == 5) return set_err(JG_ERR_ARG, "the case transports no scalar");
  const size_t N = h->ncv, ns = h->turb.ns;
  std::vector<double> cm(ns * N);
  CK(cudaMemcpyAsync(cm.data(), h->turb.phi, cm.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  const std::vector<int>& perm = h->rn.cell_old;
  for (size_t c = 0; c < N; c++) {
    const size_t o = perm.empty() ? c : (size_t)perm[c];
    for (size_t q = 0; q < ns; q++) phi[ns * o + q] = cm[q * N + c];
  }
  return JG_OK;
}

extern "C" int jg_get_turb_array(jg_case_t* h, const char* name, double* out) {
  if (!h || !name || !out) return set_err(JG_ERR_ARG, "null argument");
  if (h->bs == 5) return set_err(JG_ERR_ARG, "the case has no turbulence model");
  if (!h->primed) RC(prime(h));
  const size_t N = h->ncv, ns = h->turb.ns;
  const Turb& t = h->turb;
  const std::vector<int>&cp = h->rn.cell_old, &fp = h->rn.face_old;
  const size_t nfa = h->nfa, nfa_b = h->nfa_b;
  // name, array, order, rows, doubles per row, blocks (one per scalar)
  struct { const char* n; const double* p; const std::vector<int>* perm; size_t rows, w, nblk; } tab[] = {
      {"wallDist", t.wd, &cp, N, 1, 1}, {"strMag", t.strMag, &cp, N, 1, 1}, {"vortMag", t.vortMag, &cp, N, 1, 1},
      {"diverg", t.diverg, &cp, N, 1, 1}, {"crossDiff", t.crossDiff, &cp, N, 1, 1},
      {"blendFuncF1", t.F1, &cp, N, 1, 1}, {"blendFuncF2", t.F2, &cp, N, 1, 1},
      {"mut_fa", h->st.mut_fa, &fp, nfa, 1, 1}, {"phi_bfa", t.phi_bfa, &fp, nfa_b, 1, ns},
      {"grad_phi", t.grad_phi, &cp, N, 3, ns}, {"diff", t.diff, &fp, nfa, 1, ns}};
  for (auto& e : tab)
    if (strcmp(e.n, name) == 0) {
      if (!e.p) return set_err(JG_ERR_ARG, "%s is not an array of this model", name);
      return download_rows(h, e.p, out, *e.perm, e.rows, e.w, e.nblk);
    }
  return set_err(JG_ERR_ARG, "unknown turbulence array %s", name);
}

extern "C" int jg_calc_rhs_coupled(jg_case_t* h, double* rhs, double* A, int flagImplicit) {
  if (!h || !rhs) return set_err(JG_ERR_ARG, "null argument");
  if (h->bs == 5) return set_err(JG_ERR_ARG, "a case without a turbulence model assembles with jg_calc_rhs");
  if (!h->primed) RC(prime(h));
  int implicit = flagImplicit && A != nullptr;
  launch_flux6(h->m, h->p, h->st, h->turb, implicit, 0, h->stream);
  CKL();
  RC(download_rows(h, h->st.rhs, rhs, h->rn.cell_old, h->ncv, h->bs));
  if (implicit) RC(download_csr(h, A));
  return check_err_flags(h);
}

extern "C" int jg_get_turb(jg_case_t* h, double* wallDist, double* mut_fa, double* strMag, double* vortMag,
                           double* phi_bfa, double* grad_phi, double* diff) {
  if (!h) return set_err(JG_ERR_ARG, "null argument");
  if (h->bs == 5) return set_err(JG_ERR_ARG, "the case has no turbulence model");
  if (!h->primed) RC(prime(h));
  const size_t N = h->ncv;
  const std::vector<int>&cp = h->rn.cell_old, &fp = h->rn.face_old;
  struct { double* dst; const double* src; const std::vector<int>* perm; size_t n, w; } t[] = {
      {wallDist, h->turb.wd, &cp, N, 1}, {mut_fa, h->st.mut_fa, &fp, (size_t)h->nfa, 1},
      {strMag, h->turb.strMag, &cp, N, 1}, {vortMag, h->turb.vortMag, &cp, N, 1},
      {phi_bfa, h->turb.phi_bfa, &fp, (size_t)h->nfa_b, 1}, {grad_phi, h->turb.grad_phi, &cp, N, 3},
      {diff, h->turb.diff, &fp, (size_t)h->nfa, 1}};
  for (auto& e : t)
    if (e.dst) RC(download_rows(h, e.src, e.dst, *e.perm, e.n, e.w));
  return JG_OK;
}

// ---------------------------------------------------------------------------
// per-case operations of the serving engine (jg_serve.cu): nothing here waits
// on the device, so one host thread can keep many cases in flight
// ---------------------------------------------------------------------------
namespace jg {

int serve_case_create(const jg_mesh* mesh, const jg_params* params, jg_case** out) {
  if (!mesh || !out) return set_err(JG_ERR_ARG, "null argument");
  *out = nullptr;
  RC(check_params(params));
  if (params->lin_solver == JG_LS_BCGSTAB || params->lin_solver == JG_LS_BCGSTAB_LINELET ||
      params->lin_solver == JG_LS_LINE)
    return set_err(JG_ERR_ARG, "served cases relax with JACOBI, SGS or LUSGS (captured steps)");
  if (params->turb_model != JG_TURB_NONE) return set_err(JG_ERR_ARG, "served cases are laminar / inviscid");
  if (mesh->ncv <= 0 || mesh->nfa < mesh->nfa_b || mesh->nfa_b < 0 || mesh->nbocv_s < mesh->ncv)
    return set_err(JG_ERR_ARG, "inconsistent mesh sizes");
  jg_case* h = new jg_case();
  h->async_alloc = 1;
  int rc = build_case(h, mesh, params);
  if (rc == JG_OK) rc = dmalloc(h, &h->d_io, 5 * (size_t)mesh->ncv);
  if (rc != JG_OK) {
    std::string keep = g_err;
    jg_destroy(h);
    g_err = keep;
    return rc;
  }
  *out = h;
  return JG_OK;
}

// initial state: staged copies, then the state/face/boundary pass of jg_set_state
int serve_case_start(jg_case* h, const double* rho, const double* rhou, const double* rhoE) {
  const size_t N = h->ncv;
  CK(cudaMemcpyAsync(h->d_io, rho, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_io + N, rhou, 3 * N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CK(cudaMemcpyAsync(h->d_io + 4 * N, rhoE, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  launch_pack_state((int)N, h->d_io, h->st.q, h->d_cell_old, h->stream);
  if (h->st.jac_next) CK(cudaMemsetAsync(h->st.jac_next, 0, sizeof(long long) * h->ncases, h->stream));
  launch_state(h->m, h->p, h->st, h->stream);
  launch_face_props(h->m, h->p, h->st, h->stream);
  launch_bc(h->m, h->p, h->st, h->stream);
  CKL();
  h->primed = 1;
  return JG_OK;
}

int serve_case_ring(jg_case* h) { return h->hist_cap; }

// nsteps captured steps, then the residual ring and the error flags into
// (pinned) host memory, then ev.  Residual of step s (1-based, counted from
// the handle's creation) lands at ring[(s - 1) % ring size].
int serve_case_launch(jg_case* h, int nsteps, double* h_ring, int* h_err, cudaEvent_t ev) {
  if (nsteps < 1 || nsteps > h->hist_cap) return set_err(JG_ERR_ARG, "steps per launch must be 1..%d", h->hist_cap);
  RC(ensure_graph(h));
  for (int k = 0; k < nsteps; k++) CK(cudaGraphLaunch(h->graph, h->stream));
  CK(cudaMemcpyAsync(h_ring, h->st.resid, 5 * (size_t)h->hist_cap * sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaMemcpyAsync(h_err, h->st.err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaMemcpyAsync(h_err + 1, h->st.case_err, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaEventRecord(ev, h->stream));
  return JG_OK;
}

size_t serve_case_bytes(jg_case* h) { return h->bytes; }
int serve_case_ncv(jg_case* h) { return h->ncv; }
int serve_set_err(int code, const char* msg) { return set_err(code, "%s", msg); }
int case_restart_info(jg_case* h, int* ncv, int* nscal, int* turb_model, int* ncases, double* cfl0) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  *ncv = h->ncv;
  *nscal = h->hp.turb_model == JG_TURB_NONE ? 0 : h->hp.nscal;
  *turb_model = h->hp.turb_model;
  *ncases = h->ncases;
  *cfl0 = h->hp.cfl;
  return JG_OK;
}

}  // namespace jg

extern "C" int jg_set_profiling(jg_case_t* h, int on) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  on = on ? 1 : 0;
  if (on && !h->ev[0])
    for (int i = 0; i < 4; i++) CK(cudaEventCreate(&h->ev[i]));
  if (on != h->profiling && h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  h->profiling = on;
  return JG_OK;
}

// device time (ms) of the last completed step: [0] face loop (gradients excluded),
// [1] linear solve, waiting for that step to finish
extern "C" int jg_get_profile(jg_case_t* h, double* ms) {
  if (!h || !ms) return set_err(JG_ERR_ARG, "null argument");
  if (!h->profiling) return set_err(JG_ERR_ARG, "profiling is off");
  CK(cudaEventSynchronize(h->ev[3]));
  float a = 0.f, b = 0.f;
  CK(cudaEventElapsedTime(&a, h->ev[0], h->ev[1]));
  CK(cudaEventElapsedTime(&b, h->ev[2], h->ev[3]));
  ms[0] = a;
  ms[1] = b;
  return JG_OK;
}

// ---------------------------------------------------------------------------
// launch shapes: the lanes per cell of the 5x5 face loop and the Jacobi sweep kernel
// ---------------------------------------------------------------------------
static void drop_graph(jg_case* h) {
  if (h->graph) {
    cudaGraphExecDestroy(h->graph);
    h->graph = nullptr;
  }
  h->graph_sweeps = -1;
}

extern "C" int jg_set_launch_config(jg_case_t* h, int flux_cl, int relax_variant) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  const bool split = flux_cl == JG_FLUX_SPLIT + 1 || flux_cl == JG_FLUX_SPLIT + 2 || flux_cl == JG_FLUX_SPLIT + 4 ||
                     flux_cl == JG_FLUX_SPLIT + 8;
  if (flux_cl != 1 && flux_cl != 2 && flux_cl != 4 && flux_cl != JG_FLUX_CL1_3BLK && !split)
    return set_err(JG_ERR_ARG, "face loop shape must be 1, 2, 4 lanes per cell, JG_FLUX_CL1_3BLK or "
                               "JG_FLUX_SPLIT + 1, 2, 4 or 8");
  if (relax_variant != 0 && relax_variant != 1) return set_err(JG_ERR_ARG, "sweep kernel must be 0 or 1");
  CK(cudaStreamSynchronize(h->stream));
  h->p.flux_cl = flux_cl;
  h->p.relax_variant = relax_variant;
  drop_graph(h);  // the next step captures the new shapes
  return JG_OK;
}

extern "C" int jg_get_launch_config(jg_case_t* h, int* flux_cl, int* relax_variant) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  if (flux_cl) *flux_cl = h->p.flux_cl;
  if (relax_variant) *relax_variant = h->p.relax_variant;
  return JG_OK;
}

// Times every candidate shape on the handle's own mesh and state (trials
// launches each, CUDA events on the case stream) and keeps the fastest.  The
// timed launches only overwrite work arrays that the next step recomputes.
extern "C" int jg_autotune(jg_case_t* h, int trials, int* flux_cl, int* relax_variant, float* ms) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  if (!h->primed) RC(prime(h));
  if (h->bs == 5) {
    trials = std::max(1, trials);
    cudaStream_t S = h->stream;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    launch_dt(h->m, h->p, h->st, 1, 0.0, S);
    launch_grad(h->m, h->p, h->st, S);
    Params p = h->p;
    // every shape is timed forming the whole Jacobian (a lag schedule would skip it)
    State st = h->st;
    st.jac_lag = 1;
    // ms[0..2]: fused, 1, 2, 4 lanes per cell; ms[5]: fused, one lane with three blocks per SM;
    // ms[6..9]: split, residual with 1, 2, 4, 8 lanes per cell.  A lagged handle runs split.
    const int cls[8] = {1, 2, 4, JG_FLUX_CL1_3BLK, JG_FLUX_SPLIT + 1, JG_FLUX_SPLIT + 2, JG_FLUX_SPLIT + 4,
                        JG_FLUX_SPLIT + 8};
    const int slot[8] = {0, 1, 2, 5, 6, 7, 8, 9};
    float best = 1e30f;
    int best_cl = h->p.flux_cl, best_v = h->p.relax_variant;
    for (int i = 0; i < 8; i++) {
      if (h->st.jac_lag > 1 && cls[i] < JG_FLUX_SPLIT) {
        if (ms) ms[slot[i]] = 0.0f;
        continue;
      }
      p.flux_cl = cls[i];
      launch_flux(h->m, p, st, 1, 1, S);  // warm-up
      CK(cudaEventRecord(e0, S));
      for (int t = 0; t < trials; t++) launch_flux(h->m, p, st, 1, 1, S);
      CK(cudaEventRecord(e1, S));
      CK(cudaEventSynchronize(e1));
      float t_ms = 0.0f;
      CK(cudaEventElapsedTime(&t_ms, e0, e1));
      if (ms) ms[slot[i]] = t_ms / trials;
      if (t_ms < best) { best = t_ms; best_cl = cls[i]; }
    }
    p.flux_cl = best_cl;
    best = 1e30f;
    for (int v = 0; v < 2; v++) {
      p.relax_variant = v;
      launch_jacobi(h->m, p, h->st, 2, S);  // warm-up
      CK(cudaEventRecord(e0, S));
      launch_jacobi(h->m, p, h->st, 2 * trials, S);
      CK(cudaEventRecord(e1, S));
      CK(cudaEventSynchronize(e1));
      float t_ms = 0.0f;
      CK(cudaEventElapsedTime(&t_ms, e0, e1));
      if (ms) ms[3 + v] = t_ms / (2 * trials);
      if (t_ms < best) { best = t_ms; best_v = v; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CKL();
    h->p.flux_cl = best_cl;
    h->p.relax_variant = best_v;
    drop_graph(h);
  }
  if (flux_cl) *flux_cl = h->p.flux_cl;
  if (relax_variant) *relax_variant = h->p.relax_variant;
  return JG_OK;
}

// kernels launched by one captured step
extern "C" int jg_step_kernel_count(jg_case_t* h, int* n) {
  if (!h || !n) return set_err(JG_ERR_ARG, "null argument");
  if (h->hp.lin_solver == JG_LS_BCGSTAB || h->hp.lin_solver == JG_LS_BCGSTAB_LINELET)
    return set_err(JG_ERR_ARG, "BCGSTAB steps are not captured");
  if (!h->primed) RC(prime(h));
  RC(ensure_graph(h));
  *n = (int)h->graph_kernels;
  return JG_OK;
}

extern "C" int solveLinSysNSCoupled(jg_case_t* h, double* dq, const double* A, const double* rhs, double zeroAbs,
                                    double zeroRel, int maxIter, int* iters) {
  return jg_solve_lin_sys(h, dq, A, rhs, zeroAbs, zeroRel, maxIter, iters);
}

// calcCvVectorGrad / calcCvScalarGrad of the handle's current state on their own (UgpWithCv.h:803-1083),
// the pass calcRhs starts with: the same kernel, so the arrays equal those of jg_calc_rhs
extern "C" int jg_calc_grad(jg_case_t* h, double* grad_u, double* grad_rho, double* grad_p, double* grad_h) {
  if (!h) return set_err(JG_ERR_ARG, "null handle");
  if (h->bs != 5) return set_err(JG_ERR_ARG, "the coupled path's gradients come with jg_calc_rhs_coupled");
  if (!h->p.second_order && !h->p.viscous)
    return set_err(JG_ERR_ARG, "a first-order inviscid case computes no gradients");
  if (!h->primed) RC(prime(h));
  launch_grad(h->m, h->p, h->st, h->stream);
  CKL();
  return jg_get_gradients(h, grad_u, grad_rho, grad_p, grad_h);
}

// runBackwardEuler until a residual rule stops it, or max_steps steps.  resid_drop >= 0: the energy
// residual at or below resid_drop x the first step's (a relative drop); resid_drop < 0: doneSolver's
// rule (JoeWithModels.h:64), the absolute energy residual strictly below -resid_drop.  The residual
// is checked every check_every steps (1: step by step; more: fewer host round trips, the state then
// ends up to check_every - 1 steps past the one that met the rule).  steps / drop (may be NULL): the
// steps run and the relative drop of the last step run.
extern "C" int jg_run_to(jg_case_t* h, double resid_drop, int max_steps, int check_every, int* steps, double* drop) {
  if (!h || max_steps < 0 || check_every < 1 || !(resid_drop == resid_drop)) return set_err(JG_ERR_ARG, "bad argument");
  const bool absolute = resid_drop < 0.0;
  if (h->ncases != 1) return set_err(JG_ERR_ARG, "a batch handle: run its cases with jg_batch_step");
  const int bs = h->bs;
  std::vector<double> r((size_t)bs * check_every);
  double r0 = -1.0, last = 1.0;
  int done = 0;
  while (done < max_steps) {
    const int n = std::min(check_every, max_steps - done);
    int rc = jg_step(h, n, r.data());
    if (rc) {
      if (steps) *steps = done;
      if (drop) *drop = last;
      return rc;
    }
    bool met = false;
    for (int k = 0; k < n; k++) {
      const double e = r[(size_t)k * bs + 4];
      if (r0 < 0.0) r0 = e;
      last = r0 > 0.0 ? e / r0 : 0.0;
      if (absolute ? (e < -resid_drop) : (last <= resid_drop)) met = true;
    }
    done += n;
    if (met) break;
  }
  if (steps) *steps = done;
  if (drop) *drop = last;
  return JG_OK;
}

// new run-time settings for a live handle (the reference re-reads its parameters between runs):
// the CFL / DT settings and ramp, under-relaxation, linear-solver thresholds and sweeps, limiter
// EPS and the time-step mode.  Settings that shape the handle's arrays (flux, order, limiter on /
// off, viscosity, model, precision, solver kind, renumbering, gradient scheme, boundary kinds) must
// not change.  The CFL the ramp stands at is left as it is (jg_set_cfl_step sets it).
extern "C" int jg_set_params(jg_case_t* h, const jg_params* q) {
  if (!h || !q) return set_err(JG_ERR_ARG, "null argument");
  RC(check_params(q));
  const jg_params& o = h->hp;
  if (q->flux != o.flux || q->second_order != o.second_order || q->limiter != o.limiter ||
      q->mu_mode != o.mu_mode || q->mu_ref != o.mu_ref || q->mu_power_law != o.mu_power_law ||
      q->SL_Tref != o.SL_Tref || q->SL_Sref != o.SL_Sref || q->gamma != o.gamma || q->R_gas != o.R_gas ||
      q->Pr != o.Pr || q->PrTurb != o.PrTurb || q->T_ref != o.T_ref || q->visc_limiter != o.visc_limiter ||
      q->symm_bc != o.symm_bc || q->lin_solver != o.lin_solver || q->precision != o.precision ||
      q->nscal != o.nscal || q->turb_model != o.turb_model || q->renumber != o.renumber ||
      q->grad_scheme != o.grad_scheme || q->ausm_type != o.ausm_type || q->shock_fix != o.shock_fix ||
      q->shock_flag != o.shock_flag || q->entropy_fix != o.entropy_fix || std::max(q->jac_lag, 1) != std::max(o.jac_lag, 1))
    return set_err(JG_ERR_ARG, "jg_set_params changes run-time settings only (CFL, DT, ramp, under-relaxation, "
                               "solver thresholds and sweeps, EPS, time-step mode)");
  // a batch keeps the promise jg_batch_create makes: no setting that couples its cases
  if (h->ncases > 1 && q->time_step_mode == JG_TS_CFL_MIN)
    return set_err(JG_ERR_ARG, "CFL_MIN would couple the cases of a batch");
  CK(cudaStreamSynchronize(h->stream));
  const int cl = h->p.flux_cl, rv = h->p.relax_variant;
  h->hp = *q;
  h->p = make_params(*q);
  h->p.flux_cl = cl;
  h->p.relax_variant = rv;
  drop_graph(h);
  return JG_OK;
}

// addViscFlux per face on the GPU (per-face parity), laminar: no turbulent viscosity
extern "C" int jg_visc_flux_faces(int n, const double* S0, const double* S1, const double* gu0, const double* gu1,
                                  const double* gh0, const double* gh1, const double* mul, const double* lamOcp,
                                  const double* u_fa, const double* area, const double* nvec, const double* svec,
                                  const double* smag, double* F, double* A0, double* A1) {
  const double* host[13] = {S0, S1, gu0, gu1, gh0, gh1, mul, lamOcp, u_fa, area, nvec, svec, smag};
  const size_t width[13] = {8, 8, 9, 9, 3, 3, 1, 1, 3, 1, 3, 3, 1};
  if (n < 0 || !F) return set_err(JG_ERR_ARG, "bad argument");
  for (int k = 0; k < 13; k++)
    if (!host[k]) return set_err(JG_ERR_ARG, "null input array %d", k);
  if (n == 0) return JG_OK;
  double* dev[13] = {nullptr};
  double *dF = nullptr, *dA0 = nullptr, *dA1 = nullptr;
  int rc = JG_OK;
  auto fail = [&](cudaError_t e) {
    if (e != cudaSuccess && rc == JG_OK) rc = set_err(JG_ERR_CUDA, "%s", cudaGetErrorString(e));
  };
  for (int k = 0; k < 13 && rc == JG_OK; k++) {
    fail(cudaMalloc(&dev[k], width[k] * n * sizeof(double)));
    if (rc == JG_OK) fail(cudaMemcpy(dev[k], host[k], width[k] * n * sizeof(double), cudaMemcpyHostToDevice));
  }
  if (rc == JG_OK) fail(cudaMalloc(&dF, 4 * (size_t)n * sizeof(double)));
  if (rc == JG_OK && A0) fail(cudaMalloc(&dA0, 25 * (size_t)n * sizeof(double)));
  if (rc == JG_OK && A1) fail(cudaMalloc(&dA1, 25 * (size_t)n * sizeof(double)));
  if (rc == JG_OK) {
    const double* in[13];
    for (int k = 0; k < 13; k++) in[k] = dev[k];
    launch_visc_faces(n, in, dF, dA0, dA1, 0);
    fail(cudaGetLastError());
  }
  if (rc == JG_OK) fail(cudaMemcpy(F, dF, 4 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
  if (rc == JG_OK && A0) fail(cudaMemcpy(A0, dA0, 25 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
  if (rc == JG_OK && A1) fail(cudaMemcpy(A1, dA1, 25 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
  for (int k = 0; k < 13; k++) cudaFree(dev[k]);
  cudaFree(dF);
  cudaFree(dA0);
  cudaFree(dA1);
  return rc;
}

