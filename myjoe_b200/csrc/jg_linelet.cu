// jg_linelet.cu -- the line-implicit preconditioner of BCGSTAB_LINELET.
//
// initializeLinelet (src/joe/JoeWithModels.cpp:7471-7559) grows, from each
// cell on a WALL face, a line of cells in the direction of strong coupling;
// solveCvVectorR5BcgstabLine (src/common/UgpWithCv.cpp:3627-3992) is
// BiCGSTAB whose preconditioner solves the block-tridiagonal system of each
// line exactly (block Thomas elimination) and the block diagonal elsewhere.
//
// Here the lines are built once per handle on the host.  The LINE relaxation
// (below) uses the same rule with one relaxation: where several neighbours
// pass, the line goes on to the strongest if it is 1.1 times the next one,
// so that a line crosses from the last prism row into the hexahedron above
// (whose other lower neighbour is the quad's second prism).  On the device the
// elimination is split in two: k_line_factor runs once per linear solve (the
// matrix does not change inside BiCGSTAB) and keeps, per line cell, the
// inverse of the eliminated diagonal block, the multiplier
// A(c_i, c_{i-1}) inv_{i-1} and the upper block A(c_{i-1}, c_i); k_line_apply
// then does the forward and backward substitutions for one right-hand side
// (twice per BiCGSTAB iteration).  The reference recomputes the elimination
// inside every application; the factors are the same numbers.  One warp per
// line: the lines are independent, and inside a line the work is a chain of
// 5x5 block operations, so the warp's lanes hold the 25 entries (factor) or
// the 5 rows (substitutions) of one block step.
#include <algorithm>
#include <cmath>
#include <vector>

#include "jg_internal.h"

namespace jg {

namespace {

// findFace (JoeWithModels.cpp:7572-7587): the first face of a's list that b also has
int find_face(const jg_mesh& m, int a, int b) {
  if (a == b) return -1;
  for (int i = m.faocv_i[a]; i < m.faocv_i[a + 1]; i++)
    for (int j = m.faocv_i[b]; j < m.faocv_i[b + 1]; j++)
      if (m.faocv_v[i] == m.faocv_v[j]) return m.faocv_v[i];
  return -1;
}

double coupling(const jg_mesh& m, int a, int b) {
  int f = find_face(m, a, b);
  const double* n = &m.fa_normal[3 * f];
  double area = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  return 0.5 * area * ((1.0 / m.cv_volume[a]) + (1.0 / m.cv_volume[b]));
}

}  // namespace

int build_lines(const jg_mesh& m, const std::vector<std::vector<int>>& wall_zones, std::vector<int>& off,
                std::vector<int>& cv, bool relaxed) {
  const int N = m.ncv;
  std::vector<char> free_cv(N, 1);
  // each WALL zone replaces the sources of the one before it (relaxed: every WALL zone's cells are
  // sources, so that each case of a batch grows its own lines); all of their cells leave the pool
  std::vector<int> src;
  for (const auto& z : wall_zones) {
    if (!relaxed) src.clear();
    for (int f : z) {
      src.push_back(m.cvofa[2 * f]);
      free_cv[m.cvofa[2 * f]] = 0;
    }
  }
  off.assign(1, 0);
  cv.clear();
  for (int s : src) {
    const size_t first = cv.size();
    cv.push_back(s);
    for (;;) {
      const int icv = cv.back();
      double wmax = 0.0;
      for (int k = m.nbocv_i[icv] + 1; k < m.nbocv_i[icv + 1]; k++)
        wmax = std::max(wmax, coupling(m, icv, m.nbocv_v[k]));
      // the one free neighbour (not the cell the line came from) with more than half the largest
      // coupling; relaxed: or, among several, the strongest when it is 1.1 times the next one
      int next = -1, count = 0;
      double best_w = 0.0, second_w = 0.0;
      const int prev = cv.size() - first >= 2 ? cv[cv.size() - 2] : -1;
      for (int k = m.nbocv_i[icv] + 1; k < m.nbocv_i[icv + 1]; k++) {
        const int nb = m.nbocv_v[k];
        const double w = coupling(m, icv, nb);
        if (free_cv[nb] && w / wmax > 0.5 && nb != prev) {
          count++;
          if (w > best_w) {
            second_w = best_w;
            best_w = w;
            next = nb;
          } else if (w > second_w) {
            second_w = w;
          }
        }
      }
      if (count == 0 || (count > 1 && !(relaxed && best_w > 1.1 * second_w))) break;
      cv.push_back(next);
      free_cv[next] = 0;
    }
    off.push_back((int)cv.size());
  }
  return JG_OK;
}

namespace {

constexpr int LW = 4;  // warps (lines) per block

// ludeco (UgpWithCv.cpp:2489-2516) on a row-major 5x5 block
__device__ void ludeco5(double* A) {
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
    if (jrjc == 4) break;
#pragma unroll
    for (int jc = jrjc + 1; jc < 5; jc++) {
      double sum = A[5 * jrjc + jc];
#pragma unroll
      for (int jm = 0; jm < jrjc; jm++) sum -= A[5 * jrjc + jm] * A[5 * jm + jc];
      A[5 * jrjc + jc] = sum / A[5 * jrjc + jrjc];
    }
  }
}

// column `col` of the inverse from the ludeco factors, as luinv (UgpWithCv.cpp:2542-2577)
__device__ void luinv_col(const double* A, int col, double* c) {
#pragma unroll
  for (int i = 0; i < 5; i++) c[i] = (i == col) ? 1.0 : 0.0;
  c[0] = c[0] / A[0];
#pragma unroll
  for (int jr = 1; jr < 5; jr++) {
    double sum = c[jr];
#pragma unroll
    for (int jm = 0; jm < jr; jm++) sum -= A[5 * jr + jm] * c[jm];
    c[jr] = sum / A[5 * jr + jr];
  }
#pragma unroll
  for (int jr = 3; jr >= 0; jr--) {
    double sum = c[jr];
#pragma unroll
    for (int jm = 4; jm > jr; jm--) sum -= A[5 * jr + jm] * c[jm];
    c[jr] = sum;
  }
}

// entry e of the matrix block A(row, col): the ELL columns of `row` whose neighbour is `col`
__device__ double ell_block(const Mesh& m, const double* O, int row, int col, int e) {
  const int s = row / SLICE, lane = row % SLICE;
  double v = 0.0;
  for (int j = m.ell_off[s]; j < m.ell_off[s + 1]; j++)
    if (m.ell_nb[(size_t)j * SLICE + lane] == col) v += O[((size_t)j * 25 + e) * SLICE + lane];
  return v;
}
// the block at ELL row j (Lines::jlo / jup), or the search where the two cells share several faces
__device__ __forceinline__ double ell_block_j(const Mesh& m, const double* O, int row, int col, int j, int e) {
  if (j >= 0) return O[((size_t)j * 25 + e) * SLICE + row % SLICE];
  return j == -1 ? 0.0 : ell_block(m, O, row, col, e);
}

__global__ void __launch_bounds__(32 * LW) k_line_factor(Mesh m, State st, Lines L) {
  __shared__ double sh[LW][5][25];
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int line = blockIdx.x * LW + w;
  if (line >= L.nlines) return;
  double *b = sh[w][0], *inv = sh[w][1], *lo = sh[w][2], *up = sh[w][3], *mh = sh[w][4];
  const int p0 = L.off[line], n = L.off[line + 1] - p0;
  const int N = m.ncv;
  const double* D = (const double*)st.D;
  const double* O = (const double*)st.O;
  const int e = lane < 25 ? lane : 24, r = e / 5, k = e % 5;
  if (lane < 25) b[e] = D[(size_t)e * N + L.cv[p0]];
  __syncwarp();
  for (int i = 1;; i++) {
    // inverse of the eliminated diagonal block of position i-1
    if (lane < 5) {
      double A[25], c[5];
#pragma unroll
      for (int q = 0; q < 25; q++) A[q] = b[q];
      ludeco5(A);
      luinv_col(A, lane, c);
#pragma unroll
      for (int q = 0; q < 5; q++) inv[5 * q + lane] = c[q];
    }
    __syncwarp();
    if (lane < 25) L.inv[(size_t)(p0 + i - 1) * 25 + e] = inv[e];
    if (i == n) break;
    const int cp = L.cv[p0 + i - 1], c = L.cv[p0 + i];
    if (lane < 25) {
      lo[e] = ell_block_j(m, O, c, cp, L.jlo[p0 + i], e);
      up[e] = ell_block_j(m, O, cp, c, L.jup[p0 + i], e);
      L.up[(size_t)(p0 + i) * 25 + e] = up[e];
    }
    __syncwarp();
    // mhat = A(c, cp) inv (getMultMatrix order: sums from 0.0 over q)
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 5; q++) s += lo[5 * r + q] * inv[5 * q + k];
    if (lane < 25) {
      mh[e] = s;
      L.low[(size_t)(p0 + i) * 25 + e] = s;
    }
    __syncwarp();
    // next diagonal: A(c, c) - mhat A(cp, c)
    double a0 = 0.0;
#pragma unroll
    for (int q = 0; q < 5; q++) a0 += mh[5 * r + q] * up[5 * q + k];
    const double bn = D[(size_t)e * N + c] - a0;
    __syncwarp();
    if (lane < 25) b[e] = bn;
    __syncwarp();
  }
}

// y (cells of the lines) = the block-tridiagonal solve of x along each line; x, y are [5][N]
__global__ void __launch_bounds__(32 * LW) k_line_apply(Mesh m, Lines L, const double* x, double* y) {
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int line = blockIdx.x * LW + w;
  if (line >= L.nlines) return;
  const int p0 = L.off[line], n = L.off[line + 1] - p0;
  const size_t N = m.ncv;
  const int r = lane % 5;
  const bool row = lane < 5;
  // forward: v_0 = x_0, v_i = x_i - mhat_i v_{i-1}
  double v = x[r * N + L.cv[p0]];
  if (row) L.v[(size_t)p0 * 5 + r] = v;
  for (int i = 1; i < n; i++) {
    const double* Mi = &L.low[(size_t)(p0 + i) * 25 + 5 * r];
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 5; q++) s += Mi[q] * __shfl_sync(0xffffffffu, v, q);
    v = x[r * N + L.cv[p0 + i]] - s;
    if (row) L.v[(size_t)(p0 + i) * 5 + r] = v;
  }
  // backward: y_{n-1} = inv_{n-1} v_{n-1}, y_i = inv_i (v_i - A(c_i, c_{i+1}) y_{i+1})
  const double* I = &L.inv[(size_t)(p0 + n - 1) * 25 + 5 * r];
  double yv = 0.0;
#pragma unroll
  for (int q = 0; q < 5; q++) yv += I[q] * __shfl_sync(0xffffffffu, v, q);
  if (row) y[r * N + L.cv[p0 + n - 1]] = yv;
  for (int i = n - 2; i >= 0; i--) {
    const double* U = &L.up[(size_t)(p0 + i + 1) * 25 + 5 * r];
    double s2 = 0.0;
#pragma unroll
    for (int q = 0; q < 5; q++) s2 += U[q] * __shfl_sync(0xffffffffu, yv, q);
    const double a1 = L.v[(size_t)(p0 + i) * 5 + r] - s2;
    const double* Ii = &L.inv[(size_t)(p0 + i) * 25 + 5 * r];
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 5; q++) s += Ii[q] * __shfl_sync(0xffffffffu, a1, q);
    yv = s;
    if (row) y[r * N + L.cv[p0 + i]] = yv;
  }
}

}  // namespace

void launch_line_factor(const Mesh& m, const State& st, const Lines& L, cudaStream_t s) {
  if (L.nlines) k_line_factor<<<(L.nlines + LW - 1) / LW, 32 * LW, 0, s>>>(m, st, L);
}

void launch_line_precond(const Mesh& m, const State& st, const Lines& L, const double* x, double* y,
                         cudaStream_t s) {
  launch_precond(m, st, x, y, s);  // the block diagonal everywhere, then the lines overwrite their cells
  if (L.nlines) k_line_apply<<<(L.nlines + LW - 1) / LW, 32 * LW, 0, s>>>(m, L, x, y);
}

}  // namespace jg

// ---------------------------------------------------------------------------
// LINE relaxation: block line-Jacobi sweeps for B x B blocks (B = 5, 6, 7) in
// the matrix precision BT.  A sweep is x' = T^-1 (b - (A - T) x), T the
// block-tridiagonal part of A along the lines (the block diagonal elsewhere):
//   k_lrelax_rhs: per cell r = b - sum of the off-diagonal blocks that are not
//                 a line coupling times x; off the lines x' = Dinv r, on the
//                 lines r is left in x' for
//   k_lsolve:     the block Thomas substitutions of each line, in place.
// k_lfactor computes the line factors once per step from D and the ELL
// blocks, in FP64 arithmetic, and stores them in BT.  (The LINE relaxation has
// no reference counterpart; the reference's own line solver, BCGSTAB_LINELET,
// keeps the reference's ludeco/luinv arithmetic in k_line_factor above.)
// ---------------------------------------------------------------------------
namespace jg {
namespace {

template <typename BT, int B>
__device__ double ell_block_b(const Mesh& m, const BT* O, int row, int col, int e) {
  const int s = row / SLICE, lane = row % SLICE;
  double v = 0.0;
  for (int j = m.ell_off[s]; j < m.ell_off[s + 1]; j++)
    if (m.ell_nb[(size_t)j * SLICE + lane] == col) v += (double)O[((size_t)j * B * B + e) * SLICE + lane];
  return v;
}
template <typename BT, int B>
__device__ __forceinline__ double ell_block_bj(const Mesh& m, const BT* O, int row, int col, int j, int e) {
  if (j >= 0) return (double)O[((size_t)j * B * B + e) * SLICE + row % SLICE];
  return j == -1 ? 0.0 : ell_block_b<BT, B>(m, O, row, col, e);
}

// The block Thomas factors along one line per warp: inv_i = (the eliminated diagonal block)^-1,
// low_i = A(c_i, c_i-1) inv_i-1, up_i = A(c_i-1, c_i).  The elimination is serial along the line,
// so each step is kept short: the eliminated block is inverted in place by all lanes together
// (Gauss-Jordan without pivoting, the reference's ludeco/luinv having none either: B pivot
// steps, each one shared-memory read per entry), and the next step's blocks (its coupling
// blocks and diagonal block) are loaded while the current step computes.
template <typename BT, int B>
__global__ void __launch_bounds__(32 * LW) k_lfactor(Mesh m, State st, Lines L) {
  constexpr int BB = B * B, EP = (BB + 31) / 32;  // entries per lane
  __shared__ double sh[LW][4][BB];
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int line = blockIdx.x * LW + w;
  if (line >= L.nlines) return;
  double *b = sh[w][0], *lo = sh[w][1], *up = sh[w][2], *mh = sh[w][3];
  const int p0 = L.off[line], n = L.off[line + 1] - p0;
  const int N = m.ncv;
  const BT* D = (const BT*)st.D;
  const BT* O = (const BT*)st.O;
  BT* Linv = (BT*)L.binv;
  BT* Llow = (BT*)L.blow;
  BT* Lup = (BT*)L.bup;
  for (int e = lane; e < BB; e += 32) b[e] = (double)D[(size_t)e * N + L.cv[p0]];
  // the next step's operands, a step ahead: coupling blocks and diagonal block of position 1
  double nlo[EP], nup[EP], nd[EP];
  auto load_step = [&](int i) {
    const int cp = L.cv[p0 + i - 1], c = L.cv[p0 + i];
    const int jl = L.jlo[p0 + i], ju = L.jup[p0 + i];
#pragma unroll
    for (int t = 0; t < EP; t++) {
      const int e = lane + 32 * t;
      if (e < BB) {
        nlo[t] = ell_block_bj<BT, B>(m, O, c, cp, jl, e);
        nup[t] = ell_block_bj<BT, B>(m, O, cp, c, ju, e);
        nd[t] = (double)D[(size_t)e * N + c];
      }
    }
  };
  if (n > 1) load_step(1);
  __syncwarp();
  for (int i = 1;; i++) {
    // b <- b^-1 in place
#pragma unroll
    for (int k = 0; k < B; k++) {
      const double rp = 1.0 / b[B * k + k];
      double nv[EP];
#pragma unroll
      for (int t = 0; t < EP; t++) {
        const int e = lane + 32 * t, ri = e / B, cj = e % B;
        if (e < BB) {
          if (ri == k) nv[t] = (cj == k) ? rp : b[e] * rp;
          else nv[t] = (cj == k) ? -b[B * ri + k] * rp : b[e] - b[B * ri + k] * (b[B * k + cj] * rp);
        }
      }
      __syncwarp();
#pragma unroll
      for (int t = 0; t < EP; t++)
        if (lane + 32 * t < BB) b[lane + 32 * t] = nv[t];
      __syncwarp();
    }
    for (int e = lane; e < BB; e += 32) Linv[(size_t)(p0 + i - 1) * BB + e] = (BT)b[e];
    if (i == n) break;
    // this step's coupling blocks (loaded a step ahead), the next step's requested now
#pragma unroll
    for (int t = 0; t < EP; t++) {
      const int e = lane + 32 * t;
      if (e < BB) {
        lo[e] = nlo[t];
        up[e] = nup[t];
        Lup[(size_t)(p0 + i) * BB + e] = (BT)nup[t];
      }
    }
    double dc[EP];
#pragma unroll
    for (int t = 0; t < EP; t++) dc[t] = nd[t];
    if (i + 1 < n) load_step(i + 1);
    __syncwarp();
    for (int e = lane; e < BB; e += 32) {
      const int r = e / B, k = e % B;
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < B; q++) s += lo[B * r + q] * b[B * q + k];
      mh[e] = s;
      Llow[(size_t)(p0 + i) * BB + e] = (BT)s;
    }
    __syncwarp();
    double bn[EP];
#pragma unroll
    for (int t = 0; t < EP; t++) {
      const int e = lane + 32 * t;
      bn[t] = 0.0;
      if (e < BB) {
        const int r = e / B, k = e % B;
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < B; q++) s += mh[B * r + q] * up[B * q + k];
        bn[t] = dc[t] - s;
      }
    }
    __syncwarp();
#pragma unroll
    for (int t = 0; t < EP; t++)
      if (lane + 32 * t < BB) b[lane + 32 * t] = bn[t];
    __syncwarp();
  }
}

// one block per 32-cell slice, B rows x 32 lanes (the k_jacobi_c layout)
template <typename BT, int B>
__global__ void __launch_bounds__(B * 32) k_lrelax_rhs(Mesh m, State st, Lines L, const BT* __restrict__ xin,
                                                       BT* __restrict__ xout, int first) {
  __shared__ BT sacc[B][SLICE];
  const int row = threadIdx.x / SLICE, lane = threadIdx.x % SLICE;
  const int slice = blockIdx.x;
  const int c = slice * SLICE + lane;
  const bool active = c < m.ncv;
  const int N = m.ncv;
  BT acc = active ? (BT)st.b[(size_t)B * c + row] : (BT)0;
  if (!first && active) {
    const BT* O = (const BT*)st.O;
    for (int j = m.ell_off[slice]; j < m.ell_off[slice + 1]; j++) {
      if (L.ell_inline[(size_t)j * SLICE + lane]) continue;
      int nb = m.ell_nb[(size_t)j * SLICE + lane];
      const BT* Ob = O + ((size_t)j * B * B + B * row) * SLICE + lane;
      BT s = 0;
#pragma unroll
      for (int k = 0; k < B; k++) s += Ob[k * SLICE] * xin[(size_t)k * N + nb];
      acc -= s;
    }
  }
  sacc[row][lane] = acc;
  __syncthreads();
  if (active) {
    if (L.on_line[c]) {
      xout[(size_t)row * N + c] = acc;
    } else {
      const BT* Di = (const BT*)st.Dinv;
      BT s = 0;
#pragma unroll
      for (int k = 0; k < B; k++) s += Di[(size_t)(B * row + k) * N + c] * sacc[k][lane];
      xout[(size_t)row * N + c] = s;
    }
  }
}

// x (cells of a line) = T_line^-1 r, r read from x.  Four lines per warp, eight lanes per line
// (lanes < B of a group hold the rows of its blocks): the chain along a line is serial, so a
// warp's lines advance together, each step costing one warp's latency for four lines.  The
// operands of the steps (a matrix row, the cell id, the right-hand side) do not depend on the
// chain: they are loaded LK steps at a time into one of two register sets, the next chunk's
// loads issued before the current chunk's steps compute (and its cell ids a chunk earlier), so a
// chunk's memory latency runs under the previous chunk's arithmetic.  The shuffles run on every lane; a group past the end of its
// line only skips the update.
constexpr int LK = 4;
constexpr int LG = 8;         // lanes per line
constexpr int LPW = 32 / LG;  // lines per warp

template <typename BT, int B>
__global__ void __launch_bounds__(32 * LW) k_lsolve(Mesh m, Lines L, BT* __restrict__ x) {
  static_assert(B <= LG, "a line's rows fit its lane group");
  constexpr int BB = B * B;
  constexpr int K = sizeof(BT) * B > 48 ? LK / 2 : LK;  // steps per chunk (FP64 7x7: two register sets fit at LK / 2)
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const int r = lane % LG;
  const int line = (blockIdx.x * LW + w) * LPW + lane / LG;
  const bool has = line < L.nlines;
  const int p0 = has ? L.off[line] : 0, n = has ? L.off[line + 1] - p0 : 0;
  const bool row = has && r < B;
  const int rr = r < B ? r : 0;  // lanes past the rows mirror row 0 and never store
  int nmax = n;
  for (int o = LG; o < 32; o *= 2) nmax = max(nmax, __shfl_xor_sync(0xffffffffu, nmax, o));
  if (nmax == 0) return;  // the whole warp (no line of its own)
  const size_t N = m.ncv;
  const BT* Linv = (const BT*)L.binv;
  const BT* Llow = (const BT*)L.blow;
  const BT* Lup = (const BT*)L.bup;
  BT* Lv = (BT*)L.bv;
  // forward: v_0 = r_0, v_i = r_i - low_i v_{i-1}
  BT v = has ? x[rr * N + L.cv[p0]] : BT(0);
  if (row) Lv[(size_t)p0 * B + r] = v;
  // the operands of steps i0 .. i0 + K - 1 (past the line's end: zeros), called chunk after
  // chunk; their cell ids were loaded by the call before, and this call loads the next chunk's
  int cn[K];
#pragma unroll
  for (int t = 0; t < K; t++) cn[t] = (1 + t < n) ? L.cv[p0 + 1 + t] : 0;
  auto load_fwd = [&](int i0, BT(&mi)[K][B], BT(&xi)[K]) {
#pragma unroll
    for (int t = 0; t < K; t++) {
      const int i = i0 + t;
      if (i < n) {
#pragma unroll
        for (int q = 0; q < B; q++) mi[t][q] = Llow[(size_t)(p0 + i) * BB + B * rr + q];
        xi[t] = x[rr * N + cn[t]];
      } else {
#pragma unroll
        for (int q = 0; q < B; q++) mi[t][q] = BT(0);
        xi[t] = BT(0);
      }
    }
#pragma unroll
    for (int t = 0; t < K; t++) cn[t] = (i0 + K + t < n) ? L.cv[p0 + i0 + K + t] : 0;
  };
  auto step_fwd = [&](int i0, const BT(&mi)[K][B], const BT(&xi)[K]) {
#pragma unroll
    for (int t = 0; t < K; t++) {
      const int i = i0 + t;
      BT s = 0;
#pragma unroll
      for (int q = 0; q < B; q++) s += mi[t][q] * __shfl_sync(0xffffffffu, v, q, LG);
      if (i < n) {
        v = xi[t] - s;
        if (row) Lv[(size_t)(p0 + i) * B + r] = v;
      }
    }
  };
  {
    BT ma[K][B], xa[K], mb[K][B], xb[K];
    load_fwd(1, ma, xa);
    for (int i0 = 1; i0 < nmax; i0 += 2 * K) {
      if (i0 + K < nmax) load_fwd(i0 + K, mb, xb);
      step_fwd(i0, ma, xa);
      if (i0 + K >= nmax) break;
      if (i0 + 2 * K < nmax) load_fwd(i0 + 2 * K, ma, xa);
      step_fwd(i0 + K, mb, xb);
    }
  }
  // backward: y_{n-1} = inv_{n-1} v_{n-1}, y_i = inv_i (v_i - up_{i+1} y_{i+1}); step j of the
  // warp is position n-2-j of each line
  BT yv = 0;
  {
    BT vq[B];
#pragma unroll
    for (int q = 0; q < B; q++) vq[q] = __shfl_sync(0xffffffffu, v, q, LG);
    if (has) {
      const BT* I = &Linv[(size_t)(p0 + n - 1) * BB + B * rr];
#pragma unroll
      for (int q = 0; q < B; q++) yv += I[q] * vq[q];
      if (row) x[r * N + L.cv[p0 + n - 1]] = yv;
    }
  }
  auto load_bwd = [&](int j0, BT(&ui)[K][B], BT(&ii)[K][B], BT(&vi)[K], int(&ci)[K]) {
#pragma unroll
    for (int t = 0; t < K; t++) {
      const int i = n - 2 - (j0 + t);
      if (i >= 0) {
#pragma unroll
        for (int q = 0; q < B; q++) {
          ui[t][q] = Lup[(size_t)(p0 + i + 1) * BB + B * rr + q];
          ii[t][q] = Linv[(size_t)(p0 + i) * BB + B * rr + q];
        }
        vi[t] = Lv[(size_t)(p0 + i) * B + rr];
        ci[t] = L.cv[p0 + i];
      } else {
#pragma unroll
        for (int q = 0; q < B; q++) ui[t][q] = ii[t][q] = BT(0);
        vi[t] = BT(0);
        ci[t] = 0;
      }
    }
  };
  auto step_bwd = [&](int j0, const BT(&ui)[K][B], const BT(&ii)[K][B], const BT(&vi)[K], const int(&ci)[K]) {
#pragma unroll
    for (int t = 0; t < K; t++) {
      const int i = n - 2 - (j0 + t);
      BT s2 = 0;
#pragma unroll
      for (int q = 0; q < B; q++) s2 += ui[t][q] * __shfl_sync(0xffffffffu, yv, q, LG);
      const BT a1 = vi[t] - s2;
      BT s = 0;
#pragma unroll
      for (int q = 0; q < B; q++) s += ii[t][q] * __shfl_sync(0xffffffffu, a1, q, LG);
      if (i >= 0) {
        yv = s;
        if (row) x[r * N + ci[t]] = yv;
      }
    }
  };
  {
    BT ua[K][B], ia[K][B], va[K], ub[K][B], ib[K][B], vb[K];
    int ca[K], cb[K];
    load_bwd(0, ua, ia, va, ca);
    for (int j0 = 0; j0 < nmax - 1; j0 += 2 * K) {
      if (j0 + K < nmax - 1) load_bwd(j0 + K, ub, ib, vb, cb);
      step_bwd(j0, ua, ia, va, ca);
      if (j0 + K >= nmax - 1) break;
      if (j0 + 2 * K < nmax - 1) load_bwd(j0 + 2 * K, ua, ia, va, ca);
      step_bwd(j0 + K, ub, ib, vb, cb);
    }
  }
}

template <typename BT, int B>
void line_relax(const Mesh& m, State& st, const Lines& L, int sweeps, cudaStream_t s) {
  const int lb = (L.nlines + LW - 1) / LW;
  if (L.nlines) k_lfactor<BT, B><<<lb, 32 * LW, 0, s>>>(m, st, L);
  for (int it = 0; it < sweeps; it++) {
    BT* xin = (BT*)((it % 2 == 0) ? st.x1 : st.x0);
    BT* xout = (BT*)((it % 2 == 0) ? st.x0 : st.x1);
    k_lrelax_rhs<BT, B><<<m.nslices, B * SLICE, 0, s>>>(m, st, L, xin, xout, it == 0);
    if (L.nlines) k_lsolve<BT, B><<<(L.nlines + LW * LPW - 1) / (LW * LPW), 32 * LW, 0, s>>>(m, L, xout);
  }
}

}  // namespace

void launch_line_relax(const Mesh& m, const Params& p, State& st, const Lines& L, int bs, int sweeps,
                       cudaStream_t s) {
  sweeps = sweeps < 1 ? 1 : sweeps;
  switch (bs) {
    case 5: p.fp32 ? line_relax<float, 5>(m, st, L, sweeps, s) : line_relax<double, 5>(m, st, L, sweeps, s); break;
    case 6: p.fp32 ? line_relax<float, 6>(m, st, L, sweeps, s) : line_relax<double, 6>(m, st, L, sweeps, s); break;
    default: p.fp32 ? line_relax<float, 7>(m, st, L, sweeps, s) : line_relax<double, 7>(m, st, L, sweeps, s); break;
  }
}

}  // namespace jg
