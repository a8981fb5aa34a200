// jg_renumber.cu -- cell and face renumbering of a case for locality on the GPU.
//
// The reference renumbers the cells of its partition with reverse
// Cuthill-McKee when it loads a mesh (Ugp::init -> reorder, src/common/Ugp.cpp:
// 3389-3399) and puts boundary faces first, grouped by zone.  A caller of this
// library may hand over cells and faces in any order (a mesh from another
// tool, or one shuffled on purpose); with jg_params.renumber = JG_RENUMBER_RCM
// the handle renumbers them itself:
//
//  * cells: reverse Cuthill-McKee over the cell graph (neighbours through
//    internal faces), each connected component started from a
//    pseudo-peripheral cell found by repeated breadth-first level structures
//    (the George-Liu procedure), neighbours queued by increasing degree;
//  * boundary faces: stay inside their zone's range, sorted by their cell;
//  * internal faces: sorted by (lower, higher) new cell id.
//
// Every per-cell list keeps its order (the cell's faces in faocv order, its
// neighbours in nbocv order with the diagonal first), only the ids change.
// The arithmetic of every per-cell and per-face operation is therefore the
// same operation on the same operands as without renumbering, so the
// residual, the Jacobian and each relaxation sweep of block Jacobi give
// bit-identical results; what changes is the order of the L1 residual sum and
// the colouring of multicolour Gauss-Seidel.
//
// JG_RENUMBER_RCM_COLOR groups the RCM order by colour, so that each colour
// pass of multicolour Gauss-Seidel reads a contiguous range of slices of the
// implicit matrix instead of every slice with only some lanes active; its
// sweeps are bit-identical to the RCM order's.
//
// JG_RENUMBER_RCM_LINES makes the cells of each LINE relaxation line
// consecutive in the RCM order (a line is placed where RCM meets the first of
// its cells), so that the line kernels stream each line's blocks and the
// off-line neighbours of a line's consecutive cells are the next line's
// consecutive cells.
#include <algorithm>
#include <numeric>
#include <vector>

#include "jg_internal.h"

namespace jg {

void MeshOwned::bind() {
  m.cvofa = cvofa.data();
  m.faocv_i = faocv_i.data();
  m.faocv_v = faocv_v.data();
  m.nbocv_i = nbocv_i.data();
  m.nbocv_v = nbocv_v.data();
  m.x_cv = x_cv.data();
  m.x_fa = x_fa.data();
  m.fa_normal = fa_normal.data();
  m.cv_volume = vol.data();
  m.nbocv_lsg_coeff = lsq.data();
  m.boundary_fa_lsg_coeff = blsq.data();
  m.zones = zones.data();
  m.nzones = (int)zones.size();
}

namespace {

// breadth-first level structure from `root` over the unvisited part of the
// component; returns the cells of the last level and the number of levels
int levels(const std::vector<int>& adj_i, const std::vector<int>& adj_v, int root, std::vector<int>& level,
           std::vector<int>& touched, std::vector<int>& last) {
  for (int c : touched) level[c] = -1;
  touched.clear();
  level[root] = 0;
  touched.push_back(root);
  size_t head = 0;
  int depth = 0;
  while (head < touched.size()) {
    int c = touched[head++];
    depth = std::max(depth, level[c]);
    for (int k = adj_i[c]; k < adj_i[c + 1]; k++) {
      int nb = adj_v[k];
      if (level[nb] < 0) {
        level[nb] = level[c] + 1;
        touched.push_back(nb);
      }
    }
  }
  last.clear();
  for (int c : touched)
    if (level[c] == depth) last.push_back(c);
  return depth + 1;
}

}  // namespace

int rcm_order(const jg_mesh& m, std::vector<int>& cell_old) {
  const int N = m.ncv;
  // cell graph from nbocv (diagonal first, then the neighbours through internal faces)
  std::vector<int> adj_i(N + 1, 0), adj_v;
  adj_v.reserve((size_t)m.nbocv_s);
  for (int c = 0; c < N; c++) {
    for (int k = m.nbocv_i[c]; k < m.nbocv_i[c + 1]; k++) {
      int nb = m.nbocv_v[k];
      if (nb < 0 || nb >= N) return record_error(JG_ERR_ARG, "nbocv_v holds a cell id out of range");
      if (nb != c) adj_v.push_back(nb);
    }
    adj_i[c + 1] = (int)adj_v.size();
  }
  std::vector<int> deg(N);
  for (int c = 0; c < N; c++) deg[c] = adj_i[c + 1] - adj_i[c];
  // seeds in increasing degree (ties: lower id), so each component starts near its boundary
  std::vector<int> seeds(N);
  std::iota(seeds.begin(), seeds.end(), 0);
  std::stable_sort(seeds.begin(), seeds.end(), [&](int a, int b) { return deg[a] < deg[b]; });
  std::vector<char> done(N, 0);
  std::vector<int> level(N, -1), touched, last, order;
  order.reserve(N);
  std::vector<int> nbs;
  for (int seed : seeds) {
    if (done[seed]) continue;
    // pseudo-peripheral root: move to a least-degree cell of the deepest level while the depth grows
    int root = seed;
    int depth = levels(adj_i, adj_v, root, level, touched, last);
    for (int it = 0; it < 8; it++) {
      int cand = last[0];
      for (int c : last)
        if (deg[c] < deg[cand] || (deg[c] == deg[cand] && c < cand)) cand = c;
      int d2 = levels(adj_i, adj_v, cand, level, touched, last);
      if (d2 <= depth) break;
      root = cand;
      depth = d2;
    }
    for (int c : touched) level[c] = -1;
    touched.clear();
    // Cuthill-McKee from the root
    size_t head = order.size();
    order.push_back(root);
    done[root] = 1;
    while (head < order.size()) {
      int c = order[head++];
      nbs.clear();
      for (int k = adj_i[c]; k < adj_i[c + 1]; k++)
        if (!done[adj_v[k]]) {
          done[adj_v[k]] = 1;
          nbs.push_back(adj_v[k]);
        }
      std::stable_sort(nbs.begin(), nbs.end(),
                       [&](int a, int b) { return deg[a] < deg[b] || (deg[a] == deg[b] && a < b); });
      for (int nb : nbs) order.push_back(nb);
    }
  }
  cell_old.assign(order.rbegin(), order.rend());
  return JG_OK;
}

// Cells grouped by colour: the greedy colouring of the cell graph taken in RCM order (what a
// handle computes on the RCM-renumbered mesh), then the cells stably sorted by colour.  A handle
// colours its cells greedily in its own order; in this order that gives back the same colour
// classes (each cell's earlier-coloured neighbours all precede it), so multicolour Gauss-Seidel
// does exactly the sweeps of the RCM order, while each colour's cells are contiguous.
int rcm_color_order(const jg_mesh& m, std::vector<int>& cell_old) {
  int rc = rcm_order(m, cell_old);
  if (rc != JG_OK) return rc;
  const int N = m.ncv;
  std::vector<int> cell_new(N);
  for (int c = 0; c < N; c++) cell_new[cell_old[c]] = c;
  std::vector<std::vector<int>> adj(N);
  for (int f = m.nfa_b; f < m.nfa; f++) {
    const int a = cell_new[m.cvofa[2 * f]], b = cell_new[m.cvofa[2 * f + 1]];
    adj[a].push_back(b);
    adj[b].push_back(a);
  }
  std::vector<int> color(N, 0), mark(256, -1);
  for (int c = 0; c < N; c++) {
    for (int nb : adj[c])
      if (nb < c) mark[color[nb]] = c;
    int k = 0;
    while (k < 255 && mark[k] == c) k++;
    color[c] = k;
  }
  std::vector<int> order(N);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return color[a] < color[b]; });
  std::vector<int> out(N);
  for (int c = 0; c < N; c++) out[c] = cell_old[order[c]];
  cell_old.swap(out);
  return JG_OK;
}

// The RCM order with every line of the LINE relaxation made consecutive: walking the RCM order,
// the first cell met of a line brings in the whole line, in line order from its wall cell.  The
// lines are those a handle builds (the relaxed rule from every WALL zone's faces in the caller's
// order), which depend on the mesh's connectivity and geometry only, not on its cell ids, so a
// handle finds the same lines in the renumbered mesh.
int rcm_lines_order(const jg_mesh& m, std::vector<int>& cell_old) {
  int rc = rcm_order(m, cell_old);
  if (rc != JG_OK) return rc;
  const int N = m.ncv;
  std::vector<std::vector<int>> walls;
  for (int z = 0; z < m.nzones; z++)
    if (m.zones[z].kind == JG_BC_WALL) {
      if (m.zones[z].ifa_f < 0 || m.zones[z].ifa_l >= m.nfa_b)
        return record_error(JG_ERR_ARG, "zone face range outside the boundary faces");
      for (int i = m.zones[z].ifa_f; i <= m.zones[z].ifa_l; i++)
        if (m.cvofa[2 * i] < 0 || m.cvofa[2 * i] >= N) return record_error(JG_ERR_ARG, "a boundary face has a cell id out of range");
      std::vector<int> f;
      for (int i = m.zones[z].ifa_f; i <= m.zones[z].ifa_l; i++) f.push_back(i);
      walls.push_back(std::move(f));
    }
  std::vector<int> off, cv;
  rc = build_lines(m, walls, off, cv, true);
  if (rc != JG_OK) return rc;
  std::vector<int> line_of(N, -1);
  for (size_t l = 0; l + 1 < off.size(); l++)
    if (off[l + 1] - off[l] >= 2)
      for (int k = off[l]; k < off[l + 1]; k++) line_of[cv[k]] = (int)l;
  std::vector<char> placed(N, 0);
  std::vector<int> out;
  out.reserve(N);
  for (int c : cell_old) {
    if (placed[c]) continue;
    const int l = line_of[c];
    if (l < 0) {
      out.push_back(c);
      placed[c] = 1;
      continue;
    }
    for (int k = off[l]; k < off[l + 1]; k++) {
      out.push_back(cv[k]);
      placed[cv[k]] = 1;
    }
  }
  cell_old.swap(out);
  return JG_OK;
}

int cell_order(const jg_mesh& m, int method, std::vector<int>& cell_old) {
  switch (method) {
    case JG_RENUMBER_RCM: return rcm_order(m, cell_old);
    case JG_RENUMBER_RCM_COLOR: return rcm_color_order(m, cell_old);
    case JG_RENUMBER_RCM_LINES: return rcm_lines_order(m, cell_old);
    default: return record_error(JG_ERR_ARG, "unknown renumbering method");
  }
}

int renumber_mesh(const jg_mesh& in, int method, MeshOwned& o, Renumbering& r) {
  const int N = in.ncv, nfa = in.nfa, nfa_b = in.nfa_b, nbs = in.nbocv_s;
  if (method != JG_RENUMBER_RCM && method != JG_RENUMBER_RCM_COLOR && method != JG_RENUMBER_RCM_LINES)
    return record_error(JG_ERR_ARG, "unknown renumbering method");
  for (int f = nfa_b; f < nfa; f++) {
    int c0 = in.cvofa[2 * f], c1 = in.cvofa[2 * f + 1];
    if (c0 < 0 || c0 >= N || c1 < 0 || c1 >= N) return record_error(JG_ERR_ARG, "an internal face has a cell id out of range");
  }
  int rc = cell_order(in, method, r.cell_old);
  if (rc != JG_OK) return rc;
  std::vector<int> cell_new(N);
  for (int c = 0; c < N; c++) cell_new[r.cell_old[c]] = c;
  // faces: boundary faces by zone range, then by their (new) cell; internal by (lower, higher) new cell
  r.face_old.resize(nfa);
  std::iota(r.face_old.begin(), r.face_old.end(), 0);
  auto owner = [&](int f) { return cell_new[in.cvofa[2 * f]]; };
  for (int z = 0; z < in.nzones; z++) {
    int f0 = in.zones[z].ifa_f, f1 = in.zones[z].ifa_l + 1;
    if (f0 < 0 || f1 > nfa_b || f0 > f1) return record_error(JG_ERR_ARG, "zone face range outside the boundary faces");
    std::stable_sort(r.face_old.begin() + f0, r.face_old.begin() + f1,
                     [&](int a, int b) { return owner(a) < owner(b); });
  }
  for (int f = nfa_b; f < nfa; f++) {
    int c1 = in.cvofa[2 * f + 1];
    if (c1 < 0 || c1 >= N || in.cvofa[2 * f] < 0 || in.cvofa[2 * f] >= N)
      return record_error(JG_ERR_ARG, "an internal face has a cell id out of range");
  }
  auto lo = [&](int f) { return std::min(cell_new[in.cvofa[2 * f]], cell_new[in.cvofa[2 * f + 1]]); };
  auto hi = [&](int f) { return std::max(cell_new[in.cvofa[2 * f]], cell_new[in.cvofa[2 * f + 1]]); };
  std::stable_sort(r.face_old.begin() + nfa_b, r.face_old.end(), [&](int a, int b) {
    int la = lo(a), lb = lo(b);
    return la < lb || (la == lb && hi(a) < hi(b));
  });
  std::vector<int> face_new(nfa);
  for (int f = 0; f < nfa; f++) face_new[r.face_old[f]] = f;
  // faces: orientation kept (c0 stays c0)
  o.cvofa.assign(2 * (size_t)nfa, -1);
  o.x_fa.resize(3 * (size_t)nfa);
  o.fa_normal.resize(3 * (size_t)nfa);
  o.blsq.resize(3 * (size_t)nfa_b);
  for (int f = 0; f < nfa; f++) {
    int g = r.face_old[f];
    o.cvofa[2 * f] = cell_new[in.cvofa[2 * g]];
    o.cvofa[2 * f + 1] = in.cvofa[2 * g + 1] >= 0 ? cell_new[in.cvofa[2 * g + 1]] : -1;
    for (int i = 0; i < 3; i++) {
      o.x_fa[3 * f + i] = in.x_fa[3 * g + i];
      o.fa_normal[3 * f + i] = in.fa_normal[3 * g + i];
    }
    if (f < nfa_b)
      for (int i = 0; i < 3; i++) o.blsq[3 * f + i] = in.boundary_fa_lsg_coeff[3 * g + i];
  }
  // cells: each row keeps its order, ids mapped
  o.x_cv.resize(3 * (size_t)N);
  o.vol.resize(N);
  o.faocv_i.assign(N + 1, 0);
  o.nbocv_i.assign(N + 1, 0);
  o.faocv_v.clear();
  o.nbocv_v.clear();
  o.lsq.clear();
  o.faocv_v.reserve(in.faocv_i[N]);
  o.nbocv_v.reserve(nbs);
  o.lsq.reserve(3 * (size_t)nbs);
  r.nbs_old.clear();
  r.nbs_old.reserve(nbs);
  for (int c = 0; c < N; c++) {
    int g = r.cell_old[c];
    for (int i = 0; i < 3; i++) o.x_cv[3 * c + i] = in.x_cv[3 * g + i];
    o.vol[c] = in.cv_volume[g];
    for (int k = in.faocv_i[g]; k < in.faocv_i[g + 1]; k++) {
      int f = in.faocv_v[k];
      if (f < 0 || f >= nfa) return record_error(JG_ERR_ARG, "faocv_v holds a face id out of range");
      o.faocv_v.push_back(face_new[f]);
    }
    o.faocv_i[c + 1] = (int)o.faocv_v.size();
    for (int k = in.nbocv_i[g]; k < in.nbocv_i[g + 1]; k++) {
      o.nbocv_v.push_back(cell_new[in.nbocv_v[k]]);
      for (int i = 0; i < 3; i++) o.lsq.push_back(in.nbocv_lsg_coeff[3 * k + i]);
      r.nbs_old.push_back(k);
    }
    o.nbocv_i[c + 1] = (int)o.nbocv_v.size();
  }
  o.zones.assign(in.zones, in.zones + in.nzones);
  o.m = in;
  o.m.nbocv_s = (int)o.nbocv_v.size();
  o.bind();
  return JG_OK;
}

}  // namespace jg

extern "C" int jg_renumber_cells(const jg_mesh* mesh, int method, int* cell_old) {
  if (!mesh || !cell_old) return jg::record_error(JG_ERR_ARG, "null argument");
  if (method != JG_RENUMBER_RCM && method != JG_RENUMBER_RCM_COLOR && method != JG_RENUMBER_RCM_LINES)
    return jg::record_error(JG_ERR_ARG, "unknown renumbering method");
  if (mesh->ncv <= 0 || mesh->nbocv_s < mesh->ncv) return jg::record_error(JG_ERR_ARG, "inconsistent mesh sizes");
  for (int f = mesh->nfa_b; f < mesh->nfa; f++) {
    int c0 = mesh->cvofa[2 * f], c1 = mesh->cvofa[2 * f + 1];
    if (c0 < 0 || c0 >= mesh->ncv || c1 < 0 || c1 >= mesh->ncv)
      return jg::record_error(JG_ERR_ARG, "an internal face has a cell id out of range");
  }
  std::vector<int> order;
  int rc = jg::cell_order(*mesh, method, order);
  if (rc != JG_OK) return rc;
  std::copy(order.begin(), order.end(), cell_old);
  return JG_OK;
}
