"""Mixed prism/hex meshes and the library's cell renumbering, on the CPU.

``meshgen.channel_bump_mixed`` must give closed cells (the outward face
normals of every cell sum to zero) filling the same volume as the hex mesh of
the same domain, and write a mixed cell zone (element type 0 with one type per
cell) for the reference reader.  ``jg_renumber_cells`` (host-only entry point
of the C ABI; the order a handle uses with renumber = JG_RENUMBER_RCM) must
return a permutation whose matrix bandwidth is that of a reverse
Cuthill-McKee order: no wider than scipy's reverse_cuthill_mckee on the same
graph, from the generator's order and from a shuffled one.
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp
from scipy.sparse.csgraph import reverse_cuthill_mckee

from myjoe_b200 import case, geometry, meshgen, solver


def _bandwidth(g, new_of_old):
    fa = g.cvofa[g.nfa_b:]
    return int(np.abs(new_of_old[fa[:, 0]] - new_of_old[fa[:, 1]]).max())


def _inverse(order):
    inv = np.empty_like(order)
    inv[order] = np.arange(order.size)
    return inv


def test_mixed_mesh_cells_are_closed():
    raw = meshgen.channel_bump_mixed(10, 8, 3, n_prism=3, stretch=1.2, jitter=0.1, seed=2)
    g = geometry.build_cv_mesh(raw)
    # triangular faces: the prism caps on the wall and the 3 node rows above it, 2 per (i, k) quad
    assert (raw.fa_nno == 3).sum() == 2 * 10 * 3 * (3 + 1)
    # prisms have 5 faces, hexahedra 6, the hexahedra on the last prism row 7 (two triangles below)
    assert np.bincount(np.diff(g.faocv_i), minlength=8)[5:8].tolist() == [180, 10 * 3 * 4, 10 * 3]
    acc = np.zeros((g.ncv, 3))
    np.add.at(acc, g.cvofa[:, 0], g.fa_normal)
    internal = g.cvofa[:, 1] >= 0
    np.add.at(acc, g.cvofa[internal, 1], -g.fa_normal[internal])
    assert np.abs(acc).max() < 1e-14
    assert g.cv_volume.min() > 0.0
    hexes = geometry.build_cv_mesh(meshgen.channel_bump(10, 8, 3, stretch=1.2, jitter=0.1, seed=2))
    assert abs(g.cv_volume.sum() - hexes.cv_volume.sum()) < 1e-12
    # 3 prism rows of 2 prisms per (i, k) quad, 5 hexahedron rows above
    assert g.ncv == 2 * 10 * 3 * 3 + 10 * 3 * 5
    assert np.count_nonzero(raw.cell_types == 6) == 2 * 10 * 3 * 3


def test_mixed_mesh_file_has_a_mixed_cell_zone(tmp_path):
    raw = meshgen.channel_bump_mixed(6, 4, 2, n_prism=2)
    path = os.path.join(tmp_path, "m.msh")
    meshgen.write_msh(path, raw)
    text = open(path).read()
    head = "(12 (2 1 %x 1 0)(" % raw.ncv
    assert head in text
    body = text.split(head, 1)[1].split("))", 1)[0].split()
    assert len(body) == raw.ncv and set(body) == {"4", "6"}


@pytest.mark.parametrize("shuffle", [False, True])
def test_rcm_order_matches_scipy_bandwidth(shuffle):
    raw = meshgen.channel_bump_mixed(48, 24, 4, n_prism=6, stretch=1.1, jitter=0.1, seed=5)
    g = geometry.build_cv_mesh(raw, seed=9, shuffle=shuffle)
    _, _, prm = case.bump_case(8, 4, 2)
    order = solver.renumber_cells(g, prm)
    assert np.array_equal(np.sort(order), np.arange(g.ncv))
    fa = g.cvofa[g.nfa_b:]
    rows = np.concatenate([fa[:, 0], fa[:, 1]])
    cols = np.concatenate([fa[:, 1], fa[:, 0]])
    A = sp.csr_matrix((np.ones(rows.size), (rows, cols)), shape=(g.ncv, g.ncv))
    ref = reverse_cuthill_mckee(A, symmetric_mode=True)
    ours = _bandwidth(g, _inverse(order))
    assert ours <= _bandwidth(g, _inverse(ref))
    if shuffle:
        assert ours * 20 < _bandwidth(g, np.arange(g.ncv))


def test_rcm_order_handles_disconnected_components():
    # two copies of a mesh side by side in one handle's arrays: each component is ordered on its own
    raw = meshgen.channel_bump_mixed(8, 6, 2, n_prism=2)
    g = geometry.build_cv_mesh(raw)
    _, _, prm = case.bump_case(8, 4, 2)
    order = solver.renumber_cells(g, prm)
    n = g.ncv
    g2 = geometry.CvMesh(**{**g.__dict__})
    g2.nbocv_i = np.concatenate([g.nbocv_i, g.nbocv_i[1:] + g.nbocv_i[-1]]).astype(np.int32)
    g2.nbocv_v = np.concatenate([g.nbocv_v, g.nbocv_v + n]).astype(np.int32)
    g2.ncv = 2 * n
    g2.x_cv = np.concatenate([g.x_cv, g.x_cv])
    g2.cv_volume = np.concatenate([g.cv_volume, g.cv_volume])
    g2.faocv_i = np.concatenate([g.faocv_i, g.faocv_i[1:] + g.faocv_i[-1]]).astype(np.int32)
    g2.faocv_v = np.concatenate([g.faocv_v, g.faocv_v]).astype(np.int32)
    g2.nbocv_lsg_coeff = np.concatenate([g.nbocv_lsg_coeff, g.nbocv_lsg_coeff])
    order2 = solver.renumber_cells(g2, prm)
    assert np.array_equal(np.sort(order2), np.arange(2 * n))
    # no cell of one component between two cells of the other
    comp = order2 >= n
    assert np.count_nonzero(np.diff(comp.astype(int))) == 1
    assert sorted(order.tolist()) == sorted((order2[comp] - n).tolist())


def _greedy_colors(g, cell_old):
    """greedy colouring of the cell graph in the order cell_old (a handle's own colouring)"""
    new = _inverse(cell_old)
    fa = g.cvofa[g.nfa_b:]
    adj = [[] for _ in range(g.ncv)]
    for a, b in fa:
        adj[new[a]].append(new[b])
        adj[new[b]].append(new[a])
    col = np.zeros(g.ncv, int)
    for c in range(g.ncv):
        used = {col[nb] for nb in adj[c] if nb < c}
        k = 0
        while k in used:
            k += 1
        col[c] = k
    return col


def test_rcm_color_order_groups_the_rcm_colour_classes():
    """JG_RENUMBER_RCM_COLOR: the RCM order stably grouped by the greedy colours of
    the RCM order; colouring again in the new order gives the same classes, now
    contiguous (so each Gauss-Seidel colour pass reads a contiguous range)."""
    raw = meshgen.channel_bump_mixed(48, 24, 4, n_prism=6, stretch=1.1, jitter=0.1, seed=5)
    g = geometry.build_cv_mesh(raw, seed=9, shuffle=True)
    _, _, prm = case.bump_case(8, 4, 2)
    rcm = solver.renumber_cells(g, prm, solver.RENUMBER_RCM)
    rc = solver.renumber_cells(g, prm, solver.RENUMBER_RCM_COLOR)
    assert np.array_equal(np.sort(rc), np.arange(g.ncv))
    col_rcm = _greedy_colors(g, rcm)
    col_rc = _greedy_colors(g, rc)
    assert np.all(np.diff(col_rc) >= 0)                       # colours contiguous, in order
    by_cell_rcm = np.empty(g.ncv, int)
    by_cell_rcm[rcm] = col_rcm
    by_cell_rc = np.empty(g.ncv, int)
    by_cell_rc[rc] = col_rc
    np.testing.assert_array_equal(by_cell_rcm, by_cell_rc)    # the same class of every cell
    # inside a colour, the RCM order is kept
    pos_rcm = _inverse(rcm)
    for q in range(col_rc.max() + 1):
        assert np.all(np.diff(pos_rcm[rc[col_rc == q]]) > 0)
