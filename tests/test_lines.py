"""Lines of the line solvers, on the CPU (oracle).

BCGSTAB_LINELET uses the reference's initializeLinelet rule unchanged
(pinned against the reference by the golden fixtures); on a mixed mesh its
lines stop at the last prism row, because the hexahedron above has two
candidate neighbours below it (the quad's two prisms).  The LINE
relaxation's rule goes on to the strongest candidate when it is 1.1 times
the next, so its lines run from the wall through the prism rows into the
stretched hexahedra and stop only where the cells turn isotropic."""
import dataclasses

import numpy as np

from myjoe_b200 import case
from oracle.oracle import Oracle


def _oracle(n_prism):
    _, g, prm = case.sa_bump_case(48, 40, 2, stretch=1.1, n_prism=n_prism, bump_h=0.05, alternate=True, seed=1)
    return g, Oracle(g, dataclasses.replace(prm, TURB_MODEL="NONE", scalar_bcs={}))


def test_reference_lines_stop_at_the_prism_rows():
    g, o = _oracle(8)
    off, cv = o.linelets()
    assert np.diff(off).max() <= 8 + 1


def test_relaxed_lines_cross_into_the_hexahedra():
    g, o = _oracle(8)
    off, cv = o.relax_lines()
    L = np.diff(off)
    assert L.max() > 20 and (off[-1] / g.ncv) > 0.6
    # every cell on at most one line, consecutive cells of a line are neighbours
    assert len(np.unique(cv)) == len(cv)
    nb = {c: set(g.nbocv_v[g.nbocv_i[c] + 1:g.nbocv_i[c + 1]]) for c in range(g.ncv)}
    for l in range(len(L)):
        seg = cv[off[l]:off[l + 1]]
        assert all(b in nb[a] for a, b in zip(seg[:-1], seg[1:]))


def test_relaxed_lines_extend_the_reference_lines_on_hexahedra():
    """On a hex mesh every line of the reference rule is the start of the
    relaxed line from the same wall cell; the relaxed rule only goes on a
    little further where the cells approach isotropy."""
    g, o = _oracle(0)
    (ao, ac), (bo, bc) = o.linelets(), o.relax_lines()
    assert len(ao) == len(bo)
    for l in range(len(ao) - 1):
        ref, rel = ac[ao[l]:ao[l + 1]], bc[bo[l]:bo[l + 1]]
        assert len(rel) >= len(ref) and np.array_equal(rel[:len(ref)], ref)


def test_rcm_lines_order_makes_each_line_consecutive():
    """JG_RENUMBER_RCM_LINES: the RCM order in which the first cell met of each LINE
    relaxation line (two or more cells) brings in the whole line, in line order from its
    wall cell; the lines are those of the relaxed rule on the caller's mesh (the oracle's)."""
    from myjoe_b200 import solver
    _, g, prm = case.sa_bump_case(48, 40, 2, stretch=1.1, n_prism=8, bump_h=0.05, alternate=True,
                                  shuffle=True, seed=3)
    o = Oracle(g, dataclasses.replace(prm, TURB_MODEL="NONE", scalar_bcs={}))
    off, cv = o.relax_lines()
    rcm = solver.renumber_cells(g, prm, solver.RENUMBER_RCM)
    got = solver.renumber_cells(g, prm, solver.RENUMBER_RCM_LINES)
    assert np.array_equal(np.sort(got), np.arange(g.ncv))
    line_of = np.full(g.ncv, -1)
    for l in range(len(off) - 1):
        if off[l + 1] - off[l] >= 2:
            line_of[cv[off[l]:off[l + 1]]] = l
    want, placed = [], np.zeros(g.ncv, bool)
    for c in rcm:
        if placed[c]:
            continue
        seg = [c] if line_of[c] < 0 else list(cv[off[line_of[c]]:off[line_of[c] + 1]])
        want += seg
        placed[seg] = True
    np.testing.assert_array_equal(got, np.array(want))
    pos = np.empty(g.ncv, int)
    pos[got] = np.arange(g.ncv)
    for l in range(len(off) - 1):
        seg = pos[cv[off[l]:off[l + 1]]]
        assert np.all(np.diff(seg) == 1)
    assert (line_of >= 0).mean() > 0.6
