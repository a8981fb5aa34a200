"""Seeded synthetic meshes for the implicit finite-volume path, plus the Fluent
ASCII ``.msh`` writer the reference's ``MshFilter`` reads.

The meshes are hexahedral channels (a sinusoidal bump on the lower wall, or a
flat plate with a stretched wall-normal spacing).  A mesh is returned as a raw
polyhedral description (nodes, faces with their two cells, boundary zones);
``myjoe_b200.geometry`` turns it into the reference's control-volume arrays.

Face orientation convention (internal): the right-hand normal of a face's node
list points from ``cvofa[f][0]`` into ``cvofa[f][1]`` (outward of cell 0), the
convention of the reference's ``Ugp`` after ``MshFilter`` has read the file.
Fluent files store the opposite orientation (the right-hand normal points into
cell 0), so the writer reverses each node list (reference reader:
``src/common/MshFilter.cpp:455-472`` reverses it back).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class RawMesh:
    """Polyhedral mesh before the control-volume geometry is computed."""

    x_no: np.ndarray          # [nno, 3] node coordinates
    fa_nodes: np.ndarray      # [nfa, 4] node ids, -1 padded (triangles)
    fa_nno: np.ndarray        # [nfa] nodes per face (3 or 4)
    cvofa: np.ndarray         # [nfa, 2] cell ids, cvofa[:,1] == -1 on boundaries
    ncv: int
    zones: list               # [(name, face ids ndarray)] boundary zones, in order
    cell_type: int = 4        # Fluent cell type of the (single) cell zone: 4 = hex, 0 = mixed
    cell_types: np.ndarray | None = None   # [ncv] per-cell Fluent types of a mixed zone (6 = prism)

    @property
    def nfa(self) -> int:
        return int(self.cvofa.shape[0])


def _node_id(i, j, k, nx, ny):
    return (k * (ny + 1) + j) * (nx + 1) + i


def _cell_id(i, j, k, nx, ny):
    return (k * ny + j) * nx + i


def structured_hex(X: np.ndarray, Y: np.ndarray, z: np.ndarray,
                   zone_of_face) -> RawMesh:
    """Hex mesh from node coordinates X[i,j], Y[i,j] (extruded along z[k]).

    ``zone_of_face(side, i, j, k)`` returns the boundary zone name of the
    boundary face on ``side`` in {"imin","imax","jmin","jmax","kmin","kmax"}
    at the given face indices.
    """
    nx, ny = X.shape[0] - 1, X.shape[1] - 1
    nz = z.shape[0] - 1
    nno = (nx + 1) * (ny + 1) * (nz + 1)
    x_no = np.empty((nno, 3))
    I, J, K = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    nid = _node_id(I, J, K, nx, ny)
    x_no[nid.ravel(), 0] = np.broadcast_to(X[:, :, None], I.shape).ravel()
    x_no[nid.ravel(), 1] = np.broadcast_to(Y[:, :, None], I.shape).ravel()
    x_no[nid.ravel(), 2] = np.broadcast_to(z[None, None, :], I.shape).ravel()

    # vectorised construction per face family
    fam_nodes, fam_c0, fam_c1, fam_zone = [], [], [], []
    # x-faces (normal +x): nodes (i,j,k),(i,j+1,k),(i,j+1,k+1),(i,j,k+1)
    i, j, k = np.meshgrid(np.arange(nx + 1), np.arange(ny), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    nodes = np.stack([_node_id(i, j, k, nx, ny), _node_id(i, j + 1, k, nx, ny),
                      _node_id(i, j + 1, k + 1, nx, ny), _node_id(i, j, k + 1, nx, ny)], 1)
    c_left = np.where(i > 0, _cell_id(i - 1, j, k, nx, ny), -1)
    c_right = np.where(i < nx, _cell_id(np.minimum(i, nx - 1), j, k, nx, ny), -1)
    fam_nodes.append((nodes, c_left, c_right, ("imin", "imax"), (i, j, k), i == 0, i == nx))
    # y-faces (normal +y): (i,j,k),(i,j,k+1),(i+1,j,k+1),(i+1,j,k)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny + 1), np.arange(nz), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    nodes = np.stack([_node_id(i, j, k, nx, ny), _node_id(i, j, k + 1, nx, ny),
                      _node_id(i + 1, j, k + 1, nx, ny), _node_id(i + 1, j, k, nx, ny)], 1)
    c_left = np.where(j > 0, _cell_id(i, j - 1, k, nx, ny), -1)
    c_right = np.where(j < ny, _cell_id(i, np.minimum(j, ny - 1), k, nx, ny), -1)
    fam_nodes.append((nodes, c_left, c_right, ("jmin", "jmax"), (i, j, k), j == 0, j == ny))
    # z-faces (normal +z): (i,j,k),(i+1,j,k),(i+1,j+1,k),(i,j+1,k)
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz + 1), indexing="ij")
    i, j, k = i.ravel(), j.ravel(), k.ravel()
    nodes = np.stack([_node_id(i, j, k, nx, ny), _node_id(i + 1, j, k, nx, ny),
                      _node_id(i + 1, j + 1, k, nx, ny), _node_id(i, j + 1, k, nx, ny)], 1)
    c_left = np.where(k > 0, _cell_id(i, j, k - 1, nx, ny), -1)
    c_right = np.where(k < nz, _cell_id(i, j, np.minimum(k, nz - 1), nx, ny), -1)
    fam_nodes.append((nodes, c_left, c_right, ("kmin", "kmax"), (i, j, k), k == 0, k == nz))

    all_nodes, all_cv, zone_names = [], [], []
    for nodes, cl, cr, sides, (fi, fj, fk), at_min, at_max in fam_nodes:
        internal = ~(at_min | at_max)
        # internal faces: c0 = left, c1 = right, normal left->right as built
        all_nodes.append(nodes[internal])
        all_cv.append(np.stack([cl[internal], cr[internal]], 1))
        zone_names.extend([None] * int(internal.sum()))
        # min side: the only cell is "right"; outward normal is -axis -> reverse nodes
        idx = np.nonzero(at_min)[0]
        all_nodes.append(nodes[idx][:, ::-1])
        all_cv.append(np.stack([cr[idx], np.full(idx.size, -1)], 1))
        zone_names.extend(zone_of_face(sides[0], fi[idx], fj[idx], fk[idx]))
        # max side: the only cell is "left"; outward normal is +axis
        idx = np.nonzero(at_max)[0]
        all_nodes.append(nodes[idx])
        all_cv.append(np.stack([cl[idx], np.full(idx.size, -1)], 1))
        zone_names.extend(zone_of_face(sides[1], fi[idx], fj[idx], fk[idx]))

    fa_nodes = np.concatenate(all_nodes).astype(np.int64)
    cvofa = np.concatenate(all_cv).astype(np.int64)
    zone_names = np.array([z if z is not None else "" for z in zone_names], dtype=object)
    zones = []
    seen = []
    for z in zone_names:
        if z and z not in seen:
            seen.append(z)
    for z in seen:
        zones.append((z, np.nonzero(zone_names == z)[0]))
    return RawMesh(x_no=x_no, fa_nodes=fa_nodes, fa_nno=np.full(len(fa_nodes), 4, np.int64),
                   cvofa=cvofa, ncv=nx * ny * nz, zones=zones)


def channel_bump(nx=64, ny=32, nz=4, length=3.0, height=1.0, bump_h=0.1,
                 bump_x0=1.0, bump_x1=2.0, depth=None, jitter=0.0, seed=0, stretch=1.0) -> RawMesh:
    """Channel of length ``length`` and height ``height`` with the lower-wall
    bump y_b(x) = bump_h * sin^2(pi (x - x0) / (x1 - x0)) on [x0, x1].

    Zones: ``inlet`` (x=0), ``outlet`` (x=L), ``lower`` (bump wall),
    ``upper`` (top), ``sides`` (the two z planes).  ``jitter`` (fraction of
    the local spacing, seeded) moves interior nodes in x/y to make the mesh
    non-orthogonal.  ``stretch`` > 1 grows the row heights geometrically away
    from the lower wall by that ratio.
    """
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, length, nx + 1)
    if stretch != 1.0:
        h = stretch ** np.arange(ny)
        eta = np.concatenate([[0.0], np.cumsum(h)]) / h.sum()
    else:
        eta = np.linspace(0.0, 1.0, ny + 1)
    yb = np.where((xs >= bump_x0) & (xs <= bump_x1),
                  bump_h * np.sin(math.pi * (xs - bump_x0) / (bump_x1 - bump_x0)) ** 2, 0.0)
    X = np.repeat(xs[:, None], ny + 1, 1)
    Y = yb[:, None] + (height - yb[:, None]) * eta[None, :]
    if jitter > 0.0:
        dx = length / nx
        dy = height / ny
        X[1:-1, 1:-1] += jitter * dx * rng.uniform(-1, 1, size=(nx - 1, ny - 1))
        Y[1:-1, 1:-1] += jitter * dy * rng.uniform(-1, 1, size=(nx - 1, ny - 1))
    if depth is None:
        depth = nz * length / nx
    z = np.linspace(0.0, depth, nz + 1)

    def zone(side, i, j, k):
        name = {"imin": "inlet", "imax": "outlet", "jmin": "lower", "jmax": "upper",
                "kmin": "sides", "kmax": "sides"}[side]
        return [name] * len(i)

    return structured_hex(X, Y, z, zone)


def flat_plate(nx=256, ny=96, nz=2, plate_length=1.0, lead=0.25, stretch=1.1,
               first_dy=None, re_l=1.0e5, depth=None) -> RawMesh:
    """Flat plate on y=0 for x in [0, plate_length], preceded by a symmetry
    plane on [-lead, 0].  Wall-normal spacing grows geometrically by
    ``stretch`` from ``first_dy`` (default: y+ ~ 0.5 at the trailing edge from
    the Blasius skin friction at ``re_l``).

    Zones: ``inlet``, ``outlet``, ``lower_sym`` (x<0), ``plate`` (x>=0),
    ``upper``, ``sides``.
    """
    if first_dy is None:
        cf = 0.664 / math.sqrt(re_l)
        first_dy = 0.5 * plate_length / (re_l * math.sqrt(cf / 2.0))
    xs = np.linspace(-lead, plate_length, nx + 1)
    dys = first_dy * stretch ** np.arange(ny)
    ys = np.concatenate([[0.0], np.cumsum(dys)])
    X = np.repeat(xs[:, None], ny + 1, 1)
    Y = np.repeat(ys[None, :], nx + 1, 0)
    if depth is None:
        depth = nz * (plate_length + lead) / nx
    z = np.linspace(0.0, depth, nz + 1)
    xc = 0.5 * (xs[:-1] + xs[1:])

    def zone(side, i, j, k):
        if side == "jmin":
            return ["lower_sym" if xc[ii] < 0.0 else "plate" for ii in i]
        name = {"imin": "inlet", "imax": "outlet", "jmax": "upper",
                "kmin": "sides", "kmax": "sides"}[side]
        return [name] * len(i)

    return structured_hex(X, Y, z, zone)


def write_msh(path: str, mesh: RawMesh) -> None:
    """Write ``mesh`` as Fluent ASCII (hex integers) for the reference reader
    (``src/common/MshFilter.cpp``: sections 2, 10, 12, 13, 45)."""
    nno = mesh.x_no.shape[0]
    nfa = mesh.nfa
    # file face order: interior zone first, then boundary zones
    internal = np.nonzero(mesh.cvofa[:, 1] >= 0)[0]
    groups = [("fluid_faces", 2, internal)]   # Fluent bc type 2 = interior
    for zi, (name, fids) in enumerate(mesh.zones):
        groups.append((name, 3, fids))          # 3 = wall-type boundary (kind is set by Joe.in)
    lines = []
    lines.append('(0 "joe_b200 synthetic mesh")')
    lines.append("(2 3)")
    lines.append("(10 (0 1 %x 0 3))" % nno)
    lines.append("(10 (1 1 %x 1 3)(" % nno)
    lines.extend("%.17e %.17e %.17e" % tuple(p) for p in mesh.x_no)
    lines.append("))")
    lines.append("(12 (0 1 %x 0))" % mesh.ncv)
    if mesh.cell_types is not None:
        # mixed zone: element type 0 followed by one type per cell
        lines.append("(12 (2 1 %x 1 0)(" % mesh.ncv)
        ct = np.asarray(mesh.cell_types)
        lines.extend(" ".join("%x" % int(v) for v in ct[i:i + 16]) for i in range(0, ct.size, 16))
        lines.append("))")
    else:
        lines.append("(12 (2 1 %x 1 %x))" % (mesh.ncv, mesh.cell_type))
    lines.append("(13 (0 1 %x 0))" % nfa)
    start = 1
    zone_ids = []
    for gi, (name, bctype, fids) in enumerate(groups):
        zid = 3 + gi
        zone_ids.append((zid, name, "interior" if bctype == 2 else "wall"))
        end = start + len(fids) - 1
        lines.append("(13 (%x %x %x %x 0)(" % (zid, start, end, bctype))
        fn = mesh.fa_nodes[fids]
        nn = mesh.fa_nno[fids]
        cv = mesh.cvofa[fids]
        for r in range(len(fids)):
            n = int(nn[r])
            # Fluent stores the opposite orientation: reverse the node list
            nodes = fn[r, :n][::-1] + 1
            c0 = int(cv[r, 0]) + 1
            c1 = int(cv[r, 1]) + 1 if cv[r, 1] >= 0 else 0
            lines.append(" ".join("%x" % v for v in ([n] + list(nodes) + [c0, c1])))
        lines.append("))")
        start = end + 1
    lines.append("(45 (2 fluid fluid)())")
    for zid, name, kind in zone_ids:
        lines.append("(45 (%d %s %s)())" % (zid, kind, name))
    with open(path, "w") as f:
        f.write("\n".join(lines))
        f.write("\n")


def channel_bump_mixed(nx=64, ny=32, nz=2, n_prism=8, length=3.0, height=1.0, bump_h=0.1, bump_x0=1.0,
                       bump_x1=2.0, depth=None, jitter=0.0, seed=0, stretch=1.0, alternate=False) -> RawMesh:
    """The channel-bump domain of ``channel_bump`` with a hybrid mesh: the
    wall surface (x-z) is triangulated, each (i, k) quad split along its
    (i, k)-(i+1, k+1) diagonal (with ``alternate``, quads with i + k odd along
    the other one), and extruded wall-normal into ``n_prism`` rows of
    triangular prisms; hexahedra fill the rows above.  The hexahedra
    on the last prism row see two triangles where a hexahedron has its lower
    quad (a 7-faced polyhedron, which the face-based reader takes as it
    takes any cell).  Zones as ``channel_bump``; faces are triangles (the
    prism caps) or quadrilaterals."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, length, nx + 1)
    if stretch != 1.0:
        h = stretch ** np.arange(ny)
        eta = np.concatenate([[0.0], np.cumsum(h)]) / h.sum()
    else:
        eta = np.linspace(0.0, 1.0, ny + 1)
    yb = np.where((xs >= bump_x0) & (xs <= bump_x1),
                  bump_h * np.sin(math.pi * (xs - bump_x0) / (bump_x1 - bump_x0)) ** 2, 0.0)
    X = np.repeat(xs[:, None], ny + 1, 1)
    Y = yb[:, None] + (height - yb[:, None]) * eta[None, :]
    if jitter > 0.0:
        X[1:-1, 1:-1] += jitter * (length / nx) * rng.uniform(-1, 1, size=(nx - 1, ny - 1))
        Y[1:-1, 1:-1] += jitter * (height / ny) * rng.uniform(-1, 1, size=(nx - 1, ny - 1))
    if depth is None:
        depth = nz * length / nx
    zs = np.linspace(0.0, depth, nz + 1)
    npr = int(min(max(n_prism, 0), ny))

    # nodes (i, j, k)
    def nid(i, j, k):
        return (np.asarray(i) * (ny + 1) + j) * (nz + 1) + k

    I3, J3, K3 = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    x_no = np.stack([X[I3, J3], Y[I3, J3], zs[K3]], -1).reshape(-1, 3)

    # cells: prisms A (i,k)(i+1,k)(i+1,k+1) and B (i,k)(i+1,k+1)(i,k+1) of each (i, k) quad in rows j < npr,
    # then hexahedra, row by row
    P = 2 * nx * nz * npr

    def prism(i, j, k, t):
        return ((np.asarray(j) * nx + i) * nz + k) * 2 + t

    def hexa(i, j, k):
        return P + ((np.asarray(j) - npr) * nx + i) * nz + k

    def flip(i, k):
        return ((np.asarray(i) + k) % 2 == 1) if alternate else np.zeros(np.broadcast(i, k).shape, bool)

    def cell(i, j, k, t):
        """cell of row j at quad (i, k); in a prism row the triangle t (0: A, 1: B)"""
        return np.where(np.asarray(j) < npr, prism(i, j, k, t), hexa(i, j, k))

    # the triangle holding each edge of quad (i, k): the k edge is A's, the k+1 edge B's; the i+1 edge
    # is A's and the i edge B's, the other way round on a flipped quad (A' = (i,k) (i+1,k) (i,k+1),
    # B' = (i+1,k) (i+1,k+1) (i,k+1))
    def t_i1(i, k):
        return np.where(flip(i, k), 1, 0)

    def t_i0(i, k):
        return np.where(flip(i, k), 0, 1)

    ncv = P + nx * nz * (ny - npr)
    faces, cv, zone = [], [], []

    def add(nodes, c0, c1, name):
        nodes = np.asarray(nodes).reshape(-1, nodes.shape[-1])
        if nodes.shape[1] == 3:
            nodes = np.concatenate([nodes, -np.ones((nodes.shape[0], 1), np.int64)], 1)
        faces.append(nodes)
        c0 = np.broadcast_to(c0, (nodes.shape[0],)).ravel()
        c1 = np.broadcast_to(c1, (nodes.shape[0],)).ravel()
        cv.append(np.stack([c0, c1], 1))
        zone.extend([name] * nodes.shape[0])

    # y-faces (constant j).  Node order (i,k) (i+1,k) (i+1,k+1) [(i,k+1)] gives the normal -y:
    # c0 is the cell above, c1 the one below; on the upper boundary the order is reversed.
    Ii, Kk = np.meshgrid(np.arange(nx), np.arange(nz), indexing="ij")
    Ii, Kk = Ii.ravel(), Kk.ravel()
    for j in range(ny + 1):
        above = j < ny
        below = j > 0
        if j <= npr and npr > 0:
            fl = flip(Ii, Kk)[:, None]
            ta = np.where(fl, np.stack([nid(Ii, j, Kk), nid(Ii + 1, j, Kk), nid(Ii, j, Kk + 1)], 1),
                          np.stack([nid(Ii, j, Kk), nid(Ii + 1, j, Kk), nid(Ii + 1, j, Kk + 1)], 1))
            tb = np.where(fl, np.stack([nid(Ii + 1, j, Kk), nid(Ii + 1, j, Kk + 1), nid(Ii, j, Kk + 1)], 1),
                          np.stack([nid(Ii, j, Kk), nid(Ii + 1, j, Kk + 1), nid(Ii, j, Kk + 1)], 1))
            for t, tri in ((0, ta), (1, tb)):
                if above and below:
                    add(tri, cell(Ii, j, Kk, t), prism(Ii, j - 1, Kk, t), None)
                elif above:
                    add(tri, cell(Ii, j, Kk, t), -1, "lower")
                else:
                    add(tri[:, ::-1], prism(Ii, j - 1, Kk, t), -1, "upper")
        else:
            q = np.stack([nid(Ii, j, Kk), nid(Ii + 1, j, Kk), nid(Ii + 1, j, Kk + 1), nid(Ii, j, Kk + 1)], 1)
            if above and below:
                add(q, hexa(Ii, j, Kk), hexa(Ii, j - 1, Kk), None)
            elif above:
                add(q, hexa(Ii, j, Kk), -1, "lower")
            else:
                add(q[:, ::-1], hexa(Ii, j - 1, Kk), -1, "upper")
    # x-faces (constant i): order (i,j,k) (i,j+1,k) (i,j+1,k+1) (i,j,k+1) gives +x: c0 left, c1 right.
    # Left of column i is triangle A of quad i-1 (its i+1 edge), right is triangle B of quad i.
    Jj, Kk2 = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    Jj, Kk2 = Jj.ravel(), Kk2.ravel()
    for i in range(nx + 1):
        q = np.stack([nid(i, Jj, Kk2), nid(i, Jj + 1, Kk2), nid(i, Jj + 1, Kk2 + 1), nid(i, Jj, Kk2 + 1)], 1)
        if i == 0:
            add(q[:, ::-1], cell(0, Jj, Kk2, t_i0(0, Kk2)), -1, "inlet")
        elif i == nx:
            add(q, cell(nx - 1, Jj, Kk2, t_i1(nx - 1, Kk2)), -1, "outlet")
        else:
            add(q, cell(i - 1, Jj, Kk2, t_i1(i - 1, Kk2)), cell(i, Jj, Kk2, t_i0(i, Kk2)), None)
    # z-faces (constant k): order (i,j,k) (i+1,j,k) (i+1,j+1,k) (i,j+1,k) gives +z: c0 the cell at k-1
    # (triangle B, its k+1 edge), c1 the cell at k (triangle A, its k edge).
    Ii3, Jj3 = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    Ii3, Jj3 = Ii3.ravel(), Jj3.ravel()
    for k in range(nz + 1):
        q = np.stack([nid(Ii3, Jj3, k), nid(Ii3 + 1, Jj3, k), nid(Ii3 + 1, Jj3 + 1, k), nid(Ii3, Jj3 + 1, k)], 1)
        if k == 0:
            add(q[:, ::-1], cell(Ii3, Jj3, 0, 0), -1, "sides")
        elif k == nz:
            add(q, cell(Ii3, Jj3, nz - 1, 1), -1, "sides")
        else:
            add(q, cell(Ii3, Jj3, k - 1, 1), cell(Ii3, Jj3, k, 0), None)
    # diagonal faces inside the prism quads: (i,j,k) (i+1,j,k+1) (i+1,j+1,k+1) (i,j+1,k) points from A to B;
    # on a flipped quad (i+1,j,k) (i,j,k+1) (i,j+1,k+1) (i+1,j+1,k) points from B' to A'
    if npr:
        Ii4, Jj4, Kk4 = (a.ravel() for a in np.meshgrid(np.arange(nx), np.arange(npr), np.arange(nz), indexing="ij"))
        fl = flip(Ii4, Kk4)
        q = np.where(fl[:, None],
                     np.stack([nid(Ii4 + 1, Jj4, Kk4), nid(Ii4, Jj4, Kk4 + 1), nid(Ii4, Jj4 + 1, Kk4 + 1),
                               nid(Ii4 + 1, Jj4 + 1, Kk4)], 1),
                     np.stack([nid(Ii4, Jj4, Kk4), nid(Ii4 + 1, Jj4, Kk4 + 1), nid(Ii4 + 1, Jj4 + 1, Kk4 + 1),
                               nid(Ii4, Jj4 + 1, Kk4)], 1))
        add(q, prism(Ii4, Jj4, Kk4, np.where(fl, 1, 0)), prism(Ii4, Jj4, Kk4, np.where(fl, 0, 1)), None)
    fa_nodes = np.concatenate(faces).astype(np.int64)
    fa_nno = np.where(fa_nodes[:, 3] >= 0, 4, 3).astype(np.int64)
    cvofa = np.concatenate(cv).astype(np.int64)
    names = np.array([z if z is not None else "" for z in zone], dtype=object)
    zones = [(zname, np.nonzero(names == zname)[0]) for zname in ("inlet", "outlet", "lower", "upper", "sides")]
    cell_types = np.concatenate([np.full(P, 6), np.full(ncv - P, 4)])
    return RawMesh(x_no=x_no, fa_nodes=fa_nodes, fa_nno=fa_nno, cvofa=cvofa, ncv=ncv, zones=zones,
                   cell_type=0 if npr else 4, cell_types=cell_types if npr else None)
