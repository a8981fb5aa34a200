"""Control-volume geometry and connectivity in the reference's layout.

Turns a ``meshgen.RawMesh`` into the arrays the reference's ``UgpWithCv``
holds after ``init()``: boundary-first face order grouped by zone, ``faocv``,
``nbocv`` (CSR, diagonal first), face centroids/normals, cell centroids and
volumes, and the inverse-distance-squared least-squares gradient
coefficients.  Each function names the reference routine whose arithmetic
it restates:

* ``calc_geometry``  -- ``UgpWithCv::calcGeometry`` (src/common/UgpWithCv.cpp:842-1091)
* ``build_faocv``    -- ``Ugp::buildFaocv``          (src/common/Ugp.cpp:5452-5505)
* ``build_nbocv``    -- ``UgpWithCv::buildNbocv``    (src/common/UgpWithCv.cpp:768-834)
* ``calc_lsg_coeff`` -- ``UgpWithCv::calcLsgCoeff``  (src/common/UgpWithCv.cpp:1783-1913)

This is host-side case setup (the reference's mesh layer), not part of the
GPU hot path; the GPU library receives these arrays through ``jg_create``.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .meshgen import RawMesh


@dataclasses.dataclass
class CvMesh:
    ncv: int
    nfa: int
    nfa_b: int
    cvofa: np.ndarray            # [nfa,2] int32
    fa_nodes: np.ndarray         # [nfa,4] node ids (-1 padded)
    fa_nno: np.ndarray           # [nfa]
    x_no: np.ndarray             # [nno,3]
    faocv_i: np.ndarray          # [ncv+1] int32
    faocv_v: np.ndarray          # [faocv_s] int32
    nbocv_i: np.ndarray          # [ncv+1] int32
    nbocv_v: np.ndarray          # [nbocv_s] int32
    x_fa: np.ndarray             # [nfa,3]
    fa_normal: np.ndarray        # [nfa,3] area-weighted, points from cvofa[f,0] to cvofa[f,1]
    x_cv: np.ndarray             # [ncv,3]
    cv_volume: np.ndarray        # [ncv]
    nbocv_lsg_coeff: np.ndarray  # [nbocv_s,3]
    boundary_fa_lsg_coeff: np.ndarray  # [nfa_b,3]
    zones: list                  # [(name, ifa_f, ifa_l)] boundary zones in face order

    @property
    def nbocv_s(self) -> int:
        return int(self.nbocv_v.shape[0])


def order_faces(mesh: RawMesh, seed: int | None = None, shuffle: bool = False):
    """Boundary faces first, grouped by zone, then internal faces (the
    reference's face order after ``Ugp::init``).  With ``shuffle`` the cells
    and the faces inside each group are permuted from ``seed``."""
    rng = np.random.default_rng(seed)
    cell_perm = np.arange(mesh.ncv)
    if shuffle:
        cell_perm = rng.permutation(mesh.ncv)   # new id of old cell i
    order, zones = [], []
    pos = 0
    for name, fids in mesh.zones:
        f = np.asarray(fids)
        if shuffle:
            f = f[rng.permutation(len(f))]
        order.append(f)
        zones.append((name, pos, pos + len(f) - 1))
        pos += len(f)
    nfa_b = pos
    internal = np.nonzero(mesh.cvofa[:, 1] >= 0)[0]
    if shuffle:
        internal = internal[rng.permutation(len(internal))]
    order.append(internal)
    order = np.concatenate(order)
    cvofa = mesh.cvofa[order].copy()
    valid = cvofa >= 0
    cvofa[valid] = cell_perm[cvofa[valid]]
    return order, cvofa, nfa_b, zones


def build_faocv(cvofa: np.ndarray, ncv: int):
    """Faces of each cell in increasing face index (``Ugp::buildFaocv``)."""
    nfa = cvofa.shape[0]
    f = np.repeat(np.arange(nfa), 2)
    c = cvofa.reshape(-1)
    keep = c >= 0
    f, c = f[keep], c[keep]
    idx = np.argsort(c, kind="stable")
    faocv_v = f[idx].astype(np.int32)
    counts = np.bincount(c, minlength=ncv)
    faocv_i = np.zeros(ncv + 1, np.int32)
    faocv_i[1:] = np.cumsum(counts)
    return faocv_i, faocv_v


def build_nbocv(cvofa: np.ndarray, ncv: int, nfa_b: int):
    """CSR cell neighbours, diagonal first, neighbours in internal-face order
    (``UgpWithCv::buildNbocv``)."""
    c0 = cvofa[nfa_b:, 0]
    c1 = cvofa[nfa_b:, 1]
    rows = np.stack([c0, c1], 1).reshape(-1)
    cols = np.stack([c1, c0], 1).reshape(-1)
    # the diagonal goes first: give it a sort key ahead of every face entry
    rows = np.concatenate([np.arange(ncv), rows])
    cols = np.concatenate([np.arange(ncv), cols])
    idx = np.argsort(rows, kind="stable")
    nbocv_v = cols[idx].astype(np.int32)
    counts = np.bincount(rows, minlength=ncv)
    nbocv_i = np.zeros(ncv + 1, np.int32)
    nbocv_i[1:] = np.cumsum(counts)
    return nbocv_i, nbocv_v


def _cross(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1],
                     a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1)


def calc_face_geometry(x_no, fa_nodes, fa_nno):
    """Face normal (area-weighted) and centroid, ``UgpWithCv::calcGeometry``
    first half: normal from the node-average centre, then the fixed-point
    centroid iteration until d2/area < 1e-15."""
    nfa = fa_nodes.shape[0]
    maxn = fa_nodes.shape[1]
    xf = np.zeros((nfa, 3))
    for e in range(maxn):
        m = e < fa_nno
        xf[m] += x_no[fa_nodes[m, e]]
    xf /= fa_nno[:, None]

    def edges():
        # edge e joins node (e-1 mod n) -> node e, starting with (last, first)
        for e in range(maxn):
            m = e < fa_nno
            prev = np.where(e == 0, fa_nno - 1, e - 1)
            i1 = fa_nodes[np.arange(nfa), prev]
            i2 = fa_nodes[:, e]
            yield m, i1, i2

    normal = np.zeros((nfa, 3))
    for m, i1, i2 in edges():
        v1 = x_no[i1[m]] - xf[m]
        v2 = x_no[i2[m]] - xf[m]
        normal[m] += 0.5 * _cross(v1, v2)
    area = np.sqrt((normal ** 2).sum(1))
    un = normal / area[:, None]

    active = np.ones(nfa, bool)
    for it in range(200):
        if not active.any():
            break
        a = np.nonzero(active)[0]
        xtmp = np.zeros((a.size, 3))
        dx = np.zeros((a.size, 3))
        asum = np.zeros(a.size)
        for m, i1, i2 in edges():
            mm = m[a]
            sel = a[mm]
            v1 = x_no[i1[sel]] - xf[sel]
            v2 = x_no[i2[sel]] - xf[sel]
            tn = _cross(v1, v2)
            ta = (tn * un[sel]).sum(1)
            xtmp[mm] += ta[:, None] * (x_no[i1[sel]] + x_no[i2[sel]] + xf[sel])
            dx[mm] += ta[:, None] * (v1 + v2)
            asum[mm] += ta
        xtmp /= 3.0 * asum[:, None]
        dx /= 2.0 * asum[:, None]
        d2 = (dx ** 2).sum(1)
        xf[a] = xtmp
        active[a[d2 / asum < 1.0e-15]] = False
    else:
        raise RuntimeError("face centroid did not converge")
    return xf, normal


def calc_cv_geometry(x_no, fa_nodes, fa_nno, cvofa, x_fa, faocv_i, faocv_v, ncv):
    """Cell centroid and volume from the sub-tetrahedra (face edge, face
    centroid, approximate cell centre), ``UgpWithCv::calcGeometry`` second half."""
    counts = np.diff(faocv_i)
    cell_of = np.repeat(np.arange(ncv), counts)
    fa = faocv_v
    xca = np.zeros((ncv, 3))
    np.add.at(xca, cell_of, x_fa[fa])
    xca /= counts[:, None]
    vol = np.zeros(ncv)
    xcv = np.zeros((ncv, 3))
    outward = cvofa[fa, 0] == cell_of
    nno = fa_nno[fa]
    maxn = fa_nodes.shape[1]
    v1 = x_fa[fa] - xca[cell_of]
    for e in range(maxn):
        m = e < nno
        n = nno
        # forward: (e-1 -> e); backward (face seen from cell 1): node order reversed
        prev_f = np.where(e == 0, n - 1, e - 1)
        fwd1 = fa_nodes[fa, prev_f]
        fwd2 = fa_nodes[fa, np.minimum(e, maxn - 1)]
        # backward loop: ino2 starts at node 0, then nof = n-1 .. 0
        # edge e (0-based): ino1 = node (n-e) mod n, ino2 = node (n-1-e)
        b1 = fa_nodes[fa, np.where(e == 0, 0, n - e)]
        b2 = fa_nodes[fa, np.clip(n - 1 - e, 0, maxn - 1)]
        i1 = np.where(outward, fwd1, b1)
        i2 = np.where(outward, fwd2, b2)
        sel = np.nonzero(m)[0]
        x1 = x_no[i1[sel]]
        x2 = x_no[i2[sel]]
        c = cell_of[sel]
        v2 = x1 - xca[c]
        v3 = x2 - xca[c]
        tv = (v1[sel] * _cross(v2, v3)).sum(1)
        np.add.at(vol, c, tv)
        np.add.at(xcv, c, tv[:, None] * (xca[c] + x_fa[fa[sel]] + x1 + x2))
    xcv /= 4.0 * vol[:, None]
    vol /= 6.0
    return xcv, vol


def calc_lsg_coeff(x_cv, x_fa, cvofa, nbocv_i, nbocv_v, faocv_i, faocv_v, nfa_b, ncv):
    """Inverse-distance-squared weighted least-squares gradient coefficients
    (``UgpWithCv::calcLsgCoeff``).  Boundary faces enter as Dirichlet points
    at their centroids."""
    nbocv_s = nbocv_v.shape[0]
    row = np.repeat(np.arange(ncv), np.diff(nbocv_i))
    off = np.ones(nbocv_s, bool)
    off[nbocv_i[:-1]] = False
    dxn = x_cv[nbocv_v[off]] - x_cv[row[off]]
    wn = 1.0 / (dxn ** 2).sum(1)
    bf = np.arange(nfa_b)
    bc = cvofa[bf, 0]
    dxb = x_fa[bf] - x_cv[bc]
    wb = 1.0 / (dxb ** 2).sum(1)

    def acc(vals, rows):
        out = np.zeros(ncv)
        np.add.at(out, rows, vals)
        return out

    rn = row[off]
    sxx = acc(wn * dxn[:, 0] ** 2, rn) + acc(wb * dxb[:, 0] ** 2, bc)
    syy = acc(wn * dxn[:, 1] ** 2, rn) + acc(wb * dxb[:, 1] ** 2, bc)
    szz = acc(wn * dxn[:, 2] ** 2, rn) + acc(wb * dxb[:, 2] ** 2, bc)
    sxy = acc(wn * dxn[:, 0] * dxn[:, 1], rn) + acc(wb * dxb[:, 0] * dxb[:, 1], bc)
    sxz = acc(wn * dxn[:, 0] * dxn[:, 2], rn) + acc(wb * dxb[:, 0] * dxb[:, 2], bc)
    syz = acc(wn * dxn[:, 1] * dxn[:, 2], rn) + acc(wb * dxb[:, 1] * dxb[:, 2], bc)
    denom = 2.0 * sxy * sxz * syz + sxx * syy * szz - sxx * syz * syz - syy * sxz * sxz - szz * sxy * sxy

    def coeff(dx, w, c):
        d = denom[c]
        c0 = w * ((syy[c] * szz[c] - syz[c] ** 2) * dx[:, 0] + (sxz[c] * syz[c] - sxy[c] * szz[c]) * dx[:, 1]
                  + (sxy[c] * syz[c] - sxz[c] * syy[c]) * dx[:, 2]) / d
        c1 = w * ((sxz[c] * syz[c] - sxy[c] * szz[c]) * dx[:, 0] + (sxx[c] * szz[c] - sxz[c] ** 2) * dx[:, 1]
                  + (sxy[c] * sxz[c] - syz[c] * sxx[c]) * dx[:, 2]) / d
        c2 = w * ((sxy[c] * syz[c] - sxz[c] * syy[c]) * dx[:, 0] + (sxy[c] * sxz[c] - syz[c] * sxx[c]) * dx[:, 1]
                  + (sxx[c] * syy[c] - sxy[c] ** 2) * dx[:, 2]) / d
        return np.stack([c0, c1, c2], 1)

    nb = np.zeros((nbocv_s, 3))
    nb[off] = coeff(dxn, wn, rn)
    bcoef = coeff(dxb, wb, bc)
    diag = np.zeros((ncv, 3))
    for i in range(3):
        diag[:, i] = -acc(nb[off, i], rn) - acc(bcoef[:, i], bc)
    nb[nbocv_i[:-1]] = diag
    return nb, bcoef


def build_cv_mesh(mesh: RawMesh, seed: int | None = None, shuffle: bool = False) -> CvMesh:
    order, cvofa, nfa_b, zones = order_faces(mesh, seed, shuffle)
    fa_nodes = mesh.fa_nodes[order]
    fa_nno = mesh.fa_nno[order]
    ncv = mesh.ncv
    faocv_i, faocv_v = build_faocv(cvofa, ncv)
    nbocv_i, nbocv_v = build_nbocv(cvofa, ncv, nfa_b)
    x_fa, fa_normal = calc_face_geometry(mesh.x_no, fa_nodes, fa_nno)
    x_cv, vol = calc_cv_geometry(mesh.x_no, fa_nodes, fa_nno, cvofa, x_fa, faocv_i, faocv_v, ncv)
    nb, bcoef = calc_lsg_coeff(x_cv, x_fa, cvofa, nbocv_i, nbocv_v, faocv_i, faocv_v, nfa_b, ncv)
    return CvMesh(ncv=ncv, nfa=len(order), nfa_b=nfa_b, cvofa=cvofa.astype(np.int32),
                  fa_nodes=fa_nodes, fa_nno=fa_nno, x_no=mesh.x_no,
                  faocv_i=faocv_i, faocv_v=faocv_v, nbocv_i=nbocv_i, nbocv_v=nbocv_v,
                  x_fa=x_fa, fa_normal=fa_normal, x_cv=x_cv, cv_volume=vol,
                  nbocv_lsg_coeff=nb, boundary_fa_lsg_coeff=bcoef, zones=zones)
