"""The reference's binary restart file through libjoe_b200.so.

``Restart`` wraps a ``jg_restart_t``: the reference's restart format
(``Ugp::writeRestart`` / ``Ugp::readRestart``, src/common/Ugp.cpp:9792-13240)
held in host memory, read and written by the library's C++ code.  With it a
solution moves between the reference and a ``JoeGpu`` handle either way:

* ``Restart.read(path)`` + ``to_raw_mesh()`` give the mesh in the file's
  global order (the reference's ``initializeFromRestartFile`` for a restart,
  UgpWithCv.h:316-347); ``geometry.build_cv_mesh`` of it keeps the file's cell
  order, so ``load_state`` puts the file's RHO / RHOU / RHOE / scalars and
  STEP straight into a handle built on it.
* ``Restart.from_cv_mesh(g)`` lays out a control-volume mesh as the
  reference's writer does with one process (boundary nodes first,
  Ugp.cpp:9929-10010; face zones in face order, then the internal faces as
  one internal zone); ``save_state`` adds the handle's state and ``write``
  gives a file the reference resumes from (``RESTART = <file>``).

Reading a file and writing it back reproduces it byte for byte.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import meshgen
from .solver import _ck, lib

NAME_LEN = 52
I0, D0, FA_D1, NO_D1, NO_D3, CV_D1, CV_D3, CV_D33 = 11, 12, 24, 32, 33, 42, 43, 44
FA_ZONE_BOUNDARY, FA_ZONE_INTERNAL = 1, 6

_bound = False


def _bind():
    global _bound
    if _bound:
        return lib()
    L = lib()
    P, I, D = C.c_void_p, C.c_int, C.POINTER(C.c_double)
    IP = C.POINTER(C.c_int)
    L.jg_restart_new.argtypes = [C.POINTER(P)]
    L.jg_restart_free.argtypes = [P]
    L.jg_restart_read.argtypes = [C.c_char_p, C.POINTER(P)]
    L.jg_restart_write.argtypes = [P, C.c_char_p]
    L.jg_restart_counts.argtypes = [P, IP, IP, IP, IP, IP, IP]
    L.jg_restart_get_mesh.argtypes = [P, D, IP, IP, IP, IP]
    L.jg_restart_get_zone.argtypes = [P, I, C.c_char_p, IP, IP, IP, D]
    L.jg_restart_set_mesh.argtypes = [P, I, I, I, D, IP, IP, IP]
    L.jg_restart_add_zone.argtypes = [P, C.c_char_p, I, I, I, D]
    L.jg_restart_find.argtypes = [P, C.c_char_p, IP]
    L.jg_restart_get_record.argtypes = [P, I, C.c_char_p, IP, IP, IP, D, IP, D]
    L.jg_restart_put_record.argtypes = [P, C.c_char_p, I, D, I, C.c_double]
    L.jg_restart_save_state.argtypes = [P, P]
    L.jg_restart_load_state.argtypes = [P, P]
    L.jg_set_cfl_step.argtypes = [P, C.c_double, I]
    _bound = True
    return L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Restart:
    """One restart file's mesh and data records (see the module docstring)."""

    def __init__(self, handle=None):
        L = _bind()
        if handle is None:
            h = C.c_void_p()
            _ck(L.jg_restart_new(C.byref(h)))
            handle = h
        self._h = handle

    # -- construction -----------------------------------------------------
    @classmethod
    def read(cls, path: str) -> "Restart":
        """``Ugp::readRestart``: the whole file; byte-swapped files are swapped."""
        L = _bind()
        h = C.c_void_p()
        _ck(L.jg_restart_read(str(path).encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_cv_mesh(cls, g, internal_zone: str = "fluid_faces") -> "Restart":
        """A restart holding ``g``'s mesh (cells in ``g``'s order, faces in
        ``g``'s order: its boundary zones, then the internal faces as the zone
        ``internal_zone``), nodes renumbered boundary nodes first."""
        r = cls()
        nno = g.x_no.shape[0]
        on_b = np.zeros(nno, dtype=bool)
        fb = g.fa_nodes[: g.nfa_b]
        on_b[fb[fb >= 0]] = True
        order = np.concatenate([np.nonzero(on_b)[0], np.nonzero(~on_b)[0]])   # file node -> g node
        new_of_old = np.empty(nno, dtype=np.int64)
        new_of_old[order] = np.arange(nno)
        nn = np.asarray(g.fa_nno, dtype=np.int64)
        noofa_i = np.zeros(g.nfa + 1, dtype=np.int32)
        noofa_i[1:] = np.cumsum(nn)
        mask = np.arange(g.fa_nodes.shape[1])[None, :] < nn[:, None]
        noofa_v = new_of_old[g.fa_nodes[mask]].astype(np.int32)
        cvofa = np.ascontiguousarray(g.cvofa, dtype=np.int32)
        x_no = np.ascontiguousarray(g.x_no[order], dtype=np.float64)
        r.set_mesh(x_no, noofa_i, noofa_v, cvofa, g.ncv)
        for name, f0, f1 in g.zones:
            r.add_zone(name, FA_ZONE_BOUNDARY, f0, f1)
        r.add_zone(internal_zone, FA_ZONE_INTERNAL, g.nfa_b, g.nfa - 1)
        r.node_order = order
        return r

    def close(self):
        if self._h:
            lib().jg_restart_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- mesh -------------------------------------------------------------
    def counts(self):
        v = [C.c_int() for _ in range(6)]
        _ck(lib().jg_restart_counts(self._h, *[C.byref(x) for x in v]))
        return dict(zip(("nno", "nfa", "ncv", "noofa_count", "nzones", "nrecords"), (x.value for x in v)))

    def mesh(self):
        """(x_no[nno,3], noofa_i[nfa+1], noofa_v, cvofa[nfa,2], cv_part[ncv]) in file order."""
        n = self.counts()
        x_no = np.zeros((n["nno"], 3))
        noofa_i = np.zeros(n["nfa"] + 1, dtype=np.int32)
        noofa_v = np.zeros(n["noofa_count"], dtype=np.int32)
        cvofa = np.zeros((n["nfa"], 2), dtype=np.int32)
        cv_part = np.zeros(n["ncv"], dtype=np.int32)
        _ck(lib().jg_restart_get_mesh(self._h, _dp(x_no), _ip(noofa_i), _ip(noofa_v), _ip(cvofa), _ip(cv_part)))
        return x_no, noofa_i, noofa_v, cvofa, cv_part

    def zones(self):
        """[(name, kind, ifa_f, ifa_l, periodic[3])] in face order."""
        out = []
        for z in range(self.counts()["nzones"]):
            name = C.create_string_buffer(NAME_LEN)
            kind, f0, f1 = C.c_int(), C.c_int(), C.c_int()
            per = np.zeros(3)
            _ck(lib().jg_restart_get_zone(self._h, z, name, C.byref(kind), C.byref(f0), C.byref(f1), _dp(per)))
            out.append((name.value.decode(), kind.value, f0.value, f1.value, per))
        return out

    def set_mesh(self, x_no, noofa_i, noofa_v, cvofa, ncv):
        x_no = np.ascontiguousarray(x_no, dtype=np.float64)
        noofa_i = np.ascontiguousarray(noofa_i, dtype=np.int32)
        noofa_v = np.ascontiguousarray(noofa_v, dtype=np.int32)
        cvofa = np.ascontiguousarray(cvofa, dtype=np.int32)
        _ck(lib().jg_restart_set_mesh(self._h, x_no.shape[0], cvofa.shape[0], int(ncv), _dp(x_no), _ip(noofa_i),
                                      _ip(noofa_v), _ip(cvofa)))

    def add_zone(self, name, kind, ifa_f, ifa_l, periodic=None):
        per = None if periodic is None else _dp(np.ascontiguousarray(periodic, dtype=np.float64))
        _ck(lib().jg_restart_add_zone(self._h, name.encode(), int(kind), int(ifa_f), int(ifa_l), per))

    def to_raw_mesh(self) -> meshgen.RawMesh:
        """The file's mesh for ``geometry.build_cv_mesh`` (cells and nodes in
        file order, boundary zones in file order).  Faces with more than four
        nodes and periodic zones are refused (ValueError): the mesh builder
        takes triangles and quadrilaterals, the solver no periodic faces."""
        x_no, noofa_i, noofa_v, cvofa, _ = self.mesh()
        nn = np.diff(noofa_i)
        if nn.size and (nn.max() > 4 or nn.min() < 3):
            raise ValueError("faces with %d..%d nodes: only triangles and quadrilaterals are supported"
                             % (nn.min(), nn.max()))
        fa_nodes = -np.ones((cvofa.shape[0], 4), dtype=np.int64)
        mask = np.arange(4)[None, :] < nn[:, None]
        fa_nodes[mask] = noofa_v
        zones = []
        for name, kind, f0, f1, _ in self.zones():
            if kind == FA_ZONE_INTERNAL:
                if np.any(cvofa[f0:f1 + 1, 1] < 0):
                    raise ValueError("internal zone %s holds boundary faces" % name)
                continue
            if kind != FA_ZONE_BOUNDARY:
                raise ValueError("zone %s is periodic (kind %d): not supported" % (name, kind))
            if np.any(cvofa[f0:f1 + 1, 1] != -1):
                raise ValueError("boundary zone %s holds internal faces" % name)
            zones.append((name, np.arange(f0, f1 + 1)))
        return meshgen.RawMesh(x_no=x_no, fa_nodes=fa_nodes, fa_nno=nn.astype(np.int64),
                               cvofa=cvofa.astype(np.int64), ncv=self.counts()["ncv"], zones=zones)

    # -- records ----------------------------------------------------------
    def record_names(self):
        return [self._info(i)[0] for i in range(self.counts()["nrecords"])]

    def _info(self, i):
        name = C.create_string_buffer(NAME_LEN)
        kind, count, width = C.c_int(), C.c_int(), C.c_int()
        _ck(lib().jg_restart_get_record(self._h, i, name, C.byref(kind), C.byref(count), C.byref(width), None, None,
                                        None))
        return name.value.decode(), kind.value, count.value, width.value

    def find(self, name) -> int:
        i = C.c_int()
        _ck(lib().jg_restart_find(self._h, name.encode(), C.byref(i)))
        return i.value

    def get(self, name):
        """(kind, value): an int (I0), a float (D0) or an array [count] / [count, 3] / [count, 3, 3]."""
        i = self.find(name)
        if i < 0:
            raise KeyError(name)
        _, kind, count, width = self._info(i)
        iv, dv = C.c_int(), C.c_double()
        data = np.zeros(count * width)
        _ck(lib().jg_restart_get_record(self._h, i, None, None, None, None, _dp(data) if data.size else None,
                                        C.byref(iv), C.byref(dv)))
        if kind == I0:
            return kind, iv.value
        if kind == D0:
            return kind, dv.value
        shape = {1: (count,), 3: (count, 3), 9: (count, 3, 3)}[width]
        return kind, data.reshape(shape)

    def put(self, name, kind, value):
        if kind == I0:
            _ck(lib().jg_restart_put_record(self._h, name.encode(), kind, None, int(value), 0.0))
        elif kind == D0:
            _ck(lib().jg_restart_put_record(self._h, name.encode(), kind, None, 0, float(value)))
        else:
            a = np.ascontiguousarray(value, dtype=np.float64).ravel()
            _ck(lib().jg_restart_put_record(self._h, name.encode(), kind, _dp(a), 0, 0.0))

    def write(self, path: str):
        """``Ugp::writeRestart`` with one process."""
        _ck(lib().jg_restart_write(self._h, str(path).encode()))

    # -- handle bridge ----------------------------------------------------
    def save_state(self, joe):
        """STEP, RHO, RHOE, the model's scalars and RHOU from a ``JoeGpu``."""
        _ck(lib().jg_restart_save_state(self._h, joe.h))

    def load_state(self, joe):
        """RHO, RHOU, RHOE, the model's scalars and STEP into a ``JoeGpu``
        (CFL back at its start value, as the reference resumes)."""
        _ck(lib().jg_restart_load_state(joe.h, self._h))


def write_restart(path: str, g, joe, internal_zone: str = "fluid_faces") -> None:
    """``Ugp::writeRestart`` for a handle: ``g``'s mesh (the CvMesh the handle
    was created on) with the handle's STEP, RHO, RHOE, scalars and RHOU."""
    with Restart.from_cv_mesh(g, internal_zone) as r:
        r.save_state(joe)
        r.write(path)


def read_restart(path: str):
    """``initializeFromRestartFile`` for a restart: (CvMesh in the file's cell
    order, Restart).  Create the handle on the mesh, then ``load_state``."""
    from . import geometry
    r = Restart.read(path)
    return geometry.build_cv_mesh(r.to_raw_mesh()), r

