"""Restart files on the CPU: the library's reader and writer of the
reference's binary restart format (Ugp::writeRestart / Ugp::readRestart,
src/common/Ugp.cpp:9792-13240) against files the reference itself wrote
(tests/golden/make_restart.py), and the reference resuming from a file the
library wrote (when the reference harness is built).  Host code only: no GPU.
"""
import dataclasses
import os
import struct

import numpy as np
import pytest
from scipy.spatial import cKDTree

from myjoe_b200 import build as jbuild
from myjoe_b200 import case, geometry, meshgen, restart, solver

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
BUMP = os.path.join(GOLD, "restart_bump_step3.out")
SA = os.path.join(GOLD, "restart_sa_step2.out")


@pytest.fixture(scope="module", autouse=True)
def _lib():
    jbuild.build()


def _bump_case():
    _, g, prm = case.bump_case(8, 4, 2, jitter=0.15, seed=7)
    return g, dataclasses.replace(prm, CFL_RAMP=(1, 1, 1.5, 5.0))


@pytest.mark.parametrize("path", [BUMP, SA])
def test_reference_file_is_written_back_byte_for_byte(path, tmp_path):
    r = restart.Restart.read(path)
    out = str(tmp_path / "back.out")
    r.write(out)
    assert open(out, "rb").read() == open(path, "rb").read()


def test_reference_file_contents():
    ref = np.load(os.path.join(GOLD, "restart_bump.npz"))
    r = restart.Restart.read(BUMP)
    n = r.counts()
    assert (n["nno"], n["nfa"], n["ncv"]) == (9 * 5 * 3, 248, 64)
    assert n["noofa_count"] == 4 * 248
    zones = r.zones()
    assert [(z[0], z[1]) for z in zones] == [("inlet", 1), ("lower", 1), ("outlet", 1), ("sides", 1), ("upper", 1),
                                             ("fluid_faces", 6)]
    assert zones[0][2] == 0 and zones[-1][3] == 247
    assert r.get("STEP") == (restart.I0, 3)
    # cells are in the reference's order at the time of writing: its state after 3 steps, bit for bit
    assert np.array_equal(r.get("RHO")[1], ref["rho3"])
    assert np.array_equal(r.get("RHOU")[1], ref["rhou3"])
    assert np.array_equal(r.get("RHOE")[1], ref["rhoE3"])
    x_no, noofa_i, noofa_v, cvofa, cv_part = r.mesh()
    assert np.all(cv_part == 0)
    assert np.all(cvofa[:112, 1] == -1) and np.all(cvofa[112:, 1] >= 0)
    # the file's mesh rebuilt here has the reference's cell centroids
    g = geometry.build_cv_mesh(r.to_raw_mesh())
    assert np.abs(g.x_cv - ref["x_cv3"]).max() < 1e-14


def test_sa_file_holds_the_model_records():
    r = restart.Restart.read(SA)
    names = r.record_names()
    for k in ("nuSA", "wallDist", "muT", "RHOU", "STEP"):
        assert k in names
    kind, nu = r.get("nuSA")
    assert kind == restart.CV_D1 and nu.shape == (64,) and nu.min() > 0.0
    assert r.get("STEP") == (restart.I0, 2)


def _swapped(blob: bytes) -> bytes:
    """The file as a machine of the other byte order writes it (test helper)."""
    out = bytearray(blob)

    def sw(off, n, size):
        for k in range(n):
            a = off + k * size
            out[a:a + size] = out[a:a + size][::-1]

    sw(0, 2, 4)
    pos = 8
    while True:
        hid, skip = struct.unpack_from("<iq", blob, pos + 52)
        idata = struct.unpack_from("<16i", blob, pos + 64)
        sw(pos + 52, 1, 4)
        sw(pos + 56, 1, 8)
        sw(pos + 64, 16, 4)
        sw(pos + 128, 16, 8)
        body = pos + 256
        if hid in (20, 30, 40, 41):
            sw(body, idata[0], 4)
        elif hid in (21, 22):
            sw(body, (skip - 256) // 4, 4)
        elif hid in (24, 25, 31, 32, 33, 42, 43, 44):
            sw(body, (skip - 256) // 8, 8)
        if hid == 51:
            break
        pos += skip
    return bytes(out)


def test_byte_swapped_file_is_read(tmp_path):
    blob = open(BUMP, "rb").read()
    p = str(tmp_path / "swapped.out")
    with open(p, "wb") as f:
        f.write(_swapped(blob))
    r = restart.Restart.read(p)
    ref = restart.Restart.read(BUMP)
    assert r.record_names() == ref.record_names()
    for name in ("RHO", "RHOU", "TIME", "STEP"):
        a, b = r.get(name)[1], ref.get(name)[1]
        assert np.array_equal(np.asarray(a), np.asarray(b))
    for a, b in zip(r.mesh(), ref.mesh()):
        assert np.array_equal(a, b)
    out = str(tmp_path / "native.out")
    r.write(out)
    assert open(out, "rb").read() == blob


def test_malformed_files_fail_with_io_error(tmp_path):
    with pytest.raises(solver.JoeGpuError) as e:
        restart.Restart.read(str(tmp_path / "missing.out"))
    assert e.value.code == -6
    blob = open(BUMP, "rb").read()
    cases = {
        "magic": b"\x00\x00\x00\x00" + blob[4:],
        "version": blob[:4] + struct.pack("<i", 2) + blob[8:],
        "truncated": blob[: len(blob) // 2],
        "no_eof": blob[:-256],
        "empty": b"",
    }
    # a data record whose header claims one cell more than the mesh has
    pos = blob.index(b"RHO\x00")
    bad = bytearray(blob)
    struct.pack_into("<i", bad, pos + 64, 65)
    cases["record_size"] = bytes(bad)
    for name, data in cases.items():
        p = str(tmp_path / (name + ".out"))
        with open(p, "wb") as f:
            f.write(data)
        with pytest.raises(solver.JoeGpuError) as e:
            restart.Restart.read(p)
        assert e.value.code == -6, name


def test_written_mesh_and_records_read_back(tmp_path):
    raw = meshgen.channel_bump_mixed(6, 4, 2, n_prism=2, jitter=0.1, seed=3)
    g = geometry.build_cv_mesh(raw, seed=5, shuffle=True)
    r = restart.Restart.from_cv_mesh(g)
    rng = np.random.default_rng(0)
    fields = {"RHO": (restart.CV_D1, rng.random(g.ncv)), "RHOU": (restart.CV_D3, rng.random((g.ncv, 3))),
              "grad": (restart.CV_D33, rng.random((g.ncv, 3, 3))), "nodal": (restart.NO_D1, rng.random(len(g.x_no))),
              "facial": (restart.FA_D1, rng.random(g.nfa)), "STEP": (restart.I0, 17), "TIME": (restart.D0, 0.25)}
    for name, (kind, v) in fields.items():
        r.put(name, kind, v)
    p = str(tmp_path / "mine.out")
    r.write(p)
    back = restart.Restart.read(p)
    # records come back grouped as the reference writes them: I0, D0, D1, D3, D33
    assert back.record_names() == ["STEP", "TIME", "RHO", "nodal", "facial", "RHOU", "grad"]
    for name, (kind, v) in fields.items():
        k, got = back.get(name)
        assert k == kind and np.array_equal(np.asarray(got), np.asarray(v)), name
    x_no, noofa_i, noofa_v, cvofa, _ = back.mesh()
    assert np.array_equal(cvofa, g.cvofa)
    # boundary nodes first, every face keeps its nodes (and so its orientation)
    nn = np.diff(noofa_i)
    assert np.array_equal(nn, g.fa_nno)
    on_b = np.zeros(len(x_no), dtype=bool)
    on_b[noofa_v[: noofa_i[g.nfa_b]]] = True
    nb = int(on_b.sum())
    assert on_b[:nb].all() and not on_b[nb:].any()
    mask = np.arange(4)[None, :] < nn[:, None]
    assert np.array_equal(x_no[noofa_v], g.x_no[g.fa_nodes[mask]])
    # and the mesh rebuilt from the file is the same control-volume mesh
    g2 = geometry.build_cv_mesh(back.to_raw_mesh())
    assert np.array_equal(g2.cvofa, g.cvofa)
    assert np.abs(g2.x_cv - g.x_cv).max() < 1e-15
    assert np.abs(g2.fa_normal - g.fa_normal).max() < 1e-15
    assert [z[0] for z in g2.zones] == [z[0] for z in g.zones]


def test_writer_rejects_bad_input(tmp_path):
    g, _ = _bump_case()
    r = restart.Restart.from_cv_mesh(g)
    with pytest.raises(solver.JoeGpuError):
        r.put("X" * 60, restart.CV_D1, np.zeros(g.ncv))
    with pytest.raises(solver.JoeGpuError):
        r.put("BAD", 99, np.zeros(g.ncv))
    with pytest.raises(solver.JoeGpuError):
        r.add_zone("extra", 1, 5, 7)          # zones must follow one another
    empty = restart.Restart()
    with pytest.raises(solver.JoeGpuError):
        empty.write(str(tmp_path / "x.out"))  # no mesh
    partial = restart.Restart()
    partial.set_mesh(g.x_no, np.r_[0, np.cumsum(g.fa_nno)], g.fa_nodes[g.fa_nodes >= 0], g.cvofa, g.ncv)
    partial.add_zone("inlet", 1, 0, 3)
    with pytest.raises(solver.JoeGpuError):
        partial.write(str(tmp_path / "y.out"))  # zones do not cover every face


@pytest.mark.skipif(not __import__("oracle.refrun", fromlist=["x"]).available(),
                    reason="reference harness not built")
def test_reference_resumes_from_a_library_file(tmp_path):
    """The reference reads a restart the library wrote (cells and faces in
    this build's order) and continues exactly as from its own restart."""
    from oracle import refrun
    ref = np.load(os.path.join(GOLD, "restart_bump.npz"))
    g, prm = _bump_case()
    _, m = cKDTree(ref["x_cv3"]).query(g.x_cv)
    r = restart.Restart.from_cv_mesh(g)
    r.put("STEP", restart.I0, 3)
    r.put("RHO", restart.CV_D1, ref["rho3"][m])
    r.put("RHOE", restart.CV_D1, ref["rhoE3"][m])
    r.put("RHOU", restart.CV_D3, ref["rhou3"][m])
    p = str(tmp_path / "mine.out")
    r.write(p)
    run = refrun.run(None, dataclasses.replace(prm, NSTEPS=6).joe_in("restart.in"), "run",
                     files={"restart.in": open(p, "rb").read()})
    assert run["steps"] == 6
    _, m6 = cKDTree(run["x_cv"]).query(ref["x_cv6"])
    for k in ("rho", "rhou", "rhoE"):
        a, b = ref[k + "6"], run["final_" + k][m6]
        assert np.abs(a - b).max() <= 1e-14 * np.abs(a).max(), k
