"""Runs the reference solver (oracle/_ref/ref_harness, built from the
reference's own sources by oracle/Makefile) on a case and loads its dumps.

Test infrastructure only: tests, the golden-fixture script and bench.py's
CPU-baseline leg use it as the checker / baseline, never as the product.
"""
from __future__ import annotations

import os
import re
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "ref_harness")


def available() -> bool:
    return os.path.exists(HARNESS)


def _read_meta(d):
    meta = {"zones": []}
    with open(os.path.join(d, "meta.txt")) as f:
        for line in f:
            k, *v = line.split()
            if k == "zone":
                meta["zones"].append((v[0], int(v[1]), int(v[2])))
            elif k in ("R_gas", "GAMMA"):
                meta[k] = float(v[0])
            else:
                meta[k] = int(v[0])
    return meta


def _load(d):
    out = {"meta": _read_meta(d)}
    for fn in os.listdir(d):
        p = os.path.join(d, fn)
        if fn.endswith(".f64"):
            out[fn[:-4]] = np.fromfile(p, dtype=np.float64)
        elif fn.endswith(".i32"):
            out[fn[:-4]] = np.fromfile(p, dtype=np.int32)
    m = out["meta"]
    ncv, nfa, nfa_b, nbs = m["ncv"], m["nfa"], m["nfa_b"], m["nbocv_s"]
    shapes = {"cvofa": (nfa, 2), "x_cv": (ncv, 3), "x_fa": (nfa, 3), "fa_normal": (nfa, 3),
              "nbocv_lsg_coeff": (nbs, 3), "boundary_fa_lsg_coeff": (nfa_b, 3),
              "init_rhou": (ncv, 3), "final_rhou": (ncv, 3), "vel": (ncv, 3), "vel_bfa": (nfa_b, 3),
              "rhs_rhou": (ncv, 3), "A": (nbs, 5, 5), "A_sys": (nbs, 5, 5), "rhs_sys": (ncv, 5),
              "dq": (ncv, 5), "grad_u": (ncv, 3, 3), "grad_rho": (ncv, 3), "grad_p": (ncv, 3),
              "grad_enthalpy": (ncv, 3)}
    for k, s in shapes.items():
        if k in out:
            out[k] = out[k].reshape(s)
    return out


BINDING = os.path.join(HERE, "_ref", "joe_gpu_case")


def run(mesh_writer, joe_in: str, mode: str = "dump", run_kind: int = 0, timeout: float = 600.0,
        files: dict | None = None, collect: tuple = (), harness: str | None = None):
    """Write the mesh (``mesh_writer(path)``, may be None) and ``Joe.in`` into a
    temp directory, plus ``files`` (name -> bytes), run the harness there and
    return its dumps; the files named in ``collect`` that the run wrote (e.g.
    the restart.out runBackwardEuler leaves) come back as bytes in
    dumps["files"]."""
    harness = harness or HARNESS
    if not os.path.exists(harness):
        raise FileNotFoundError("%s not built: make -C oracle ref binding REF=<the reference src directory>" % harness)
    with tempfile.TemporaryDirectory(prefix="joe_ref_") as d:
        if mesh_writer is not None:
            mesh_writer(os.path.join(d, "mesh.msh"))
        for name, data in (files or {}).items():
            with open(os.path.join(d, name), "wb") as f:
                f.write(data)
        with open(os.path.join(d, "Joe.in"), "w") as f:
            f.write(joe_in)
        out = os.path.join(d, "out")
        os.mkdir(out)
        p = subprocess.run([harness, "Joe.in", str(run_kind), mode, out], cwd=d,
                           capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError("reference harness failed (%d):\n%s\n%s" % (
                p.returncode, p.stdout[-3000:], p.stderr[-3000:]))
        dumps = _load(out)
        dumps["files"] = {}
        for name in collect:
            fp = os.path.join(d, name)
            if os.path.exists(fp):
                with open(fp, "rb") as f:
                    dumps["files"][name] = f.read()
        dumps["stdout"] = p.stdout
        m = re.search(r"HARNESS_SECONDS ([0-9.eE+-]+)", p.stdout)
        if m:
            dumps["seconds"] = float(m.group(1))
        m = re.search(r"HARNESS_STEPS (\d+)", p.stdout)
        if m:
            dumps["steps"] = int(m.group(1))
        dumps["resid"] = np.array([[float(v) for v in line.split()[2:]]
                                   for line in p.stdout.splitlines() if line.startswith("RESID:")])
        return dumps
