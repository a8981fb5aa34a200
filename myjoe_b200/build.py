"""Builds libjoe_b200.so in-tree with nvcc for sm_100a (no GPU needed)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libjoe_b200.so")
SOURCES = ["jg_kernels.cu", "jg_faceloop.cu", "jg_fused.cu", "jg_api.cu", "jg_noalloc.cu", "jg_serve.cu", "jg_coupled.cu", "jg_renumber.cu", "jg_linelet.cu", "jg_restart.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-Xcompiler", "-O2"]


def _nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "joe_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    objs, cmds = [], []
    for src in SOURCES:
        obj = os.path.join(CSRC, src.replace(".cu", ".o"))
        cmds.append([_nvcc(), *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj])
        objs.append(obj)
    if verbose:
        for cmd in cmds:
            print(" ".join(cmd))
    # the translation units compile independently: one nvcc per source, in parallel
    with ThreadPoolExecutor(max_workers=min(len(cmds), os.cpu_count() or 1)) as ex:
        for r in list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise subprocess.CalledProcessError(r.returncode, r.args)
    cmd = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
