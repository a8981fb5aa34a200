"""CPU checks of the drop-in boundary: the C-ABI library loads and exports
every entry point include/joe_b200.h declares; without a GPU every call
fails cleanly with JG_ERR_NODEVICE (no CPU fallback exists)."""
import ctypes as C
import os
import re

import pytest

from myjoe_b200 import build as jbuild
from myjoe_b200 import solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "joe_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(\w+)\s*\([^;{]*\)\s*;", txt, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    jbuild.build()
    return solver.lib()


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ["jg_create", "jg_destroy", "jg_set_state", "jg_calc_rhs", "jg_solve_lin_sys", "jg_step",
                     "jg_calc_dt", "jg_euler_flux_faces", "solveLinSysNSCoupled"]:
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_version(lib):
    assert lib.jg_version() == 1


def test_no_device_fails_cleanly(lib):
    n = C.c_int(-1)
    rc = lib.jg_device_count(C.byref(n))
    if n.value > 0:
        pytest.skip("a GPU is present")
    assert rc == -5 and n.value == 0
    from myjoe_b200 import case
    _, g, prm = case.bump_case(4, 2, 2)
    with pytest.raises(solver.JoeGpuError) as e:
        solver.JoeGpu(g, prm)
    assert e.value.code == -5


def test_null_arguments_rejected(lib):
    assert lib.jg_create(None, None, None) == -1
    assert lib.jg_step(None, 1, None) == -1
