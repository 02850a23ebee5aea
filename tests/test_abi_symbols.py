"""The C-ABI library loads and exports every entry point declared in
include/fourphonon_b200.h (CPU; no compute call is made)."""
import ctypes as ct
import os
import re

import pytest

from fourphonon_b200 import abi, build

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "fourphonon_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(fp4_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_driver_set():
    names = declared_symbols()
    for must in ("fp4_np_driver", "fp4_np_driver_4ph", "fp4_rta_driver", "fp4_rta_driver_4ph", "fp4_ind_driver",
                 "fp4_ind_only_driver", "fp4_ind_only_driver_4ph", "fp4_iteration", "fp4_tconduct"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = abi.load(build_if_missing=True)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_create_without_device_fails_cleanly():
    lib = abi.load()
    h = ct.c_void_p()
    rc = lib.fp4_create(ct.byref(h), 0)
    if rc == 0:
        lib.fp4_destroy(h)
        pytest.skip("a CUDA device is present")
    assert rc in (-1, -2)


def test_null_context_is_refused():
    """Entry points called with a null context return FP4_E_ARG (after opening and
    closing their NVTX range, which does nothing without a profiler)."""
    lib = abi.load()
    f = lib.fp4_iteration0
    f.restype = ct.c_int
    f.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int32, ct.c_void_p, ct.c_void_p, ct.c_int32, ct.c_void_p,
                  ct.c_void_p, ct.c_void_p, ct.c_void_p]
    assert f(None, None, 0, None, None, 0, None, None, None, None) == abi.FP4_E_ARG
    t = lib.fp4_server_tick
    t.restype = ct.c_int
    t.argtypes = [ct.c_void_p, ct.c_int64, ct.c_void_p, ct.c_void_p]
    assert t(None, 1, None, None) == abi.FP4_E_ARG
