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
