"""The ctypes binding hands every C entry point the arguments its prototype in
include/fourphonon_b200.h declares (CPU, no device).

ctypes calls here carry no argtypes, so a wrong argument would not be caught
by Python: a bare Python int given to an int64_t travels as a 32-bit int, an
int given to a double lands in the wrong register.  Every method of
abi.Context, serve.Server and abi.tc_selftest is called with a fake library
that records its arguments, and each recorded call is checked against the
prototype: the argument count, a pointer (or None) for every pointer
parameter, a Python int or c_int for int/int32_t, a c_int64/c_uint64 for
int64_t/uint64_t, and a float or c_double for double.
"""
import ctypes as ct
import os
import re
import sys

import numpy as np
import pytest

import helpers as H
from fourphonon_b200 import abi, serve

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
sys.path.insert(0, os.path.join(ROOT, "include"))
import make_fortran_module as M  # noqa: E402  (its header parser)

PROTOS = {name: params for _, name, params in M.prototypes(open(M.HEADER).read())}
CARG = type(ct.byref(ct.c_int()))


class Recorder:
    def __init__(self):
        self.calls = []

    def __getattr__(self, name):
        if not name.startswith("fp4_"):
            raise AttributeError(name)

        def call(*args):
            self.calls.append((name, args))
            return 0

        return call


def _ok(ctype, extent, arg):
    if "*" in ctype or extent is not None:
        return arg is None or isinstance(arg, (ct.c_void_p, ct.Array, ct._Pointer, CARG))
    base = ctype.replace("const ", "").strip()
    if base in ("int", "int32_t"):
        return (isinstance(arg, int) and not isinstance(arg, bool)) or isinstance(arg, (ct.c_int, ct.c_int32))
    if base in ("int64_t", "uint64_t"):
        return isinstance(arg, (ct.c_int64, ct.c_uint64, ct.c_longlong, ct.c_ulonglong))
    if base == "double":
        return isinstance(arg, (float, ct.c_double))
    raise AssertionError(f"unhandled C type {ctype}")


def _check(calls):
    assert calls
    for name, args in calls:
        params = PROTOS[name]
        assert len(args) == len(params), (name, len(args), len(params))
        for (ctype, pname, extent), a in zip(params, args):
            assert _ok(ctype, extent, a), (name, pname, ctype, type(a).__name__)


@pytest.fixture(scope="module")
def cell():
    return H.cached_solve("diamond", (3, 3, 3), temperatures=(300.0, 500.0))


def test_context_methods(cell):
    s = cell
    rec = Recorder()
    c = abi.Context.__new__(abi.Context)
    c.lib, c.h, c._keep = rec, ct.c_void_p(1), []
    nm = s.nmodes
    small = np.ones(nm, np.int32)
    small64 = np.ones(nm, np.int64)
    c.set_precision(abi.FP4_PREC_MIXED)
    c.stats()
    c.counters()
    c.phase_cycles(full=True)
    c.set_stream(0)
    c.set_stream(12345)
    c.set_upload_cache(False)
    c.np_driver(s)
    c.ind_only_driver(s, small, small)
    c.rta_driver(s, T=300.0)
    lists = c.ind_driver(s, small, small, T=300.0)
    c.np_driver_4ph(s)
    c.ind_only_driver_4ph(s, small64, small64, small64)
    c.rta_driver_4ph(s)
    c.rta4_partials(s, 0, 0, 2, 1)
    ind4 = c.ind_driver_4ph(s, small64, small64, small64, T=500.0)
    c.np_driver_sample(s, 1000, 7)
    c.rta_driver_sample(s, 1000, 7, T=500.0)
    c.np_driver_4ph_sample(s, 1000, 7)
    c.rta_driver_4ph_sample(s, 1000, 7)
    tau = np.ones(nm)
    F = c.iteration0(s, tau)
    c.iteration(s, F, tau, small, small, lists)
    c.iteration(s, F, tau, small, small, lists, ind4=ind4)
    c.iteration_jacobi(s, F, tau, small, small, lists)
    c.symmetrize_fn(s, F)
    cr = s.crystal
    fc = np.zeros((cr.natoms, 3, *cr.scell, cr.natoms, 3))
    c.eigen_dm(cr, fc, s.ngrid, s.sym.symmetrizers)
    c.cumulative_tconduct(s, F, T=300.0)
    c.cumulative_tconduct(s, F, T=300.0, omega_mode=True)
    c.tconduct(s, F, T=500.0)
    c.tconduct(s, F, T=500.0, with_modes=True)
    _check(rec.calls)
    used = {n for n, _ in rec.calls}
    src = open(os.path.join(ROOT, "fourphonon_b200", "abi.py")).read()
    named = set(re.findall(r"lib\.(fp4_\w+)\(", src)) - {"fp4_create", "fp4_destroy", "fp4_last_error",
                                                          "fp4_tc_selftest"}
    assert named <= used, sorted(named - used)


def test_server_methods(cell, monkeypatch):
    s = cell
    rec = Recorder()
    monkeypatch.setattr(serve, "_lib", lambda: rec)
    serve.footprint(s)
    srv = serve.Server(0, abi.FP4_PREC_FP64, max_slots=2, max_bands=6)
    slot = srv.admit(s, 300.0)
    srv.tick(1000)
    srv.collect(slot)
    srv.status()
    _check(rec.calls)
    assert {n for n, _ in rec.calls} >= {"fp4_server_footprint", "fp4_server_create", "fp4_server_admit",
                                          "fp4_server_tick", "fp4_server_collect", "fp4_server_status"}


def test_tc_selftest_binding(monkeypatch):
    rec = Recorder()
    monkeypatch.setattr(abi, "load", lambda build_if_missing=True: rec)
    abi.tc_selftest(np.zeros((128, 16), np.uint16), np.zeros((16, 16), np.uint16))
    _check(rec.calls)
