"""fp4_np_driver_4ph_noalloc: the four-phonon process counts for callers that
cannot allocate device memory (hosts whose device memory all comes from their
own pool, or code embedded in a process whose allocator it must not touch).

The entry point takes device arrays and keeps its scratch in a fixed device
array of the library, so it never calls cudaMalloc.  Its results must equal
those of the context-based fp4_np_driver_4ph on the same solve, on two calls
in a row (the second call reuses the scratch the first one left behind), and
a call must leave the device's free memory unchanged.  Calls beyond the
scratch size must be refused with FP4_E_CAPACITY and a List entry outside the
grid with FP4_E_ARG.  A host that resets the device between calls gets the
array of its new context (checked in a child process that uses only the CUDA
runtime, so the reset touches no other test's state).
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as ct
import os
import subprocess
import sys

import numpy as np
import pytest

from fourphonon_b200 import abi
from fourphonon_b200 import system as S

pytestmark = pytest.mark.gpu

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))


def _call(lib, g, de, dv, nlist, dl, dn, dp, stream):
    ptr = lambda t: ct.c_void_p(t.data_ptr())  # noqa: E731
    return lib.fp4_np_driver_4ph_noalloc(ct.byref(g), ptr(de), ptr(dv), ct.c_int32(nlist), ptr(dl), ptr(dn[0]),
                                         ptr(dp[0]), ptr(dn[1]), ptr(dp[1]), ptr(dn[2]), ptr(dp[2]),
                                         ct.c_void_p(stream))


def test_noalloc_counts_equal_context_entry_point():
    import torch

    s = S.cached_solve("diamond", (6, 6, 6))
    lib = abi.load()
    ctx = abi.Context(0)
    try:
        n_ref, p_ref = ctx.np_driver_4ph(s)
        g = ctx.globals_of(s)
        e, v, _, lst, _ = ctx._arrays(s)
        dev = torch.device("cuda", 0)
        de = torch.from_numpy(e).to(dev)
        dv = torch.from_numpy(v).to(dev)
        dl = torch.from_numpy(lst).to(dev)
        nm = s.nmodes
        dn = [torch.full((nm,), -1, dtype=torch.int64, device=dev) for _ in range(3)]
        dp = [torch.full((nm,), -1.0, dtype=torch.float64, device=dev) for _ in range(3)]
        stream = torch.cuda.current_stream(dev).cuda_stream
        for call in range(2):
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info(dev)[0]
            rc = _call(lib, g, de, dv, s.nlist, dl, dn, dp, stream)
            assert rc == 0, (call, rc)
            torch.cuda.synchronize()
            if call == 1:  # the first call may load the module; a later one must allocate nothing
                assert torch.cuda.mem_get_info(dev)[0] == free0
            for ch in range(3):
                assert np.array_equal(dn[ch].cpu().numpy(), n_ref[ch]), (call, ch)
                got, ref = dp[ch].cpu().numpy(), p_ref[ch]
                assert np.allclose(got, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max()), (call, ch)

        # a grid whose packed mode table alone exceeds the scratch: refused before any device work
        big = ctx.globals_of(s)
        for d in range(3):
            big.ngrid[d] = 64
        assert _call(lib, big, de, dv, s.nlist, dl, dn, dp, stream) == abi.FP4_E_CAPACITY

        # a List entry outside [1, nptk]: the kernel flags it and the call reports FP4_E_ARG
        bad = lst.copy()
        bad[-1] = s.nptk + 1
        dbad = torch.from_numpy(bad).to(dev)
        assert _call(lib, g, de, dv, s.nlist, dbad, dn, dp, stream) == abi.FP4_E_ARG
        # and the next good call is unaffected by what the refused one left in the scratch
        assert _call(lib, g, de, dv, s.nlist, dl, dn, dp, stream) == 0
        torch.cuda.synchronize()
        for ch in range(3):
            assert np.array_equal(dn[ch].cpu().numpy(), n_ref[ch]), ch
    finally:
        ctx.close()


_RESET_CHILD = r"""
import ctypes as ct, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from fourphonon_b200 import abi
from fourphonon_b200 import system as S

s = S.cached_solve("diamond", (6, 6, 6))
lib = abi.load()
ctx = abi.Context(0)
n_ref, p_ref = ctx.np_driver_4ph(s)
g = ctx.globals_of(s)
e, v, _, lst, _ = ctx._arrays(s)
ctx.close()
rt = ct.CDLL("libcudart.so.12")
H2D, D2H = 1, 2
nm = s.nmodes

def dev_copy(a):
    p = ct.c_void_p()
    assert rt.cudaMalloc(ct.byref(p), ct.c_size_t(a.nbytes)) == 0
    assert rt.cudaMemcpy(p, a.ctypes.data_as(ct.c_void_p), ct.c_size_t(a.nbytes), H2D) == 0
    return p

def run_once():
    bufs = [dev_copy(e), dev_copy(v), dev_copy(lst)]
    outs = [dev_copy(np.zeros(nm, np.int64)) for _ in range(3)] + [dev_copy(np.zeros(nm)) for _ in range(3)]
    rc = lib.fp4_np_driver_4ph_noalloc(ct.byref(g), bufs[0], bufs[1], ct.c_int32(s.nlist), bufs[2], outs[0],
                                       outs[3], outs[1], outs[4], outs[2], outs[5], None)
    assert rc == 0, rc
    for ch in range(3):
        n = np.zeros(nm, np.int64)
        assert rt.cudaMemcpy(n.ctypes.data_as(ct.c_void_p), outs[ch], ct.c_size_t(n.nbytes), D2H) == 0
        assert np.array_equal(n, n_ref[ch]), ch
    for b in bufs + outs:
        assert rt.cudaFree(b) == 0

run_once()
assert rt.cudaDeviceReset() == 0  # ends this process's context; the next call runs in a new one
run_once()
print("RESET-OK")
"""


def test_noalloc_after_device_reset():
    r = subprocess.run([sys.executable, "-c", _RESET_CHILD, ROOT], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "RESET-OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]
