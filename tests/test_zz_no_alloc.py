"""fp4_np_driver_4ph_noalloc: the four-phonon process counts for callers that
cannot allocate device memory (hosts whose device memory all comes from their
own pool, or code embedded in a process whose allocator it must not touch).

The entry point takes device arrays and keeps its scratch in a fixed device
array of the library, so it never calls cudaMalloc.  Its results must equal
those of the context-based fp4_np_driver_4ph on the same solve, on two calls
in a row (the second call reuses the scratch the first one left behind).
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as ct

import numpy as np
import pytest

from fourphonon_b200 import abi
from fourphonon_b200 import system as S

pytestmark = pytest.mark.gpu


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
        ptr = lambda t: ct.c_void_p(t.data_ptr())  # noqa: E731
        for call in range(2):
            rc = lib.fp4_np_driver_4ph_noalloc(ct.byref(g), ptr(de), ptr(dv), ct.c_int32(s.nlist), ptr(dl),
                                               ptr(dn[0]), ptr(dp[0]), ptr(dn[1]), ptr(dp[1]), ptr(dn[2]), ptr(dp[2]),
                                               ct.c_void_p(stream))
            assert rc == 0, (call, rc)
            torch.cuda.synchronize()
            for ch in range(3):
                assert np.array_equal(dn[ch].cpu().numpy(), n_ref[ch]), (call, ch)
                got, ref = dp[ch].cpu().numpy(), p_ref[ch]
                assert np.allclose(got, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max()), (call, ch)
    finally:
        ctx.close()
