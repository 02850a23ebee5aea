"""The tensor-core contraction of the mixed-precision four-phonon RTA path.

* fp4_tc_selftest: one tcgen05 product through the shared-memory layout,
  mbarrier and TMEM read-back the contraction uses, against an FP64 product of
  the same bf16 values (exact for small integers, 1e-5 otherwise);
* the mixed RTA driver on the tensor cores against the FP64 oracle: per-mode
  rates within 1e-3 (the error is printed), WP4 within 1e-10 (the weights stay
  FP64), kappa within 1e-4 of the FP64 driver's, and the work counters show
  that the products ran on the tensor cores.
"""
import numpy as np
import pytest

import helpers as H
import oracle as O
from fourphonon_b200 import abi

pytestmark = pytest.mark.gpu

CH = ("rate_plusplus", "rate_plusminus", "rate_minusminus")
WP = ("wp4_plusplus", "wp4_plusminus", "wp4_minusminus")


def to_bf16(x):
    """Round float32 values to bf16 (nearest even); returns the raw bits."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return r.astype(np.uint16)


def from_bf16(bits):
    return (bits.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("K,N", [(16, 16), (64, 80), (96, 128), (48, 256)])
def test_selftest_small_integers_exact(K, N):
    rng = np.random.default_rng(K * 1000 + N)
    A = to_bf16(rng.integers(-4, 5, size=(128, K)).astype(np.float32))
    B = to_bf16(rng.integers(-4, 5, size=(N, K)).astype(np.float32))
    D = abi.tc_selftest(A, B)
    ref = from_bf16(A) @ from_bf16(B).T
    assert np.array_equal(D.astype(np.float64), ref)


def test_selftest_random_values():
    rng = np.random.default_rng(7)
    K, N = 64, 128
    A = to_bf16(rng.standard_normal((128, K)).astype(np.float32))
    B = to_bf16(rng.standard_normal((N, K)).astype(np.float32))
    D = abi.tc_selftest(A, B).astype(np.float64)
    a, b = from_bf16(A), from_bf16(B)
    ref = a @ b.T
    scale = np.abs(a) @ np.abs(b).T
    assert np.all(np.abs(D - ref) <= 1e-5 * scale + 1e-30)


def close(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max() if b.size else 0.0
    err = np.abs(a - b)
    ok = err <= rtol * np.abs(b) + 1e-3 * rtol * scale
    rel = err / np.maximum(np.abs(b), 1e-300)
    rel = rel[np.abs(b) > 1e-6 * scale] if scale > 0 else rel
    return bool(ok.all()), float(rel.max() if rel.size else 0.0)


def _tau(rate):
    t = np.zeros_like(rate)
    t[rate != 0] = 1.0 / rate[rate != 0]
    return t


def test_tc_rates_against_oracle():
    s = H.cached_solve("diamond", (6, 6, 6), temperatures=(300.0, 700.0))
    c = abi.Context(0, abi.FP4_PREC_MIXED)
    c64 = abi.Context(0, abi.FP4_PREC_FP64)
    try:
        g = c.rta_driver_4ph(s)
        cnt = c.counters()
        assert cnt[7] == 1 and cnt[6] > 0 and cnt[5] > 0, cnt  # the products ran on the tensor cores
        assert cnt[1] == cnt[0] or cnt[1] > 0
        r64 = c64.rta_driver_4ph(s)
        mm0, mm1 = 6, 30
        errs = []
        for t, T in enumerate(s.temperatures):
            o = O.Oracle(s, T=T).rta4(mm0, mm1)
            for x, name in enumerate(CH):
                ok, e = close(g[name][t][mm0:mm1], o[x][mm0:mm1], 1e-3)
                errs.append(e)
                assert ok, (T, name, e)
            for x, name in enumerate(WP):
                ok, e = close(g[name][t][mm0:mm1], o[3 + x][mm0:mm1], 1e-10)
                assert ok, (T, name, e)
            # kappa (RTA, 4ph rates alone) against the FP64 driver's
            o0 = O.Oracle(s, T=T)
            k64 = np.trace(o0.tconduct(o0.iteration0(_tau(r64["rate_4ph"][t]))).reshape(3, 3, s.nb).sum(axis=2))
            kmx = np.trace(o0.tconduct(o0.iteration0(_tau(g["rate_4ph"][t]))).reshape(3, 3, s.nb).sum(axis=2))
            assert abs(kmx - k64) <= 1e-4 * abs(k64), (T, k64, kmx)
        print("tensor-core per-mode rate error vs oracle:", max(errs))
    finally:
        c.close()
        c64.close()
