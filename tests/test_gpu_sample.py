"""Sampled four-phonon drivers (NP_*_sample, RTA_*_sample) on the device
against the oracle drawing the same samples from the same seeded stream:
sampled counts exact, P4, rates and WP4 within 1e-10; the estimate agrees
with the full enumeration within its sampling error."""
import numpy as np
import pytest

import helpers as H
import oracle as O
from fourphonon_b200 import abi

pytestmark = pytest.mark.gpu


def close(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max() if b.size else 0.0
    return bool((np.abs(a - b) <= rtol * np.abs(b) + 1e-3 * rtol * scale).all())


@pytest.fixture(scope="module")
def ctx():
    c = abi.Context(0)
    yield c
    c.close()


def test_sampled_np_matches_oracle(ctx):
    s = H.cached_solve("zincblende", (4, 4, 4), (500.0,))
    ns, seed = 50_000, 20240604
    n, p = ctx.np_driver_4ph_sample(s, ns, seed)
    o = O.Oracle(s).sample4(ns, seed, mode=0)
    for ch in range(3):
        assert np.array_equal(n[ch], o["n"][ch]), ch
        assert close(p[ch], o["p"][ch], 1e-10), ch


def test_sampled_rta_matches_oracle_two_temperatures(ctx):
    s = H.cached_solve("diamond", (4, 4, 4))
    ns, seed = 20_000, 7
    g = ctx.rta_driver_4ph_sample(s, ns, seed, temperatures=[300.0, 700.0])
    for t, T in enumerate((300.0, 700.0)):
        o = O.Oracle(s, T=T).sample4(ns, seed, mode=2)
        for ch, name in enumerate(("plusplus", "plusminus", "minusminus")):
            assert close(g["rate_" + name][t], o["rate"][ch], 1e-10), (T, name)
            assert close(g["wp4_" + name][t], o["wp"][ch], 1e-10), (T, name)


def test_sampled_rates_estimate_full_enumeration(ctx):
    s = H.cached_solve("diamond", (4, 4, 4))
    full = ctx.rta_driver_4ph(s)
    g = ctx.rta_driver_4ph_sample(s, 400_000, 11)
    for name in ("rate_plusplus", "rate_plusminus", "rate_minusminus"):
        a, b = full[name][0].sum(), g[name][0].sum()
        assert abs(b / a - 1) < 0.05, (name, a, b)


def test_sampled_rta_mixed_precision_matches_oracle():
    """The mixed-precision sampled driver (FP32 V(4) sums, FP64 draws, filter,
    weights and sums) against the FP64 oracle on the same draws: per-mode rates
    within 1e-3 (the error is printed), WP4 within 1e-10 and the RTA kappa of the
    sampled 4ph rates within 1e-4."""
    s = H.cached_solve("zincblende", (4, 4, 4), (100.0, 300.0, 500.0, 1000.0))
    ns, seed = 20_000, 20240605
    cmx = abi.Context(0, abi.FP4_PREC_MIXED)
    try:
        g = cmx.rta_driver_4ph_sample(s, ns, seed)
        worst = 0.0
        for t, T in enumerate(s.temperatures):
            o = O.Oracle(s, T=T).sample4(ns, seed, mode=2)
            for ch, name in enumerate(("plusplus", "plusminus", "minusminus")):
                ref, got = o["rate"][ch], g["rate_" + name][t]
                assert close(got, ref, 1e-3), (T, name)
                m = ref > 1e-6 * ref.max()
                worst = max(worst, float(np.max(np.abs(got[m] - ref[m]) / ref[m])))
                assert close(g["wp4_" + name][t], o["wp"][ch], 1e-10), (T, name)
            rate_o = o["rate"][0] + o["rate"][1] + o["rate"][2]
            rate_g = g["rate_plusplus"][t] + g["rate_plusminus"][t] + g["rate_minusminus"][t]
            oo = O.Oracle(s, T=T)
            kap = []
            for r in (rate_o, rate_g):
                tau = np.zeros_like(r)
                tau[r != 0] = 1.0 / r[r != 0]
                kap.append(np.trace(oo.tconduct(oo.iteration0(tau)).reshape(3, 3, s.nb).sum(axis=2)))
            assert abs(kap[1] - kap[0]) <= 1e-4 * abs(kap[0]), (T, kap)
        print("mixed sampled per-mode rate error vs oracle:", worst)
    finally:
        cmx.close()
