"""Five to eight temperatures fused in one RTA_driver_4ph call: the kernels'
eight-temperature instantiation (the matrix element is contracted once and
weighted for every temperature), against the oracle run once per temperature.

Bars: FP64 rates within 1e-10, mixed-precision rates within 1e-3 per mode,
WP4 within 1e-10 in every precision (its weights are FP64 in all paths).
"""
import numpy as np
import pytest

import helpers as H
import oracle as O
from fourphonon_b200 import abi

pytestmark = pytest.mark.gpu

TEMPS = (100.0, 250.0, 400.0, 600.0, 800.0, 1000.0)
CH = ("rate_plusplus", "rate_plusminus", "rate_minusminus")
WP = ("wp4_plusplus", "wp4_plusminus", "wp4_minusminus")


def close(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max() if b.size else 0.0
    err = np.abs(a - b)
    ok = err <= rtol * np.abs(b) + 1e-3 * rtol * scale
    rel = err / np.maximum(np.abs(b), 1e-300)
    rel = rel[np.abs(b) > 1e-6 * scale] if scale > 0 else rel
    return bool(ok.all()), float(rel.max() if rel.size else 0.0)


@pytest.fixture(scope="module")
def six():
    s = H.cached_solve("zincblende", (4, 4, 4), temperatures=TEMPS)
    return s, [O.Oracle(s, T=T).rta4() for T in TEMPS]


@pytest.mark.parametrize("precision", [abi.FP4_PREC_FP64, abi.FP4_PREC_MIXED, abi.FP4_PREC_MIXED_SIMT])
def test_six_temperatures_fused(six, precision):
    s, ref = six
    c = abi.Context(0, precision)
    try:
        g = c.rta_driver_4ph(s)
    finally:
        c.close()
    rtol = 1e-10 if precision == abi.FP4_PREC_FP64 else 1e-3
    errs = []
    for t, T in enumerate(TEMPS):
        o = ref[t]
        for x, name in enumerate(CH):
            assert (o[x] > 0).any(), (T, name)
            ok, e = close(g[name][t], o[x], rtol)
            errs.append(e)
            assert ok, (T, name, e)
        for x, name in enumerate(WP):
            ok, e = close(g[name][t], o[3 + x], 1e-10)
            assert ok, (T, name, e)
    print("six fused temperatures, rate error vs oracle:", precision, max(errs))
