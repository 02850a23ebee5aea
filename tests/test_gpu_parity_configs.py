"""Parity of the kernel variants that the larger workloads run, against the
CPU oracle (through the C-ABI):

* a 12-branch layered cell with 2nd-shell quartic clusters, whose reciprocal
  cluster tables are built one branch at a time (FP64 and mixed precision);
* four temperatures fused in one call (the NT=4 instantiation);
* a finite omega_max, which gates modes in the NP, Ind_only and RTA drivers
  (processes.f90:1032, 1277, 1735, 2806, 3170, 5256);
* the 16^3 diamond grid, checked through the per-q' partial sums of a few
  modes (the full 16^3 oracle sums take hours on a CPU).

Bars: counts and lists bit-exact, FP64 rates within 1e-10, mixed-precision
rates within 1e-3 per mode (the per-mode error is reported in the message).
"""
import numpy as np
import pytest

import helpers as H
import oracle as O
from fourphonon_b200 import abi

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-10
RTOL_MIXED_RATE = 1e-3
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
def c64():
    c = abi.Context(0, abi.FP4_PREC_FP64)
    yield c
    c.close()


@pytest.fixture(scope="module")
def cmx():
    c = abi.Context(0, abi.FP4_PREC_MIXED)
    yield c
    c.close()


@pytest.fixture(scope="module")
def csimt():
    c = abi.Context(0, abi.FP4_PREC_MIXED_SIMT)
    yield c
    c.close()


MIXED_MODES = [abi.FP4_PREC_MIXED, abi.FP4_PREC_MIXED_SIMT]
ALL_MODES = [abi.FP4_PREC_FP64] + MIXED_MODES


def pick(precision, c64, cmx, csimt):
    return {abi.FP4_PREC_FP64: c64, abi.FP4_PREC_MIXED: cmx, abi.FP4_PREC_MIXED_SIMT: csimt}[precision]


# ---------------------------------------------------------------------------- 12 branches, per-branch tables


@pytest.fixture(scope="module")
def layered():
    s = H.cached_solve("layered", (4, 4, 4))
    mm0, mm1 = s.nb, s.nb + 4  # four modes of the second irreducible point
    return s, mm0, mm1, O.Oracle(s).rta4(mm0, mm1)


def test_layered_rta4_fp64(c64, layered):
    s, mm0, mm1, o = layered
    assert s.nb == 12 and s.ifc4.ntri > 100
    g = c64.rta_driver_4ph(s)
    for x, name in enumerate(CH + WP):
        ok, e = close(g[name][0][mm0:mm1], o[x][mm0:mm1], RTOL_FP64)
        assert ok, (name, e)


@pytest.mark.parametrize("precision", MIXED_MODES)
def test_layered_rta4_mixed(cmx, csimt, layered, precision):
    s, mm0, mm1, o = layered
    ctx = cmx if precision == abi.FP4_PREC_MIXED else csimt
    g = ctx.rta_driver_4ph(s)
    errs = {}
    for x, name in enumerate(CH):
        ok, e = close(g[name][0][mm0:mm1], o[x][mm0:mm1], RTOL_MIXED_RATE)
        errs[name] = e
        assert ok, (name, e)
    for x, name in enumerate(WP):  # the weights stay FP64 in the mixed path
        ok, e = close(g[name][0][mm0:mm1], o[3 + x][mm0:mm1], RTOL_FP64)
        assert ok, (name, e)
    print("layered mixed per-mode rate error vs oracle:", precision, errs, "tensor cores:", ctx.counters()[7])


# ---------------------------------------------------------------------------- four fused temperatures


@pytest.mark.parametrize("precision", ALL_MODES)
def test_four_temperatures_fused(c64, cmx, csimt, precision):
    temps = (100.0, 300.0, 500.0, 1000.0)
    s = H.cached_solve("zincblende", (4, 4, 4), temperatures=temps)
    ctx = pick(precision, c64, cmx, csimt)
    g = ctx.rta_driver_4ph(s)
    rtol = RTOL_FP64 if precision == abi.FP4_PREC_FP64 else RTOL_MIXED_RATE
    for t, T in enumerate(temps):
        o = O.Oracle(s, T=T).rta4()
        for x, name in enumerate(CH):
            ok, e = close(g[name][t], o[x], rtol)
            assert ok, (T, name, e)
        for x, name in enumerate(WP):
            ok, e = close(g[name][t], o[3 + x], RTOL_FP64)
            assert ok, (T, name, e)


# ---------------------------------------------------------------------------- omega_max gate


@pytest.fixture(scope="module")
def gated():
    import copy

    base = H.cached_solve("diamond", (4, 4, 4))
    s = copy.copy(base)
    w = np.array([base.energy[q - 1, b] for q in base.wedge.list for b in range(base.nb)])
    s.omega_max = float(np.median(w[w > 0]))
    assert (w > s.omega_max).sum() > 0 and ((w <= s.omega_max) & (w > 0)).sum() > 0
    return s


def test_omega_max_gate_np_and_ind_only(c64, gated):
    s = gated
    o = O.Oracle(s)
    n_p, n_m, p_p, p_m = c64.np_driver(s)
    on = o.np3()
    assert np.array_equal(n_p, on[0]) and np.array_equal(n_m, on[1])
    gate = np.array([s.energy[q - 1, b] > s.omega_max for q in s.wedge.list for b in range(s.nb)])
    assert (n_p[gate] == 0).all() and (n_m[gate] == 0).all() and n_p[~gate].sum() > 0
    n4, p4 = c64.np_driver_4ph(s)
    on4, op4 = o.np4()
    for ch in range(3):
        assert np.array_equal(n4[ch], on4[ch]), ch
        assert (n4[ch][gate] == 0).all()
        ok, e = close(p4[ch], op4[ch], 1e-11)
        assert ok, (ch, e)
    a, b, c, d = c64.ind_only_driver(s, n_p, n_m)
    assert a.size == n_p.sum() and c.size == n_m.sum()
    lists = c64.ind_only_driver_4ph(s, *n4)
    for ch in range(3):
        assert lists[ch][0].size == n4[ch].sum()


def test_omega_max_gate_rta(c64, gated):
    s = gated
    o = O.Oracle(s)
    g3 = c64.rta_driver(s)
    rp, rm, wpp, wpm = o.rta3()
    for a, b in ((g3["rate_plus"], rp), (g3["rate_minus"], rm), (g3["wp3_plus"], wpp), (g3["wp3_minus"], wpm)):
        ok, e = close(a, b, RTOL_FP64)
        assert ok, e
    g4 = c64.rta_driver_4ph(s)
    o4 = o.rta4()
    gate = np.array([s.energy[q - 1, b] > s.omega_max for q in s.wedge.list for b in range(s.nb)])
    for x, name in enumerate(CH + WP):
        ok, e = close(g4[name][0], o4[x], RTOL_FP64)
        assert ok, (name, e)
        assert (g4[name][0][gate] == 0).all(), name


# ---------------------------------------------------------------------------- the 16^3 grid


@pytest.fixture(scope="module")
def grid16():
    s = H.cached_solve("diamond", (16, 16, 16), temperatures=(300.0, 700.0))
    ll, ii0, ii1 = 3, 0, 8  # irreducible point 4, the first 8 q' points
    mm0, mm1 = ll * s.nb, (ll + 1) * s.nb
    ref = {t: O.Oracle(s, T=T).rta4_range(mm0, mm1, ii0, ii1) for t, T in enumerate(s.temperatures)}
    return s, ll, ii0, ii1, mm0, mm1, ref


@pytest.mark.parametrize("precision", ALL_MODES)
def test_grid16_partials(c64, cmx, csimt, grid16, precision):
    s, ll, ii0, ii1, mm0, mm1, ref = grid16
    ctx = pick(precision, c64, cmx, csimt)
    full = ctx.rta_driver_4ph(s)
    rtol = RTOL_FP64 if precision == abi.FP4_PREC_FP64 else RTOL_MIXED_RATE
    errs = []
    for t in range(len(s.temperatures)):
        g = ctx.rta4_partials(s, ll, ii0, ii1, t)
        o = ref[t]
        for x, name in enumerate(CH):
            assert (o[x][mm0:mm1] > 0).any(), name
            ok, e = close(g[name], o[x][mm0:mm1], rtol)
            errs.append(e)
            assert ok, (t, name, e)
        for x, name in enumerate(WP):
            ok, e = close(g[name], o[3 + x][mm0:mm1], RTOL_FP64)
            assert ok, (t, name, e)
        # the partials over the whole grid are the driver's output
        tot = ctx.rta4_partials(s, ll, 0, s.nptk, t)
        for name in CH + WP:
            ok, e = close(tot[name], full[name][t][mm0:mm1], 1e-12)
            assert ok, (t, name, e)
    print("16^3 partial-sum rate error vs oracle:", precision, max(errs))
