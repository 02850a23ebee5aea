"""Ind_driver_4ph and iteration_4ph on the device (through the C-ABI) against
the oracle (processes.f90:3254-3822, iterations.f90:95-215).

Bars: index lists bit-exact; per-process Gamma, rates and WP4 within 1e-10
relative (FP64 path); Gauss-Seidel sweeps with the 4-phonon lists within 1e-9.
"""
import numpy as np
import pytest

import helpers as H
import oracle as O
from fourphonon_b200 import abi

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-10


@pytest.fixture(scope="module")
def ctx():
    c = abi.Context(0)
    yield c
    c.close()


def close(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max() if b.size else 0.0
    err = np.abs(a - b)
    ok = err <= rtol * np.abs(b) + 1e-3 * rtol * scale
    return bool(ok.all()), float((err / np.maximum(np.abs(b), 1e-300)).max() if b.size else 0.0)


CASES = [("diamond", (4, 4, 4), 300.0), ("zincblende", (4, 4, 4), 500.0), ("diamond", (5, 5, 5), 200.0)]


@pytest.mark.parametrize("kind,grid,T", CASES)
def test_ind_driver_4ph_lists_and_gamma(ctx, kind, grid, T):
    s = H.cached_solve(kind, grid, temperatures=(T,))
    n4, _ = ctx.np_driver_4ph(s)
    g = ctx.ind_driver_4ph(s, *n4)
    o = O.Oracle(s, T=T).ind4(*n4)
    for ch in ("pp", "pm", "mm"):
        for k in ("ind2_", "ind3_", "ind4_"):
            assert np.array_equal(g[k + ch], o[k + ch]), k + ch
        for k in ("gamma_", "rate_", "wp_"):
            ok, e = close(g[k + ch], o[k + ch], RTOL_FP64)
            assert ok, (k + ch, e)
    ok, e = close(g["rate_4ph"], o["rate_pp"] + o["rate_pm"] + o["rate_mm"], RTOL_FP64)
    assert ok, e


def test_ind_driver_4ph_rates_equal_rta(ctx):
    s = H.cached_solve("diamond", (4, 4, 4))
    n4, _ = ctx.np_driver_4ph(s)
    g = ctx.ind_driver_4ph(s, *n4)
    r = ctx.rta_driver_4ph(s)
    for a, b in (("rate_pp", "rate_plusplus"), ("rate_pm", "rate_plusminus"), ("rate_mm", "rate_minusminus"),
                 ("wp_pp", "wp4_plusplus"), ("wp_pm", "wp4_plusminus"), ("wp_mm", "wp4_minusminus")):
        ok, e = close(g[a], r[b][0], 1e-12)
        assert ok, (a, e)
    off = np.concatenate([[0], np.cumsum(n4[0])])
    sums = np.add.reduceat(g["gamma_pp"], off[:-1][n4[0] > 0])
    ok, e = close(sums, g["rate_pp"][n4[0] > 0], 1e-12)
    assert ok, e


def _tau_zero(rate):
    t = np.zeros_like(rate)
    nz = rate != 0
    t[nz] = 1.0 / rate[nz]
    return t


def test_iteration_4ph_sweeps(ctx):
    s = H.cached_solve("diamond", (4, 4, 4))
    o = O.Oracle(s)
    n_p, n_m, _, _ = o.np3()
    lists = o.ind3(n_p, n_m)
    n4, _ = o.np4()
    ind4 = o.ind4(*n4)
    tau = _tau_zero(lists["rate_plus"] + lists["rate_minus"] + ind4["rate_pp"] + ind4["rate_pm"] + ind4["rate_mm"])
    Fg = ctx.iteration0(s, tau)
    Fo = o.iteration0(tau)
    assert np.array_equal(Fg, Fo)
    for it in range(3):
        Fg = ctx.iteration(s, Fg, tau, n_p, n_m, lists, ind4=ind4)
        Fg = ctx.symmetrize_fn(s, Fg)
        Fo = o.iteration(Fo, tau, n_p, n_m, lists, ind4=ind4)
        Fo = o.symmetrize_fn(Fo)
        ok, e = close(Fg, Fo, 1e-9)
        assert ok, (it, e)
    # the 4-phonon terms change the sweep
    F3 = ctx.iteration(s, ctx.iteration0(s, tau), tau, n_p, n_m, lists)
    F4 = ctx.iteration(s, ctx.iteration0(s, tau), tau, n_p, n_m, lists, ind4=ind4)
    assert np.abs(F4 - F3).max() > 1e-6 * np.abs(F3).max()


def test_ind_driver_4ph_wrong_counts_raise(ctx):
    s = H.cached_solve("diamond", (4, 4, 4))
    n4, _ = ctx.np_driver_4ph(s)
    bad = [x.copy() for x in n4]
    m = int(np.argmax(bad[1]))
    bad[1][m] += 1
    with pytest.raises(abi.FP4Error):
        ctx.ind_driver_4ph(s, *bad)
    g = ctx.ind_driver_4ph(s, *n4)  # the context stays usable
    assert g["rate_4ph"].max() > 0
