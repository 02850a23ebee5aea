"""Twenty-four branches: an 8-atom cell, the largest cell of the serving
stream, through the multi-solve serving kernel and the single-solve drivers.

* the server (max_bands=24) serves the 8-atom cell in the same ticks as a
  2-atom one, and each result equals the single-solve drivers' (rates 1e-12,
  kappa 1e-10);
* the single-solve four-phonon rates of the 8-atom cell equal the oracle's on
  the per-q' partial sums of six modes of one irreducible point (FP64 1e-10,
  mixed precision 1e-3 per mode, WP4 1e-10 in every precision);
* the mixed-precision server's kappa is within 1e-4 of the FP64 server's.
"""
import numpy as np
import pytest

import helpers as H
import oracle as O
from fourphonon_b200 import abi, serve

pytestmark = pytest.mark.gpu

RTOL = 1e-12
BUDGET = 32 << 30  # the queues of 24-branch bins take 11 GB on 148 SMs
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
def cells():
    big = H.cached_solve("random8", (4, 4, 4), seed=108)
    small = H.cached_solve("diamond", (4, 4, 4))
    assert big.nb == 24
    return {0: (big, 300.0), 1: (small, 500.0)}


@pytest.fixture(scope="module")
def ctx():
    c = abi.Context(0)
    yield c
    c.close()


def _single(ctx, s, T):
    r3 = ctx.rta_driver(s, T=T)
    r4 = ctx.rta_driver_4ph(s, temperatures=[T])
    rate = r3["rate_plus"] + r3["rate_minus"] + (r4["rate_plusplus"][0] + r4["rate_plusminus"][0]) + \
        r4["rate_minusminus"][0]
    tau = np.zeros_like(rate)
    tau[rate != 0] = 1.0 / rate[rate != 0]
    F = ctx.iteration0(s, tau)
    kap = ctx.tconduct(s, F, T=T).reshape(3, 3, s.nb)
    R = s.sym.crotations
    sym = lambda t: sum(R[r] @ t @ R[r].T for r in range(len(R))) / len(R)  # noqa: E731
    return r3, r4, sum(sym(kap[:, :, b].T) for b in range(s.nb))


def _serve(precision, cells, tick_items):
    srv = serve.Server(0, precision, max_slots=4, max_bands=24, hbm_budget=BUDGET)
    try:
        slots = {srv.admit(s, T): name for name, (s, T) in cells.items()}
        assert None not in slots
        out = {}
        while slots:
            for slot in srv.tick(tick_items):
                out[slots.pop(slot)] = srv.collect(slot)
    finally:
        srv.close()
    return out


def test_server_24_branches_matches_single_solve(ctx, cells):
    got = _serve(abi.FP4_PREC_FP64, cells, tick_items=4000)
    for name, (s, T) in cells.items():
        r3, r4, k = _single(ctx, s, T)
        g = got[name]
        pairs = (("rate3_plus", r3["rate_plus"]), ("rate3_minus", r3["rate_minus"]),
                 ("rate4_pp", r4["rate_plusplus"][0]), ("rate4_pm", r4["rate_plusminus"][0]),
                 ("rate4_mm", r4["rate_minusminus"][0]))
        for key, ref in pairs:
            ok, e = close(g[key], ref, RTOL)
            assert ok, (name, key, e)
        ok, e = close(g["kappa"], k, 1e-10)
        assert ok, (name, "kappa", e)
        assert g["n_processes"] > 0


def test_mixed_server_24_branches_kappa(cells):
    a = _serve(abi.FP4_PREC_FP64, cells, tick_items=20000)
    b = _serve(abi.FP4_PREC_MIXED, cells, tick_items=20000)
    for name in cells:
        ka, kb = a[name]["kappa"], b[name]["kappa"]
        err = np.abs(kb - ka).max() / np.abs(ka).max()
        assert err <= 1e-4, (name, err)


@pytest.fixture(scope="module")
def slice24(cells):
    s = cells[0][0]
    ll, ii0, ii1 = 1, 0, 6  # the second irreducible point, the first six q' points
    b0, b1 = 9, 15  # six optical branches
    mm0 = ll * s.nb
    o = O.Oracle(s, T=300.0).rta4_range(mm0 + b0, mm0 + b1, ii0, ii1)
    return s, ll, ii0, ii1, b0, b1, mm0, o


@pytest.mark.parametrize("precision", [abi.FP4_PREC_FP64, abi.FP4_PREC_MIXED, abi.FP4_PREC_MIXED_SIMT])
def test_rates_24_branches_against_oracle(slice24, precision):
    s, ll, ii0, ii1, b0, b1, mm0, o = slice24
    c = abi.Context(0, precision)
    try:
        c.rta_driver_4ph(s, temperatures=[300.0])
        g = c.rta4_partials(s, ll, ii0, ii1, 0)
    finally:
        c.close()
    rtol = 1e-10 if precision == abi.FP4_PREC_FP64 else 1e-3
    errs = []
    for x, name in enumerate(CH):
        ref = o[x][mm0 + b0:mm0 + b1]
        assert (ref > 0).any(), name
        ok, e = close(g[name][b0:b1], ref, rtol)
        errs.append(e)
        assert ok, (name, e)
    for x, name in enumerate(WP):
        ok, e = close(g[name][b0:b1], o[3 + x][mm0 + b0:mm0 + b1], 1e-10)
        assert ok, (name, e)
    print("24-branch rate error vs oracle:", precision, max(errs))
