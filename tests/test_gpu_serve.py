"""The serving path on the device: several solves resident at once, their
4ph work packed into shared launches of the multi-solve kernel.

* each result equals the single-solve drivers' (fp4_rta_driver, fp4_rta_driver_4ph,
  iteration0 + TConduct + symmetrize_tensor) within 1e-12 relative;
* a solve's result is the same alone and in a mix with others (1e-12);
* admission waits for HBM budget and slots;
* the mixed-precision server's kappa is within 1e-4 of the FP64 one.
"""
import numpy as np
import pytest

import helpers as H
from fourphonon_b200 import abi, serve

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def close(a, b, rtol):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = np.abs(b).max() if b.size else 0.0
    return bool((np.abs(a - b) <= rtol * np.abs(b) + 1e-3 * rtol * scale).all())


def _solves():
    return [(H.cached_solve("diamond", (4, 4, 4)), 300.0), (H.cached_solve("zincblende", (4, 4, 4), (500.0,)), 500.0),
            (H.cached_solve("layered", (4, 4, 4)), 300.0)]


def _reference(ctx, s, T):
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
    kb = np.stack([sym(kap[:, :, b].T) for b in range(s.nb)])
    return r3, r4, kb, kb.sum(axis=0)


def _serve_all(srv, items, tick_items):
    slots = {}
    for name, (s, T) in items.items():
        slot = srv.admit(s, T)
        assert slot is not None
        slots[slot] = name
    out = {}
    while slots:
        for slot in srv.tick(tick_items):
            out[slots.pop(slot)] = srv.collect(slot)
    return out


@pytest.fixture(scope="module")
def ctx():
    c = abi.Context(0)
    yield c
    c.close()


def test_server_matches_single_solve_drivers(ctx):
    srv = serve.Server(0, abi.FP4_PREC_FP64, max_slots=4, max_bands=12)
    items = {i: st for i, st in enumerate(_solves())}
    got = _serve_all(srv, items, tick_items=5000)
    srv.close()
    for i, (s, T) in items.items():
        r3, r4, kb, k = _reference(ctx, s, T)
        g = got[i]
        assert close(g["rate3_plus"], r3["rate_plus"], RTOL)
        assert close(g["rate3_minus"], r3["rate_minus"], RTOL)
        assert close(g["rate4_pp"], r4["rate_plusplus"][0], RTOL)
        assert close(g["rate4_pm"], r4["rate_plusminus"][0], RTOL)
        assert close(g["rate4_mm"], r4["rate_minusminus"][0], RTOL)
        assert close(g["kappa_branch"], kb, 1e-10)
        assert close(g["kappa"], k, 1e-10)
        assert g["n_processes"] > 0


def test_same_result_alone_and_in_the_mix():
    srv = serve.Server(0, abi.FP4_PREC_FP64, max_slots=4, max_bands=12)
    sol = _solves()
    alone = {i: _serve_all(srv, {i: sol[i]}, tick_items=3000)[i] for i in range(len(sol))}
    mixed = _serve_all(srv, {i: sol[i] for i in range(len(sol))}, tick_items=3000)
    srv.close()
    for i in range(len(sol)):
        for k in ("rate3_plus", "rate3_minus", "rate4_pp", "rate4_pm", "rate4_mm", "kappa"):
            assert close(mixed[i][k], alone[i][k], RTOL), (i, k)


def test_admission_waits_for_budget():
    s, T = _solves()[0]
    fp = serve.footprint(s)
    probe = serve.Server(0, abi.FP4_PREC_FP64, max_slots=4, max_bands=6, hbm_budget=64 << 30)
    fixed = probe.status()["bytes_in_use"]
    probe.close()
    srv = serve.Server(0, abi.FP4_PREC_FP64, max_slots=4, max_bands=6, hbm_budget=fixed + fp + fp // 2)
    a = srv.admit(s, T)
    assert a is not None
    assert srv.admit(s, T) is None  # the second copy does not fit until the first is collected
    done = []
    while not done:
        done = srv.tick(10 ** 9)
    srv.collect(done[0])
    assert srv.admit(s, T) is not None
    srv.close()


def test_mixed_server_kappa_within_1e_4():
    sol = _solves()
    s64 = serve.Server(0, abi.FP4_PREC_FP64, max_slots=4, max_bands=12)
    smx = serve.Server(0, abi.FP4_PREC_MIXED, max_slots=4, max_bands=12)
    a = _serve_all(s64, dict(enumerate(sol)), 20000)
    b = _serve_all(smx, dict(enumerate(sol)), 20000)
    s64.close()
    smx.close()
    for i in range(len(sol)):
        ka, kb = a[i]["kappa"], b[i]["kappa"]
        assert np.abs(kb - ka).max() <= 1e-4 * np.abs(ka).max()


def test_run_stream_latencies():
    sol = _solves()
    rng = np.random.default_rng(7)
    arrivals = np.cumsum(rng.exponential(0.02, size=6))
    reqs = [serve.Request(float(t), *sol[i % 3], tag=i) for i, t in enumerate(arrivals)]
    srv = serve.Server(0, abi.FP4_PREC_MIXED, max_slots=3, max_bands=12)
    done, summary = serve.run_stream(srv, reqs, tick_items=4000)
    srv.close()
    assert all(r.finished >= r.admitted >= r.arrival for r in done)
    assert summary["p99_ms"] >= summary["p50_ms"] > 0
    assert summary["processes"] > 0
