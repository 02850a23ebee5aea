"""Sampled three-phonon drivers (NP_plus/minus_sample, RTA_plus/minus_sample)
on the device against the oracle drawing the same samples from the same
seeded stream: sampled counts exact, P3, rates and WP3 within 1e-10."""
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


def test_sampled_3ph_np_matches_oracle(ctx):
    s = H.cached_solve("diamond", (4, 4, 4))
    ns, seed = 100_000, 31
    n_p, n_m, p_p, p_m = ctx.np_driver_sample(s, ns, seed)
    o = O.Oracle(s).sample3(ns, seed, mode=0)
    assert np.array_equal(n_p, o["n"][0]) and np.array_equal(n_m, o["n"][1])
    assert close(p_p, o["p"][0], 1e-10) and close(p_m, o["p"][1], 1e-10)
    assert n_p.sum() > 0 and n_m.sum() > 0


def test_sampled_3ph_rta_matches_oracle(ctx):
    s = H.cached_solve("diamond", (4, 4, 4))
    ns, seed = 20_000, 5
    g = ctx.rta_driver_sample(s, ns, seed)
    o = O.Oracle(s).sample3(ns, seed, mode=2)
    assert close(g["rate_plus"], o["rate"][0], 1e-10) and close(g["rate_minus"], o["rate"][1], 1e-10)
    assert close(g["wp3_plus"], o["wp"][0], 1e-10) and close(g["wp3_minus"], o["wp"][1], 1e-10)
    assert np.allclose(g["rate"], g["rate_plus"] + g["rate_minus"], rtol=0, atol=0)
    full = ctx.rta_driver(s)
    # an estimate of the full enumeration: ~9 draws per point of the sample space
    assert abs(g["rate"].sum() / full["rate"].sum() - 1) < 0.05


def test_sampled_3ph_rejects_bad_sample_count(ctx):
    s = H.cached_solve("diamond", (4, 4, 4))
    with pytest.raises(abi.FP4Error):
        ctx.np_driver_sample(s, 0, 1)
