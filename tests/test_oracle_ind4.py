"""Oracle restatement of Ind_driver_4ph (processes.f90:3254-3822) and of the
four-phonon Gauss-Seidel sweep iteration_4ph (iterations.f90:95-215), checked
on the CPU against the oracle's own Ind_only and RTA restatements:

* the index lists are the Ind_only_plusplus/plusminus/minusminus lists;
* sum(Gamma) per mode equals the RTA rate (same processes, per-process
  scaling instead of one scaling of the sum) and WP4 is identical;
* a sweep with the 4ph lists differs from the 3ph-only sweep by exactly the
  4ph terms of iteration_4ph, which vanish when every Gamma is zero.
"""
import numpy as np
import pytest

import helpers as H
import oracle as O


@pytest.fixture(scope="module")
def setup():
    s = H.cached_solve("diamond", (4, 4, 4), temperatures=(300.0,))
    o = O.Oracle(s, T=300.0)
    n4, _ = o.np4()
    return s, o, n4, o.ind4(*n4)


def test_ind4_lists_are_ind_only_lists(setup):
    s, o, n4, r = setup
    for ch, key in enumerate(("pp", "pm", "mm")):
        off = np.concatenate([[0], np.cumsum(n4[ch])])
        for mm in range(1, s.nmodes + 1, 5):
            n = int(n4[ch][mm - 1])
            if n == 0:
                continue
            a, b, c, cnt = o.ind_only4(mm, ch, n)
            assert cnt == n
            seg = slice(off[mm - 1], off[mm])
            assert np.array_equal(r["ind2_" + key][seg], a)
            assert np.array_equal(r["ind3_" + key][seg], b)
            assert np.array_equal(r["ind4_" + key][seg], c)


def test_ind4_rates_equal_rta(setup):
    s, o, n4, r = setup
    rta = o.rta4()
    for x, key in enumerate(("pp", "pm", "mm")):
        ref = rta[x]
        assert np.allclose(r["rate_" + key], ref, rtol=1e-12, atol=1e-15 * np.abs(ref).max())
        assert np.array_equal(r["wp_" + key], rta[3 + x])
        off = np.concatenate([[0], np.cumsum(n4[x])])
        sums = np.array([r["gamma_" + key][off[m]:off[m + 1]].sum() for m in range(s.nmodes)])
        assert np.allclose(sums, r["rate_" + key], rtol=1e-13, atol=0)


def test_iteration_4ph_terms(setup):
    s, o, n4, r = setup
    n_p, n_m, _, _ = o.np3()
    lists = o.ind3(n_p, n_m)
    rate = lists["rate_plus"] + lists["rate_minus"] + r["rate_pp"] + r["rate_pm"] + r["rate_mm"]
    tau = np.zeros_like(rate)
    tau[rate != 0] = 1.0 / rate[rate != 0]
    F0 = o.iteration0(tau)
    F3 = o.iteration(F0.copy(), tau, n_p, n_m, lists)
    zero = dict(r)
    for key in ("pp", "pm", "mm"):
        zero["gamma_" + key] = np.zeros_like(r["gamma_" + key])
    F3z = o.iteration(F0.copy(), tau, n_p, n_m, lists, ind4=zero)
    assert np.array_equal(F3, F3z)
    F4 = o.iteration(F0.copy(), tau, n_p, n_m, lists, ind4=r)
    assert np.isfinite(F4).all()
    assert np.abs(F4 - F3).max() > 1e-6 * np.abs(F3).max()
