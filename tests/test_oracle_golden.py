"""The oracle against the reference's own golden outputs (CPU).

The harmonic inputs are the reference's printed BTE.omega / BTE.v_full of its
example runs (10 significant digits), so a handful of candidates that sit
within rounding of the filter threshold may flip; everything else must match
the reference's log.out counts, BTE.Numprocess_4ph and phase spaces.
"""
import numpy as np
import pytest

import helpers as H
import oracle as O


def test_licoo2_3ph_counts_exact():
    g = H.GoldenSolve("LiCoO2")
    n_p, n_m, p_p, p_m = O.Oracle(g).np3()
    assert int(n_p.sum()) == int(g.z["ntotal_plus"]) == 93181
    assert int(n_m.sum()) == int(g.z["ntotal_minus"]) == 126112
    for mine, key in ((p_p, "P3_plus"), (p_m, "P3_minus")):
        ref = g.z[key].ravel()
        assert np.abs(mine - ref).max() <= 1e-5 * ref.max()


def test_bas_3ph_counts_with_run_broadening():
    # The BAs example outputs were produced with scalebroad=1 (its CONTROL says 0.1).
    g = H.GoldenSolve("BAs")
    g.scalebroad = 1.0
    n_p, n_m, _, _ = O.Oracle(g).np3()
    assert abs(int(n_p.sum()) - int(g.z["ntotal_plus"])) <= 4
    assert int(n_m.sum()) == int(g.z["ntotal_minus"])


def test_licoo2_4ph_counts_per_mode():
    g = H.GoldenSolve("LiCoO2")
    mm0, mm1 = 16, 20  # modes 17..20 (1-based)
    n, p = O.Oracle(g).np4(mm0, mm1)
    gold = g.z["numprocess_4ph"]  # line L holds mode L
    for ch in range(3):
        for m in range(mm0, mm1):
            ref = int(gold[m, ch])
            assert abs(int(n[ch][m]) - ref) <= max(2, int(1e-5 * ref)), (ch, m, int(n[ch][m]), ref)
    for ch, key in enumerate(("P4_pp", "P4_pm", "P4_mm")):
        ref = g.z[key].ravel()[mm0:mm1]
        assert np.abs(p[ch][mm0:mm1] - ref).max() <= 1e-5 * ref.max()
