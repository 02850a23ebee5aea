"""Oracle restatement of the sampled 3ph drivers (NP_plus/minus_sample,
processes.f90:828-979; RTA_plus/minus_sample, 1474-1672) on the CPU: the
seeded stream is reproducible, and the sampled counts, P3 and rates estimate
the full NP_driver / RTA_driver ones within their sampling error."""
import numpy as np

import helpers as H
import oracle as O


def test_sampled_3ph_counts_and_rates_estimate_full_ones():
    s = H.cached_solve("diamond", (4, 4, 4))
    o = O.Oracle(s)
    nm = s.nmodes
    n_p, n_m, p_p, p_m = o.np3()
    a = o.sample3(200_000, 7, mode=0)
    b = o.sample3(200_000, 7, mode=0)
    c = o.sample3(200_000, 8, mode=0)
    assert np.array_equal(a["n"], b["n"]) and np.array_equal(a["p"], b["p"])
    assert not np.array_equal(a["p"], c["p"])
    # the sample space per mode is nb*nptk*nb = 2304 points: 200k draws cover it ~87 times
    for ch, (nf, pf) in enumerate(((n_p, p_p), (n_m, p_m))):
        assert abs(a["n"][ch].sum() / nf.sum() - 1) < 0.01, ch
        assert abs(a["p"][ch].sum() / pf.sum() - 1) < 0.01, ch
    rp, rm, wp, wm = o.rta3()
    r = o.sample3(30_000, 7, mode=2)  # ~13 draws per point of the sample space: ~1% error
    for ch, (rf, wf) in enumerate(((rp, wp), (rm, wm))):
        assert abs(r["rate"][ch].sum() / rf.sum() - 1) < 0.03, ch
        assert abs(r["wp"][ch].sum() / wf.sum() - 1) < 0.03, ch
    assert r["rate"].shape == (2, nm)


def test_sampled_3ph_mode_range_and_gate():
    s = H.cached_solve("diamond", (4, 4, 4))
    o = O.Oracle(s)
    full = o.sample3(2000, 3, mode=2)
    part = o.sample3(2000, 3, mode=2, mm0=6, mm1=12)
    # a mode's draws do not depend on which other modes run
    assert np.array_equal(part["rate"][:, 6:12], full["rate"][:, 6:12])
    assert np.all(part["rate"][:, :6] == 0) and np.all(part["rate"][:, 12:] == 0)
