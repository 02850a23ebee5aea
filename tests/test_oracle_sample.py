"""Oracle restatement of the sampled 4ph drivers (NP_*_sample,
processes.f90:2480-2746) on the CPU: the seeded stream is reproducible, and
the sampled counts and P4 estimate the full NP_driver_4ph ones within their
sampling error."""
import numpy as np

import helpers as H
import oracle as O


def test_sampled_counts_estimate_full_counts():
    s = H.cached_solve("diamond", (4, 4, 4))
    o = O.Oracle(s)
    n4, p4 = o.np4()
    a = o.sample4(200_000, 99, mode=0)
    b = o.sample4(200_000, 99, mode=0)
    c = o.sample4(200_000, 100, mode=0)
    assert np.array_equal(a["n"], b["n"]) and np.array_equal(a["p"], b["p"])
    assert not np.array_equal(a["n"], c["n"])
    for ch in range(3):
        full, est = n4[ch].sum(), a["n"][ch].sum()
        # the draws cover ~23% of the sample space here: a few per mille statistical error
        assert abs(est / full - 1) < 0.03, (ch, full, est)
        assert abs(a["p"][ch].sum() / p4[ch].sum() - 1) < 0.03
