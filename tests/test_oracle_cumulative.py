"""Oracle restatement of CumulativeTConduct / CumulativeTConductOmega
(conductivity.f90:64-148) on the CPU: thresholds as the reference computes
them, monotone accumulation, and the last omega tick (above every frequency)
giving exactly TConduct's kappa."""
import numpy as np

import helpers as H
import oracle as O


def test_cumulative_kappa_properties():
    s = H.cached_solve("diamond", (4, 4, 4))
    o = O.Oracle(s)
    n_p, n_m, _, _ = o.np3()
    rp, rm, _, _ = o.rta3()
    rate = rp + rm
    tau = np.zeros_like(rate)
    tau[rate != 0] = 1.0 / rate[rate != 0]
    F = o.iteration0(tau)
    k = o.tconduct(F)
    nt = 100
    ticks, res = o.cumulative_tconduct(F, nt, omega_mode=False)
    ref = np.array([np.float32(10.0) ** np.float32(np.float32(8.0) * (np.float32(i) - np.float32(1.0)) /
                                                    (np.float32(nt) - np.float32(1.0)) - np.float32(2.0))
                    for i in range(1, nt + 1)], dtype=np.float32).astype(np.float64)
    assert np.allclose(ticks, ref, rtol=2e-7, atol=0)
    r = res.reshape(nt, 9 * s.nb)
    # mean free paths (nm) of every mode lie below the last tick (1e6 nm) here
    assert np.allclose(r[-1], k, rtol=1e-12, atol=1e-14 * np.abs(k).max())
    tw, resw = o.cumulative_tconduct(F, nt, omega_mode=True)
    assert np.isclose(tw[-1], 1.1 * s.energy.max(), rtol=1e-15)
    assert np.array_equal(resw.reshape(nt, -1)[-1], k)
    # thresholds grow, and each tick adds whole modes (diagonal kappa never decreases)
    diag = resw.reshape(nt, 3, 3, s.nb)[:, [0, 1, 2], [0, 1, 2], :].sum(axis=(1, 2))
    assert (np.diff(tw) > 0).all() and (np.diff(diag) >= -1e-12 * abs(diag).max()).all()
