"""CumulativeTConduct / CumulativeTConductOmega on the device (C-ABI) against
the oracle: thresholds bit-exact, cumulative kappa within 1e-12."""
import numpy as np
import pytest

import helpers as H
import oracle as O
from fourphonon_b200 import abi

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("omega_mode", [False, True])
def test_cumulative_tconduct(omega_mode):
    s = H.cached_solve("diamond", (6, 6, 6), temperatures=(300.0, 700.0))
    o = O.Oracle(s, T=700.0)
    rp, rm, _, _ = o.rta3()
    rate = rp + rm
    tau = np.zeros_like(rate)
    tau[rate != 0] = 1.0 / rate[rate != 0]
    F = o.iteration0(tau)
    c = abi.Context(0)
    tg, rg = c.cumulative_tconduct(s, F, T=700.0, nticks=100, omega_mode=omega_mode)
    c.close()
    to, ro = o.cumulative_tconduct(F, 100, omega_mode=omega_mode)
    assert np.array_equal(tg, to)
    scale = np.abs(ro).max()
    assert np.all(np.abs(rg - ro) <= 1e-12 * np.abs(ro) + 1e-14 * scale)
