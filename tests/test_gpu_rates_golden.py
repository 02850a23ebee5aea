"""The device path end to end against the reference's printed three-phonon
rates: fp4_eigen_dm from the example's FORCE_CONSTANTS_2ND, then fp4_rta_driver
with its FORCE_CONSTANTS_3RD; summed over each degenerate set the rates equal
T300K/BTE.w_3ph_plus, _minus and BTE.w_3ph to their 10 printed digits."""
import numpy as np
import pytest

import harmonic_cases as HC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from fourphonon_b200 import abi
    return abi.Context(0)


@pytest.mark.parametrize("name", ["LiCoO2", "BAs"])
def test_device_harmonic_and_3ph_rates_match_reference_output(ctx, name):
    gh = HC.GoldenHarmonic(name)
    om, vel, eig = ctx.eigen_dm(gh.cr, gh.fc, gh.ngrid, gh.symmetrizers, **gh.kwargs())
    s = gh.solve(om, vel, eig, HC.RUN_SCALEBROAD.get(name))
    r = ctx.rta_driver(s, T=300.0)
    nb = s.nb
    worst, nsets = HC.check_w3(gh, om, r["rate_plus"].reshape(s.nlist, nb), r["rate_minus"].reshape(s.nlist, nb))
    assert nsets > 500 and worst < 1e-9
