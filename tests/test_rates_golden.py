"""Three-phonon RTA rates against the reference's own printed rates.

The harmonic stage (the numpy restatement of eigenDM, itself pinned to the
examples' BTE.omega and BTE.v_full) and the example's FORCE_CONSTANTS_3RD feed
the oracle's RTA_driver restatement; its rates, summed over each degenerate
set, must equal T300K/BTE.w_3ph_plus, _minus and BTE.w_3ph to their 10 printed
digits.  This pins the three-phonon matrix elements, weights and constants to
reference data.
"""
import numpy as np
import pytest

import harmonic_cases as HC
import oracle as O
from fourphonon_b200 import harmonic as HM


@pytest.mark.parametrize("name,points", [("LiCoO2", None), ("BAs", 24)])
def test_oracle_3ph_rates_match_reference_output(name, points):
    gh = HC.GoldenHarmonic(name)
    om, vel, eig = HM.eigen_dm(gh.cr, gh.fc, gh.ngrid, gh.symmetrizers, **gh.kwargs())
    s = gh.solve(om, vel, eig, HC.RUN_SCALEBROAD.get(name))
    assert np.array_equal(s.wedge.list, gh.z["list"])  # the same irreducible points, in the same order
    nb = s.nb
    rp, rm, _, _ = O.Oracle(s).rta3(0, None if points is None else points * nb)
    worst, nsets = HC.check_w3(gh, om, rp.reshape(s.nlist, nb), rm.reshape(s.nlist, nb), points)
    assert nsets > 100 and worst < 1e-9
