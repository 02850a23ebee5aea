"""A non-cubic grid (3x3x4 on the diamond cell) through the host side and the
oracle (CPU): the symmetry operations kept are those that map the grid onto
itself, the irreducible wedge covers every grid point once, and the oracle's
Ind_driver_4ph restatement agrees with its RTA restatement there (lists and
per-mode sums), as it does on cubic grids."""
import numpy as np

import oracle as O
from fourphonon_b200 import system as S


def test_noncubic_wedge_and_oracle_consistency():
    s = S.diamond_solve(ngrid=(3, 3, 4), temperatures=(300.0,))
    assert s.nptk == 36
    assert 1 < s.sym.nsymm_rot < 48  # the cubic operations that mix z with x or y are gone
    assert int(np.sum(s.wedge.nequi)) == s.nptk
    # ALLEquiList(nlist, nsymm_rot): the first nequi entries of each row are its star
    seen = np.zeros(s.nptk, int)
    for ll in range(s.nlist):
        for kk in range(int(s.wedge.nequi[ll])):
            seen[int(s.wedge.allequi[ll, kk]) - 1] += 1
    assert (seen == 1).all()
    o = O.Oracle(s)
    n4, _ = o.np4()
    r = o.rta4()
    ind4 = o.ind4(*n4)
    for x, k in enumerate(("pp", "pm", "mm")):
        assert int(n4[x].sum()) > 0
        assert np.allclose(ind4["rate_" + k], r[x], rtol=1e-12, atol=1e-15 * np.abs(r[x]).max())
        assert np.array_equal(ind4["wp_" + k], r[3 + x])
