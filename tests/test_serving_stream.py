"""The request stream of the serving workload and its random cells (CPU).

* system.config4_stream draws the 512 requests reproducibly: 2-8 atoms, grids
  from {6,8,10,12,14}^3, T in [100, 1000] K;
* every random cell is mechanically stable under the seeded BvK springs (the
  per-atom spring shells bond every atom): three zero modes at Gamma only;
* the cost model that picks the served prefix grows with the grid and the
  branch count.
"""
import numpy as np
import pytest

import helpers  # noqa: F401  (puts the repository on the path)
from fourphonon_b200 import system as S


def test_stream_is_reproducible_and_in_range():
    a = S.config4_stream(512)
    b = S.config4_stream(512)
    assert a == b and len(a) == 512
    nat = np.array([r[0] for r in a])
    grid = np.array([r[1] for r in a])
    T = np.array([r[2] for r in a])
    assert nat.min() >= 2 and nat.max() <= 8 and len(set(nat)) == 7
    assert set(grid) == {6, 8, 10, 12, 14}
    assert T.min() >= 100.0 and T.max() <= 1000.0
    assert S.config4_stream(512, seed=1) != a


@pytest.mark.parametrize("natoms", [2, 3, 5, 7, 8])
def test_random_cells_are_stable(natoms):
    s = S.random_solve(natoms=natoms, ngrid=(4, 4, 4), seed=100 + natoms)
    w = np.asarray(s.energy)  # (nptk, nb), q = 0 is Gamma
    assert np.all(np.abs(w[0, :3]) < 1e-6)
    assert w[0, 3:].min() > 0.5
    assert w[1:].min() > 0.5, w[1:].min()
    assert s.ifc3.ntri > 0 and s.ifc4.ntri > 0


def test_cost_model_grows_with_grid_and_branches():
    t = [S.request_seconds(2, g) for g in (6, 8, 10, 12, 14)]
    assert all(x < y for x, y in zip(t, t[1:]))
    u = [S.request_seconds(n, 8) for n in range(2, 9)]
    assert all(x < y for x, y in zip(u, u[1:]))
    # the 16^3 diamond step the constants come from: about 10 s
    assert 5.0 < S.request_seconds(2, 16, nlist=145) < 20.0
