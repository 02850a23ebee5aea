"""End to end: the ShengBTE rate/BTE/kappa section on the device path
(fourphonon_b200.driver.run) against the same sequence driven through the
oracle (counts, Ind_driver lists, 4ph RTA or, with four_phonon_iteration,
the Ind_driver_4ph lists and iteration_4ph sweeps, tau_zero, iteration0,
TConduct, symmetrize_tensor, Gauss-Seidel sweeps until the relative change
< eps)."""
import os

import numpy as np
import pytest

import helpers as H
import oracle as O
from fourphonon_b200 import driver

pytestmark = pytest.mark.gpu


def _oracle_sequence(s, T, maxiter=50, eps=float(np.float32(1e-5)), it4=False):
    o = O.Oracle(s, T=T)
    n_p, n_m, _, _ = o.np3()
    lists = o.ind3(n_p, n_m)
    ind4 = None
    if it4:
        ind4 = o.ind4(*o.np4()[0])
        r4 = (ind4["rate_pp"], ind4["rate_pm"], ind4["rate_mm"])
    else:
        r4 = o.rta4()
    rate = lists["rate_plus"] + lists["rate_minus"] + r4[0] + r4[1] + r4[2]
    tau = np.zeros_like(rate)
    tau[rate != 0] = 1.0 / rate[rate != 0]
    F = o.iteration0(tau)

    def kappa(F):
        k = o.tconduct(F).reshape(3, 3, s.nb)
        return sum(o.symmetrize_tensor(k[:, :, b].T) for b in range(s.nb))

    k_rta = kappa(F)
    k = k_rta
    it = 0
    for it in range(1, maxiter + 1):
        kold = k
        F = o.iteration(F, tau, n_p, n_m, lists, ind4=ind4)
        F = o.symmetrize_fn(F)
        k = kappa(F)
        rel = np.linalg.svd(k - kold, compute_uv=False)[0] / np.linalg.svd(kold, compute_uv=False)[0]
        if rel < eps:
            break
    return k_rta, k, it


@pytest.mark.parametrize("it4", [False, True])
def test_driver_matches_oracle_sequence(tmp_path, it4):
    s = H.cached_solve("diamond", (4, 4, 4), temperatures=(300.0,))
    res = driver.run(s, str(tmp_path), convergence=True, four_phonon=True, maxiter=50, log=lambda *a: None,
                     four_phonon_iteration=it4)
    k_rta, k_conv, it = _oracle_sequence(s, 300.0, it4=it4)
    r = res[0]
    assert np.allclose(r["kappa_rta"], k_rta, rtol=1e-9, atol=1e-12 * np.abs(k_rta).max())
    assert r["iterations"] == it
    assert np.allclose(r["kappa_conv"], k_conv, rtol=1e-8, atol=1e-11 * np.abs(k_conv).max())
    for name in ("BTE.Numprocess_4ph", "BTE.P3", "BTE.P4", "BTE.KappaTensorVsT_RTA", "BTE.KappaTensorVsT_CONV",
                 os.path.join("T300K", "BTE.w_3ph"), os.path.join("T300K", "BTE.w_4ph"),
                 os.path.join("T300K", "BTE.kappa"), os.path.join("T300K", "BTE.kappa_scalar")):
        assert os.path.getsize(os.path.join(str(tmp_path), name)) > 0, name
    # BTE.w_4ph holds (omega, rate) pairs in E20.10, branch-major like the reference
    rows = open(os.path.join(str(tmp_path), "T300K", "BTE.w_4ph")).read().splitlines()
    assert len(rows) == s.nmodes and all(len(x) == 40 for x in rows)
