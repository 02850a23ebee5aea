"""The host side of fourphonon_b200.driver.run on the CPU.

driver.run strings the C-ABI calls together the way ShengBTE.f90 strings the
Fortran routines (counts, rates per temperature, tau, iteration0, TConduct,
the Gauss-Seidel loop and its stop test, the BTE.* files).  Here every call
is answered by the oracle instead of the device (OracleContext, test-only),
so the sequencing, the convergence loop, the file formats and the metrics
stream are checked without a GPU.  The device path itself is checked by
tests/test_gpu_driver.py.
"""
import io
import json
import os

import numpy as np
import pytest

import helpers as H
import oracle as O
from fourphonon_b200 import driver


class OracleContext:
    """The abi.Context calls that driver.run makes, answered by the oracle."""

    def __init__(self, s):
        self.s = s
        self._o = {}

    def _at(self, T=None):
        T = float(self.s.temperatures[0] if T is None else T)
        if T not in self._o:
            self._o[T] = O.Oracle(self.s, T=T)
        return self._o[T]

    def np_driver(self, s):
        return self._at().np3()

    def np_driver_4ph(self, s):
        return self._at().np4()

    def rta_driver(self, s, T=None):
        r = self._at(T).rta3()
        return dict(rate=r[0] + r[1], rate_plus=r[0], rate_minus=r[1], wp3_plus=r[2], wp3_minus=r[3])

    def ind_driver(self, s, n_plus, n_minus, T=None):
        d = self._at(T).ind3(n_plus, n_minus)
        d["rate"] = d["rate_plus"] + d["rate_minus"]
        return d

    def rta_driver_4ph(self, s, temperatures=None):
        temps = s.temperatures if temperatures is None else temperatures
        per_t = [self._at(T).rta4() for T in temps]
        names = ("rate_plusplus", "rate_plusminus", "rate_minusminus", "wp4_plusplus", "wp4_plusminus",
                 "wp4_minusminus")
        d = {k: np.stack([r[x] for r in per_t]) for x, k in enumerate(names)}
        d["rate_4ph"] = d["rate_plusplus"] + d["rate_plusminus"] + d["rate_minusminus"]
        return d

    def ind_driver_4ph(self, s, n_pp, n_pm, n_mm, T=None):
        return self._at(T).ind4(n_pp, n_pm, n_mm)

    def iteration0(self, s, tau_zero):
        return self._at().iteration0(tau_zero)

    def iteration(self, s, F, tau_zero, n_plus, n_minus, lists, ind4=None):
        return self._at().iteration(F, tau_zero, n_plus, n_minus, lists, ind4=ind4)

    def symmetrize_fn(self, s, F):
        return self._at().symmetrize_fn(F)

    def tconduct(self, s, F, T=None):
        return self._at(T).tconduct(F)

    def cumulative_tconduct(self, s, F, T=None, nticks=100, omega_mode=False):
        return self._at(T).cumulative_tconduct(F, nticks=nticks, omega_mode=omega_mode)


def _by_hand(s, T, it4, maxiter=50, eps=float(np.float32(1e-5))):
    """The ShengBTE sequence written out directly against the oracle."""
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

    k_rta = k = kappa(F)
    it = 0
    for it in range(1, maxiter + 1):
        kold = k
        F = o.symmetrize_fn(o.iteration(F, tau, n_p, n_m, lists, ind4=ind4))
        k = kappa(F)
        if np.linalg.svd(k - kold, compute_uv=False)[0] / np.linalg.svd(kold, compute_uv=False)[0] < eps:
            break
    return k_rta, k, it


@pytest.fixture(scope="module")
def cell():
    return H.cached_solve("diamond", (3, 3, 3), temperatures=(300.0, 500.0))


@pytest.mark.parametrize("it4", [False, True])
def test_driver_sequence_files_and_metrics(tmp_path, cell, it4):
    s = cell
    out = io.StringIO()
    res = driver.run(s, str(tmp_path), convergence=True, four_phonon=True, maxiter=50, ctx=OracleContext(s),
                     log=lambda *a: None, four_phonon_iteration=it4, metrics=out)
    assert [r["T"] for r in res] == list(s.temperatures)
    for t, T in enumerate(s.temperatures):
        k_rta, k_conv, it = _by_hand(s, T, it4)
        r = res[t]
        assert np.allclose(r["kappa_rta"], k_rta, rtol=1e-12, atol=1e-14 * np.abs(k_rta).max())
        assert r["iterations"] == it
        assert np.allclose(r["kappa_conv"], k_conv, rtol=1e-12, atol=1e-14 * np.abs(k_conv).max())
        tdir = os.path.join(str(tmp_path), f"T{int(T)}K")
        for name in ("BTE.w_3ph", "BTE.w_4ph", "BTE.w", "BTE.w_final", "BTE.WP3", "BTE.WP4"):
            rows = open(os.path.join(tdir, name)).read().splitlines()
            assert len(rows) == s.nmodes, name
        assert all(len(x) == 40 for x in open(os.path.join(tdir, "BTE.w_4ph")).read().splitlines())
        kap = open(os.path.join(tdir, "BTE.kappa_scalar")).read().splitlines()
        assert len(kap) == it + 1 and kap[0].startswith(f"{0:9d}")
        assert len(open(os.path.join(tdir, "BTE.cumulative_kappa_tensor")).read().splitlines()) == 100
    for name, n in (("BTE.KappaTensorVsT_RTA", 2), ("BTE.KappaTensorVsT_CONV", 2)):
        rows = open(os.path.join(str(tmp_path), name)).read().splitlines()
        assert len(rows) == n and rows[0].startswith(f"{300.0:7.1f}")
    assert os.path.getsize(os.path.join(str(tmp_path), "BTE.Numprocess_4ph")) > 0
    events = [json.loads(x) for x in out.getvalue().splitlines()]
    assert all(e["event"] == "stage" and e["seconds"] >= 0 for e in events)
    names = [e["stage"] for e in events]
    assert names[:2] == ["np_driver", "np_driver_4ph"]
    assert ("rta_driver_4ph" in names) != it4 and ("ind_driver_4ph" in names) == it4
    its = [e for e in events if e["stage"] == "iterations"]
    assert [e["iterations"] for e in its] == [r["iterations"] for r in res]
    assert names.count("outputs") == len(s.temperatures)


def test_driver_rta_only_three_phonon(tmp_path, cell):
    """convergence=.false. and four_phonon=.false.: RTA_driver per temperature,
    no BTE loop, no four-phonon files and no KappaTensorVsT_CONV."""
    s = cell
    res = driver.run(s, str(tmp_path), convergence=False, four_phonon=False, ctx=OracleContext(s),
                     log=lambda *a: None)
    for t, T in enumerate(s.temperatures):
        o = O.Oracle(s, T=T)
        r3 = o.rta3()
        assert np.array_equal(res[t]["rate3"], r3[0] + r3[1])
        assert not res[t]["rate4"].any()
        assert "kappa_conv" not in res[t]
        tdir = os.path.join(str(tmp_path), f"T{int(T)}K")
        assert not os.path.exists(os.path.join(tdir, "BTE.w_4ph"))
        assert len(open(os.path.join(tdir, "BTE.kappa_scalar")).read().splitlines()) == 1
    assert not os.path.exists(os.path.join(str(tmp_path), "BTE.KappaTensorVsT_CONV"))
    assert len(open(os.path.join(str(tmp_path), "BTE.KappaTensorVsT_RTA")).read().splitlines()) == 2


def test_input_directory_to_outputs(tmp_path):
    """A FourPhonon input directory (CONTROL, FORCE_CONSTANTS_2ND/3RD/4TH) through
    system.load_inputs (numpy harmonic stage) and driver.run to the BTE.* files,
    as a user runs it; the rates come from the oracle here, from the device in
    production."""
    from fourphonon_b200 import crystal as C
    from fourphonon_b200 import ifcgen as G
    from fourphonon_b200 import inputs as I
    from fourphonon_b200 import system as S

    cr = C.diamond(5.43, (28.085, 28.085))
    cr.scell = (3, 3, 3)
    blocks = G.bvk_fc2(cr, [3.0, 0.45])
    shells = G.shell_distances(cr, 4)
    cl3 = G.generate_anharmonic(cr, 3, 0.5 * (shells[2] + shells[3]), 5.0, 11)
    cl4 = G.generate_anharmonic(cr, 4, 0.5 * (shells[0] + shells[1]), 2.0, 12)
    inp = tmp_path / "input"
    inp.mkdir()
    I.write_control(inp / "CONTROL", cr, (3, 3, 3), T=300.0, scalebroad=1.0, four_phonon=True)
    G.write_fc2_phonopy(inp / "FORCE_CONSTANTS_2ND", cr, blocks)
    G.write_fc_anharmonic(inp / "FORCE_CONSTANTS_3RD", cr, cl3)
    G.write_fc_anharmonic(inp / "FORCE_CONSTANTS_4TH", cr, cl4)
    s = S.load_inputs(str(inp))
    out = tmp_path / "output"
    res = driver.run(s, str(out), convergence=True, four_phonon=True, maxiter=50, ctx=OracleContext(s),
                     log=lambda *a: None)
    k_rta, k_conv, it = _by_hand(s, 300.0, it4=False)
    assert np.allclose(res[0]["kappa_conv"], k_conv, rtol=1e-12, atol=1e-14 * np.abs(k_conv).max())
    assert res[0]["iterations"] == it
    assert np.isfinite(res[0]["kappa_conv"]).all() and np.trace(res[0]["kappa_conv"]) > 0
    for name in ("BTE.Numprocess_4ph", "BTE.P3", "BTE.P4", "BTE.KappaTensorVsT_RTA", "BTE.KappaTensorVsT_CONV",
                 os.path.join("T300K", "BTE.w_4ph"), os.path.join("T300K", "BTE.kappa_tensor")):
        assert os.path.getsize(os.path.join(str(out), name)) > 0, name
