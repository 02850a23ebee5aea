"""The device eigenDM (fp4_eigen_dm) against the reference's printed outputs
and against the numpy restatement (LAPACK eigensolver)."""
import numpy as np
import pytest

import harmonic_cases as HC

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from fourphonon_b200 import abi
    return abi.Context(0)


@pytest.mark.parametrize("name", ["LiCoO2", "BAs"])
def test_device_eigen_dm_matches_reference_output(ctx, name):
    gh = HC.GoldenHarmonic(name)
    om, vel, eig = ctx.eigen_dm(gh.cr, gh.fc, gh.ngrid, gh.symmetrizers, **gh.kwargs())
    HC.check_against_golden(gh, om, vel)
    ref = HC.numpy_eigen_dm(gh.cr, gh.fc, gh.ngrid, gh.symmetrizers, **gh.kwargs())
    HC.compare_harmonic((om, vel, eig), ref, omega_rtol=1e-11, vec_tol=1e-7, vel_rtol=1e-8)
    nb = om.shape[1]
    g = np.einsum("qnc,qmc->qnm", eig.conj(), eig)
    assert np.abs(g - np.eye(nb)[None]).max() < 1e-12


@pytest.mark.parametrize("kind,ngrid,seed", [("diamond", (6, 6, 6), 11), ("layered", (4, 4, 4), 12),
                                             ("random4", (4, 4, 4), 13), ("random8", (3, 3, 3), 14)])
def test_device_eigen_dm_matches_numpy(ctx, kind, ngrid, seed):
    cr, fc, sym = HC.synthetic(kind, ngrid, seed)
    dev = ctx.eigen_dm(cr, fc, ngrid, sym)
    ref = HC.numpy_eigen_dm(cr, fc, ngrid, sym)
    HC.compare_harmonic(dev, ref, omega_rtol=1e-11, vec_tol=1e-7, vel_rtol=1e-8)
    assert np.all(dev[0][0, :3] == 0.0) and np.all(dev[1][0, :3] == 0.0)


def test_device_eigen_dm_dielectric_synthetic(ctx):
    # random Born charges (acoustic sum over atoms zero) and a random epsilon
    cr, fc, sym = HC.synthetic("random3", (4, 4, 4), 21)
    rng = np.random.default_rng(5)
    born = rng.normal(scale=0.8, size=(3, 3, cr.natoms))
    born -= born.mean(axis=2, keepdims=True)
    a = rng.normal(size=(3, 3))
    eps = 4.0 * np.eye(3) + 0.5 * (a + a.T)
    kw = dict(born=born, epsilon=eps, nonanalytic=True)
    dev = ctx.eigen_dm(cr, fc, (4, 4, 4), sym, **kw)
    ref = HC.numpy_eigen_dm(cr, fc, (4, 4, 4), sym, **kw)
    HC.compare_harmonic(dev, ref, omega_rtol=1e-11, vec_tol=1e-7, vel_rtol=1e-8)


def test_device_eigen_dm_rejects_bad_arguments(ctx):
    from fourphonon_b200 import abi
    cr, fc, sym = HC.synthetic("diamond", (2, 2, 2), 1)
    with pytest.raises(abi.FP4Error):
        ctx.eigen_dm(cr, fc, (2, 2, 2), sym, nonanalytic=True, V=-1.0)
