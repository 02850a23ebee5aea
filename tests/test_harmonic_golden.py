"""The numpy restatement of eigenDM / phonon_phonopy against the reference's
printed frequencies and velocities of its LiCoO2 (no dielectric correction:
its CONTROL gives no Born charges) and BAs (dielectric correction) examples."""
import numpy as np
import pytest

import harmonic_cases as HC
from fourphonon_b200 import harmonic as HM


@pytest.mark.parametrize("name", ["LiCoO2", "BAs"])
def test_eigen_dm_matches_reference_output(name):
    gh = HC.GoldenHarmonic(name)
    om, vel, eig = HM.eigen_dm(gh.cr, gh.fc, gh.ngrid, gh.symmetrizers, **gh.kwargs())
    HC.check_against_golden(gh, om, vel)
    # eigenvectors are orthonormal at every q
    nb = om.shape[1]
    g = np.einsum("qnc,qmc->qnm", eig.conj(), eig)
    assert np.abs(g - np.eye(nb)[None]).max() < 1e-12


def test_bas_dielectric_correction_is_needed():
    # without the correction the LO-TO splitting near Gamma is missing
    gh = HC.GoldenHarmonic("BAs")
    kw = gh.kwargs()
    kw["nonanalytic"] = False
    om, vel, _ = HM.eigen_dm(gh.cr, gh.fc, gh.ngrid, gh.symmetrizers, **kw)
    lst = gh.z["list"] - 1
    assert np.abs(om[lst] - gh.z["energy"][lst]).max() > 1e-3


def test_first_zone_image_ties_follow_the_reference():
    # q points with two images of equal length: the extended-precision norm
    # keeps the reference's choice; count them so the golden test above covers ties
    gh = HC.GoldenHarmonic("BAs")
    k = HM.kspace(gh.cr, gh.ngrid, gh.rl)
    norms = []
    for ix in range(-2, 3):
        for iy in range(-2, 3):
            for iz in range(-2, 3):
                norms.append(np.linalg.norm(k + ix * gh.rl[:, 0] + iy * gh.rl[:, 1] + iz * gh.rl[:, 2], axis=1))
    norms = np.array(norms)
    mn = norms.min(0)
    ties = ((norms <= mn * (1 + 1e-12)).sum(0) > 1).sum()
    assert ties > 200
