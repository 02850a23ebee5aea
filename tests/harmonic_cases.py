"""Inputs of the harmonic stage for the tests: the reference's examples with a
Phonopy FORCE_CONSTANTS_2ND (stored in the golden fixtures) and seeded
synthetic cells, with the comparisons that tolerate LAPACK's freedom in the
eigenvectors (a phase per branch, a basis per degenerate set)."""
import os

import numpy as np

from fourphonon_b200 import crystal as C
from fourphonon_b200 import harmonic as HM
from fourphonon_b200 import ifcgen as G
from fourphonon_b200 import system as S

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class GoldenHarmonic:
    """Crystal, fc array, dielectric inputs and the reference's printed
    omega / v_full of one example."""

    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
        self.z = z
        self.cr = C.Crystal(z["lattvec"], z["positions"], z["types"].astype(np.int64), z["masses"], [],
                            tuple(int(x) for x in z["scell"]))
        self.ngrid = tuple(int(x) for x in z["ngrid"])
        self.fc = z["fc2"]
        self.born = z["born"]
        self.epsilon = z["epsilon"]
        self.nonanalytic = bool(z["nonanalytic"])
        self.V = float(z["volume"])
        self.rl = z["rlattvec"]
        self.symmetrizers = C.build_symmetry(self.cr, self.ngrid).symmetrizers

    def kwargs(self):
        return dict(born=self.born, epsilon=self.epsilon, nonanalytic=self.nonanalytic, V=self.V, rl=self.rl)

    def ifc3(self):
        """The example's FORCE_CONSTANTS_3RD as read3fc stores it."""
        cl = G.Clusters(order=3, phi=self.z["fc3_phi"], cells=self.z["fc3_cells"].astype(np.int64),
                        atoms=self.z["fc3_atoms"].astype(np.int32))
        return S.IFC.from_clusters(cl, self.cr.lattvec)

    def solve(self, omega, vel, eig, scalebroad=None):
        """A rate solve on the example's grid, wedge and clusters with the given
        harmonic arrays; T = 300 K as in the example's T300K outputs."""
        sym = C.build_symmetry(self.cr, self.ngrid)
        wd = C.wedge(sym)
        sb = float(self.z["scalebroad"]) if scalebroad is None else scalebroad
        return S.Solve(self.cr, self.ngrid, np.asfortranarray(omega), np.asfortranarray(vel), np.asfortranarray(eig),
                       sym, wd, [300.0], scalebroad=sb, ifc3=self.ifc3())

    def w3(self):
        """BTE.w_3ph_plus, _minus and the total at 300 K as [ll, branch] arrays
        (the files list branch-major: line (i-1)*Nlist+ll)."""
        nb = self.z["energy"].shape[1]
        nl = len(self.z["list"])
        return tuple(self.z[k][:, 1].reshape(nb, nl).T for k in ("w3_plus", "w3_minus", "w3"))


# The BAs example's outputs were produced with scalebroad = 1 (its CONTROL says 0.1):
# its 3ph counts in log.out match at 1, not at 0.1.
RUN_SCALEBROAD = {"BAs": 1.0}


def check_w3(gh, omega, rate_plus, rate_minus, modes=None):
    """Rates per irreducible point summed over each degenerate set (the basis inside a
    set is LAPACK's choice; the sum is basis-free) against BTE.w_3ph*, all three
    printed with 10 significant digits.  rate_* are [ll, branch]; modes limits the
    check to the first `modes` irreducible points."""
    gp, gm, g3 = gh.w3()
    lst = gh.z["list"] - 1
    nl = gp.shape[0] if modes is None else modes
    scale = g3.max()
    worst = 0.0
    nsets = 0
    for ll in range(nl):
        w = omega[lst[ll]]
        for (a, b) in degenerate_sets(np.sign(w) * w * w, 1e-9 * float(np.max(omega) ** 2)):
            for mine, ref in ((rate_plus, gp), (rate_minus, gm), (rate_plus + rate_minus, g3)):
                r = ref[ll, a:b].sum()
                m = mine[ll, a:b].sum()
                err = abs(m - r)
                assert err <= 2e-9 * abs(r) + 1e-14 * scale, (ll, a, b, m, r)
                if r > 1e-6 * scale:
                    worst = max(worst, err / r)
            nsets += 1
    return worst, nsets


def check_against_golden(gh, omega, vel):
    """omega on the irreducible points (BTE.omega lists those; the reference's
    own omega is not exactly symmetric under the dielectric correction) and
    the velocities on the full grid (BTE.v_full), both printed with 10
    significant digits."""
    lst = gh.z["list"] - 1
    e0 = gh.z["energy"][lst]
    d = np.abs(omega[lst] - e0)
    assert np.all(d <= 1e-9 * np.abs(e0) + 1e-10), float(d.max())
    v0 = gh.z["velocity"]
    dv = np.abs(vel - v0)
    assert np.all(dv <= 1e-9 * np.abs(v0) + 1e-9), float(dv.max())


def synthetic(kind, ngrid, seed):
    """(crystal, fc, symmetrizers) of a seeded synthetic cell."""
    if kind == "diamond":
        cr = C.diamond(5.43, (28.085, 28.085))
    elif kind == "layered":
        cr = C.layered_rhombohedral()
    else:
        cr = C.random_cell(np.random.default_rng(seed), int(kind[len("random"):]))
    fc, _ = S.spring_fc(cr, seed)
    return cr, fc, C.build_symmetry(cr, ngrid).symmetrizers


def degenerate_sets(w_q, tol):
    """[start, end) ranges of the ascending eigenvalues w_q (omega^2) that lie
    within tol of their neighbour."""
    out, b, nb = [], 0, w_q.size
    while b < nb:
        e = b + 1
        while e < nb and abs(w_q[e] - w_q[e - 1]) <= tol:
            e += 1
        out.append((b, e))
        b = e
    return out


def compare_harmonic(a, b, omega_rtol=1e-10, vec_tol=1e-7, vel_rtol=1e-7):
    """Compare two (omega, vel, eig) triples: the eigenvalues sign(omega)
    omega^2 pointwise (two Hermitian solvers agree to rounding times the norm
    of D; near omega = 0 the square root magnifies that), the projector onto
    every degenerate set, and the velocity summed over every set whose omega
    is not at the rounding floor (v divides by 2 omega)."""
    om, vel, eig = a
    om0, vel0, eig0 = b
    w, w0 = np.sign(om) * om * om, np.sign(om0) * om0 * om0
    scale = np.abs(w0).max()
    assert np.abs(w - w0).max() <= omega_rtol * scale, float(np.abs(w - w0).max() / scale)
    floor = 1e-3 * np.abs(om0).max()
    vs = max(np.abs(vel0).max(), 1e-30)
    worst_p = worst_v = 0.0
    for q in range(om0.shape[0]):
        if q == 0:
            w0q = w0[q].copy()
            w0q[:3] = 0.0  # the acoustic branches at Gamma are zeroed after the solve
        else:
            w0q = w0[q]
        for (s, e) in degenerate_sets(w0q, 1e-9 * scale):
            P = eig[q, s:e].T @ eig[q, s:e].conj()  # sum over the set of e e^+
            P0 = eig0[q, s:e].T @ eig0[q, s:e].conj()
            worst_p = max(worst_p, float(np.abs(P - P0).max()))
            if np.abs(om0[q, s:e]).min() > floor:
                worst_v = max(worst_v, float(np.abs(vel[q, s:e].sum(0) - vel0[q, s:e].sum(0)).max()))
    assert worst_p <= vec_tol, worst_p
    assert worst_v <= vel_rtol * vs, worst_v
    return worst_p, worst_v


def numpy_eigen_dm(cr, fc, ngrid, symmetrizers, **kw):
    return HM.eigen_dm(cr, fc, ngrid, symmetrizers, **kw)
