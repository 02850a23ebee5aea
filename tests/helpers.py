"""Shared test helpers: golden reference fixtures and cached synthetic solves."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
if os.path.join(ROOT, "oracle") not in sys.path:
    sys.path.insert(0, os.path.join(ROOT, "oracle"))

from fourphonon_b200 import crystal as C  # noqa: E402
from fourphonon_b200 import system as S  # noqa: E402


class GoldenSolve:
    """The counting-stage inputs of a reference example, as the reference
    wrote them (no eigenvectors, so only the filter/count path applies)."""

    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, f"ref_{name}.npz"))
        self.z = z
        self.ngrid = tuple(int(x) for x in z["ngrid"])
        self.energy = np.asfortranarray(z["energy"])
        self.velocity = np.asfortranarray(z["velocity"])
        self.nb = self.energy.shape[1]
        self.eig = np.zeros((self.nptk, self.nb, self.nb), dtype=np.complex128, order="F")
        self.rlattvec = z["rlattvec"]
        self.scalebroad = float(z["scalebroad"])
        self.temperatures = [300.0]
        self.omega_max = 1.0e100
        self.onlyharmonic = False
        self.ifc3 = None
        self.ifc4 = None
        lst = z["list"]
        self.wedge = C.Wedge(len(lst), lst, z["nequi"], None, None, None)
        natoms = self.nb // 3
        self.crystal = C.Crystal(z["lattvec"], np.zeros((3, natoms)), np.ones(natoms, dtype=np.int64),
                                 np.ones(1), [], (1, 1, 1))

    nptk = property(lambda self: int(np.prod(self.ngrid)))
    nlist = property(lambda self: self.wedge.nlist)
    nmodes = property(lambda self: self.nb * self.wedge.nlist)
    ijk = property(lambda self: C.id2ind(self.ngrid))

    def flat(self):
        return (np.asfortranarray(self.energy).ravel(order="F"), np.asfortranarray(self.velocity).ravel(order="F"),
                np.asfortranarray(self.eig).ravel(order="F"))


def cached_solve(kind="diamond", ngrid=(4, 4, 4), temperatures=(300.0,), seed=None):
    return S.cached_solve(kind, ngrid, temperatures, seed)
