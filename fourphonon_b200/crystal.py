"""Crystal cells, space-group operations and the irreducible wedge of the q grid.

Host-side set-up of the scattering-rate path.  The reference obtains its
symmetry operations from spglib (Src/symmetry.f90:11-150) and builds the
irreducible wedge in Src/wedgetc.f90:20-75; spglib is not available here, so
the operations are found by a direct search over integer rotation matrices
that preserve the lattice metric and map the basis onto itself.  The derived
tables (rotations with time reversal, Cartesian and reciprocal forms, grid
maps, symmetrizers, List/Nequi/ALLEquiList/TypeofSymmetry) follow
Src/config.f90:271-376 and 397-478 step by step.

Conventions: ``lattvec`` holds the lattice vectors as columns in nm (the
reference's lattvec after the lfactor scaling); ``positions`` are fractional
coordinates, shape (3, natoms); ``types`` are 1-based element indices.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Crystal:
    lattvec: np.ndarray  # (3,3) columns, nm
    positions: np.ndarray  # (3, natoms) fractional
    types: np.ndarray  # (natoms,) 1-based
    masses: np.ndarray  # (nelements,) amu
    elements: list = field(default_factory=list)
    scell: tuple = (4, 4, 4)

    @property
    def natoms(self) -> int:
        return self.positions.shape[1]

    @property
    def nbands(self) -> int:
        return 3 * self.natoms

    @property
    def cartesian(self) -> np.ndarray:
        return self.lattvec @ self.positions

    def rlattvec(self) -> np.ndarray:
        """Reciprocal lattice vectors as columns in nm^-1 (config.f90:238-244)."""
        lv = self.lattvec
        r = np.zeros((3, 3))
        for i in range(3):
            j = (i + 1) % 3
            k = (j + 1) % 3
            a, b = lv[:, j], lv[:, k]
            r[:, i] = [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]
        V = abs(float(np.dot(lv[:, 0], r[:, 0])))
        rV = 2.0 * np.pi / V
        return rV * r

    def volume(self) -> float:
        return abs(float(np.linalg.det(self.lattvec)))


# ---------------------------------------------------------------------------
# Space-group operations
# ---------------------------------------------------------------------------

def find_operations(cr: Crystal, symprec: float = 1e-5):
    """Return (rotations[n,3,3] int, translations[n,3]) acting on fractional
    coordinates as x' = R x + t, like spg_get_symmetry (symmetry.f90:118-125).

    Order: identity first, then the remaining operations sorted
    lexicographically by (R, t); the order only affects which image the wedge
    records first, never a rate.
    """
    lv = cr.lattvec
    G = lv.T @ lv
    scale = np.sqrt(np.abs(np.diag(G))).max()
    rots = []
    for ent in itertools.product((-1, 0, 1), repeat=9):
        R = np.array(ent, dtype=np.int64).reshape(3, 3)
        if round(abs(np.linalg.det(R))) != 1:
            continue
        if np.abs(R.T @ G @ R - G).max() > 1e-6 * scale * scale:
            continue
        rots.append(R)
    pos = cr.positions
    nat = pos.shape[1]
    ops = []
    for R in rots:
        rp = R @ pos
        for a in range(nat):
            if cr.types[a] != cr.types[0]:
                continue
            t = pos[:, a] - rp[:, 0]
            t = t - np.round(t)
            ok = True
            for b in range(nat):
                x = rp[:, b] + t
                found = False
                for c in range(nat):
                    if cr.types[c] != cr.types[b]:
                        continue
                    d = x - pos[:, c]
                    d = d - np.round(d)
                    if np.linalg.norm(lv @ d) < symprec * max(1.0, scale):
                        found = True
                        break
                if not found:
                    ok = False
                    break
            if ok:
                t = np.where(np.abs(t) < 1e-12, 0.0, t)
                t = t - np.floor(t + 1e-9)
                ops.append((R, t))
    ident = [o for o in ops if np.array_equal(o[0], np.eye(3, dtype=np.int64)) and np.allclose(o[1], 0)]
    rest = [o for o in ops if not (np.array_equal(o[0], np.eye(3, dtype=np.int64)) and np.allclose(o[1], 0))]
    rest.sort(key=lambda o: (tuple(o[0].ravel()), tuple(np.round(o[1], 8))))
    ops = ident + rest
    rotations = np.array([o[0] for o in ops], dtype=np.int64)
    translations = np.array([o[1] for o in ops], dtype=np.float64)
    return rotations, translations


@dataclass
class Symmetry:
    """Tables derived from the operations exactly as read_config builds them."""

    rotations: np.ndarray  # (nsymm_rot,3,3) int, lattice coords (after filtering)
    crotations: np.ndarray  # (nsymm_rot,3,3) Cartesian
    qrotations: np.ndarray  # (nsymm_rot,3,3) reciprocal basis
    symmetrizers: np.ndarray  # (nptk,3,3)
    nsymm: int  # operations before time reversal doubling
    ngrid: tuple

    @property
    def nsymm_rot(self) -> int:
        return self.rotations.shape[0]


def id2ind(ngrid):
    """IJK(3,nptk): config.f90:458-468 (G1 index fastest)."""
    n1, n2, n3 = ngrid
    nptk = n1 * n2 * n3
    ii = np.arange(nptk)
    i1 = ii % n1
    t = ii // n1
    i2 = t % n2
    i3 = t // n2
    return np.stack([i1, i2, i3], axis=0).astype(np.int32)


def _symm_images(qrot, ijk, ngrid):
    """r_out = ngrid*matmul(qrotations, r_in/ngrid) for every op and point
    (config.f90:381-393).  Returns (nsym, 3, nptk)."""
    ng = np.asarray(ngrid, dtype=np.float64)[:, None]
    x = ijk.astype(np.float64) / ng  # (3,nptk)
    return np.einsum("sij,jq->siq", qrot, x) * ng[None]


def _ind2id(ivec, ngrid):
    return 1 + ivec[0] + (ivec[1] + ivec[2] * ngrid[1]) * ngrid[0]


def symmetry_map(qrot, ngrid):
    """ID_equi(nsymm_rot,nptk) of config.f90:397-419 (1-based, -1 = off grid)."""
    ijk = id2ind(ngrid)
    vec = _symm_images(qrot, ijk, ngrid)
    iv = np.rint(vec).astype(np.int64)
    off = np.sqrt(((np.abs(vec - iv)) ** 2).sum(axis=1)) > 1e-2
    ng = np.asarray(ngrid)[None, :, None]
    ivm = np.mod(iv, ng)
    ids = _ind2id(ivm.transpose(1, 0, 2), ngrid)  # (nsym,nptk)
    ids = np.where(off, -1, ids)
    return ids.astype(np.int32)


def symmetry_map_notransl(qrot, ngrid):
    """config.f90:422-443: ID_equi(isym,i)=i if the op maps q to itself."""
    ijk = id2ind(ngrid)
    vec = _symm_images(qrot, ijk, ngrid)
    d = np.sqrt(((np.abs(ijk[None].astype(np.float64) - vec)) ** 2).sum(axis=1))
    nptk = ijk.shape[1]
    ids = np.where(d <= 1e-5, np.arange(1, nptk + 1)[None, :], -1)
    return ids.astype(np.int32)


def build_symmetry(cr: Crystal, ngrid) -> Symmetry:
    """config.f90:271-376: time-reversal doubling, Cartesian/reciprocal
    forms, symmetrizers, then removal of grid-incompatible and duplicated
    rotations."""
    rot0, tr0 = find_operations(cr)
    nsymm = rot0.shape[0]
    lv = cr.lattvec
    crot0 = np.array([lv @ R @ np.linalg.inv(lv) for R in rot0.astype(np.float64)])
    G = lv.T @ lv
    qrot0 = np.array([(np.linalg.solve(G, R.T.astype(np.float64)) @ G).T for R in rot0])
    rotations = np.concatenate([rot0, -rot0])
    crot = np.concatenate([crot0, -crot0])
    qrot = np.concatenate([qrot0, -qrot0])
    nptk = int(np.prod(ngrid))
    # symmetrizers from the full (unfiltered) list
    ide = symmetry_map_notransl(qrot, ngrid)
    symm = np.zeros((nptk, 3, 3))
    for q in range(nptk):
        sel = np.nonzero(ide[:, q] == q + 1)[0]
        if len(sel):
            symm[q] = crot[sel].sum(axis=0)
            if len(sel) > 1:
                symm[q] /= len(sel)
    idm = symmetry_map(qrot, ngrid)
    valid = np.ones(rotations.shape[0], dtype=bool)
    for s in range(rotations.shape[0]):
        if valid[s] and np.any(idm[s] == -1):
            valid[s] = False
    for s in range(1, rotations.shape[0]):
        for t in range(s):
            if not valid[t]:
                continue
            if np.array_equal(rotations[s], rotations[t]):
                valid[s] = False
                break
    return Symmetry(rotations=rotations[valid], crotations=crot[valid], qrotations=qrot[valid],
                    symmetrizers=symm, nsymm=nsymm, ngrid=tuple(ngrid))


@dataclass
class Wedge:
    nlist: int
    list: np.ndarray  # (nlist,) 1-based
    nequi: np.ndarray  # (nlist,)
    allequi: np.ndarray  # (nlist, nsymm_rot) 1-based, padded with 0
    typeofsym: np.ndarray  # (nlist, nsymm_rot) 1-based op index, padded with 0
    id_equi: np.ndarray  # (nsymm_rot, nptk) symmetry_map, 1-based


def wedge(sym: Symmetry) -> Wedge:
    """wedgetc.f90:20-75."""
    ngrid = sym.ngrid
    nptk = int(np.prod(ngrid))
    idm = symmetry_map(sym.qrotations, ngrid)
    nsr = sym.nsymm_rot
    seen = np.zeros(nptk + 1, dtype=bool)
    lst, neq, alle, tos = [], [], [], []
    for ii in range(1, nptk + 1):
        if seen[ii]:
            continue
        eq = []
        ty = []
        for s in range(nsr):
            x = int(idm[s, ii - 1])
            if x not in eq:
                eq.append(x)
                ty.append(s + 1)
                seen[x] = True
        lst.append(ii)
        neq.append(len(eq))
        alle.append(eq + [0] * (nsr - len(eq)))
        tos.append(ty + [0] * (nsr - len(ty)))
    if sum(neq) != nptk:
        raise ValueError("wedge: ntot != nptk")
    return Wedge(nlist=len(lst), list=np.array(lst, dtype=np.int32), nequi=np.array(neq, dtype=np.int32),
                 allequi=np.array(alle, dtype=np.int32), typeofsym=np.array(tos, dtype=np.int32),
                 id_equi=idm.astype(np.int32))


# ---------------------------------------------------------------------------
# Cells used by the workloads
# ---------------------------------------------------------------------------

def diamond(a_angstrom: float = 5.43, masses=(28.085, 28.085)) -> Crystal:
    """Two-atom diamond / zincblende primitive cell (fcc lattice)."""
    a = a_angstrom / 10.0
    lv = 0.5 * a * np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]]).T
    pos = np.array([[0.0, 0.25], [0.0, 0.25], [0.0, 0.25]])
    m = np.asarray(masses, dtype=np.float64)
    if m[0] == m[1]:
        return Crystal(lv, pos, np.array([1, 1]), m[:1].copy(), ["X"])
    return Crystal(lv, pos, np.array([1, 2]), m.copy(), ["A", "B"])


def layered_rhombohedral(a_angstrom: float = 2.82, c_over_a: float = 5.0,
                         masses=(6.94, 58.93, 16.00, 16.00)) -> Crystal:
    """Four-atom R-3m layered cell (LiCoO2-like primitive rhombohedral
    setting): Li at 0, Co at 1/2, O at +-u along the rhombohedral diagonal."""
    a = a_angstrom / 10.0
    c = c_over_a * a
    # rhombohedral primitive vectors of the hexagonal (a,c) lattice
    lv = np.zeros((3, 3))
    lv[:, 0] = [a / np.sqrt(3.0), 0.0, c / 3.0]
    lv[:, 1] = [-a / (2.0 * np.sqrt(3.0)), a / 2.0, c / 3.0]
    lv[:, 2] = [-a / (2.0 * np.sqrt(3.0)), -a / 2.0, c / 3.0]
    u = 0.2396
    pos = np.array([[0.0, 0.5, 1.0 - u, u]] * 3)
    m = np.asarray(masses, dtype=np.float64)
    return Crystal(lv, pos, np.array([1, 2, 3, 3]), np.array([m[0], m[1], m[2]]), ["Li", "Co", "O"])


def random_cell(rng: np.random.Generator, natoms: int) -> Crystal:
    """A random 2-8 atom cell: an fcc host of lattice constant ~5 A with the
    basis placed on a jittered simple sublattice; masses U[6,120] amu."""
    a = rng.uniform(4.8, 6.0) / 10.0
    lv = 0.5 * a * np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]]).T
    lv = lv * np.array([1.0, 1.0, max(1, (natoms + 1) // 2)])[None, :]
    base = []
    for n in range(natoms):
        base.append([(n % 2) * 0.25 + 0.0, (n % 2) * 0.25, (n // 2 + (n % 2) * 0.25) / max(1, (natoms + 1) // 2)])
    pos = np.array(base).T
    pos = pos + rng.uniform(-0.02, 0.02, size=pos.shape)
    pos[:, 0] = 0.0
    pos = np.mod(pos, 1.0)
    masses = rng.uniform(6.0, 120.0, size=natoms)
    return Crystal(lv, pos, np.arange(1, natoms + 1), masses, [f"E{i}" for i in range(natoms)])
