"""Seeded synthetic force constants for the workloads, written in the
reference's own input formats.

* 2nd order: central-force Born-von Karman springs, one spring constant per
  neighbour shell (so the crystal symmetry is kept), written as a Phonopy
  FORCE_CONSTANTS_2ND for a supercell (read by Src/input.f90:18-79).
* 3rd / 4th order: every site set whose pairwise distances are within the
  cutoff carries a random homogeneous cubic (quartic) form in the
  displacement differences of its sites.  The force constants are the third
  (fourth) derivatives of the sum of these forms, averaged over the space
  group.  Derivatives of a scalar of displacement differences are
  permutation-symmetric and satisfy the acoustic sum rule exactly; the
  space-group average makes them crystal-symmetric.  The cluster list is every
  ordered site tuple with its first atom in the home cell and all pairwise
  distances within the cutoff, as thirdorder/fourthorder write it, in
  FORCE_CONSTANTS_3RD / FORCE_CONSTANTS_4TH format (Src/input.f90:102-182,
  Manual.md "4th-IFCs files").
Entries are in eV/A^n, cell vectors in A.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np

from .crystal import Crystal, find_operations


@dataclass
class Clusters:
    """Anharmonic IFC in the reference's in-memory layout.

    phi: (ntri, 3,...,3) with axis order (atom1 axis, atom2 axis, ...) -- i.e.
         phi[c, t, s, r] == Phi(t,s,r,c) of the reference.
    cells: (ntri, order-1, 3) integer lattice coordinates of atoms 2..order.
    atoms: (ntri, order) 1-based atom indices.
    """

    order: int
    phi: np.ndarray
    cells: np.ndarray
    atoms: np.ndarray

    @property
    def ntri(self) -> int:
        return self.phi.shape[0]


def _sites_within(cr: Crystal, radius_nm: float, reach: int = 4):
    cart = cr.cartesian
    out = []
    for n in itertools.product(range(-reach, reach + 1), repeat=3):
        nn = np.array(n, dtype=np.float64)
        for a in range(cr.natoms):
            p = cr.lattvec @ (nn + cr.positions[:, a])
            if np.min(np.linalg.norm(cart.T - p[None, :], axis=1)) <= radius_nm + 1e-9:
                out.append((a, n, p))
    return out


def shell_distances(cr: Crystal, nshell: int = 6, rel_tol: float = 0.0):
    """Sorted distinct interatomic distances (nm) from the basis atoms.  With
    rel_tol > 0 a distance within rel_tol of the current shell's first one joins
    that shell (the bonds of a jittered cell), and a shell is represented by its
    largest member so that every bond of it lies within the shell's radius."""
    sites = _sites_within(cr, 2.0 * np.max(np.linalg.norm(cr.lattvec, axis=0)), reach=3)
    cart = cr.cartesian
    ds = []
    for a in range(cr.natoms):
        for (b, n, p) in sites:
            d = np.linalg.norm(p - cart[:, a])
            if d > 1e-6:
                ds.append(d)
    ds = np.sort(np.array(ds))
    if rel_tol > 0.0:
        shells, first = [ds[0]], ds[0]
        for d in ds[1:]:
            if d > first * (1.0 + rel_tol):
                if len(shells) >= nshell:
                    break
                shells.append(d)
                first = d
            else:
                shells[-1] = d
        return np.array(shells)
    shells = [ds[0]]
    for d in ds[1:]:
        if d - shells[-1] > 1e-4:
            shells.append(d)
        if len(shells) >= nshell:
            break
    return np.array(shells)


def _image(cr: Crystal, R, t, site):
    """Apply the space-group op x' = R x + t to site (a, n)."""
    a, n = site
    x = R @ (np.asarray(n, dtype=np.float64) + cr.positions[:, a]) + t
    for b in range(cr.natoms):
        d = x - cr.positions[:, b]
        r = np.round(d)
        if np.abs(d - r).max() < 1e-5 and cr.types[b] == cr.types[a]:
            return (b, tuple(int(v) for v in r))
    raise ValueError("symmetry image not found")


def generate_anharmonic(cr: Crystal, order: int, cutoff_nm: float, std: float, seed: int,
                        symmetrize: bool = True) -> Clusters:
    """Random order-3 or order-4 force constants (see module docstring)."""
    rng = np.random.default_rng(seed)
    cart = cr.cartesian
    sites = _sites_within(cr, cutoff_nm, reach=3)
    pos = {(a, tuple(n)): p for (a, n, p) in sites}

    def within(group):
        for x, y in itertools.combinations(group, 2):
            if np.linalg.norm(pos[x] - pos[y]) > cutoff_nm + 1e-6:
                return False
        return True

    # translation classes of site sets (size 2..order) containing a home-cell site
    home = [(a, (0, 0, 0)) for a in range(cr.natoms)]
    keys = list(pos.keys())
    sets = set()
    for h in home:
        near = [k for k in keys if np.linalg.norm(pos[k] - pos[h]) <= cutoff_nm + 1e-6 and k != h]
        for size in range(1, order):
            for comb in itertools.combinations(near, size):
                g = (h,) + comb
                if within(g):
                    # canonical representative: translate so the smallest site is home
                    canon = _canon_set(g)
                    sets.add(canon)
    sets = sorted(sets)
    if symmetrize:
        rots, trs = find_operations(cr)
        crots = np.array([cr.lattvec @ R @ np.linalg.inv(cr.lattvec) for R in rots.astype(np.float64)])
    else:
        rots, trs = np.eye(3, dtype=np.int64)[None], np.zeros((1, 3))
        crots = np.eye(3)[None]
    nop = len(rots)
    acc: dict = {}
    ndim = 3 ** order
    for S in sets:
        m = len(S)
        nvar = 3 * (m - 1)
        # random symmetric derivative tensor in the difference coordinates
        W = rng.normal(0.0, 1.0, size=(nvar,) * order)
        Wsym = np.zeros_like(W)
        for perm in itertools.permutations(range(order)):
            Wsym += np.transpose(W, perm)
        Wsym /= _fact(order)
        # site-level tensor: M maps site displacements (3m) to differences (nvar)
        M = np.zeros((nvar, 3 * m))
        for x in range(m - 1):
            for al in range(3):
                M[3 * x + al, 3 * x + al] = 1.0
                M[3 * x + al, 3 * (m - 1) + al] = -1.0
        T = Wsym
        for ax in range(order):
            T = np.tensordot(T, M, axes=([0], [0]))  # contracts leading axis, appends a site axis
        # T: (3m,)*order, axes in site-coordinate order
        T = T.reshape((m, 3) * order)
        T = np.transpose(T, [2 * i for i in range(order)] + [2 * i + 1 for i in range(order)])
        # T[s0..s_{o-1}, a0..a_{o-1}]
        for g in range(nop):
            img = [_image(cr, rots[g], trs[g], s) for s in S]
            Rc = crots[g]
            Tg = T
            for ax in range(order):
                Tg = np.moveaxis(np.tensordot(Tg, Rc, axes=([order + ax], [1])), -1, order + ax)
            for idx in itertools.product(range(m), repeat=order):
                tup = [img[i] for i in idx]
                n0 = np.array(tup[0][1])
                key = (tup[0][0],) + tuple((b, tuple(int(v) for v in (np.array(n) - n0))) for (b, n) in tup[1:])
                blk = Tg[idx].reshape(ndim) / nop
                if key in acc:
                    acc[key] += blk
                else:
                    acc[key] = blk.copy()
    # enumerate the cluster list (all ordered tuples within the cutoff)
    clusters = []
    for a in range(cr.natoms):
        h = (a, (0, 0, 0))
        near = [k for k in keys if np.linalg.norm(pos[k] - pos[h]) <= cutoff_nm + 1e-6]
        for tup in itertools.product(near, repeat=order - 1):
            if within((h,) + tup):
                clusters.append((a,) + tuple(tup))
    clusters.sort(key=lambda k: (k[0],) + tuple((b, n) for (b, n) in k[1:]))
    raw = np.array([acc.get(k, np.zeros(ndim)) for k in clusters])
    scale = std / max(1e-30, raw.std()) if raw.size else 1.0
    phi = (raw * scale).reshape((len(clusters),) + (3,) * order)
    cells = np.array([[n for (b, n) in k[1:]] for k in clusters], dtype=np.int64)
    atoms = np.array([[k[0] + 1] + [b + 1 for (b, n) in k[1:]] for k in clusters], dtype=np.int32)
    return Clusters(order=order, phi=phi, cells=cells, atoms=atoms)


def _fact(n):
    r = 1
    for i in range(2, n + 1):
        r *= i
    return r


def _canon_set(g):
    best = None
    for s in g:
        n0 = np.array(s[1])
        tr = tuple(sorted((b, tuple(int(v) for v in np.array(n) - n0)) for (b, n) in g))
        if best is None or tr < best:
            best = tr
    return best


def bvk_fc2(cr: Crystal, constants, seed_note: str = "", rel_tol: float = 0.0) -> dict:
    """Central-force springs on the first len(constants) neighbour shells
    (shells grouped with shell_distances' rel_tol).

    Returns {(a, b, n): 3x3 block} of Phi(a at 0, b at cell n) in eV/A^2.
    """
    shells = shell_distances(cr, len(constants), rel_tol)
    cart = cr.cartesian
    if rel_tol > 0.0:
        # per-atom shells: every atom keeps springs to its own nearest neighbours, and a
        # bond takes the shell that the more distant-neighboured of its two atoms gives it
        probe = _sites_within(cr, 2.0 * np.max(np.linalg.norm(cr.lattvec, axis=0)), reach=3)
        own = []
        for a in range(cr.natoms):
            ds = np.sort([np.linalg.norm(p - cart[:, a]) for (b, n, p) in probe if np.linalg.norm(p - cart[:, a]) > 1e-6])
            radii, first = [ds[0]], ds[0]
            for d in ds[1:]:
                if d > first * (1.0 + rel_tol):
                    if len(radii) >= len(constants):
                        break
                    radii.append(d)
                    first = d
                else:
                    radii[-1] = d
            own.append(radii + [radii[-1]] * (len(constants) - len(radii)))
        own = np.array(own)
        rmax = float(own.max())
        shell_of = lambda a, b, r: next((x for x in range(len(constants))  # noqa: E731
                                         if r <= max(own[a, x], own[b, x]) + 1e-9), None)
    else:
        rmax = shells[len(constants) - 1] + 1e-4
        shell_of = lambda a, b, r: int(np.argmin(np.abs(shells - r))) if r <= rmax else None  # noqa: E731
    sites = _sites_within(cr, rmax + 0.5, reach=3)
    fc: dict = {}
    for a in range(cr.natoms):
        self_blk = np.zeros((3, 3))
        for (b, n, p) in sites:
            d = p - cart[:, a]
            r = np.linalg.norm(d)
            if r < 1e-6 or r > rmax + 1e-9:
                continue
            sh = shell_of(a, b, r)
            if sh is None:
                continue
            e = d / r
            k = constants[sh]
            blk = -k * np.outer(e, e)
            fc[(a, b, tuple(n))] = fc.get((a, b, tuple(n)), 0) + blk
            self_blk -= blk
        fc[(a, a, (0, 0, 0))] = fc.get((a, a, (0, 0, 0)), 0) + self_blk
    return fc


def write_fc2_phonopy(path, cr: Crystal, fc: dict, scell=None):
    """FORCE_CONSTANTS_2ND in Phonopy's full format (input.f90:18-79 reads it):
    supercell atom index = 1 + ix + iy*nx + iz*nx*ny + iatom*nx*ny*nz."""
    nx, ny, nz = scell or cr.scell
    nat = cr.natoms
    ntot = nx * ny * nz * nat

    def split(idx):
        t = idx
        ix = t % nx
        t //= nx
        iy = t % ny
        t //= ny
        iz = t % nz
        ia = t // nz
        return ia, np.array([ix, iy, iz])

    folded: dict = {}
    for (a, b, n), blk in fc.items():
        m = (np.mod(n[0], nx), np.mod(n[1], ny), np.mod(n[2], nz))
        folded[(a, b, m)] = folded.get((a, b, m), 0) + blk
    lines = [f"{ntot:4d} {ntot:4d}"]
    zero = np.zeros((3, 3))
    for i in range(ntot):
        ia, ci = split(i)
        for j in range(ntot):
            ja, cj = split(j)
            d = cj - ci
            m = (int(np.mod(d[0], nx)), int(np.mod(d[1], ny)), int(np.mod(d[2], nz)))
            blk = folded.get((ia, ja, m), zero)
            lines.append(f"{i + 1:4d} {j + 1:4d}")
            for r in range(3):
                lines.append(" ".join(f"{blk[r, c]:22.15f}" for c in range(3)))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_fc_anharmonic(path, cr: Crystal, cl: Clusters):
    """FORCE_CONSTANTS_3RD / FORCE_CONSTANTS_4TH sparse format."""
    lv_a = cr.lattvec * 10.0
    out = [f"{cl.ntri}"]
    o = cl.order
    for c in range(cl.ntri):
        out.append("")
        out.append(f"{c + 1}")
        for x in range(o - 1):
            R = lv_a @ cl.cells[c, x].astype(np.float64)
            out.append(" ".join(f"{v:.10e}" for v in R))
        out.append(" ".join(f"{int(v):6d}" for v in cl.atoms[c]))
        for idx in itertools.product(range(3), repeat=o):
            out.append(" ".join(f"{i + 1:2d}" for i in idx) + f" {cl.phi[(c,) + idx]:20.10f}")
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")
