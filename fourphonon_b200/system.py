"""One solve of the scattering-rate path: every array the hot path consumes,
in the reference's column-major layout, plus builders for the synthetic
workloads.

A :class:`Solve` carries what the Fortran host holds in module globals and
local arrays when it calls the rate drivers (Src/ShengBTE.f90:140-260 and
698-703): grid, reciprocal lattice, temperatures, scalebroad, omega_max,
masses/types, the harmonic arrays energy/velocity/eigenvect, IJK, the wedge
(List, Nequi, ALLEquiList, TypeofSymmetry), the grid map ID_equi, the
symmetrizers and the 3rd/4th-order clusters.
"""
from __future__ import annotations

import os
import tempfile
from dataclasses import dataclass, field

import numpy as np

from . import crystal as C
from . import harmonic as H
from . import ifcgen as G
from . import inputs as I


@dataclass
class IFC:
    """Anharmonic clusters in the reference's in-memory layout (input.f90)."""

    order: int
    ntri: int
    phi: np.ndarray  # flat, Phi(t,s,r,c) column-major (3ph) / Psi(u,t,s,r,c) (4ph)
    R: np.ndarray  # (order-1, ntri, 3) nm: R_j, R_k[, R_l]
    cells: np.ndarray  # (order-1, ntri, 3) integer lattice coordinates
    atoms: np.ndarray  # (order, ntri) 1-based Index_i, Index_j, ...

    @staticmethod
    def from_clusters(cl: G.Clusters, lattvec):
        o = cl.order
        perm = (0,) + tuple(range(o, 0, -1))
        phi = np.ascontiguousarray(np.transpose(cl.phi, perm)).ravel()
        cells = np.ascontiguousarray(np.transpose(cl.cells, (1, 0, 2)))
        R = np.einsum("ij,xcj->xci", lattvec, cells.astype(np.float64))
        atoms = np.ascontiguousarray(cl.atoms.T.astype(np.int32))
        return IFC(o, cl.ntri, phi, np.ascontiguousarray(R), cells, atoms)


@dataclass
class Solve:
    crystal: C.Crystal
    ngrid: tuple
    energy: np.ndarray  # (nptk, nb) Fortran order
    velocity: np.ndarray  # (nptk, nb, 3)
    eig: np.ndarray  # (nptk, nb, nb) complex128
    sym: C.Symmetry
    wedge: C.Wedge
    temperatures: list
    scalebroad: float = 1.0
    omega_max: float = 1.0e100
    ifc3: IFC | None = None
    ifc4: IFC | None = None
    onlyharmonic: bool = False
    meta: dict = field(default_factory=dict)

    @property
    def nptk(self) -> int:
        return int(np.prod(self.ngrid))

    @property
    def nb(self) -> int:
        return self.crystal.nbands

    @property
    def nlist(self) -> int:
        return self.wedge.nlist

    @property
    def nmodes(self) -> int:
        return self.nb * self.nlist

    @property
    def ijk(self) -> np.ndarray:
        return C.id2ind(self.ngrid)

    @property
    def rlattvec(self) -> np.ndarray:
        return self.crystal.rlattvec()

    @property
    def volume(self) -> float:
        """V of config.f90:243 in nm^3."""
        lv = self.crystal.lattvec
        r = self.crystal.rlattvec() / (2.0 * np.pi)
        return abs(float(np.dot(lv[:, 0], np.cross(lv[:, 1], lv[:, 2]))))

    def flat(self):
        """Column-major buffers exactly as the Fortran arrays are laid out."""
        e = np.asfortranarray(self.energy).ravel(order="F")
        v = np.asfortranarray(self.velocity).ravel(order="F")
        z = np.asfortranarray(self.eig).ravel(order="F")
        return e, v, z


def fc2_array(cr: C.Crystal, blocks: dict):
    """The fc array of read2fc built directly from spring blocks (same values
    a written-and-read FORCE_CONSTANTS_2ND yields)."""
    sx, sy, sz = cr.scell
    nat = cr.natoms
    fc = np.zeros((nat, 3, sx, sy, sz, nat, 3))
    for (a, b, n), blk in blocks.items():
        fc[a, :, n[0] % sx, n[1] % sy, n[2] % sz, b, :] += blk
    mm = np.zeros((nat, nat))
    for i in range(nat):
        for j in range(nat):
            mm[i, j] = cr.masses[cr.types[i] - 1] if i == j else np.sqrt(
                cr.masses[cr.types[i] - 1] * cr.masses[cr.types[j] - 1])
    for a in range(nat):
        for b in range(nat):
            fc[a, :, :, :, :, b, :] /= mm[a, b]
    return H.UNITFACTOR * fc


def spring_fc(cr: C.Crystal, seed: int, spring_shells: int = 2, alpha_range=(2.5, 3.5), beta_range=(0.3, 0.6),
              shell_tol: float = 0.0):
    """The seeded BvK second-order constants of build_solve: (fc array of
    read2fc, spring constants)."""
    rng = np.random.default_rng(seed)
    consts = [rng.uniform(*alpha_range)]
    for s in range(1, spring_shells):
        consts.append(rng.uniform(*beta_range) * (1.0 if s == 1 else 0.25))
    return fc2_array(cr, G.bvk_fc2(cr, consts, rel_tol=shell_tol)), consts


def build_solve(cr: C.Crystal, ngrid, temperatures, seed: int, fc3_shell: int = 3, fc4_shell: int = 1,
                scalebroad: float = 1.0, with_4ph: bool = True, with_3ph: bool = True, spring_shells: int = 2,
                alpha_range=(2.5, 3.5), beta_range=(0.3, 0.6), shell_tol: float = 0.0) -> Solve:
    """Seeded synthetic solve: BvK springs (alpha per 1NN shell, beta per 2NN
    shell, further shells with beta/4), N(0,5) cubic and N(0,2) quartic
    clusters within the given neighbour-shell cutoffs.  shell_tol groups the
    scattered bond lengths of a jittered cell into shells (relative tolerance)."""
    fc, consts = spring_fc(cr, seed, spring_shells, alpha_range, beta_range, shell_tol)
    sym = C.build_symmetry(cr, ngrid)
    wd = C.wedge(sym)
    omega, vel, eig = H.eigen_dm(cr, fc, ngrid, sym.symmetrizers)
    shells = G.shell_distances(cr, max(fc3_shell, fc4_shell) + 1, shell_tol)
    ifc3 = ifc4 = None
    if with_3ph:
        cut3 = 0.5 * (shells[fc3_shell - 1] + shells[fc3_shell])
        cl3 = G.generate_anharmonic(cr, 3, cut3, 5.0, seed + 1)
        ifc3 = IFC.from_clusters(cl3, cr.lattvec)
    if with_4ph:
        cut4 = 0.5 * (shells[fc4_shell - 1] + shells[fc4_shell])
        cl4 = G.generate_anharmonic(cr, 4, cut4, 2.0, seed + 2)
        ifc4 = IFC.from_clusters(cl4, cr.lattvec)
    s = Solve(cr, tuple(ngrid), np.asfortranarray(omega), np.asfortranarray(vel), np.asfortranarray(eig), sym, wd,
              list(temperatures), scalebroad=scalebroad, ifc3=ifc3, ifc4=ifc4)
    s.meta = dict(seed=seed, springs=consts, fc3_shell=fc3_shell, fc4_shell=fc4_shell)
    return s


def load_inputs(directory, ctx=None) -> Solve:
    """A solve from a FourPhonon input directory: CONTROL, a Phonopy
    FORCE_CONSTANTS_2ND, FORCE_CONSTANTS_3RD and, when four_phonon is set and the
    file is there, FORCE_CONSTANTS_4TH (the readers of Src/config.f90 and
    Src/input.f90).  The harmonic stage (eigenDM) runs on the device through
    ctx.eigen_dm when a context is given, else in the numpy restatement.
    CONTROL must list masses(:): the isotope table that autoisotopes averages
    is not part of this package."""
    path = lambda name: os.path.join(directory, name)  # noqa: E731
    ctl = I.read_control(path("CONTROL"))
    cr = ctl.crystal()
    if not np.all(np.asarray(cr.masses) > 0):
        raise I.InputError("CONTROL must give masses(:) (autoisotopes needs the isotope table)")
    fc = H.read_fc2_phonopy(path("FORCE_CONSTANTS_2ND"), cr)
    sym = C.build_symmetry(cr, ctl.ngrid)
    wd = C.wedge(sym)
    nac = bool(ctl.flags["nonanalytic"])
    if ctx is not None:
        omega, vel, eig = ctx.eigen_dm(cr, fc, ctl.ngrid, sym.symmetrizers, born=ctl.born, epsilon=ctl.epsilon,
                                       nonanalytic=nac)
    else:
        omega, vel, eig = H.eigen_dm(cr, fc, ctl.ngrid, sym.symmetrizers, ctl.born, ctl.epsilon, nac)
    cl3, _ = I.read_fc_anharmonic(path("FORCE_CONSTANTS_3RD"), cr.lattvec, 3)
    ifc4 = None
    if ctl.flags["four_phonon"]:
        # the reference stops when four_phonon is set and read4fc finds no file
        if not os.path.exists(path("FORCE_CONSTANTS_4TH")):
            raise I.InputError("four_phonon=.TRUE. but FORCE_CONSTANTS_4TH is missing")
        cl4, _ = I.read_fc_anharmonic(path("FORCE_CONSTANTS_4TH"), cr.lattvec, 4)
        ifc4 = IFC.from_clusters(cl4, cr.lattvec)
    return Solve(cr, tuple(ctl.ngrid), np.asfortranarray(omega), np.asfortranarray(vel), np.asfortranarray(eig), sym,
                 wd, list(ctl.temperatures()), scalebroad=ctl.scalebroad, omega_max=ctl.omega_max,
                 ifc3=IFC.from_clusters(cl3, cr.lattvec), ifc4=ifc4, onlyharmonic=bool(ctl.flags["onlyharmonic"]))


def diamond_solve(ngrid=(6, 6, 6), temperatures=(300.0,), seed=20240601, **kw) -> Solve:
    """2-atom diamond, fcc a=5.43 A, masses 28.085 (workload of the 6^3 and 16^3 cases)."""
    return build_solve(C.diamond(5.43, (28.085, 28.085)), ngrid, temperatures, seed, fc3_shell=3, fc4_shell=1, **kw)


def zincblende_solve(ngrid=(24, 24, 24), temperatures=(100.0, 300.0, 500.0, 1000.0), seed=20240603, **kw) -> Solve:
    """2-atom zincblende, a=4.78 A, masses 10.81 / 74.92."""
    return build_solve(C.diamond(4.78, (10.81, 74.92)), ngrid, temperatures, seed, fc3_shell=3, fc4_shell=1, **kw)


def layered_solve(ngrid=(12, 12, 12), temperatures=(300.0,), seed=20240602, **kw) -> Solve:
    """4-atom R-3m layered cell, 4th-order cutoff at the 2nd neighbour shell."""
    return build_solve(C.layered_rhombohedral(), ngrid, temperatures, seed, fc3_shell=3, fc4_shell=2, **kw)


def random_solve(natoms=2, ngrid=(6, 6, 6), temperatures=(300.0,), seed=1, **kw) -> Solve:
    """A random 2-8 atom cell (crystal.random_cell: masses U[6,120] amu) with the
    same seeded BvK + Gaussian cluster generator; the request cells of serving."""
    cr = C.random_cell(np.random.default_rng(seed), natoms)
    # the jittered basis scatters the bond lengths: group them into shells within 15 %, and
    # spring three shells per atom (two leave some 7-8 atom cells with zero-energy mechanisms)
    kw.setdefault("spring_shells", 3)
    return build_solve(cr, ngrid, temperatures, seed, fc3_shell=3, fc4_shell=1, shell_tol=0.15, **kw)


def config4_stream(n=512, seed=20240604, grids=(6, 8, 10, 12, 14), natoms=(2, 8), temps=(100.0, 1000.0)):
    """The request stream of the serving workload: n requests, each a random cell of
    natoms[0]..natoms[1] atoms (crystal.random_cell: masses U[6,120] amu, the seeded
    BvK + Gaussian cluster generator of the diamond workload), a grid edge drawn from
    `grids` and T ~ U[temps].  Returns (natoms, grid edge, T, cell seed) per request,
    in arrival order."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        na = int(rng.integers(natoms[0], natoms[1] + 1))
        g = int(rng.choice(grids))
        T = float(rng.uniform(*temps))
        out.append((na, g, T, int(rng.integers(1, 1 << 30))))
    return out


def request_candidates(natoms, grid, nlist=None):
    """Four-phonon candidate (q', q'', k, l) slots of one RTA solve: 3 channels x
    nlist x nptk work items of nptk x nbands^2 candidates (nlist ~ nptk/2 for a cell
    with inversion only when not given)."""
    nptk = grid ** 3
    nl = nlist if nlist is not None else nptk // 2 + 4
    return 3 * nl * nptk * nptk * (3 * natoms) ** 2


def request_seconds(natoms, grid, nlist=None):
    """Rough plain-FP64 time of one four-phonon RTA solve on one B200: the filter
    per candidate slot plus the contraction per surviving process, whose number
    grows as nbands^4 (the windows of the nbands^2 sorted pair sums fill up).
    Constants from the 16^3 diamond workload (1.6e-11 s per slot, 2.2 % of
    nptk^2 nlist nbands^4 survive, 9e-11 s per survivor).  The contraction's
    cost per survivor also grows with the number of displacement classes,
    which this leaves out, so it underestimates many-atom cells: the first
    five requests of config4_stream come to 45 s here and took 185 s on a
    B200, one at a time in FP64."""
    nptk = grid ** 3
    nl = nlist if nlist is not None else nptk // 2 + 4
    nb = 3 * natoms
    return 1.6e-11 * request_candidates(natoms, grid, nl) + 9e-11 * 0.0217 * nptk * nptk * nl * nb ** 4


def serving_pool(n=8, seed=4242, grids=(4, 6, 8), natoms=(2, 3, 4), max_cost=8 ** 3 * 6):
    """n cached random solves for a request stream: cells of natoms atoms on
    grids drawn from `grids`, keeping nptk * nbands <= max_cost so that one
    solve stays a short request."""
    rng = np.random.default_rng(seed)
    pool = []
    while len(pool) < n:
        na = int(rng.choice(natoms))
        g = int(rng.choice(grids))
        if g ** 3 * 3 * na > max_cost:
            continue
        pool.append(cached_solve(f"random{na}", (g, g, g), (300.0,), seed=int(rng.integers(1, 1 << 30))))
    return pool


# ---------------------------------------------------------------------------
# compact on-disk form (npz) for fixtures and caches
# ---------------------------------------------------------------------------

def save_solve(path, s: Solve):
    d = dict(lattvec=s.crystal.lattvec, positions=s.crystal.positions, types=s.crystal.types,
             masses=s.crystal.masses, scell=np.array(s.crystal.scell), ngrid=np.array(s.ngrid),
             energy=np.asarray(s.energy), velocity=np.asarray(s.velocity), eig=np.asarray(s.eig),
             rotations=s.sym.rotations, crotations=s.sym.crotations, qrotations=s.sym.qrotations,
             symmetrizers=s.sym.symmetrizers, nsymm=np.array(s.sym.nsymm),
             w_list=s.wedge.list, w_nequi=s.wedge.nequi, w_allequi=s.wedge.allequi, w_typeofsym=s.wedge.typeofsym,
             w_id_equi=s.wedge.id_equi, temperatures=np.array(s.temperatures), scalebroad=np.array(s.scalebroad),
             omega_max=np.array(s.omega_max))
    for name, ifc in (("ifc3", s.ifc3), ("ifc4", s.ifc4)):
        if ifc is not None:
            d[name + "_phi"] = ifc.phi
            d[name + "_cells"] = ifc.cells
            d[name + "_atoms"] = ifc.atoms
    np.savez_compressed(path, **d)


def load_solve(path) -> Solve:
    z = np.load(path)
    cr = C.Crystal(z["lattvec"], z["positions"], z["types"], z["masses"], [], tuple(int(x) for x in z["scell"]))
    ngrid = tuple(int(x) for x in z["ngrid"])
    sym = C.Symmetry(z["rotations"], z["crotations"], z["qrotations"], z["symmetrizers"], int(z["nsymm"]), ngrid)
    wd = C.Wedge(int(z["w_list"].shape[0]), z["w_list"], z["w_nequi"], z["w_allequi"], z["w_typeofsym"],
                 z["w_id_equi"])
    ifcs = {}
    for name, order in (("ifc3", 3), ("ifc4", 4)):
        if name + "_phi" in z:
            cells = z[name + "_cells"]
            R = np.einsum("ij,xcj->xci", cr.lattvec, cells.astype(np.float64))
            ifcs[name] = IFC(order, int(z[name + "_atoms"].shape[1]), z[name + "_phi"], np.ascontiguousarray(R),
                             cells, z[name + "_atoms"])
    return Solve(cr, ngrid, np.asfortranarray(z["energy"]), np.asfortranarray(z["velocity"]),
                 np.asfortranarray(z["eig"]), sym, wd, [float(t) for t in z["temperatures"]],
                 scalebroad=float(z["scalebroad"]), omega_max=float(z["omega_max"]), ifc3=ifcs.get("ifc3"),
                 ifc4=ifcs.get("ifc4"))


_CACHE: dict = {}


def cached_solve(kind: str = "diamond", ngrid=(4, 4, 4), temperatures=(300.0,), seed=None) -> Solve:
    """Synthetic solve built once and cached in memory and under _build/solves
    (rebuilt from the seed when the file is absent)."""
    key = (kind, tuple(ngrid), tuple(temperatures), seed)
    if key in _CACHE:
        return _CACHE[key]
    root = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
    d = os.path.join(root, "_build", "solves")
    os.makedirs(d, exist_ok=True)
    fn = os.path.join(d, f"{kind}_{'x'.join(map(str, ngrid))}_{'-'.join(str(int(t)) for t in temperatures)}_{seed}.npz")
    if os.path.exists(fn):
        s = load_solve(fn)
    else:
        kw = {} if seed is None else {"seed": seed}
        if kind.startswith("random"):
            s = random_solve(int(kind[6:]), ngrid=tuple(ngrid), temperatures=tuple(temperatures), **kw)
        else:
            builder = {"diamond": diamond_solve, "zincblende": zincblende_solve, "layered": layered_solve}[kind]
            s = builder(ngrid=tuple(ngrid), temperatures=tuple(temperatures), **kw)
        tmp = fn + f".{os.getpid()}.tmp.npz"
        save_solve(tmp, s)
        os.replace(tmp, fn)
    _CACHE[key] = s
    return s
