"""The reference's input formats: the CONTROL namelists and the sparse
FORCE_CONSTANTS_3RD / FORCE_CONSTANTS_4TH files.

* CONTROL: the four namelist groups ``allocations``, ``crystal``,
  ``parameters`` and ``flags`` with the defaults and checks of
  Src/config.f90:56-249 (the subset of Fortran namelist syntax these files
  use: scalars, whole arrays, ``name(:,k)=`` column sections, strings,
  logicals, ``&end`` or ``/`` terminators, ``!`` comments).
* FORCE_CONSTANTS_3RD/4TH: read3fc / read4fc (Src/input.f90:102-182),
  including the rounding of every cell vector to the nearest lattice vector
  and the conversion from A to nm.
"""
from __future__ import annotations

import re
from dataclasses import dataclass, field

import numpy as np

from .crystal import Crystal
from .ifcgen import Clusters


class InputError(ValueError):
    pass


_TOKEN = re.compile(r'"[^"]*"|\'[^\']*\'|[^\s,]+')


def _parse_value(tok: str):
    t = tok.strip()
    if t[:1] in "\"'":
        return t[1:-1]
    tl = t.lower()
    if tl in (".true.", "t", ".t.", "true"):
        return True
    if tl in (".false.", "f", ".f.", "false"):
        return False
    try:
        if re.fullmatch(r"[+-]?\d+", t):
            return int(t)
        return float(t.replace("d", "e").replace("D", "e"))
    except ValueError:
        raise InputError(f"cannot parse namelist value {tok!r}")


def parse_namelists(text: str) -> dict:
    """Return {group: [(name, index_spec or None, [values])...]}."""
    groups: dict = {}
    lines = []
    for raw in text.splitlines():
        line = raw.split("!")[0]
        lines.append(line)
    body = "\n".join(lines)
    for m in re.finditer(r"&(\w+)(.*?)(?:&end|/\s*$|/\s*\n)", body, flags=re.S | re.I | re.M):
        name = m.group(1).lower()
        content = m.group(2)
        items = []
        for am in re.finditer(r"([A-Za-z_]\w*)\s*(\([^)]*\))?\s*=\s*(.*?)(?=(?:[A-Za-z_]\w*\s*(?:\([^)]*\))?\s*=)|\Z)",
                              content, flags=re.S):
            vals = [_parse_value(t) for t in _TOKEN.findall(am.group(3))]
            items.append((am.group(1).lower(), am.group(2), vals))
        groups[name] = items
    return groups


@dataclass
class Control:
    nelements: int
    natoms: int
    ngrid: tuple
    lfactor: float
    lattvec: np.ndarray  # nm (lfactor applied)
    elements: list
    types: np.ndarray
    positions: np.ndarray
    masses: np.ndarray
    scell: tuple
    epsilon: np.ndarray
    born: np.ndarray
    T: float = 0.0
    T_min: float = 0.0
    T_max: float = 0.0
    T_step: float = 0.0
    scalebroad: float = 1.0
    maxiter: int = 1000
    eps: float = float(np.float32(1e-5))
    omega_max: float = 1.0e100
    num_sample_process_3ph: int = -1
    num_sample_process_3ph_phase_space: int = -1
    num_sample_process_4ph: int = -1
    num_sample_process_4ph_phase_space: int = -1
    flags: dict = field(default_factory=dict)

    def crystal(self) -> Crystal:
        return Crystal(self.lattvec.copy(), self.positions.copy(), self.types.copy(), self.masses.copy(),
                       list(self.elements), tuple(self.scell))

    def temperatures(self):
        """The temperature loop of ShengBTE.f90:262-266."""
        out = []
        import math
        n = math.ceil((self.T_max - self.T_min) / self.T_step) + 1 if self.T_step > 0 else 1
        for c in range(1, n + 1):
            T = self.T_min + (c - 1) * self.T_step
            if T > self.T_max and T < self.T_max + 1.0:
                break
            if T > self.T_max + 1.0:
                T = self.T_max
            out.append(T)
        return out


def _assign(arr, spec, vals):
    if spec is None:
        flat = np.asarray(vals, dtype=arr.dtype)
        arr.reshape(-1, order="F")[: flat.size] = flat
        if arr.ndim > 1:
            arr[...] = arr.reshape(-1, order="F").reshape(arr.shape, order="F")
        return
    parts = [p.strip() for p in spec.strip("()").split(",")]
    idx = []
    for p in parts:
        if p == ":":
            idx.append(slice(None))
        else:
            idx.append(int(p) - 1)
    tgt = arr[tuple(idx)]
    v = np.asarray(vals, dtype=arr.dtype)
    if np.ndim(tgt) == 0:
        arr[tuple(idx)] = v[0]
    else:
        arr[tuple(idx)] = v.reshape(np.shape(tgt), order="F")


def read_control(path_or_text: str, is_text: bool = False) -> Control:
    text = path_or_text if is_text else open(path_or_text).read()
    g = parse_namelists(text)
    al = {k: (s, v) for (k, s, v) in g.get("allocations", [])}
    nelements = int(al.get("nelements", (None, [0]))[1][0])
    natoms = int(al.get("natoms", (None, [0]))[1][0])
    ngrid = np.zeros(3, dtype=np.int64)
    if "ngrid" in al:
        _assign(ngrid, None, al["ngrid"][1])
    if nelements < 1 or natoms < 1 or natoms < nelements:
        raise InputError("nelements,natoms must be >0, natoms must be >=nelements")
    if np.any(ngrid < 1):
        raise InputError("all components of ngrid must be must be >0")
    lfactor = 1.0
    lattvec = np.zeros((3, 3))
    types = np.zeros(natoms, dtype=np.int64)
    positions = np.zeros((3, natoms))
    masses = np.zeros(nelements)
    elements = [""] * nelements
    scell = np.full(3, -1, dtype=np.int64)
    epsilon = np.eye(3)
    born = np.zeros((3, 3, natoms))
    for (k, s, v) in g.get("crystal", []):
        if k == "lfactor":
            lfactor = float(v[0])
        elif k == "lattvec":
            _assign(lattvec, s, v)
        elif k == "types":
            _assign(types, s, v)
        elif k == "positions":
            _assign(positions, s, v)
        elif k == "masses":
            _assign(masses, s, v)
        elif k == "elements":
            elements = [str(x) for x in v]
        elif k == "scell":
            _assign(scell, s, v)
        elif k == "epsilon":
            _assign(epsilon, s, v)
        elif k == "born":
            _assign(born, s, v)
    if not np.all(scell > 0):
        raise InputError("all supercell sizes must be >0")
    if not np.all(types != 0):
        raise InputError("atom types must be initialized correctly")
    c = Control(nelements, natoms, tuple(int(x) for x in ngrid), lfactor, lfactor * lattvec, elements, types,
                positions, masses, tuple(int(x) for x in scell), epsilon, born)
    # namelist names are case-insensitive; map them onto the Control fields
    pmap = {"t": "T", "t_min": "T_min", "t_max": "T_max", "t_step": "T_step", "scalebroad": "scalebroad",
            "maxiter": "maxiter", "eps": "eps", "omega_max": "omega_max",
            "num_sample_process_3ph": "num_sample_process_3ph",
            "num_sample_process_3ph_phase_space": "num_sample_process_3ph_phase_space",
            "num_sample_process_4ph": "num_sample_process_4ph",
            "num_sample_process_4ph_phase_space": "num_sample_process_4ph_phase_space"}
    for (k, s, v) in g.get("parameters", []):
        if k in pmap:
            cur = getattr(c, pmap[k])
            val = v[0]
            if k == "eps" and isinstance(val, float):
                val = float(np.float32(val))  # eps is a default-REAL literal in CONTROL's reader
            setattr(c, pmap[k], type(cur)(val))
    if c.T <= 0.0 and c.T_min <= 0:
        raise InputError("T must be >0 K")
    if c.T > 0:
        c.T_min = c.T_max = c.T_step = c.T
    flags = dict(nonanalytic=True, convergence=True, isotopes=True, autoisotopes=True, nanowires=False,
                 onlyharmonic=False, espresso=False, tdep=False, four_phonon=False, four_phonon_iteration=False)
    for (k, s, v) in g.get("flags", []):
        flags[k] = bool(v[0])
    if flags["four_phonon_iteration"] and not flags["convergence"]:
        raise InputError("four_phonon_iteration=.TRUE. but convergence=.FALSE.")
    if flags["four_phonon_iteration"] and not flags["four_phonon"]:
        raise InputError("four_phonon_iteration=.TRUE. but four_phonon=.FALSE.")
    # the sampling checks of read_config (config.f90:204-221)
    if not flags["four_phonon"] and (c.num_sample_process_4ph > 0 or c.num_sample_process_4ph_phase_space > 0):
        raise InputError("four_phonon=.false. but num_sample_process_4ph.gt.0 or "
                         "num_sample_process_4ph_phase_space.gt.0")
    if flags["convergence"] and c.num_sample_process_3ph > 0:
        raise InputError("convergence=.true. but num_sample_process_3ph.gt.0")
    if flags["four_phonon_iteration"] and c.num_sample_process_4ph > 0:
        raise InputError("four_phonon_iteration=.true. but num_sample_process_4ph.gt.0")
    c.flags = flags
    return c


def write_control(path, cr: Crystal, ngrid, T=None, T_min=None, T_max=None, T_step=None, scalebroad=1.0,
                  convergence=False, four_phonon=True, eps=None, maxiter=None):
    lv = cr.lattvec
    out = ["&allocations", f"        nelements={len(cr.masses)},", f"        natoms={cr.natoms},",
           f"        ngrid(:)={ngrid[0]} {ngrid[1]} {ngrid[2]}", "&end", "&crystal", "        lfactor=1.0,"]
    for i in range(3):
        out.append(f"        lattvec(:,{i + 1})={lv[0, i]:.16f} {lv[1, i]:.16f} {lv[2, i]:.16f},")
    names = cr.elements if cr.elements else [f"E{i}" for i in range(len(cr.masses))]
    out.append("        elements=" + " ".join(f'"{e}"' for e in names) + ",")
    out.append("        types=" + " ".join(str(int(t)) for t in cr.types) + ",")
    for a in range(cr.natoms):
        p = cr.positions[:, a]
        out.append(f"        positions(:,{a + 1})={p[0]:.16f} {p[1]:.16f} {p[2]:.16f},")
    out.append("        masses=" + " ".join(f"{m:.10f}" for m in cr.masses) + ",")
    out.append(f"        scell(:)={cr.scell[0]} {cr.scell[1]} {cr.scell[2]}")
    out.append("&end")
    out.append("&parameters")
    if T is not None:
        out.append(f"        T={T}")
    else:
        out.append(f"        T_min={T_min}, T_max={T_max}, T_step={T_step}")
    out.append(f"        scalebroad={scalebroad}")
    if eps is not None:
        out.append(f"        eps={eps}")
    if maxiter is not None:
        out.append(f"        maxiter={maxiter}")
    out.append("&end")
    out.append("&flags")
    out.append("        nonanalytic=.FALSE.")
    out.append(f"        convergence={'.TRUE.' if convergence else '.FALSE.'}")
    out.append("        isotopes=.FALSE.")
    out.append("        autoisotopes=.FALSE.")
    out.append(f"        four_phonon={'.TRUE.' if four_phonon else '.FALSE.'}")
    out.append("&end")
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")


def read_fc_anharmonic(path, lattvec_nm, order: int):
    """read3fc / read4fc.  Returns (Clusters, R) with R (ntri, order-1, 3) in
    nm, each rounded to the nearest lattice vector as
    R=matmul(lattvec,anint(solve(lattvec,R_A)/10.))."""
    with open(path) as fh:
        toks = fh.read().split()
    p = 0
    ntri = int(toks[p]); p += 1
    nent = 3 ** order
    phi = np.zeros((ntri, nent))
    Rraw = np.zeros((ntri, order - 1, 3))
    atoms = np.zeros((ntri, order), dtype=np.int32)
    for c in range(ntri):
        p += 1  # sequential index
        for x in range(order - 1):
            Rraw[c, x] = [float(t) for t in toks[p:p + 3]]; p += 3
        atoms[c] = [int(t) for t in toks[p:p + order]]; p += order
        for e in range(nent):
            p += order
            phi[c, e] = float(toks[p].replace("d", "e").replace("D", "e")); p += 1
    inv = np.linalg.inv(lattvec_nm)
    cells = np.rint(np.einsum("ij,cxj->cxi", inv, Rraw) / 10.0).astype(np.int64)
    R = np.einsum("ij,cxj->cxi", lattvec_nm, cells.astype(np.float64))
    cl = Clusters(order=order, phi=phi.reshape((ntri,) + (3,) * order), cells=cells, atoms=atoms)
    return cl, R
