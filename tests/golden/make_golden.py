"""Builds the golden fixtures of the reference's example runs.

Run in the development container (it reads the reference tree, which is not
present on GPU machines):

    python tests/golden/make_golden.py /path/to/FourPhonon

For each example with phonopy/espresso inputs (Example-LiCoO2, Example-BAs,
Example-Si) it stores, in ``<name>.npz``:

* the harmonic arrays exactly as the reference itself wrote them:
  omega on the irreducible points (BTE.omega, expanded to the full grid through
  BTE.qpoints_full's equivalence classes), the full-grid group velocities
  (BTE.v_full), the wedge's List and Nequi (BTE.qpoints);
* the lattice from CONTROL (rlattvec is recomputed from it in the
  reference's operation order, so the energy filter sees the same sigma);
* where the example ships a Phonopy FORCE_CONSTANTS_2ND (LiCoO2, BAs), the
  inputs of the harmonic stage: the read2fc array (mass-reduced, times
  unitfactor), positions, types, scell, epsilon, born, the nonanalytic flag and
  the element masses that data_calc_mandg (Src/data.f90:907-930) averages
  from the isotope table of Src/data.f90, and the FORCE_CONSTANTS_3RD clusters
  as read3fc (Src/input.f90:102-141) stores them;
* the golden outputs of the counting stage: Ntotal_plus/minus and
  Ntotal_plusplus/plusminus/minusminus (log.out), per-mode four-phonon counts
  (BTE.Numprocess_4ph, whose line L holds the count of mode L), per-mode phase
  spaces (BTE.P3_plus, BTE.P3_minus, BTE.P4_plusplus, BTE.P4_plusmius,
  BTE.P4_minusminus) and the per-mode RTA rates (T300K/BTE.w_3ph_plus/minus).

All values are the reference's own printed numbers (10 significant digits).
"""
from __future__ import annotations

import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from fourphonon_b200 import harmonic as H  # noqa: E402
from fourphonon_b200 import inputs as I  # noqa: E402


def _floats(path):
    with open(path) as fh:
        return np.array([float(x) for x in fh.read().split()])


def rlattvec_ref(lattvec):
    """config.f90:238-244 in the reference's operation order."""
    r = np.zeros((3, 3))
    for i in range(3):
        j = (i + 1) % 3
        k = (j + 1) % 3
        a, b = lattvec[:, j], lattvec[:, k]
        for ii in range(3):
            jj = (ii + 1) % 3
            kk = (jj + 1) % 3
            r[ii, i] = a[jj] * b[kk] - a[kk] * b[jj]
    V = abs(lattvec[0, 0] * r[0, 0] + lattvec[1, 0] * r[1, 0] + lattvec[2, 0] * r[2, 0])
    rV = 2.0 * np.pi / V
    return rV * r, V


def element_masses(ref_root: str, elements):
    """data_calc_mandg: the abundance-weighted mean of the isotope masses of
    each element, in the table's order, divided by 100."""
    txt = open(os.path.join(ref_root, "Src", "data.f90")).read()
    el = {int(a): b for a, b in re.findall(r'isotope_element\((\d+)\)="(\w+)"', txt)}
    ms = {int(a): float(b.replace("d", "e")) for a, b in re.findall(r"isotope_mass\((\d+)\)=([\d.d+-]+)", txt)}
    ab = {int(a): float(b.replace("d", "e")) for a, b in re.findall(r"isotope_abundance\((\d+)\)=([\d.d+-]+)", txt)}
    out = []
    for e in elements:
        m = 0.0
        for i in sorted(el):
            if el[i] == e:
                m = m + ms[i] * ab[i]
        out.append(m / 100.0)
    return np.array(out)


def build(ref_root: str, name: str):
    base = os.path.join(ref_root, name)
    ctl = I.read_control(os.path.join(base, "input", "CONTROL"))
    out = os.path.join(base, "output")
    ngrid = ctl.ngrid
    nptk = int(np.prod(ngrid))
    nb = 3 * ctl.natoms
    qp = np.loadtxt(os.path.join(out, "BTE.qpoints"))
    qf = np.loadtxt(os.path.join(out, "BTE.qpoints_full"))
    lst = qp[:, 1].astype(np.int32)
    nequi = qp[:, 2].astype(np.int32)
    nlist = len(lst)
    eqc = qf[:, 1].astype(np.int64)
    om_irr = _floats(os.path.join(out, "BTE.omega")).reshape(nlist, nb)
    energy = om_irr[eqc - 1]  # (nptk, nb)
    vfull = _floats(os.path.join(out, "BTE.v_full")).reshape(nb, nptk, 3)
    velocity = np.transpose(vfull, (1, 0, 2))  # (nptk, nb, 3)
    rl, V = rlattvec_ref(ctl.lattvec)
    log = open(os.path.join(out, "log.out")).read()
    m3 = re.search(r"Ntotal_plus\s*=\s*(\d+).*?Ntotal_minus\s*=\s*(\d+)", log, re.S)
    m4 = re.search(r"Ntotal_plusplus,Ntotal_plusminus,Ntotal_minusminus=\s*(\d+)\s+(\d+)\s+(\d+)", log, re.S)
    d = dict(ngrid=np.array(ngrid), rlattvec=rl, volume=np.array(V), lattvec=ctl.lattvec, list=lst, nequi=nequi,
             energy=energy, velocity=velocity, scalebroad=np.array(ctl.scalebroad),
             ntotal_plus=np.array(int(m3.group(1))), ntotal_minus=np.array(int(m3.group(2))))
    if m4:
        d["ntotal_4ph"] = np.array([int(m4.group(i)) for i in (1, 2, 3)], dtype=np.int64)
    npf = os.path.join(out, "BTE.Numprocess_4ph")
    if os.path.exists(npf):
        d["numprocess_4ph"] = np.loadtxt(npf, dtype=np.int64).reshape(-1, 3)
    for key, fn in (("P3_plus", "BTE.P3_plus"), ("P3_minus", "BTE.P3_minus"), ("P4_pp", "BTE.P4_plusplus"),
                    ("P4_pm", "BTE.P4_plusmius"), ("P4_mm", "BTE.P4_minusminus")):
        f = os.path.join(out, fn)
        if os.path.exists(f):
            d[key] = _floats(f).reshape(nlist, nb)
    for key, fn in (("w3_plus", "BTE.w_3ph_plus"), ("w3_minus", "BTE.w_3ph_minus"), ("w3", "BTE.w_3ph")):
        f = os.path.join(out, "T300K", fn)
        if os.path.exists(f):
            d[key] = _floats(f).reshape(-1, 2)
    fc2 = os.path.join(base, "input", "FORCE_CONSTANTS_2ND")
    if os.path.exists(fc2):
        cr = ctl.crystal()
        cr.masses = element_masses(ref_root, ctl.elements)
        d.update(fc2=H.read_fc2_phonopy(fc2, cr), masses=cr.masses, positions=ctl.positions,
                 types=np.asarray(ctl.types, dtype=np.int32), scell=np.array(ctl.scell), epsilon=ctl.epsilon,
                 born=ctl.born, nonanalytic=np.array(bool(ctl.flags["nonanalytic"])))
        # the third-order clusters as read3fc leaves them (lattice-rounded cells)
        cl, _ = I.read_fc_anharmonic(os.path.join(base, "input", "FORCE_CONSTANTS_3RD"), ctl.lattvec, 3)
        d.update(fc3_phi=cl.phi, fc3_cells=cl.cells.astype(np.int8), fc3_atoms=cl.atoms.astype(np.int8))
    np.savez_compressed(os.path.join(HERE, name.replace("Example-", "ref_") + ".npz"), **d)
    return d


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("FOURPHONON_REF", "")
    if not root or not os.path.isdir(root):
        raise SystemExit("usage: make_golden.py <reference root>")
    for ex in ("Example-LiCoO2", "Example-BAs", "Example-Si"):
        d = build(root, ex)
        print(ex, "nptk", d["energy"].shape[0], "nlist", len(d["list"]), "Ntotal 3ph",
              int(d["ntotal_plus"]), int(d["ntotal_minus"]), "4ph", d.get("ntotal_4ph"))
