"""Harmonic inputs of the scattering path: frequencies, group velocities and
eigenvectors on the full q grid.

The reference computes them in eigenDM / phonon_phonopy
(Src/phonon_routines.f90:12-81, 84-307) from a Phonopy FORCE_CONSTANTS_2ND
with LAPACK zheev.  This module restates phonon_phonopy (Wigner-Seitz image
weights, analytic group velocities from the derivative of the dynamical
matrix, the dielectric correction of lines 140-247), the velocity
symmetrization and the zeroing of the acoustic branches at Gamma (lines
62-80).  The eigen-solver is numpy's LAPACK Hermitian solver; the harmonic
stage sits upstream of the accelerated path, whose kernels and whose oracle
both consume the same (omega, v, e) arrays produced here.
"""
from __future__ import annotations

import numpy as np

from .crystal import Crystal

# input.f90:13 unitfactor=9648.53336213 (default REAL literal)
UNITFACTOR = float(np.float32(9648.53336213))
# phonon_routines.f90:91 prefactor=1745.91429109 (default REAL literal)
NAC_PREFACTOR = float(np.float32(1745.91429109))


def read_fc2_phonopy(path, cr: Crystal):
    """read2fc (input.f90:18-79): fc(natoms,3,sx,sy,sz,natoms,3), mass-reduced
    and multiplied by unitfactor."""
    sx, sy, sz = cr.scell
    nat = cr.natoms
    mm = np.zeros((nat, nat))
    for i in range(nat):
        mm[i, i] = cr.masses[cr.types[i] - 1]
        for j in range(i + 1, nat):
            mm[i, j] = np.sqrt(cr.masses[cr.types[i] - 1] * cr.masses[cr.types[j] - 1])
            mm[j, i] = mm[i, j]
    fc = np.zeros((nat, 3, sx, sy, sz, nat, 3))
    with open(path) as fh:
        toks = fh.read().split()
    p = 0
    ntot = int(toks[p]); p += 1
    if len(toks) > 1 and toks[1].lstrip("-").isdigit() and int(toks[1]) == ntot and len(toks) > 2 + 11 * ntot * ntot - 5:
        p += 1  # "ntot ntot" header form
    if ntot != sx * sy * sz * nat:
        raise ValueError("wrong number of force constants for the specified scell")

    def split(index):
        t = index - 1
        ix = t % sx; t //= sx
        iy = t % sy; t //= sy
        iz = t % sz; ia = t // sz
        return ix, iy, iz, ia

    for _ in range(ntot * ntot):
        a1 = int(toks[p]); a2 = int(toks[p + 1]); p += 2
        blk = np.array([float(x) for x in toks[p:p + 9]]).reshape(3, 3); p += 9
        ix1, iy1, iz1, ia1 = split(a1)
        ix2, iy2, iz2, ia2 = split(a2)
        if ix1 == 0 and iy1 == 0 and iz1 == 0:
            fc[ia1, :, ix2, iy2, iz2, ia2, :] = blk
    for a in range(nat):
        for b in range(nat):
            fc[a, :, :, :, :, b, :] /= mm[a, b]
    return UNITFACTOR * fc


def _images(cr: Crystal):
    """Per (a1, a2, cell) the Wigner-Seitz images rr (phonon_routines.f90:224-251)."""
    sx, sy, sz = cr.scell
    lv = cr.lattvec
    cart = cr.cartesian
    out = {}
    for a1 in range(cr.natoms):
        for a2 in range(cr.natoms):
            for ix in range(sx):
                for iy in range(sy):
                    for iz in range(sz):
                        rcell = lv @ np.array([ix, iy, iz], dtype=np.float64)
                        r = cart[:, a1] - cart[:, a2] + rcell
                        dmin = np.inf
                        rr = []
                        for jx in range(-2, 3):
                            for jy in range(-2, 3):
                                for jz in range(-2, 3):
                                    rl = jx * sx * lv[:, 0] + jy * sy * lv[:, 1] + jz * sz * lv[:, 2]
                                    rn = np.linalg.norm(rl + r)
                                    if abs(rn - dmin) > 1e-5:
                                        if rn < dmin:
                                            dmin = rn
                                            rr = [rl + rcell]
                                    else:
                                        rr.append(rl + rcell)
                        out[(a1, a2, ix, iy, iz)] = np.array(rr)
    return out


def kspace(cr: Crystal, ngrid, rl=None):
    """kspace(nptk,3) of eigenDM (phonon_routines.f90:27-35), nm^-1, in the
    reference's operation order rlattvec(:,d)*(i-1)/ngrid(d) summed over d."""
    rl = cr.rlattvec() if rl is None else rl
    n1, n2, n3 = ngrid
    nptk = n1 * n2 * n3
    idx = np.arange(nptk)
    i1 = (idx % n1).astype(np.float64)
    i2 = ((idx // n1) % n2).astype(np.float64)
    i3 = (idx // (n1 * n2)).astype(np.float64)
    return (np.outer(i1, rl[:, 0]) / n1 + np.outer(i2, rl[:, 1]) / n2) + np.outer(i3, rl[:, 2]) / n3


def _norms(r):
    """Euclidean norms of the rows of r, correctly rounded: the squares are
    summed in extended precision before the square root.  The reference's
    dnrm2 behaves so (its results on the BAs example pick the same first-zone
    image at every one of the 4096 points, ties included), while a double
    sum of squares breaks some of the ties between images of equal length the
    other way."""
    x = np.asarray(r, dtype=np.longdouble)
    return np.sqrt((x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1]) + x[:, 2] * x[:, 2]).astype(np.float64)


def shortest_images(kpoints, rl):
    """The first-Brillouin-zone image of each q point used by the dielectric
    correction (phonon_routines.f90:140-156): starting from q itself, an image
    of the (-2..2)^3 scan replaces the current one when its norm is strictly
    smaller."""
    best = kpoints.copy()
    bn = _norms(best)
    for ix in range(-2, 3):
        for iy in range(-2, 3):
            for iz in range(-2, 3):
                r = ((kpoints + ix * rl[:, 0]) + iy * rl[:, 1]) + iz * rl[:, 2]
                n = _norms(r)
                m = n < bn
                best[m] = r[m]
                bn[m] = n[m]
    return best


def nac_terms(cr: Crystal, kpoints, born, epsilon, V, rl):
    """dyn_nac (nk,nb,nb) and ddyn_nac (nk,nb,nb,3) of the dielectric
    correction (phonon_routines.f90:158-198); zero where the shortest image is
    Gamma."""
    nat = cr.natoms
    nb = 3 * nat
    nk = kpoints.shape[0]
    q = shortest_images(kpoints, rl)
    mm = np.zeros((nat, nat))
    for i in range(nat):
        for j in range(nat):
            mm[i, j] = cr.masses[cr.types[i] - 1] if i == j else np.sqrt(
                cr.masses[cr.types[i] - 1] * cr.masses[cr.types[j] - 1])
    on = ~np.all(q == 0.0, axis=1)
    tmp3 = np.einsum("ka,ka->k", q, q @ epsilon.T)
    t3 = np.where(on, tmp3, 1.0)
    qb = np.einsum("ka,aib->kbi", q, born).reshape(nk, nb)  # tmp1 of row (a, i): q . born(:, i, a)
    qe = q @ epsilon.T  # (nk, 3): epsilon(ip,:) . q
    mmx = np.repeat(np.repeat(mm, 3, axis=0), 3, axis=1)
    bornx = np.transpose(born, (2, 1, 0)).reshape(nb, 3)  # bornx[(a,i), ip] = born(ip, i, a)
    dyn = qb[:, :, None] * qb[:, None, :] / mmx[None]
    dd = (qb[:, :, None, None] * bornx[None, None, :, :] + qb[:, None, :, None] * bornx[None, :, None, :]
          - 2.0 * (qb[:, :, None] * qb[:, None, :])[..., None] * qe[:, None, None, :] / t3[:, None, None, None])
    dd = dd / mmx[None, :, :, None]
    pref = NAC_PREFACTOR
    dyn = pref * dyn / t3[:, None, None] / V
    dd = pref * dd / t3[:, None, None, None] / V
    dyn[~on] = 0.0
    dd[~on] = 0.0
    return dyn, dd


def phonon_phonopy(cr: Crystal, fc, kpoints, born=None, epsilon=None, nonanalytic=False, V=None, rl=None):
    """Frequencies (rad/ps), velocities (km/s) and eigenvectors for kpoints (nk,3).

    Returns omega (nk,nb), vel (nk,nb,3), eig (nk,nb,nb) with eig[k,band,comp].
    With nonanalytic, the dielectric correction of phonon_routines.f90:158-247
    is added (born(3,3,natoms), epsilon(3,3)); V is the cell volume in nm^3.
    """
    nat = cr.natoms
    nb = 3 * nat
    sx, sy, sz = cr.scell
    ncell = sx * sy * sz
    nk = kpoints.shape[0]
    rl = cr.rlattvec() if rl is None else rl
    V = cr.volume() if V is None else V
    imgs = _images(cr)
    dyn = np.zeros((nk, nb, nb), dtype=np.complex128)
    ddyn = np.zeros((nk, nb, nb, 3), dtype=np.complex128)
    if nonanalytic:
        born = np.zeros((3, 3, nat)) if born is None else np.asarray(born, dtype=np.float64)
        epsilon = np.eye(3) if epsilon is None else np.asarray(epsilon, dtype=np.float64)
        dnac, ddnac = nac_terms(cr, kpoints, born, epsilon, V, rl)
        kon = ~np.all(kpoints == 0.0, axis=1)
    for (a1, a2, ix, iy, iz), rr in imgs.items():
        neq = rr.shape[0]
        qr = kpoints @ rr.T  # (nk, neq)
        z = np.exp(-1j * qr) / neq  # (nk, neq)
        star = z.sum(axis=1)
        blk = fc[a2, :, ix, iy, iz, a1, :].T  # blk[i,j] = fc(a2,j,cell,a1,i)
        zr = -1j * np.einsum("kn,nd->kd", z, rr)  # (nk,3)
        if nonanalytic:
            # fc_total(a2,j,cell,a1,i) = fc + real(dyn_nac(3*a2+j, 3*a1+i)) / ncell
            ft = blk[None] + np.transpose(dnac[:, 3 * a2:3 * a2 + 3, 3 * a1:3 * a1 + 3], (0, 2, 1)).real / ncell
            dyn[:, 3 * a1:3 * a1 + 3, 3 * a2:3 * a2 + 3] += star[:, None, None] * ft
            ddyn[:, 3 * a1:3 * a1 + 3, 3 * a2:3 * a2 + 3, :] += ft[..., None] * zr[:, None, None, :]
            ddyn[:, 3 * a1:3 * a1 + 3, 3 * a2:3 * a2 + 3, :] += np.where(
                kon[:, None, None, None],
                star[:, None, None, None] * ddnac[:, 3 * a1:3 * a1 + 3, 3 * a2:3 * a2 + 3, :] / ncell, 0.0)
        else:
            dyn[:, 3 * a1:3 * a1 + 3, 3 * a2:3 * a2 + 3] += star[:, None, None] * blk[None]
            ddyn[:, 3 * a1:3 * a1 + 3, 3 * a2:3 * a2 + 3, :] += blk[None, :, :, None] * zr[:, None, None, :]
    w2, vecs = np.linalg.eigh(dyn)
    omega = np.sign(w2) * np.sqrt(np.abs(w2))
    eig = np.transpose(vecs, (0, 2, 1))  # eig[k, band, comp] = Z(comp, band)
    vel = np.zeros((nk, nb, 3))
    for ip in range(3):
        t = np.einsum("kab,kbn->kan", ddyn[..., ip], vecs)
        vel[:, :, ip] = np.real(np.einsum("kan,kan->kn", np.conj(vecs), t))
    with np.errstate(divide="ignore", invalid="ignore"):
        vel = vel / (2.0 * omega[:, :, None])
    vel = np.where(np.isfinite(vel), vel, 0.0)
    return omega, vel, eig


def eigen_dm(cr: Crystal, fc, ngrid, symmetrizers, born=None, epsilon=None, nonanalytic=False, V=None, rl=None):
    """eigenDM (phonon_routines.f90:12-81) for the full grid, arrays in the
    reference's (nptk, nb[, ...]) order."""
    k = kspace(cr, ngrid, rl)
    omega, vel, eig = phonon_phonopy(cr, fc, k, born, epsilon, nonanalytic, V, rl)
    # velocity(ii,:,:)=transpose(matmul(symmetrizers(:,:,ii),transpose(velocity(ii,:,:))))
    vel = np.einsum("qab,qnb->qna", symmetrizers, vel)
    omega[0, 0:3] = 0.0
    vel[0, 0:3, :] = 0.0
    return omega, vel, eig


def to_fortran_arrays(omega, vel, eig):
    """Flatten to the column-major buffers of the C-ABI:
    energy(nptk,nb), velocity(nptk,nb,3), eigenvect(nptk,nb,nb) complex."""
    energy = np.asfortranarray(omega)
    velocity = np.asfortranarray(vel)
    eigenvect = np.asfortranarray(eig)
    return energy, velocity, eigenvect
