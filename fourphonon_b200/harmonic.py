"""Harmonic inputs of the scattering path: frequencies, group velocities and
eigenvectors on the full q grid.

The reference computes them in eigenDM / phonon_phonopy
(Src/phonon_routines.f90:12-81, 84-307) from a Phonopy FORCE_CONSTANTS_2ND
with LAPACK zheev.  This module restates phonon_phonopy (Wigner-Seitz image
weights, analytic group velocities from the derivative of the dynamical
matrix, the optional dielectric correction of lines 170-210), the velocity
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


def kspace(cr: Crystal, ngrid):
    """kspace(nptk,3) of eigenDM (phonon_routines.f90:27-35), nm^-1."""
    rl = cr.rlattvec()
    n1, n2, n3 = ngrid
    nptk = n1 * n2 * n3
    k = np.zeros((nptk, 3))
    idx = np.arange(nptk)
    i1 = idx % n1
    i2 = (idx // n1) % n2
    i3 = idx // (n1 * n2)
    k = (np.outer(i1 / n1, rl[:, 0]) + np.outer(i2 / n2, rl[:, 1]) + np.outer(i3 / n3, rl[:, 2]))
    return k


def phonon_phonopy(cr: Crystal, fc, kpoints, born=None, epsilon=None, nonanalytic=False):
    """Frequencies (rad/ps), velocities (km/s) and eigenvectors for kpoints (nk,3).

    Returns omega (nk,nb), vel (nk,nb,3), eig (nk,nb,nb) with eig[k,band,comp].
    """
    nat = cr.natoms
    nb = 3 * nat
    sx, sy, sz = cr.scell
    nk = kpoints.shape[0]
    rl = cr.rlattvec()
    V = cr.volume()
    imgs = _images(cr)
    dyn = np.zeros((nk, nb, nb), dtype=np.complex128)
    ddyn = np.zeros((nk, nb, nb, 3), dtype=np.complex128)
    use_nac = nonanalytic and born is not None and np.any(born != 0)
    for (a1, a2, ix, iy, iz), rr in imgs.items():
        neq = rr.shape[0]
        qr = kpoints @ rr.T  # (nk, neq)
        z = np.exp(-1j * qr) / neq  # (nk, neq)
        blk = fc[a2, :, ix, iy, iz, a1, :].T  # blk[i,j] = fc(a2,j,cell,a1,i)
        dyn[:, 3 * a1:3 * a1 + 3, 3 * a2:3 * a2 + 3] += z.sum(axis=1)[:, None, None] * blk[None]
        zr = -1j * np.einsum("kn,nd->kd", z, rr)  # (nk,3)
        ddyn[:, 3 * a1:3 * a1 + 3, 3 * a2:3 * a2 + 3, :] += blk[None, :, :, None] * zr[:, None, None, :]
    if use_nac:
        raise NotImplementedError("dielectric correction with Born charges is not needed by the workloads")
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


def eigen_dm(cr: Crystal, fc, ngrid, symmetrizers):
    """eigenDM (phonon_routines.f90:12-81) for the full grid, arrays in the
    reference's (nptk, nb[, ...]) order."""
    k = kspace(cr, ngrid)
    omega, vel, eig = phonon_phonopy(cr, fc, k)
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
