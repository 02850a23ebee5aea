"""The factored matrix-element formula used by the CUDA kernels, evaluated in
numpy, against the oracle's literal restatement of Vp_plus/Vp_minus and
Vp_pp/Vp_pm/Vp_mm (processes.f90:25-330) on random processes (CPU).

Kernel formula (4ph, channel ch, q = grid point n, q' = n', q'' = n''):
    kappa_c = mu_c exp(2 pi i (-n.m_l + s_j n'.(m_j - m_l))/N)       s_j = -1 for --
    Z_p[s][r] = sum_{c in class p} kappa_c sum_{u,t} Psi_c[u,t,s,r] e_i[u] e~'_j[t]
    V = sum_p exp(2 pi i s_d n''.D_p/N) sum_{s,r} e~''_k[s] Z_p[s][r] conj(e'''_l[r])
with D_p = m_k - m_l and s_d = +1 for ++, -1 for +- and --.
"""
import numpy as np
import pytest

import helpers as H
import oracle as O


def _phase(s, n, m):
    ng = np.asarray(s.ngrid)
    return np.exp(2j * np.pi * np.sum((np.asarray(n) * np.asarray(m)) % ng / ng))


def _vp4_factored(s, ch, i, j, k, l, q, qp, qdp, qtp):
    f = s.ifc4
    ijk = s.ijk
    n, n1, n2 = ijk[:, q - 1], ijk[:, qp - 1], ijk[:, qdp - 1]
    masses = s.crystal.masses[s.crystal.types - 1]
    psi = f.phi.reshape(f.ntri, 3, 3, 3, 3)  # [c][r][s][t][u] (Fortran Psi(u,t,s,r,c))
    psi = np.transpose(psi, (0, 4, 3, 2, 1))  # [c][u][t][s][r]
    e = s.eig
    V = 0j
    sj = -1 if ch == 2 else 1
    sd = 1 if ch == 0 else -1
    for c in range(f.ntri):
        a1, a2, a3, a4 = (f.atoms[x, c] - 1 for x in range(4))
        mj, mk, ml = f.cells[0, c], f.cells[1, c], f.cells[2, c]
        mu = 1.0 / np.sqrt(masses[a1] * masses[a2] * masses[a3] * masses[a4])
        kap = mu * _phase(s, n, -ml) * _phase(s, n1, sj * (mj - ml))
        ei = e[q - 1, i - 1, 3 * a1:3 * a1 + 3]
        ej = e[qp - 1, j - 1, 3 * a2:3 * a2 + 3]
        ek = e[qdp - 1, k - 1, 3 * a3:3 * a3 + 3]
        el = np.conj(e[qtp - 1, l - 1, 3 * a4:3 * a4 + 3])
        if ch == 2:
            ej = np.conj(ej)
        if ch != 0:
            ek = np.conj(ek)
        Z = kap * np.einsum("utsr,u,t->sr", psi[c], ei, ej)
        V += _phase(s, n2, sd * (mk - ml)) * np.einsum("s,sr,r->", ek, Z, el)
    return V


def _vp3_factored(s, which, i, j, k, q, qp, qdp):
    f = s.ifc3
    ijk = s.ijk
    n, n1 = ijk[:, q - 1], ijk[:, qp - 1]
    masses = s.crystal.masses[s.crystal.types - 1]
    phi = np.transpose(f.phi.reshape(f.ntri, 3, 3, 3), (0, 3, 2, 1))  # [c][t][s][r]
    e = s.eig
    V = 0j
    for c in range(f.ntri):
        a1, a2, a3 = (f.atoms[x, c] - 1 for x in range(3))
        mj, mk = f.cells[0, c], f.cells[1, c]
        mu = 1.0 / np.sqrt(masses[a1] * masses[a2] * masses[a3])
        Z = mu * _phase(s, n, -mk) * np.einsum("tsr,t->sr", phi[c], e[q - 1, i - 1, 3 * a1:3 * a1 + 3])
        ej = e[qp - 1, j - 1, 3 * a2:3 * a2 + 3]
        if which < 0:
            ej = np.conj(ej)
        ek = np.conj(e[qdp - 1, k - 1, 3 * a3:3 * a3 + 3])
        V += _phase(s, n1, which * (mj - mk)) * np.einsum("s,sr,r->", ej, Z, ek)
    return V


@pytest.fixture(scope="module")
def solve():
    return H.cached_solve("diamond", (4, 4, 4))


def _qidx(s, v):
    ng = np.asarray(s.ngrid)
    v = np.mod(v, ng)
    return int(1 + v[0] + (v[1] + v[2] * ng[1]) * ng[0])


def test_vp4_factored_matches_literal(solve):
    s = solve
    o = O.Oracle(s)
    rng = np.random.default_rng(7)
    ijk = s.ijk
    for trial in range(24):
        ch = trial % 3
        q = int(s.wedge.list[rng.integers(s.nlist)])
        qp, qdp = (int(x) for x in rng.integers(1, s.nptk + 1, size=2))
        n, n1, n2 = ijk[:, q - 1], ijk[:, qp - 1], ijk[:, qdp - 1]
        t = n + n1 + n2 if ch == 0 else (n + n1 - n2 if ch == 1 else n - n1 - n2)
        qtp = _qidx(s, t)
        i, j, k, l = (int(x) for x in rng.integers(1, s.nb + 1, size=4))
        ref = o.vp4(ch, i, j, k, l, q, qp, qdp, qtp)
        mine = _vp4_factored(s, ch, i, j, k, l, q, qp, qdp, qtp)
        assert abs(mine - ref) <= 1e-11 * max(1.0, abs(ref)), (ch, ref, mine)


def test_vp3_factored_matches_literal(solve):
    s = solve
    o = O.Oracle(s)
    rng = np.random.default_rng(11)
    ijk = s.ijk
    for trial in range(16):
        which = 1 if trial % 2 == 0 else -1
        q = int(s.wedge.list[rng.integers(s.nlist)])
        qp = int(rng.integers(1, s.nptk + 1))
        qdp = _qidx(s, ijk[:, q - 1] + which * ijk[:, qp - 1])
        i, j, k = (int(x) for x in rng.integers(1, s.nb + 1, size=3))
        ref = o.vp3(which, i, j, k, q, qp, qdp)
        mine = _vp3_factored(s, which, i, j, k, q, qp, qdp)
        assert abs(mine - ref) <= 1e-11 * max(1.0, abs(ref)), (which, ref, mine)
