"""ctypes front end of the CPU oracle (libfp4_oracle.so built from fp4_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker; the product path never uses it.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "libfp4_oracle.so")
# FP4_ORACLE_LIB names another build of the same source (the sanitizer build of
# `make sanitize`); it is used as it is, without the rebuild check below.
_LIB_OVERRIDE = os.environ.get("FP4_ORACLE_LIB")
_lib = None


class _Sys(ct.Structure):
    _fields_ = [("ngrid", ct.c_int * 3), ("nptk", ct.c_int), ("nb", ct.c_int), ("nlist", ct.c_int),
                ("rlattvec", ct.c_double * 9), ("scalebroad", ct.c_double), ("T", ct.c_double),
                ("omega_max", ct.c_double), ("onlyharmonic", ct.c_int),
                ("energy", ct.c_void_p), ("velocity", ct.c_void_p), ("eig", ct.c_void_p),
                ("list", ct.c_void_p), ("ijk", ct.c_void_p), ("masses", ct.c_void_p), ("types", ct.c_void_p)]


class _Ifc(ct.Structure):
    _fields_ = [("ntri", ct.c_int), ("phi", ct.c_void_p), ("rj", ct.c_void_p), ("rk", ct.c_void_p),
                ("rl", ct.c_void_p), ("ii", ct.c_void_p), ("ij", ct.c_void_p), ("ik", ct.c_void_p),
                ("il", ct.c_void_p)]


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if _LIB_OVERRIDE:
            _lib = ct.CDLL(_LIB_OVERRIDE)
        else:
            if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(
                    os.path.join(_HERE, "fp4_oracle.c")):
                build()
            _lib = ct.CDLL(_LIB)
        _lib.fp4o_base_sigma.restype = ct.c_double
        _lib.fp4o_ind_only3.restype = ct.c_int64
        _lib.fp4o_ind_only4.restype = ct.c_int64
        _lib.fp4o_num_threads.restype = ct.c_int
        _lib.fp4o_rta4_sample.restype = ct.c_int64
        _lib.fp4o_rta4_strided.restype = ct.c_int64
        _lib.fp4o_rta4_pairs.restype = ct.c_int64
    return _lib


def _p(a):
    return a.ctypes.data_as(ct.c_void_p)


class Oracle:
    """Binds one Solve (and one temperature) to the oracle."""

    def __init__(self, solve, T=None):
        self.s = solve
        self.keep = []
        e, v, z = solve.flat()
        self.energy = np.ascontiguousarray(e, dtype=np.float64)
        self.velocity = np.ascontiguousarray(v, dtype=np.float64)
        self.eig = np.ascontiguousarray(z.view(np.float64))
        self.list = np.ascontiguousarray(solve.wedge.list, dtype=np.int32)
        self.ijk = np.ascontiguousarray(solve.ijk.T, dtype=np.int32)  # IJK(3,nptk) column-major
        self.masses = np.ascontiguousarray(solve.crystal.masses, dtype=np.float64)
        self.types = np.ascontiguousarray(solve.crystal.types, dtype=np.int32)
        sy = _Sys()
        for d in range(3):
            sy.ngrid[d] = int(solve.ngrid[d])
        sy.nptk = solve.nptk
        sy.nb = solve.nb
        sy.nlist = solve.nlist
        rl = np.asfortranarray(solve.rlattvec).ravel(order="F")
        for x in range(9):
            sy.rlattvec[x] = float(rl[x])
        sy.scalebroad = float(solve.scalebroad)
        sy.T = float(T if T is not None else solve.temperatures[0])
        sy.omega_max = float(solve.omega_max)
        sy.onlyharmonic = int(bool(solve.onlyharmonic))
        sy.energy, sy.velocity, sy.eig = _p(self.energy), _p(self.velocity), _p(self.eig)
        sy.list, sy.ijk, sy.masses, sy.types = _p(self.list), _p(self.ijk), _p(self.masses), _p(self.types)
        self.sys = sy
        self.ifc3 = self._ifc(solve.ifc3) if solve.ifc3 is not None else None
        self.ifc4 = self._ifc(solve.ifc4) if solve.ifc4 is not None else None

    def _ifc(self, ifc):
        f = _Ifc()
        f.ntri = ifc.ntri
        arrs = [np.ascontiguousarray(ifc.phi, dtype=np.float64)]
        arrs += [np.ascontiguousarray(ifc.R[x], dtype=np.float64) for x in range(ifc.order - 1)]
        arrs += [np.ascontiguousarray(ifc.atoms[x], dtype=np.int32) for x in range(ifc.order)]
        self.keep.append(arrs)
        f.phi = _p(arrs[0])
        f.rj = _p(arrs[1])
        f.rk = _p(arrs[2])
        f.rl = _p(arrs[3]) if ifc.order == 4 else None
        f.ii = _p(arrs[ifc.order])
        f.ij = _p(arrs[ifc.order + 1])
        f.ik = _p(arrs[ifc.order + 2])
        f.il = _p(arrs[ifc.order + 3]) if ifc.order == 4 else None
        return f

    # -- counting --------------------------------------------------------------
    def np3(self, mm0=0, mm1=None):
        nm = self.s.nmodes
        mm1 = nm if mm1 is None else mm1
        n_p = np.zeros(nm, np.int32); n_m = np.zeros(nm, np.int32)
        p_p = np.zeros(nm); p_m = np.zeros(nm)
        lib().fp4o_np3(ct.byref(self.sys), mm0, mm1, _p(n_p), _p(n_m), _p(p_p), _p(p_m))
        return n_p, n_m, p_p, p_m

    def np4(self, mm0=0, mm1=None):
        nm = self.s.nmodes
        mm1 = nm if mm1 is None else mm1
        n = [np.zeros(nm, np.int64) for _ in range(3)]
        p = [np.zeros(nm) for _ in range(3)]
        lib().fp4o_np4(ct.byref(self.sys), mm0, mm1, *[_p(x) for x in n], *[_p(x) for x in p])
        return n, p

    def ind_only3(self, mm, which, cap):
        a = np.zeros(cap, np.int32); b = np.zeros(cap, np.int32)
        n = lib().fp4o_ind_only3(ct.byref(self.sys), mm, which, ct.c_int64(cap), _p(a), _p(b))
        return a[:n], b[:n], n

    def ind_only4(self, mm, ch, cap):
        a = np.zeros(cap, np.int64); b = np.zeros(cap, np.int64); c = np.zeros(cap, np.int64)
        n = lib().fp4o_ind_only4(ct.byref(self.sys), mm, ch, ct.c_int64(cap), _p(a), _p(b), _p(c))
        return a[:n], b[:n], c[:n], n

    # -- rates -----------------------------------------------------------------
    def rta3(self, mm0=0, mm1=None):
        nm = self.s.nmodes
        mm1 = nm if mm1 is None else mm1
        out = [np.zeros(nm) for _ in range(4)]
        lib().fp4o_rta3(ct.byref(self.sys), ct.byref(self.ifc3), mm0, mm1, *[_p(x) for x in out])
        return out  # rate_plus, rate_minus(x0.5), wp3_plus, wp3_minus

    def rta4(self, mm0=0, mm1=None):
        nm = self.s.nmodes
        mm1 = nm if mm1 is None else mm1
        out = [np.zeros(nm) for _ in range(6)]
        lib().fp4o_rta4(ct.byref(self.sys), ct.byref(self.ifc4), mm0, mm1, *[_p(x) for x in out])
        return out  # rate_pp, rate_pm, rate_mm, wp_pp, wp_pm, wp_mm

    def rta4_range(self, mm0, mm1, ii0, ii1):
        """RTA_driver_4ph over modes [mm0,mm1) restricted to q' in [ii0,ii1) (0-based),
        normalised as the full driver: rate_pp, rate_pm, rate_mm, wp_pp, wp_pm, wp_mm."""
        nm = self.s.nmodes
        out = [np.zeros(nm) for _ in range(6)]
        lib().fp4o_rta4_range(ct.byref(self.sys), ct.byref(self.ifc4), mm0, mm1, ii0, ii1, *[_p(x) for x in out])
        return out

    def rta4_strided(self, modes, ii_stride, ii_offset=0):
        """Timing sample: RTA_driver_4ph work of the listed modes (0-based) over the
        q' points ii_offset, ii_offset + ii_stride, ...; returns the surviving
        processes visited."""
        m = np.ascontiguousarray(modes, dtype=np.int32)
        return int(lib().fp4o_rta4_strided(ct.byref(self.sys), ct.byref(self.ifc4), _p(m), int(m.size),
                                             int(ii_stride), int(ii_offset)))

    def rta4_pairs(self, modes, qps):
        """Timing sample: RTA_driver_4ph work at the (mode, q') pairs (0-based);
        returns the surviving processes visited."""
        m = np.ascontiguousarray(modes, dtype=np.int32)
        q = np.ascontiguousarray(qps, dtype=np.int32)
        return int(lib().fp4o_rta4_pairs(ct.byref(self.sys), ct.byref(self.ifc4), _p(m), _p(q), int(m.size)))

    def rta4_sample(self, mm0, mm1, ii0, ii1):
        """Timing sample: RTA_driver_4ph work for modes [mm0,mm1) restricted to
        q' in [ii0,ii1); returns the number of surviving processes visited."""
        return int(lib().fp4o_rta4_sample(ct.byref(self.sys), ct.byref(self.ifc4), mm0, mm1, ii0, ii1))

    def ind3(self, n_plus, n_minus):
        tp, tm = int(n_plus.sum()), int(n_minus.sum())
        nm = self.s.nmodes
        i2p = np.zeros(tp, np.int32); i3p = np.zeros(tp, np.int32); gp = np.zeros(tp)
        i2m = np.zeros(tm, np.int32); i3m = np.zeros(tm, np.int32); gm = np.zeros(tm)
        outs = [np.zeros(nm) for _ in range(4)]
        lib().fp4o_ind3(ct.byref(self.sys), ct.byref(self.ifc3), _p(np.ascontiguousarray(n_plus, np.int32)),
                        _p(np.ascontiguousarray(n_minus, np.int32)), _p(i2p), _p(i3p), _p(gp), _p(i2m), _p(i3m),
                        _p(gm), *[_p(x) for x in outs])
        return dict(ind2_plus=i2p, ind3_plus=i3p, gamma_plus=gp, ind2_minus=i2m, ind3_minus=i3m, gamma_minus=gm,
                    rate_plus=outs[0], rate_minus=outs[1], wp3_plus=outs[2], wp3_minus=outs[3])

    def ind4(self, n_pp, n_pm, n_mm):
        """Ind_driver_4ph: per-process Gamma lists, rates and WP4 of the three channels.
        Returns a dict usable as the `ind4` argument of iteration()."""
        nm = self.s.nmodes
        N = [np.ascontiguousarray(x, np.int64) for x in (n_pp, n_pm, n_mm)]
        out = dict(n_pp=N[0], n_pm=N[1], n_mm=N[2])
        args = [ct.byref(self.sys), ct.byref(self.ifc4)] + [_p(x) for x in N]
        for ch, n in zip(("pp", "pm", "mm"), N):
            tot = int(n.sum())
            for key in ("ind2_", "ind3_", "ind4_"):
                out[key + ch] = np.zeros(tot, np.int64)
            out["gamma_" + ch] = np.zeros(tot)
            args += [_p(out["ind2_" + ch]), _p(out["ind3_" + ch]), _p(out["ind4_" + ch]), _p(out["gamma_" + ch])]
        for key in ("rate_pp", "rate_pm", "rate_mm", "wp_pp", "wp_pm", "wp_mm"):
            out[key] = np.zeros(nm)
        args += [_p(out[k]) for k in ("rate_pp", "rate_pm", "rate_mm", "wp_pp", "wp_pm", "wp_mm")]
        lib().fp4o_ind4(*args)
        return out

    def vp3(self, which, i, j, k, q, qp, qdp):
        rq = self._realq(qp); rqd = self._realq(qdp)
        re = ct.c_double(); im = ct.c_double()
        lib().fp4o_vp3(ct.byref(self.sys), ct.byref(self.ifc3), which, i, j, k, q, qp, qdp, _p(rq), _p(rqd),
                       ct.byref(re), ct.byref(im))
        return complex(re.value, im.value)

    def vp4(self, ch, i, j, k, l, q, qp, qdp, qtp):
        a, b, c = self._realq(qp), self._realq(qdp), self._realq(qtp)
        re = ct.c_double(); im = ct.c_double()
        lib().fp4o_vp4(ct.byref(self.sys), ct.byref(self.ifc4), ch, i, j, k, l, q, qp, qdp, qtp, _p(a), _p(b), _p(c),
                       ct.byref(re), ct.byref(im))
        return complex(re.value, im.value)

    def _realq(self, q1):
        n = self.s.ijk[:, q1 - 1].astype(np.float64) / np.asarray(self.s.ngrid, np.float64)
        rl = self.s.rlattvec
        out = np.zeros(3)
        for i in range(3):
            acc = 0.0
            acc = acc + rl[i, 0] * n[0]
            acc = acc + rl[i, 1] * n[1]
            acc = acc + rl[i, 2] * n[2]
            out[i] = acc
        return out

    # -- BTE -------------------------------------------------------------------
    def iteration0(self, tau_zero):
        F = np.zeros(self.s.nb * self.s.nptk * 3)
        w = self.s.wedge
        lib().fp4o_iteration0(ct.byref(self.sys), self.s.sym.nsymm_rot, _p(np.ascontiguousarray(w.nequi, np.int32)),
                              _p(np.ascontiguousarray(w.allequi, np.int32)),
                              _p(np.ascontiguousarray(tau_zero, np.float64)), _p(F))
        return F

    def iteration(self, F, tau_zero, n_plus, n_minus, ind3_lists, ind4=None):
        w = self.s.wedge
        symm = np.ascontiguousarray(np.transpose(self.s.sym.symmetrizers, (0, 2, 1))).ravel()
        idq = np.ascontiguousarray(w.id_equi.T, np.int32)  # ID_equi(nsymm_rot,nptk) column-major
        args = [ct.byref(self.sys), self.s.sym.nsymm_rot, _p(np.ascontiguousarray(w.nequi, np.int32)),
                _p(np.ascontiguousarray(w.allequi, np.int32)), _p(np.ascontiguousarray(w.typeofsym, np.int32)),
                _p(idq), _p(symm), _p(np.ascontiguousarray(n_plus, np.int32)), _p(np.ascontiguousarray(n_minus, np.int32)),
                _p(ind3_lists["ind2_plus"]), _p(ind3_lists["ind3_plus"]), _p(ind3_lists["gamma_plus"]),
                _p(ind3_lists["ind2_minus"]), _p(ind3_lists["ind3_minus"]), _p(ind3_lists["gamma_minus"])]
        if ind4 is None:
            args += [None] * 15
        else:
            args += [_p(ind4["n_pp"]), _p(ind4["n_pm"]), _p(ind4["n_mm"])]
            for ch in ("pp", "pm", "mm"):
                args += [_p(ind4["ind2_" + ch]), _p(ind4["ind3_" + ch]), _p(ind4["ind4_" + ch]), _p(ind4["gamma_" + ch])]
        args += [_p(np.ascontiguousarray(tau_zero, np.float64)), _p(F)]
        lib().fp4o_iteration(*args)
        return F

    def symmetrize_fn(self, F):
        symm = np.ascontiguousarray(np.transpose(self.s.sym.symmetrizers, (0, 2, 1))).ravel()
        lib().fp4o_symmetrize_fn(ct.byref(self.sys), _p(symm), _p(F))
        return F

    def tconduct(self, F):
        k = np.zeros(self.s.nb * 9)
        lib().fp4o_tconduct(ct.byref(self.sys), ct.c_double(self.s.volume), _p(F), _p(k))
        return k

    def sample4(self, nsamples, seed, mode=2, mm0=0, mm1=None):
        """Seeded NP_*_sample (mode 0) / RTA_*_sample (mode 2): arrays [ch][mode]."""
        nm = self.s.nmodes
        mm1 = nm if mm1 is None else mm1
        n = np.zeros(3 * nm, np.int64)
        p = np.zeros(3 * nm)
        r = np.zeros(3 * nm)
        w = np.zeros(3 * nm)
        lib().fp4o_sample4(ct.byref(self.sys), ct.byref(self.ifc4) if self.ifc4 is not None else None, mm0, mm1,
                           ct.c_int64(nsamples), ct.c_uint64(seed), mode, _p(n), _p(p), _p(r), _p(w))
        return dict(n=n.reshape(3, nm), p=p.reshape(3, nm), rate=r.reshape(3, nm), wp=w.reshape(3, nm))

    def sample3(self, nsamples, seed, mode=2, mm0=0, mm1=None):
        """Seeded NP_plus/minus_sample (mode 0) / RTA_plus/minus_sample (mode 2):
        arrays [ch][mode], ch 0 absorption, 1 emission (rate with the driver's x0.5)."""
        nm = self.s.nmodes
        mm1 = nm if mm1 is None else mm1
        n = np.zeros(2 * nm, np.int32)
        p = np.zeros(2 * nm)
        r = np.zeros(2 * nm)
        w = np.zeros(2 * nm)
        lib().fp4o_sample3(ct.byref(self.sys), ct.byref(self.ifc3) if self.ifc3 is not None else None, mm0, mm1,
                           ct.c_int64(nsamples), ct.c_uint64(seed), mode, _p(n), _p(p), _p(r), _p(w))
        return dict(n=n.reshape(2, nm), p=p.reshape(2, nm), rate=r.reshape(2, nm), wp=w.reshape(2, nm))

    def cumulative_tconduct(self, F, nticks=100, omega_mode=False):
        ticks = np.zeros(nticks)
        res = np.zeros(self.s.nb * 9 * nticks)
        lib().fp4o_cumulative_tconduct(ct.byref(self.sys), ct.c_double(self.s.volume), _p(F), nticks,
                                       1 if omega_mode else 0, _p(ticks), _p(res))
        return ticks, res

    def symmetrize_tensor(self, t33):
        crot = np.ascontiguousarray(np.transpose(self.s.sym.crotations, (0, 2, 1))).ravel()
        t = np.asfortranarray(t33).ravel(order="F").copy()
        lib().fp4o_symmetrize_tensor(self.s.sym.nsymm_rot, _p(crot), _p(t))
        return t.reshape(3, 3, order="F")
