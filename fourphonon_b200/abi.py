"""ctypes binding of libfp4b200.so, mirroring the reference's driver interface.

Each method takes a :class:`fourphonon_b200.system.Solve` (the arrays the
Fortran host holds when it calls the driver) and returns what the Fortran
subroutine writes into its intent(out) arguments, under the same names:

    np_driver            -> NP_driver          (processes.f90:983)
    np_driver_4ph        -> NP_driver_4ph      (processes.f90:2749)
    ind_only_driver      -> Ind_only_driver    (processes.f90:1198)
    ind_only_driver_4ph  -> Ind_only_driver_4ph(processes.f90:3080)
    rta_driver           -> RTA_driver         (processes.f90:1676)
    rta_driver_4ph       -> RTA_driver_4ph     (processes.f90:5174)
    ind_driver           -> Ind_driver         (processes.f90:524)
    iteration0/iteration -> iterations.f90:13 / 34
    tconduct             -> TConduct           (conductivity.f90:11)
    eigen_dm             -> eigenDM / phonon_phonopy (phonon_routines.f90:12 / 84)
    np_driver_sample / rta_driver_sample         -> NP_/RTA_plus/minus_sample (processes.f90:828 / 1474)
    np_driver_4ph_sample / rta_driver_4ph_sample -> NP_/RTA_plusplus..._sample (processes.f90:2480 / 4811)

The library is required: loading fails with an error if it is missing or was
not built, and every failing call raises :class:`FP4Error` with the
library's message.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

from . import build as _build

_lib = None

FP4_PREC_FP64 = 0
FP4_PREC_MIXED = 1
FP4_PREC_MIXED_SIMT = 2
FP4_OK = 0
FP4_E_ARG = -1
FP4_E_CUDA = -2
FP4_E_CAPACITY = -3
FP4_E_TIMEOUT = -4
FP4_E_STATE = -5


class FP4Error(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"fp4 error {code}: {msg}")
        self.code = code


class Globals(ct.Structure):
    _fields_ = [("ngrid", ct.c_int32 * 3), ("nbands", ct.c_int32), ("rlattvec", ct.c_double * 9), ("T", ct.c_double),
                ("scalebroad", ct.c_double), ("omega_max", ct.c_double), ("onlyharmonic", ct.c_int32),
                ("nelements", ct.c_int32), ("natoms", ct.c_int32), ("masses", ct.c_void_p), ("types", ct.c_void_p)]


def library_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load the CUDA library (building it with nvcc when asked and absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_build.LIB):
        if not build_if_missing:
            raise FP4Error(-5, f"{_build.LIB} is missing; build it with python -m fourphonon_b200.build")
        _build.build()
    lib = ct.CDLL(_build.LIB)
    lib.fp4_last_error.restype = ct.c_char_p
    lib.fp4_last_error.argtypes = [ct.c_void_p]
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


def tc_selftest(A_bf16: np.ndarray, B_bf16: np.ndarray) -> np.ndarray:
    """D = A B^T on the tensor cores (fp4_tc_selftest): A (128, K) and B (N, K)
    as raw bf16 bits (uint16), D (128, N) float32."""
    lib = load()
    A = np.ascontiguousarray(A_bf16, dtype=np.uint16)
    B = np.ascontiguousarray(B_bf16, dtype=np.uint16)
    assert A.shape[0] == 128 and A.shape[1] == B.shape[1]
    D = np.zeros((128, B.shape[0]), dtype=np.float32)
    rc = lib.fp4_tc_selftest(ct.c_int32(A.shape[1]), ct.c_int32(B.shape[0]), _p(A), _p(B), _p(D))
    if rc != 0:
        raise FP4Error(rc, "fp4_tc_selftest failed")
    return D


class Context:
    """One fp4_ctx (one CUDA stream and its device-resident buffers)."""

    def __init__(self, device: int = 0, precision: int = FP4_PREC_FP64):
        self.lib = load()
        h = ct.c_void_p()
        rc = self.lib.fp4_create(ct.byref(h), device)
        if rc != 0:
            raise FP4Error(rc, "fp4_create failed (no CUDA device?)")
        self.h = h
        self._keep = []
        self.set_precision(precision)

    def close(self):
        if self.h:
            self.lib.fp4_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        if rc != 0:
            raise FP4Error(rc, self.lib.fp4_last_error(self.h).decode())

    def set_precision(self, precision: int):
        self._chk(self.lib.fp4_set_precision(self.h, precision))

    def stats(self):
        """(surviving processes, contracted processes, call ms, main-kernel ms, kernel launches)
        of the last call."""
        n = ct.c_int64()
        k = ct.c_int64()
        ms = ct.c_double()
        kms = ct.c_double()
        nl = ct.c_int64()
        self._chk(self.lib.fp4_last_stats(self.h, ct.byref(n), ct.byref(k), ct.byref(ms), ct.byref(kms),
                                          ct.byref(nl)))
        return n.value, k.value, ms.value, kms.value, nl.value

    def counters(self):
        """Work counters of the last four-phonon call (see fp4_last_counters)."""
        a = (ct.c_int64 * 8)()
        self._chk(self.lib.fp4_last_counters(self.h, a))
        return list(a)

    def phase_cycles(self, full=False):
        """(work-item cycles, phase-B cycles) of the last four-phonon work kernel,
        summed over its CTAs; full=True: all eight fields of fp4_last_phase_cycles."""
        a = (ct.c_int64 * 8)()
        self._chk(self.lib.fp4_last_phase_cycles(self.h, a))
        return [int(x) for x in a] if full else (int(a[0]), int(a[1]))

    def set_stream(self, stream_handle):
        """Run on an existing cudaStream_t (an int handle, e.g. torch's stream.cuda_stream)."""
        self._chk(self.lib.fp4_set_stream(self.h, ct.c_void_p(stream_handle) if stream_handle else None))

    def set_upload_cache(self, enable: bool):
        self._chk(self.lib.fp4_set_upload_cache(self.h, 1 if enable else 0))

    # -- argument marshalling ----------------------------------------------------
    def globals_of(self, s, T=None) -> Globals:
        g = Globals()
        for d in range(3):
            g.ngrid[d] = int(s.ngrid[d])
        g.nbands = int(s.nb)
        rl = np.asfortranarray(s.rlattvec).ravel(order="F")
        for x in range(9):
            g.rlattvec[x] = float(rl[x])
        g.T = float(T if T is not None else s.temperatures[0])
        g.scalebroad = float(s.scalebroad)
        g.omega_max = float(s.omega_max)
        g.onlyharmonic = int(bool(s.onlyharmonic))
        masses = np.ascontiguousarray(s.crystal.masses, dtype=np.float64)
        types = np.ascontiguousarray(s.crystal.types, dtype=np.int32)
        self._keep = [masses, types]
        g.nelements = masses.size
        g.natoms = types.size
        g.masses = _p(masses)
        g.types = _p(types)
        return g

    @staticmethod
    def _arrays(s):
        e, v, z = s.flat()
        e = np.ascontiguousarray(e, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        z = np.ascontiguousarray(z, dtype=np.complex128)
        lst = np.ascontiguousarray(s.wedge.list, dtype=np.int32)
        ijk = np.ascontiguousarray(s.ijk.T, dtype=np.int32)
        return e, v, z, lst, ijk

    @staticmethod
    def _ifc(ifc):
        arrs = [np.ascontiguousarray(ifc.phi, dtype=np.float64)]
        arrs += [np.ascontiguousarray(ifc.R[x], dtype=np.float64) for x in range(ifc.order - 1)]
        arrs += [np.ascontiguousarray(ifc.atoms[x], dtype=np.int32) for x in range(ifc.order)]
        return arrs

    # -- three-phonon drivers ------------------------------------------------------
    def np_driver(self, s):
        g = self.globals_of(s)
        e, v, _, lst, ijk = self._arrays(s)
        nm = s.nmodes
        n_p = np.zeros(nm, np.int32); n_m = np.zeros(nm, np.int32)
        p_p = np.zeros(nm); p_m = np.zeros(nm)
        self._chk(self.lib.fp4_np_driver(self.h, ct.byref(g), _p(e), _p(v), s.nlist, _p(lst), _p(ijk), _p(n_p), _p(p_p),
                                         _p(n_m), _p(p_m)))
        return n_p, n_m, p_p, p_m

    def ind_only_driver(self, s, n_plus, n_minus):
        g = self.globals_of(s)
        e, v, _, lst, ijk = self._arrays(s)
        n_plus = np.ascontiguousarray(n_plus, np.int32)
        n_minus = np.ascontiguousarray(n_minus, np.int32)
        tp, tm = int(n_plus.sum()), int(n_minus.sum())
        a = np.zeros(tp, np.int32); b = np.zeros(tp, np.int32)
        c = np.zeros(tm, np.int32); d = np.zeros(tm, np.int32)
        self._chk(self.lib.fp4_ind_only_driver(self.h, ct.byref(g), _p(e), _p(v), s.nlist, _p(lst), _p(ijk),
                                               _p(n_plus), _p(n_minus), _p(a), _p(b), _p(c), _p(d)))
        return a, b, c, d

    def rta_driver(self, s, T=None):
        g = self.globals_of(s, T)
        e, v, z, lst, ijk = self._arrays(s)
        f = self._ifc(s.ifc3)
        nm = s.nmodes
        out = [np.zeros(nm) for _ in range(5)]
        self._chk(self.lib.fp4_rta_driver(self.h, ct.byref(g), _p(e), _p(v), _p(z), s.nlist, _p(lst), _p(ijk),
                                          s.ifc3.ntri, *[_p(x) for x in f], *[_p(x) for x in out]))
        return dict(rate=out[0], rate_plus=out[1], rate_minus=out[2], wp3_plus=out[3], wp3_minus=out[4])

    def ind_driver(self, s, n_plus, n_minus, T=None):
        g = self.globals_of(s, T)
        e, v, z, lst, ijk = self._arrays(s)
        f = self._ifc(s.ifc3)
        n_plus = np.ascontiguousarray(n_plus, np.int32)
        n_minus = np.ascontiguousarray(n_minus, np.int32)
        tp, tm = int(n_plus.sum()), int(n_minus.sum())
        i2p = np.zeros(tp, np.int32); i3p = np.zeros(tp, np.int32); gp = np.zeros(tp)
        i2m = np.zeros(tm, np.int32); i3m = np.zeros(tm, np.int32); gm = np.zeros(tm)
        nm = s.nmodes
        out = [np.zeros(nm) for _ in range(5)]
        self._chk(self.lib.fp4_ind_driver(self.h, ct.byref(g), _p(e), _p(v), _p(z), s.nlist, _p(lst), _p(ijk),
                                          _p(n_plus), _p(n_minus), s.ifc3.ntri, *[_p(x) for x in f], _p(i2p), _p(i3p),
                                          _p(gp), _p(i2m), _p(i3m), _p(gm), *[_p(x) for x in out]))
        return dict(ind2_plus=i2p, ind3_plus=i3p, gamma_plus=gp, ind2_minus=i2m, ind3_minus=i3m, gamma_minus=gm,
                    rate=out[0], rate_plus=out[1], rate_minus=out[2], wp3_plus=out[3], wp3_minus=out[4])

    # -- four-phonon drivers -------------------------------------------------------
    def np_driver_4ph(self, s):
        g = self.globals_of(s)
        e, v, _, lst, ijk = self._arrays(s)
        nm = s.nmodes
        n = [np.zeros(nm, np.int64) for _ in range(3)]
        p = [np.zeros(nm) for _ in range(3)]
        self._chk(self.lib.fp4_np_driver_4ph(self.h, ct.byref(g), _p(e), _p(v), s.nlist, _p(lst), _p(ijk),
                                             _p(n[0]), _p(p[0]), _p(n[1]), _p(p[1]), _p(n[2]), _p(p[2])))
        return n, p

    def ind_only_driver_4ph(self, s, n_pp, n_pm, n_mm):
        g = self.globals_of(s)
        e, v, _, lst, ijk = self._arrays(s)
        ns = [np.ascontiguousarray(x, np.int64) for x in (n_pp, n_pm, n_mm)]
        outs = [[np.zeros(int(x.sum()), np.int64) for _ in range(3)] for x in ns]
        self._chk(self.lib.fp4_ind_only_driver_4ph(self.h, ct.byref(g), _p(e), _p(v), s.nlist, _p(lst), _p(ijk),
                                                   *[_p(x) for x in ns], *[_p(a) for ch in outs for a in ch]))
        return outs

    def rta_driver_4ph(self, s, temperatures=None):
        """RTA_driver_4ph at each temperature (multi-temperature fused call).

        Returns dict of arrays shaped (nT, nmodes)."""
        temps = np.ascontiguousarray(s.temperatures if temperatures is None else temperatures, dtype=np.float64)
        g = self.globals_of(s, float(temps[0]))
        e, v, z, lst, ijk = self._arrays(s)
        f = self._ifc(s.ifc4)
        nm = s.nmodes
        nT = temps.size
        out = [np.zeros(nm * nT) for _ in range(6)]
        self._chk(self.lib.fp4_rta_driver_4ph_multi_t(self.h, ct.byref(g), nT, _p(temps), _p(e), _p(v), _p(z),
                                                      s.nlist, _p(lst), _p(ijk), s.ifc4.ntri, *[_p(x) for x in f],
                                                      *[_p(x) for x in out]))
        names = ("rate_plusplus", "rate_plusminus", "rate_minusminus", "wp4_plusplus", "wp4_plusminus",
                 "wp4_minusminus")
        d = {k: o.reshape(nT, nm) for k, o in zip(names, out)}
        d["rate_4ph"] = d["rate_plusplus"] + d["rate_plusminus"] + d["rate_minusminus"]
        return d

    def rta4_partials(self, s, ll, ii0, ii1, t=0):
        """The last rta_driver_4ph call's rates and WP4 of irreducible point ll
        (0-based) at temperature index t from the q' in [ii0, ii1): arrays of
        nbands per channel, keyed like rta_driver_4ph's result."""
        out = [np.zeros(s.nb) for _ in range(6)]
        self._chk(self.lib.fp4_rta4_partials(self.h, ll, ii0, ii1, t, *[_p(x) for x in out]))
        names = ("rate_plusplus", "rate_plusminus", "rate_minusminus", "wp4_plusplus", "wp4_plusminus",
                 "wp4_minusminus")
        return dict(zip(names, out))

    def ind_driver_4ph(self, s, n_pp, n_pm, n_mm, T=None):
        """Ind_driver_4ph: the three channels' index lists and per-process Gamma,
        rates and WP4 per mode.  Keys follow the oracle's ind4(), so the result
        is also the `ind4` argument of iteration()."""
        g = self.globals_of(s, T)
        e, v, z, lst, ijk = self._arrays(s)
        f = self._ifc(s.ifc4)
        nm = s.nmodes
        N = [np.ascontiguousarray(x, np.int64) for x in (n_pp, n_pm, n_mm)]
        d = dict(n_pp=N[0], n_pm=N[1], n_mm=N[2])
        lists = []
        for ch, n in zip(("pp", "pm", "mm"), N):
            tot = int(n.sum())
            for key in ("ind2_", "ind3_", "ind4_"):
                d[key + ch] = np.zeros(tot, np.int64)
            d["gamma_" + ch] = np.zeros(tot)
            lists += [d["ind2_" + ch], d["ind3_" + ch], d["ind4_" + ch], d["gamma_" + ch]]
        names = ("rate_4ph", "rate_pp", "rate_pm", "rate_mm", "wp_pp", "wp_pm", "wp_mm")
        for k in names:
            d[k] = np.zeros(nm)
        self._chk(self.lib.fp4_ind_driver_4ph(self.h, ct.byref(g), _p(e), _p(v), _p(z), s.nlist, _p(lst), _p(ijk),
                                              *[_p(x) for x in N], s.ifc4.ntri, *[_p(x) for x in f],
                                              *[_p(x) for x in lists], *[_p(d[k]) for k in names]))
        return d

    def np_driver_sample(self, s, nsamples, seed):
        """Sampled NP_driver: (n_plus, n_minus, p_plus, p_minus), as np_driver returns them."""
        g = self.globals_of(s)
        e, v, _, lst, ijk = self._arrays(s)
        nm = s.nmodes
        n_p = np.zeros(nm, np.int32); n_m = np.zeros(nm, np.int32)
        p_p = np.zeros(nm); p_m = np.zeros(nm)
        self._chk(self.lib.fp4_np_driver_sample(self.h, ct.byref(g), _p(e), _p(v), s.nlist, _p(lst), _p(ijk),
                                                ct.c_int64(nsamples), ct.c_uint64(seed), _p(n_p), _p(p_p), _p(n_m),
                                                _p(p_m)))
        return n_p, n_m, p_p, p_m

    def rta_driver_sample(self, s, nsamples, seed, T=None):
        """Sampled RTA_driver at T (default: the solve's first temperature)."""
        g = self.globals_of(s, T)
        e, v, z, lst, ijk = self._arrays(s)
        f = self._ifc(s.ifc3)
        nm = s.nmodes
        out = [np.zeros(nm) for _ in range(5)]
        self._chk(self.lib.fp4_rta_driver_sample(self.h, ct.byref(g), _p(e), _p(v), _p(z), s.nlist, _p(lst), _p(ijk),
                                                 s.ifc3.ntri, *[_p(x) for x in f], ct.c_int64(nsamples),
                                                 ct.c_uint64(seed), *[_p(x) for x in out]))
        return dict(rate=out[0], rate_plus=out[1], rate_minus=out[2], wp3_plus=out[3], wp3_minus=out[4])

    def np_driver_4ph_sample(self, s, nsamples, seed):
        """Sampled NP_driver_4ph: (N, P) per channel, as np_driver_4ph returns them."""
        g = self.globals_of(s)
        e, v, _, lst, ijk = self._arrays(s)
        nm = s.nmodes
        n = [np.zeros(nm, np.int64) for _ in range(3)]
        p = [np.zeros(nm) for _ in range(3)]
        self._chk(self.lib.fp4_np_driver_4ph_sample(self.h, ct.byref(g), _p(e), _p(v), s.nlist, _p(lst), _p(ijk),
                                                    ct.c_int64(nsamples), ct.c_uint64(seed), _p(n[0]), _p(p[0]),
                                                    _p(n[1]), _p(p[1]), _p(n[2]), _p(p[2])))
        return n, p

    def rta_driver_4ph_sample(self, s, nsamples, seed, temperatures=None):
        """Sampled RTA_driver_4ph at each temperature; dict of (nT, nmodes) arrays."""
        temps = np.ascontiguousarray(s.temperatures if temperatures is None else temperatures, dtype=np.float64)
        g = self.globals_of(s, float(temps[0]))
        e, v, z, lst, ijk = self._arrays(s)
        f = self._ifc(s.ifc4)
        nm = s.nmodes
        nT = temps.size
        out = [np.zeros(nm * nT) for _ in range(6)]
        self._chk(self.lib.fp4_rta_driver_4ph_sample_multi_t(
            self.h, ct.byref(g), nT, _p(temps), _p(e), _p(v), _p(z), s.nlist, _p(lst), _p(ijk), s.ifc4.ntri,
            *[_p(x) for x in f], ct.c_int64(nsamples), ct.c_uint64(seed), *[_p(x) for x in out]))
        names = ("rate_plusplus", "rate_plusminus", "rate_minusminus", "wp4_plusplus", "wp4_plusminus",
                 "wp4_minusminus")
        d = {k: o.reshape(nT, nm) for k, o in zip(names, out)}
        d["rate_4ph"] = d["rate_plusplus"] + d["rate_plusminus"] + d["rate_minusminus"]
        return d

    # -- BTE -------------------------------------------------------------------------
    def iteration0(self, s, tau_zero):
        g = self.globals_of(s)
        e, v, _, _, _ = self._arrays(s)
        w = s.wedge
        nsr = s.sym.nsymm_rot
        F = np.zeros(s.nb * s.nptk * 3)
        self._chk(self.lib.fp4_iteration0(self.h, ct.byref(g), s.nlist, _p(np.ascontiguousarray(w.nequi, np.int32)),
                                          _p(np.ascontiguousarray(w.allequi, np.int32)), nsr, _p(e), _p(v),
                                          _p(np.ascontiguousarray(tau_zero, np.float64)), _p(F)))
        return F

    def iteration(self, s, F, tau_zero, n_plus, n_minus, lists, ind4=None):
        """One sweep: iteration, or iteration_4ph when the 4-phonon lists
        `ind4` (from ind_driver_4ph) are given."""
        if ind4 is not None:
            return self._iteration_4ph(s, F, tau_zero, n_plus, n_minus, lists, ind4)
        g = self.globals_of(s)
        e, v, _, _, _ = self._arrays(s)
        w = s.wedge
        nsr = s.sym.nsymm_rot
        symm = np.ascontiguousarray(np.transpose(s.sym.symmetrizers, (0, 2, 1))).ravel()
        idq = np.ascontiguousarray(w.id_equi.T, np.int32)
        n_plus = np.ascontiguousarray(n_plus, np.int32)
        n_minus = np.ascontiguousarray(n_minus, np.int32)
        self._chk(self.lib.fp4_iteration(
            self.h, ct.byref(g), s.nlist, _p(np.ascontiguousarray(w.nequi, np.int32)),
            _p(np.ascontiguousarray(w.allequi, np.int32)), _p(np.ascontiguousarray(w.typeofsym, np.int32)), nsr,
            _p(idq), _p(symm), _p(n_plus), _p(n_minus), int(n_plus.sum()), int(n_minus.sum()),
            _p(lists["ind2_plus"]), _p(lists["ind3_plus"]), _p(lists["ind2_minus"]), _p(lists["ind3_minus"]), _p(e),
            _p(v), _p(lists["gamma_plus"]), _p(lists["gamma_minus"]), _p(np.ascontiguousarray(tau_zero, np.float64)),
            _p(F)))
        return F

    def iteration_jacobi(self, s, F, tau_zero, n_plus, n_minus, lists):
        """One Jacobi sweep (fp4_iteration_jacobi): every step reads F, the new
        F_n (site symmetrizers applied) is returned."""
        g = self.globals_of(s)
        e, v, _, _, _ = self._arrays(s)
        w = s.wedge
        nsr = s.sym.nsymm_rot
        symm = np.ascontiguousarray(np.transpose(s.sym.symmetrizers, (0, 2, 1))).ravel()
        idq = np.ascontiguousarray(w.id_equi.T, np.int32)
        n_plus = np.ascontiguousarray(n_plus, np.int32)
        n_minus = np.ascontiguousarray(n_minus, np.int32)
        out = np.array(F, dtype=np.float64, copy=True)
        self._chk(self.lib.fp4_iteration_jacobi(
            self.h, ct.byref(g), s.nlist, _p(np.ascontiguousarray(w.nequi, np.int32)),
            _p(np.ascontiguousarray(w.allequi, np.int32)), _p(np.ascontiguousarray(w.typeofsym, np.int32)), nsr,
            _p(idq), _p(symm), _p(n_plus), _p(n_minus), int(n_plus.sum()), int(n_minus.sum()),
            _p(lists["ind2_plus"]), _p(lists["ind3_plus"]), _p(lists["ind2_minus"]), _p(lists["ind3_minus"]), _p(e),
            _p(v), _p(lists["gamma_plus"]), _p(lists["gamma_minus"]), _p(np.ascontiguousarray(tau_zero, np.float64)),
            _p(out)))
        return out

    def _iteration_4ph(self, s, F, tau_zero, n_plus, n_minus, lists, ind4):
        g = self.globals_of(s)
        e, v, _, _, _ = self._arrays(s)
        w = s.wedge
        nsr = s.sym.nsymm_rot
        symm = np.ascontiguousarray(np.transpose(s.sym.symmetrizers, (0, 2, 1))).ravel()
        idq = np.ascontiguousarray(w.id_equi.T, np.int32)
        n_plus = np.ascontiguousarray(n_plus, np.int32)
        n_minus = np.ascontiguousarray(n_minus, np.int32)
        N = [np.ascontiguousarray(ind4["n_" + ch], np.int64) for ch in ("pp", "pm", "mm")]
        L = {k: np.ascontiguousarray(ind4[k], np.int64) for ch in ("pp", "pm", "mm")
             for k in ("ind2_" + ch, "ind3_" + ch, "ind4_" + ch)}
        G = [np.ascontiguousarray(ind4["gamma_" + ch], np.float64) for ch in ("pp", "pm", "mm")]
        self._chk(self.lib.fp4_iteration_4ph(
            self.h, ct.byref(g), s.nlist, _p(np.ascontiguousarray(w.nequi, np.int32)),
            _p(np.ascontiguousarray(w.allequi, np.int32)), _p(np.ascontiguousarray(w.typeofsym, np.int32)), nsr,
            _p(idq), _p(symm), _p(n_plus), _p(n_minus), int(n_plus.sum()), int(n_minus.sum()),
            *[_p(x) for x in N], *[ct.c_int64(int(x.sum())) for x in N],
            _p(lists["ind2_plus"]), _p(lists["ind3_plus"]), _p(lists["ind2_minus"]), _p(lists["ind3_minus"]),
            *[_p(L[k + ch]) for ch in ("pp", "pm", "mm") for k in ("ind2_", "ind3_", "ind4_")],
            _p(e), _p(v), _p(lists["gamma_plus"]), _p(lists["gamma_minus"]), *[_p(x) for x in G],
            _p(np.ascontiguousarray(tau_zero, np.float64)), _p(F)))
        return F

    def symmetrize_fn(self, s, F):
        g = self.globals_of(s)
        symm = np.ascontiguousarray(np.transpose(s.sym.symmetrizers, (0, 2, 1))).ravel()
        self._chk(self.lib.fp4_symmetrize_fn(self.h, ct.byref(g), _p(symm), _p(F)))
        return F

    def eigen_dm(self, cr, fc, ngrid, symmetrizers, born=None, epsilon=None, nonanalytic=False, V=None, rl=None):
        """eigenDM on the device: omega (nptk,nb), velocity (nptk,nb,3) and
        eigenvect (nptk,nb,nb) [q, band, component] for the crystal `cr`, the
        read2fc array `fc` (natoms,3,sx,sy,sz,natoms,3) and symmetrizers
        (nptk,3,3); with nonanalytic, the dielectric correction from born
        (3,3,natoms) and epsilon (3,3). V and rl default to the crystal's
        volume and reciprocal lattice."""
        g = Globals()
        for d in range(3):
            g.ngrid[d] = int(ngrid[d])
        nb = 3 * cr.natoms
        g.nbands = nb
        rl = cr.rlattvec() if rl is None else np.asarray(rl)
        rlf = np.asfortranarray(rl).ravel(order="F")
        for x in range(9):
            g.rlattvec[x] = float(rlf[x])
        masses = np.ascontiguousarray(cr.masses, dtype=np.float64)
        types = np.ascontiguousarray(cr.types, dtype=np.int32)
        self._keep = [masses, types]
        g.nelements, g.natoms = masses.size, types.size
        g.masses, g.types = _p(masses), _p(types)
        nptk = int(np.prod(ngrid))
        lv = np.asfortranarray(cr.lattvec, dtype=np.float64).ravel(order="F")
        cart = np.asfortranarray(cr.cartesian, dtype=np.float64).ravel(order="F")
        scell = np.array(cr.scell, dtype=np.int32)
        fcf = np.asfortranarray(fc, dtype=np.float64).ravel(order="F")
        symm = np.ascontiguousarray(np.transpose(symmetrizers, (0, 2, 1))).ravel()
        eps = np.asfortranarray(np.eye(3) if epsilon is None else epsilon, dtype=np.float64).ravel(order="F")
        bo = np.asfortranarray(np.zeros((3, 3, cr.natoms)) if born is None else born, dtype=np.float64).ravel(order="F")
        vol = float(cr.volume() if V is None else V)
        om = np.zeros(nptk * nb)
        vel = np.zeros(nptk * nb * 3)
        eig = np.zeros(nptk * nb * nb, dtype=np.complex128)
        self._chk(self.lib.fp4_eigen_dm(self.h, ct.byref(g), _p(lv), _p(cart), _p(scell), _p(fcf),
                                        int(bool(nonanalytic)), _p(eps), _p(bo), ct.c_double(vol), _p(symm), _p(om),
                                        _p(vel), _p(eig)))
        return (om.reshape((nptk, nb), order="F"), vel.reshape((nptk, nb, 3), order="F"),
                eig.reshape((nptk, nb, nb), order="F"))

    def cumulative_tconduct(self, s, F, T=None, nticks=100, omega_mode=False):
        """CumulativeTConduct (or CumulativeTConductOmega): (ticks, results(nb,3,3,nticks) flat)."""
        g = self.globals_of(s, T)
        e, v, _, _, _ = self._arrays(s)
        ticks = np.zeros(nticks)
        res = np.zeros(s.nb * 9 * nticks)
        fn = self.lib.fp4_cumulative_tconduct_omega if omega_mode else self.lib.fp4_cumulative_tconduct
        self._chk(fn(self.h, ct.byref(g), ct.c_double(s.volume), _p(e), _p(v), _p(F), nticks, _p(ticks), _p(res)))
        return ticks, res

    def tconduct(self, s, F, T=None, with_modes=False):
        g = self.globals_of(s, T)
        e, v, _, _, _ = self._arrays(s)
        k = np.zeros(s.nb * 9)
        km = np.zeros(s.nptk * s.nb * 9) if with_modes else None
        self._chk(self.lib.fp4_tconduct(self.h, ct.byref(g), ct.c_double(s.volume), _p(e), _p(v), _p(F), _p(k),
                                        _p(km)))
        return (k, km) if with_modes else k
