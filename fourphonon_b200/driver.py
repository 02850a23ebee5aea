"""The rate/BTE/kappa section of the ShengBTE main program, on the device path.

`run(solve, outdir)` follows Src/ShengBTE.f90 from the counting stage to the
converged conductivity, calling the C-ABI for every hot step:

* NP_driver / NP_driver_4ph (ShengBTE.f90:436-488) -> BTE.Numprocess_4ph,
  BTE.P3_plus/minus, BTE.P3, BTE.P4_* and the *_total files (500-587);
* per temperature (787-1027): Ind_driver (convergence) or RTA_driver, and
  RTA_driver_4ph for all temperatures in one fused call, or Ind_driver_4ph
  per temperature with four_phonon_iteration; BTE.w_3ph*, BTE.w_4ph*,
  BTE.WP3*, BTE.WP4*, BTE.w (1030-1230);
* tau_zero, iteration0, TConduct, symmetrize_tensor, the Gauss-Seidel
  iteration loop (iteration, or iteration_4ph with four_phonon_iteration)
  with twonorm3x3 relative change < eps (1232-1307);
  BTE.kappa, BTE.kappa_tensor, BTE.kappa_scalar, BTE.KappaTensorVsT_RTA/CONV;
* BTE.w_final and the cumulative kappa files of CumulativeTConduct and
  CumulativeTConductOmega (1315-1404).

Numbers are written in the reference's Fortran edit descriptors (E20.10,
E14.5, F7.1, I9, I0), so the files read the same way.
"""
from __future__ import annotations

import json
import math
import os
import time

import numpy as np

from . import abi


def fortran_e(x: float, w: int, d: int) -> str:
    """Fortran Ew.d: 0.ddddE+xx right-justified in w columns."""
    x = float(x)
    if math.isnan(x):
        return "NaN".rjust(w)
    if math.isinf(x):
        return ("-Infinity" if x < 0 else "Infinity").rjust(w)
    if x == 0.0:
        return f"0.{'0' * d}E+00".rjust(w)
    sign = "-" if x < 0 else ""
    a = abs(x)
    e = math.floor(math.log10(a)) + 1
    m = a / 10.0 ** e
    digits = round(m * 10 ** d)
    if digits >= 10 ** d:
        digits //= 10
        e += 1
    if digits < 10 ** (d - 1):
        digits *= 10
        e -= 1
    ex = f"{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100 else f"{'+' if e >= 0 else '-'}{abs(e):03d}"
    return f"{sign}0.{digits:0{d}d}E{ex}".rjust(w)


def _rows(path, rows):
    with open(path, "w") as fh:
        fh.write("".join(r + "\n" for r in rows))


def write_counts(outdir, s, n3, p3, n4, p4):
    """BTE.Numprocess_4ph and the phase-space files of ShengBTE.f90:500-587."""
    nb, nl = s.nb, s.nlist
    nequi = np.asarray(s.wedge.nequi, dtype=np.float64)
    n_p, n_m = n3
    pp, pm = p3
    if n4 is not None:
        # the file's line L holds N(L): the loop writes N(ll+Nlist*(i-1)) with i outer, ll inner
        _rows(os.path.join(outdir, "BTE.Numprocess_4ph"),
              [f" {int(n4[0][m])} {int(n4[1][m])} {int(n4[2][m])}" for m in range(nb * nl)])
    P = lambda v: v.reshape(nl, nb)  # noqa: E731  Pspace(nb,nlist) in mode order
    _rows(os.path.join(outdir, "BTE.P3_plus"), ["".join(fortran_e(x, 20, 10) for x in r) for r in P(pp)])
    _rows(os.path.join(outdir, "BTE.P3_minus"), ["".join(fortran_e(x, 20, 10) for x in r) for r in P(pm)])
    _rows(os.path.join(outdir, "BTE.P3"),
          ["".join(fortran_e(2.0 * (a + b / 2.0) / 3.0, 20, 10) for a, b in zip(ra, rb)) for ra, rb in zip(P(pp), P(pm))])
    tp = float((P(pp) * nequi[:, None]).sum())
    tm = float((P(pm) * nequi[:, None]).sum())
    _rows(os.path.join(outdir, "BTE.P3_plus_total"), [f"  {tp!r}"])
    _rows(os.path.join(outdir, "BTE.P3_minus_total"), [f"  {tm!r}"])
    _rows(os.path.join(outdir, "BTE.P3_total"), [f"  {2.0 * (tp + tm / 2.0) / 3.0!r}"])
    if p4 is not None:
        names = ("BTE.P4_plusplus", "BTE.P4_plusmius", "BTE.P4_minusminus")
        for name, v in zip(names, p4):
            _rows(os.path.join(outdir, name), ["".join(fortran_e(x, 20, 10) for x in r) for r in P(v)])
        _rows(os.path.join(outdir, "BTE.P4"), ["".join(fortran_e(6.0 * (a + b + c) / 7.0, 20, 10)
                                                        for a, b, c in zip(ra, rb, rc))
                                                for ra, rb, rc in zip(P(p4[0]), P(p4[1]), P(p4[2]))])
        tots = [float((P(v) * nequi[:, None]).sum()) for v in p4]
        for name, t in zip(("BTE.P4_plusplus_total", "BTE.P4_plusminus_total", "BTE.P4_minusminus_total"), tots):
            _rows(os.path.join(outdir, name), [f"  {t!r}"])
        _rows(os.path.join(outdir, "BTE.P4_total"), [f"  {6.0 * sum(tots) / 7.0!r}"])


def _mode_lines(s, values, fmt_w=20, fmt_d=10):
    """Lines of (energy(list(ll),i), value(i,ll)) with i outer, ll inner."""
    nb, nl = s.nb, s.nlist
    out = []
    for i in range(nb):
        for ll in range(nl):
            w = s.energy[s.wedge.list[ll] - 1, i]
            out.append(fortran_e(w, fmt_w, fmt_d) + fortran_e(values[ll * nb + i], fmt_w, fmt_d))
    return out


def twonorm3x3(a):
    """Largest singular value (misc.f90:53-67, dgesdd)."""
    return float(np.linalg.svd(np.asarray(a), compute_uv=False)[0])


def symmetrize_tensor(s, t):
    """config.f90:503-518."""
    acc = np.zeros((3, 3))
    for R in s.sym.crotations:
        acc += R @ t @ R.T
    return acc / s.sym.nsymm_rot


def write_final(tdir, s, F, ctx, T, nticks=100):
    """BTE.w_final and the cumulative kappa files (ShengBTE.f90:1315-1404)."""
    Fq = np.asarray(F).reshape(3, s.nptk, s.nb)  # F_n(b,q,d) as [d][q][b]
    lines = []
    for i in range(s.nb):
        for ll in range(s.nlist):
            q = s.wedge.list[ll] - 1
            v = s.velocity[q, i, :]
            f = Fq[:, q, i]
            w = s.energy[q, i]
            with np.errstate(divide="ignore", invalid="ignore"):
                tau = np.float64(np.dot(f, v)) / (np.float64(np.dot(v, v)) * w)
                inv = np.float64(1.0) / tau
            lines.append(fortran_e(w, 20, 10) + fortran_e(inv, 20, 10))
    _rows(os.path.join(tdir, "BTE.w_final"), lines)
    for omega_mode, name in ((False, "BTE.cumulative_kappa_tensor"), (True, "BTE.cumulative_kappaVsOmega_tensor")):
        ticks, res = ctx.cumulative_tconduct(s, F, T=T, nticks=nticks, omega_mode=omega_mode)
        r = res.reshape(nticks, 3, 3, s.nb)  # [k][d2][d1][b]
        tens, scal = [], []
        for k in range(nticks):
            tot = sum(symmetrize_tensor(s, r[k, :, :, b].T) for b in range(s.nb))
            tens.append(fortran_e(ticks[k], 20, 10) + "".join(fortran_e(x, 20, 10) for x in tot.ravel(order="F")))
            scal.append(fortran_e(ticks[k], 20, 10) + fortran_e(np.trace(tot) / 3.0, 20, 10))
        _rows(os.path.join(tdir, name), tens)
        if not omega_mode:
            _rows(os.path.join(tdir, "BTE.cumulative_kappa_scalar"), scal)


def run(s, outdir, convergence=True, four_phonon=True, maxiter=1000, eps=float(np.float32(1e-5)),
        ctx=None, log=print, four_phonon_iteration=False, metrics=None):
    """The hot-path section of ShengBTE for solve `s`; returns per-T results.

    metrics: a writable text stream that receives one JSON line per stage
    (counting, rates, the BTE loop, the output files) with its wall-clock
    seconds, and the temperature and process counts where they apply; the
    reference prints MPI_Wtime differences around the same stages."""
    os.makedirs(outdir, exist_ok=True)
    own = ctx is None
    ctx = ctx or abi.Context(0)
    files = []

    def stage(name, t0, **fields):
        if metrics is not None:
            metrics.write(json.dumps({"event": "stage", "stage": name, "seconds": time.perf_counter() - t0,
                                      **fields}) + "\n")
            metrics.flush()

    try:
        t0 = time.perf_counter()
        n3 = ctx.np_driver(s)
        stage("np_driver", t0, processes=int(n3[0].sum()) + int(n3[1].sum()))
        n4 = p4 = None
        if four_phonon:
            t0 = time.perf_counter()
            n4, p4 = ctx.np_driver_4ph(s)
            stage("np_driver_4ph", t0, processes=int(sum(int(x.sum()) for x in n4)))
        write_counts(outdir, s, (n3[0], n3[1]), (n3[2], n3[3]), n4, p4)
        log(f"Info: Ntotal_plus = {int(n3[0].sum())}  Ntotal_minus = {int(n3[1].sum())}")
        if four_phonon:
            log(f"Info: Ntotal_plusplus,Ntotal_plusminus,Ntotal_minusminus= "
                f"{int(n4[0].sum())} {int(n4[1].sum())} {int(n4[2].sum())}")
        it4 = four_phonon and four_phonon_iteration and convergence
        r4 = None
        if four_phonon and not it4:
            t0 = time.perf_counter()
            r4 = ctx.rta_driver_4ph(s)
            stage("rta_driver_4ph", t0, temperatures=[float(x) for x in s.temperatures],
                  processes=int(sum(int(x.sum()) for x in n4)))
        results = []
        f303 = open(os.path.join(outdir, "BTE.KappaTensorVsT_RTA"), "w")
        f403 = open(os.path.join(outdir, "BTE.KappaTensorVsT_CONV"), "w") if convergence else None
        files += [f for f in (f303, f403) if f is not None]
        for t, T in enumerate(s.temperatures):
            tdir = os.path.join(outdir, f"T{int(round(T))}K")
            os.makedirs(tdir, exist_ok=True)
            t0 = time.perf_counter()
            if convergence:
                lists = ctx.ind_driver(s, n3[0], n3[1], T=T)
                r3 = lists
            else:
                r3 = ctx.rta_driver(s, T=T)
            stage("ind_driver" if convergence else "rta_driver", t0, T=float(T),
                  processes=int(n3[0].sum()) + int(n3[1].sum()))
            rate3 = r3["rate_plus"] + r3["rate_minus"]
            _rows(os.path.join(tdir, "BTE.w_3ph"), _mode_lines(s, rate3))
            _rows(os.path.join(tdir, "BTE.w_3ph_plus"), _mode_lines(s, r3["rate_plus"]))
            _rows(os.path.join(tdir, "BTE.w_3ph_minus"), _mode_lines(s, r3["rate_minus"]))
            _rows(os.path.join(tdir, "BTE.WP3_plus"), _mode_lines(s, r3["wp3_plus"], 14, 5))
            _rows(os.path.join(tdir, "BTE.WP3_minus"), _mode_lines(s, r3["wp3_minus"], 14, 5))
            _rows(os.path.join(tdir, "BTE.WP3"), _mode_lines(s, r3["wp3_plus"] + r3["wp3_minus"], 14, 5))
            rate4 = np.zeros_like(rate3)
            ind4 = None
            if four_phonon:
                if it4:
                    t0 = time.perf_counter()
                    ind4 = ctx.ind_driver_4ph(s, n4[0], n4[1], n4[2], T=T)
                    stage("ind_driver_4ph", t0, T=float(T), processes=int(sum(int(x.sum()) for x in n4)))
                    rates = [ind4["rate_pp"], ind4["rate_pm"], ind4["rate_mm"]]
                    wps = [ind4["wp_pp"], ind4["wp_pm"], ind4["wp_mm"]]
                else:
                    rates = [r4[f"rate_{ch}"][t] for ch in ("plusplus", "plusminus", "minusminus")]
                    wps = [r4[f"wp4_{ch}"][t] for ch in ("plusplus", "plusminus", "minusminus")]
                rate4 = rates[0] + rates[1] + rates[2]
                _rows(os.path.join(tdir, "BTE.w_4ph"), _mode_lines(s, rate4))
                for x, ch in enumerate(("plusplus", "plusminus", "minusminus")):
                    _rows(os.path.join(tdir, f"BTE.w_4ph_{ch}"), _mode_lines(s, rates[x]))
                    _rows(os.path.join(tdir, f"BTE.WP4_{ch}"), _mode_lines(s, wps[x], 14, 5))
                _rows(os.path.join(tdir, "BTE.WP4"), _mode_lines(s, wps[0] + wps[1] + wps[2], 14, 5))
            rate = rate3 + rate4  # isotope scattering is outside this path
            _rows(os.path.join(tdir, "BTE.w"), _mode_lines(s, rate))
            tau = np.zeros_like(rate)
            nz = rate != 0
            tau[nz] = 1.0 / rate[nz]
            t0 = time.perf_counter()
            F = ctx.iteration0(s, tau)
            kap = ctx.tconduct(s, F, T=T).reshape(3, 3, s.nb)  # [d2][d1][branch]
            kb = np.stack([symmetrize_tensor(s, kap[:, :, b].T) for b in range(s.nb)])  # (nb,3,3)
            ktot = kb.sum(axis=0)
            kappa_lines = [f"{0:9d}" + "".join(fortran_e(x, 20, 10) for x in kb.ravel(order="F"))]
            tensor_lines = [f"{0:9d}" + "".join(fortran_e(x, 20, 10) for x in ktot.ravel(order="F"))]
            scalar_lines = [f"{0:9d}" + fortran_e(np.trace(ktot) / 3.0, 20, 10)]
            f303.write(f"{T:7.1f}" + "".join(fortran_e(x, 14, 5) for x in ktot.ravel(order="F")) + "\n")
            res = {"T": T, "kappa_rta": ktot.copy(), "rate3": rate3, "rate4": rate4}
            stage("kappa_rta", t0, T=float(T))
            if convergence:
                t0 = time.perf_counter()
                it = 0
                for it in range(1, maxiter + 1):
                    kold = ktot.copy()
                    F = ctx.iteration(s, F, tau, n3[0], n3[1], lists, ind4=ind4)
                    F = ctx.symmetrize_fn(s, F)
                    kap = ctx.tconduct(s, F, T=T).reshape(3, 3, s.nb)
                    kb = np.stack([symmetrize_tensor(s, kap[:, :, b].T) for b in range(s.nb)])
                    ktot = kb.sum(axis=0)
                    kappa_lines.append(f"{it:9d}" + "".join(fortran_e(x, 20, 10) for x in kb.ravel(order="F")))
                    tensor_lines.append(f"{it:9d}" + "".join(fortran_e(x, 20, 10) for x in ktot.ravel(order="F")))
                    scalar_lines.append(f"{it:9d}" + fortran_e(np.trace(ktot) / 3.0, 20, 10))
                    rel = twonorm3x3(ktot - kold) / twonorm3x3(kold)
                    log(f"Info: Iteration {it}  Relative change = {rel!r}")
                    if rel < eps:
                        break
                f403.write(f"{T:7.1f}" + "".join(fortran_e(x, 14, 5) for x in ktot.ravel(order="F")) + f"{it:6d}\n")
                res["kappa_conv"] = ktot.copy()
                res["iterations"] = it
                stage("iterations", t0, T=float(T), iterations=int(it))
            t0 = time.perf_counter()
            write_final(tdir, s, F, ctx, T)
            _rows(os.path.join(tdir, "BTE.kappa"), kappa_lines)
            _rows(os.path.join(tdir, "BTE.kappa_tensor"), tensor_lines)
            _rows(os.path.join(tdir, "BTE.kappa_scalar"), scalar_lines)
            stage("outputs", t0, T=float(T))
            results.append(res)
        return results
    finally:
        for f in files:
            f.close()
        if own:
            ctx.close()
