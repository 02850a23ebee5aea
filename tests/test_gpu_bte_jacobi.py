"""The Jacobi form of the BTE sweep (fp4_iteration_jacobi) against the
reference's Gauss-Seidel sweep (fp4_iteration, iterations.f90:34-92).

Both iterate the same linear map, so they share its fixed point: the F_n that
the Jacobi sweeps converge to is left unchanged by one in-order sweep (within
1e-8), and the converged kappa of the two agree (within 1e-6).  A Jacobi sweep
is also deterministic (fixed summation order).
"""
import numpy as np
import pytest

import helpers as H
from fourphonon_b200 import abi

pytestmark = pytest.mark.gpu


def _kappa(ctx, s, F):
    k = ctx.tconduct(s, F).reshape(3, 3, s.nb).sum(axis=2)
    return np.trace(k) / 3.0


def test_jacobi_and_gauss_seidel_share_the_fixed_point():
    s = H.cached_solve("diamond", (6, 6, 6))
    ctx = abi.Context(0)
    try:
        n_p, n_m, _, _ = ctx.np_driver(s)
        lists = ctx.ind_driver(s, n_p, n_m)
        rate = lists["rate_plus"] + lists["rate_minus"]
        tau = np.zeros_like(rate)
        tau[rate != 0] = 1.0 / rate[rate != 0]
        F0 = ctx.iteration0(s, tau)
        # Gauss-Seidel to a tight tolerance
        Fg = F0.copy()
        kg = _kappa(ctx, s, Fg)
        for it in range(200):
            Fg = ctx.iteration(s, Fg, tau, n_p, n_m, lists)
            Fg = ctx.symmetrize_fn(s, Fg)
            knew = _kappa(ctx, s, Fg)
            done = abs(knew - kg) <= 1e-12 * abs(knew)
            kg = knew
            if done:
                break
        # Jacobi to the same tolerance
        Fj = F0.copy()
        kj = _kappa(ctx, s, Fj)
        nj = 0
        for nj in range(1, 1000):
            Fj = ctx.iteration_jacobi(s, Fj, tau, n_p, n_m, lists)
            knew = _kappa(ctx, s, Fj)
            done = abs(knew - kj) <= 1e-12 * abs(knew)
            kj = knew
            if done:
                break
        assert abs(kj - kg) <= 1e-6 * abs(kg), (kj, kg, nj)
        # the Jacobi fixed point is a fixed point of the in-order sweep
        Fs = ctx.iteration(s, Fj.copy(), tau, n_p, n_m, lists)
        Fs = ctx.symmetrize_fn(s, Fs)
        scale = np.abs(Fj).max()
        assert np.abs(Fs - Fj).max() <= 1e-8 * scale
        # a sweep's sums run in a fixed order: the same input gives the same output, bit for bit
        a = ctx.iteration_jacobi(s, F0.copy(), tau, n_p, n_m, lists)
        b = ctx.iteration_jacobi(s, F0.copy(), tau, n_p, n_m, lists)
        assert np.array_equal(a, b)
        print("converged kappa: Gauss-Seidel", kg, "Jacobi", kj, "Jacobi sweeps", nj)
    finally:
        ctx.close()
