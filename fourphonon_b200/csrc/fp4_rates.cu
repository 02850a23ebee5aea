// Three-phonon kernels, ordered four-phonon index lists and occupation tables (sm_100a).
//
// Three-phonon path (one CTA per irreducible mode and channel):
//   enumerate the candidates of the mode in the reference's list order
//   (j outer, q' middle, k inner; Ind_only_plus, processes.f90:1105-1110),
//   apply the bit-exact energy filter, compact survivors in order with warp
//   ballots and a block scan, then contract each survivor's matrix element
//   against the mode's reciprocal-space cluster table held in shared memory:
//       Z_p[s][r] = sum_{c in p} mu_c exp(-2 pi i n.m_k/N) sum_t Phi_c[t][s][r] e_i[t]
//       V+- = sum_p exp(+-2 pi i n'.D_p/N) e~'_j[s] Z_p[s][r] conj(e''_k[r]),
//   classes p = (m_j - m_k, atom_j, atom_k); this is Vp_plus/Vp_minus
//   (processes.f90:25-139) with the phases factored through lattice coordinates.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp4_device.cuh"
#include "fp4_internal.h"

namespace fp4 {

template <int MODE>  // 0 NP, 1 Ind_only, 2 RTA, 3 Ind
__global__ void __launch_bounds__(256) k3_mode(P3Params p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const DevSys& S = p.S;
    const DevIfc& F = p.F;
    const int nb = S.nb, nptk = S.nptk;
    const int N0 = S.n[0], N1 = S.n[1], N2 = S.n[2];
    const int mm = blockIdx.x, w = blockIdx.y, sign = (w == 0) ? 1 : -1;
    const int ll = mm / nb, i = mm % nb;
    const int q0 = S.list0[ll];
    int n0, n1, n2;
    q_coords_t(S, q0, n0, n1, n2);
    const double omega = S.wv[q0 * nb + i].w;

    double2* Z = reinterpret_cast<double2*>(smem_raw);  // npi*9
    const bool need_v = (MODE == 3) || (MODE == 2 && !S.onlyharmonic);
    const size_t zbytes = need_v ? (size_t)F.npi * 9 * sizeof(double2) : 0;
    int* queue = reinterpret_cast<int*>(smem_raw + zbytes);  // kQ3 entries: candidate index
    int* qpos = queue + kQ3;                                  // position in the mode's list
    int* warp_tot = qpos + kQ3;                               // 33 (+1 pad)
    double* red = reinterpret_cast<double*>(warp_tot + 34);   // 32

    bool active = (omega != 0.0);
    if (MODE == 0 || MODE == 2) active = active && (omega <= S.omega_max);
    if (MODE == 1 || MODE == 3) active = active && (p.nlist_counts[w][mm] != 0);
    if (!active) {
        if (threadIdx.x == 0) {
            if (MODE == 0) {
                p.n_out[w][mm] = 0;
                p.p_out[w][mm] = 0.0;
            } else if (MODE >= 2) {
                p.rate[w][mm] = 0.0;
                p.wp[w][mm] = 0.0;
            }
        }
        return;
    }
    if (need_v) {
        const double2* ei = S.eig + (size_t)(q0 * nb + i) * nb;
        for (int idx = threadIdx.x; idx < F.npi * 9; idx += blockDim.x) {
            const int pc = idx / 9, sr = idx % 9;
            double2 acc = make_double2(0.0, 0.0);
            for (int x = F.cl_start[pc]; x < F.cl_start[pc + 1]; x++) {
                const int c = F.cl_index[x];
                const int4 at = F.atoms[c];
                const int4 mk = F.mk[c];
                double2 kap = lattice_phase(S, n0, n1, n2, -mk.x, -mk.y, -mk.z);
                kap.x *= F.mu[c];
                kap.y *= F.mu[c];
                const double* ph = F.phi + (size_t)c * 27 + sr;
                double2 t1 = make_double2(0.0, 0.0);
#pragma unroll
                for (int t = 0; t < 3; t++) {
                    const double2 e = ei[3 * at.x + t];
                    const double f = ph[t * 9];
                    t1.x = fma(f, e.x, t1.x);
                    t1.y = fma(f, e.y, t1.y);
                }
                acc = cmac(acc, kap, t1);
            }
            Z[idx] = acc;
        }
    }
    __syncthreads();

    const int per_j = nptk * nb;
    const long long total = (long long)nb * per_j;
    long long running = 0;
    int qn = 0;
    Comp accP = {0.0, 0.0}, accR = {0.0, 0.0}, accW = {0.0, 0.0};
    const long long list_base = (MODE == 1 || MODE == 3) ? p.list_off[w][mm] : 0;
    const long long list_cap = (MODE == 1 || MODE == 3) ? p.nlist_counts[w][mm] : 0;
    const double sqrtpi = sqrt(3.141592653589793238);

    for (long long base = 0; base < total; base += blockDim.x) {
        const int x = (int)(base + threadIdx.x);
        bool ok = false;
        int j = 0, ii = 0, k = 0, ss = 0;
        if (base + threadIdx.x < total) {
            j = x / per_j;
            const int rem = x - j * per_j;
            ii = rem / nb;
            k = rem - ii * nb;
            int a, b, c;
            q_coords_t(S, ii, a, b, c);
            ss = q_index(S, wrapN(n0 + sign * a, N0), wrapN(n1 + sign * b, N1), wrapN(n2 + sign * c, N2));
            const double4 wp = S.wv[ii * nb + j];
            const double4 wd = S.wv[ss * nb + k];
            if (wp.w != 0.0 && wd.w != 0.0) {
                const double sigma = sigma_exact(S, wp, wd);
                const double delta = (sign > 0) ? __dadd_rn(__dadd_rn(omega, wp.w), -wd.w)
                                                : __dadd_rn(__dadd_rn(omega, -wp.w), -wd.w);
                ok = fabs(delta) <= 2.0 * sigma;
            }
        }
        int cnt;
        const int pos = block_exclusive_scan_flag(ok, warp_tot, cnt);
        if (ok) {
            if (MODE == 1) {
                if (running + pos < list_cap) {
                    const long long o = list_base + running + pos;
                    p.ind2[w][o] = ii * nb + j + 1;
                    p.ind3[w][o] = ss * nb + k + 1;
                } else {
                    atomicOr(p.err, kErrQueue);
                }
            } else {
                queue[qn + pos] = x;
                qpos[qn + pos] = (int)(running + pos);
            }
        }
        running += cnt;
        if (MODE != 1) qn += cnt;
        const bool last = (base + blockDim.x >= total);
        if (MODE != 1 && (qn > kQ3 - (int)blockDim.x || last)) {
            // every thread's queue write of this pass must be visible before any thread
            // reads the queue (the condition is uniform over the block)
            __syncthreads();
            for (int e = threadIdx.x; e < qn; e += blockDim.x) {
                const int xx = queue[e];
                const int jj = xx / per_j, rem = xx - jj * per_j, q1 = rem / nb, kk = rem - q1 * nb;
                int a, b, c;
                q_coords_t(S, q1, a, b, c);
                const int s2 =
                    q_index(S, wrapN(n0 + sign * a, N0), wrapN(n1 + sign * b, N1), wrapN(n2 + sign * c, N2));
                const double4 wp = S.wv[q1 * nb + jj];
                const double4 wd = S.wv[s2 * nb + kk];
                const double sigma = sigma_exact(S, wp, wd);
                const double delta = (sign > 0) ? __dadd_rn(__dadd_rn(omega, wp.w), -wd.w)
                                                : __dadd_rn(__dadd_rn(omega, -wp.w), -wd.w);
                const double g = exp(-(delta * delta) / (sigma * sigma));
                if (MODE == 0) {
                    accP.add(g / (sigma * sqrtpi * (double)((long long)nptk * nptk) * (double)(nb * nb * nb)));
                    continue;
                }
                if (MODE == 3 && qpos[e] >= list_cap) {
                    atomicOr(p.err, kErrQueue);
                    continue;
                }
                const double fp = p.bose[q1 * nb + jj], fd = p.bose[s2 * nb + kk];
                const double bose = (sign > 0) ? (fp - fd) : (fp + fd + 1.0);
                const double wp3 = bose * g / sigma / sqrtpi / (omega * wp.w * wd.w);
                accW.add(wp3);
                if (!need_v) continue;
                double2 V = make_double2(0.0, 0.0);
                const double2* e1 = S.eig + (size_t)(q1 * nb + jj) * nb;
                const double2* e2 = S.eig + (size_t)(s2 * nb + kk) * nb;
                for (int blk = 0; blk < F.nblk; blk++) {
                    const int p0 = F.blk_start[blk], p1 = F.blk_start[blk + 1];
                    if (p0 == p1) continue;
                    const int a2 = blk / S.natoms, a3 = blk - a2 * S.natoms;
                    double2 u[3], v[3];
#pragma unroll
                    for (int s = 0; s < 3; s++) {
                        u[s] = e1[3 * a2 + s];
                        if (sign < 0) u[s] = cconj(u[s]);
                        v[s] = cconj(e2[3 * a3 + s]);
                    }
                    for (int pc = p0; pc < p1; pc++) {
                        const int4 D = F.pi_d[pc];
                        const double2 ph = lattice_phase(S, a, b, c, sign * D.x, sign * D.y, sign * D.z);
                        const double2* z = Z + pc * 9;
                        double2 t = make_double2(0.0, 0.0);
#pragma unroll
                        for (int s = 0; s < 3; s++) {
                            double2 h = make_double2(0.0, 0.0);
#pragma unroll
                            for (int r = 0; r < 3; r++) h = cmac(h, z[s * 3 + r], v[r]);
                            t = cmac(t, u[s], h);
                        }
                        V = cmac(V, ph, t);
                    }
                }
                const double av2 = V.x * V.x + V.y * V.y;
                const double gam = p.scale * wp3 * av2;
                if (MODE == 3) {
                    const long long o = list_base + qpos[e];
                    p.ind2[w][o] = q1 * nb + jj + 1;
                    p.ind3[w][o] = s2 * nb + kk + 1;
                    p.gamma[w][o] = gam * p.unit / (double)nptk;
                } else {
                    accR.add(gam);
                }
            }
            __syncthreads();
            qn = 0;
        }
    }
    if (MODE == 0) {
        const double P = block_sum(accP.val(), red);
        if (threadIdx.x == 0) {
            p.n_out[w][mm] = (int)running;
            p.p_out[w][mm] = P;
        }
    } else if (MODE >= 2) {
        double W = block_sum(accW.val(), red);
        const double R = block_sum(accR.val(), red);
        if (threadIdx.x == 0) {
            W = (sign > 0) ? W / nptk : W * 5.e-1 / nptk;
            p.wp[w][mm] = W;
            if (MODE == 2) p.rate[w][mm] = R * p.unit / (double)nptk * (sign > 0 ? 1.0 : 5.e-1);
        }
    }
    if (MODE == 1 || MODE == 3) {
        if (threadIdx.x == 0 && running != list_cap) atomicOr(p.err, kErrQueue);
    }
    if (MODE == 3) {
        // rate = sum of the mode's Gamma list (Ind_driver), the minus channel halved
        __syncthreads();
        Comp acc = {0.0, 0.0};
        const long long n = running < list_cap ? running : list_cap;
        for (long long e = threadIdx.x; e < n; e += blockDim.x) acc.add(p.gamma[w][list_base + e]);
        const double R = block_sum(acc.val(), red);
        if (threadIdx.x == 0) p.rate[w][mm] = (sign > 0) ? R : R * 5.e-1;
    }
    if (threadIdx.x == 0 && (MODE == 2 || MODE == 3)) {
        atomicAdd(&p.stats[0], (unsigned long long)running);
        if (need_v) atomicAdd(&p.stats[1], (unsigned long long)running);
    }
}

// ---------------------------------------------------------------------------
// Ordered four-phonon index lists (Ind_only_plusplus/plusminus/minusminus,
// processes.f90:2854-3074): one CTA per mode, candidates walked in the
// reference's loop order (q', q'', j, k, l) and compacted in order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k4_order(P4OrderParams p) {
    __shared__ int warp_tot[34];
    const DevSys& S = p.S;
    const int nb = S.nb, nptk = S.nptk, ch = p.ch;
    const int N0 = S.n[0], N1 = S.n[1], N2 = S.n[2];
    const int mm = blockIdx.x, ll = mm / nb, i = mm % nb;
    const int q0 = S.list0[ll];
    int n0, n1, n2;
    q_coords_t(S, q0, n0, n1, n2);
    const double omega = S.wv[q0 * nb + i].w;
    if (!(omega != 0.0 && omega <= S.omega_max) || p.counts[mm] == 0) return;
    const long long nb3 = (long long)nb * nb * nb;
    const long long total = (long long)nptk * nptk * nb3;
    long long running = 0;
    const long long off = p.list_off[mm], cap = p.counts[mm];
    for (long long base = 0; base < total; base += blockDim.x) {
        const long long x = base + threadIdx.x;
        bool ok = false;
        int ii = 0, jj = 0, j = 0, k = 0, l = 0, ss = 0;
        if (x < total) {
            const long long pr = x / nb3;
            const int br = (int)(x - pr * nb3);
            ii = (int)(pr / nptk);
            jj = (int)(pr - (long long)ii * nptk);
            j = br / (nb * nb);
            k = (br / nb) % nb;
            l = br % nb;
            bool go = (ch == 1) || (jj >= ii);
            int m0, m1, m2, a, b, c;
            q_coords_t(S, ii, m0, m1, m2);
            q_coords_t(S, jj, a, b, c);
            int t0, t1, t2;
            if (ch == 0) {
                t0 = n0 + m0 + a; t1 = n1 + m1 + b; t2 = n2 + m2 + c;
            } else if (ch == 1) {
                t0 = n0 + m0 - a; t1 = n1 + m1 - b; t2 = n2 + m2 - c;
            } else {
                t0 = n0 - m0 - a; t1 = n1 - m1 - b; t2 = n2 - m2 - c;
            }
            ss = q_index(S, wrapN(t0, N0), wrapN(t1, N1), wrapN(t2, N2));
            if (ch != 0 && ss < jj) go = false;
            if (ch != 1 && jj == ii && k < j) go = false;
            if (ch != 0 && ss == jj && l < k) go = false;
            if (go) {
                const double4 w1 = S.wv[ii * nb + j], w2 = S.wv[jj * nb + k], w3 = S.wv[ss * nb + l];
                if (w1.w != 0.0 && w2.w != 0.0 && w3.w != 0.0) {
                    bool excl = false;
                    if (ch == 1)
                        excl = !((q0 != jj || i != k) && (q0 != ss || i != l) && (ii != jj || j != k) &&
                                 (ii != ss || j != l));
                    if (!excl) {
                        const double sigma = sigma_exact(S, w2, w3);
                        const double s = (ch == 2) ? __dadd_rn(omega, -w1.w) : __dadd_rn(omega, w1.w);
                        const double delta = (ch == 0) ? __dadd_rn(__dadd_rn(s, w2.w), -w3.w)
                                                       : __dadd_rn(__dadd_rn(s, -w2.w), -w3.w);
                        ok = fabs(delta) <= sigma;
                    }
                }
            }
        }
        int cnt;
        const int pos = block_exclusive_scan_flag(ok, warp_tot, cnt);
        if (ok) {
            const long long r = running + pos;
            if (r < cap) {
                p.ind2[off + r] = (long long)ii * nb + j + 1;
                p.ind3[off + r] = (long long)jj * nb + k + 1;
                p.ind4[off + r] = (long long)ss * nb + l + 1;
            } else {
                atomicOr(p.err, kErrQueue);
            }
        }
        running += cnt;
    }
    if (threadIdx.x == 0 && running != cap) atomicOr(p.err, kErrQueue);
}

// Bose-Einstein occupations for every mode and temperature.
__global__ void k_bose(DevSys S, const double* T, int nT, double* bose) {
    const size_t plane = (size_t)S.nptk * S.nb;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < plane * nT; x += (size_t)gridDim.x * blockDim.x) {
        const int t = (int)(x / plane);
        const size_t qb = x % plane;
        bose[x] = bose_of(S.wv[qb].w, T[t]);
    }
}

// omega and the Bose factors of every mode in one record per mode
__global__ void k_wbose(DevSys S, const double* T, int nT, int stride, double* wb) {
    const size_t plane = (size_t)S.nptk * S.nb;
    for (size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x; m < plane; m += (size_t)gridDim.x * blockDim.x) {
        const double w = S.wv[m].w;
        double* r = wb + m * stride;
        r[0] = w;
        for (int t = 1; t < stride; t++) r[t] = (t <= nT) ? bose_of(w, T[t - 1]) : 0.0;
    }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
size_t k3_smem(int mode, const DevIfc& F, bool onlyharmonic) {
    const bool need_v = (mode == 3) || (mode == 2 && !onlyharmonic);
    const size_t z = need_v ? (size_t)F.npi * 9 * sizeof(double2) : 0;
    return z + 2 * kQ3 * sizeof(int) + 34 * sizeof(int) + 32 * sizeof(double);
}

template <int MODE>
static cudaError_t launch_k3_t(const P3Params& p, int nmodes, cudaStream_t st) {
    const size_t sm = k3_smem(MODE, p.F, p.S.onlyharmonic);
    cudaError_t e = cudaFuncSetAttribute(k3_mode<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k3_mode<MODE><<<dim3(nmodes, 2), 256, sm, st>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_k3(int mode, const P3Params& p, int nmodes, cudaStream_t st) {
    switch (mode) {
        case 0: return launch_k3_t<0>(p, nmodes, st);
        case 1: return launch_k3_t<1>(p, nmodes, st);
        case 2: return launch_k3_t<2>(p, nmodes, st);
        default: return launch_k3_t<3>(p, nmodes, st);
    }
}

cudaError_t launch_k4_order(const P4OrderParams& p, int nmodes, cudaStream_t st) {
    k4_order<<<nmodes, 256, 0, st>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_wbose(const DevSys& S, const double* T, int nT, int stride, double* wb, cudaStream_t st) {
    if (nT + 1 > stride) return cudaErrorInvalidValue;
    const size_t n = (size_t)S.nptk * S.nb;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    k_wbose<<<blocks, 256, 0, st>>>(S, T, nT, stride, wb);
    return cudaGetLastError();
}

cudaError_t launch_bose(const DevSys& S, const double* T, int nT, double* bose, cudaStream_t st) {
    const size_t n = (size_t)S.nptk * S.nb * nT;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    k_bose<<<blocks, 256, 0, st>>>(S, T, nT, bose);
    return cudaGetLastError();
}

}  // namespace fp4
