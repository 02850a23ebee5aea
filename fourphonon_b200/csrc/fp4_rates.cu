// Scattering-rate kernels for sm_100a.
//
// Three-phonon path (one CTA per irreducible mode and channel):
//   enumerate the candidates of the mode in the reference's list order
//   (j outer, q' middle, k inner; Ind_only_plus, processes.f90:1105-1110),
//   apply the bit-exact energy filter, compact survivors in order with warp
//   ballots and a block scan, then contract each survivor's matrix element
//   against the mode's reciprocal-space cluster table held in shared memory.
//
// Four-phonon path (persistent CTAs pulling work items (q, q', channel)):
//   phase A enumerates every q'' and branch pair (k,l) once, computes the
//   broadening sigma(v''-v''') once for all (i,j) branch pairs, and finds the
//   surviving (i,j) with a window search in the sorted sums w_i+-w'_j; the
//   survivors go to per-(i,j) device queues.  Phase B builds, for one branch
//   i at a time, the reciprocal cluster table
//       Z_p^{(ij)}[s][r] = sum_{c in class p} kappa_c sum_{u,t} Psi_c[u][t][s][r] e_i[u] e'_j[t]
//   and contracts each queued process as
//       V = sum_p exp(2 pi i n''.D_p/N) e''_k[s] Z_p[s][r] e'''_l[r],
//   which equals Vp_pp/Vp_pm/Vp_mm (processes.f90:142-330) term by term after
//   the cluster phases are factored through integer lattice coordinates.
//   Per-(work item, branch, temperature) partial sums are reduced afterwards
//   in a fixed order with compensated summation.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp4_device.cuh"
#include "fp4_internal.h"

namespace fp4 {

// ---------------------------------------------------------------------------
// block-wide ordered compaction helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ int block_exclusive_scan_flag(bool flag, int* warp_tot, int& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = (blockDim.x + 31) >> 5;
    unsigned bal = __ballot_sync(0xffffffffu, flag);
    int pre = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[warp] = __popc(bal);
    __syncthreads();
    if (warp == 0) {
        int v = lane < nwarp ? warp_tot[lane] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane < nwarp) warp_tot[lane] = incl - v;
        if (lane == 31) warp_tot[32] = incl;
    }
    __syncthreads();
    int r = warp_tot[warp] + pre;
    total = warp_tot[32];
    __syncthreads();
    return r;
}

__device__ __forceinline__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < nwarp; w++) t += red[w];
    __syncthreads();
    return t;  // valid in thread 0
}

// Neumaier two-sum accumulation
struct Comp {
    double s, c;
    __device__ __forceinline__ void add(double x) {
        double t = s + x;
        if (fabs(s) >= fabs(x))
            c += (s - t) + x;
        else
            c += (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ double val() const { return s + c; }
};

// ---------------------------------------------------------------------------
// Three-phonon per-mode kernel
// ---------------------------------------------------------------------------
template <int MODE>  // 0 NP, 1 Ind_only, 2 RTA, 3 Ind
__global__ void __launch_bounds__(256) k3_mode(P3Params p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const DevSys& S = p.S;
    const DevIfc& F = p.F;
    const int nb = S.nb, nptk = S.nptk;
    const int mm = blockIdx.x, w = blockIdx.y, sign = (w == 0) ? 1 : -1;
    const int ll = mm / nb, i = mm % nb;
    const int q0 = S.list0[ll];
    int n0, n1, n2;
    q_coords(S, q0, n0, n1, n2);
    const double omega = S.wv[q0 * nb + i].w;

    double2* Z = reinterpret_cast<double2*>(smem_raw);  // npi*9
    const bool need_v = (MODE == 3) || (MODE == 2 && !S.onlyharmonic);
    size_t zbytes = need_v ? (size_t)F.npi * 9 * sizeof(double2) : 0;
    int* queue = reinterpret_cast<int*>(smem_raw + zbytes);  // kQ3 entries: candidate x
    int* qpos = queue + kQ3;                                  // position in the mode's list
    int* warp_tot = qpos + kQ3;                               // 33
    double* red = reinterpret_cast<double*>(warp_tot + 34);   // 32 (8-aligned: 34 ints after 2*kQ3)

    bool active = (omega != 0.0);
    if (MODE == 0 || MODE == 2) active = active && (omega <= S.omega_max);
    if (MODE == 3) active = active && (p.nlist_counts[w][mm] != 0);
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
    // reciprocal cluster table of this mode: Z_p[s][r] = sum_c mu_c e^{-2pi i n.m_k/N} sum_t Phi_c[t][s][r] e_i[t]
    if (need_v) {
        const double2* ei = S.eig + (size_t)(q0 * nb + i) * nb;
        for (int idx = threadIdx.x; idx < F.npi * 9; idx += blockDim.x) {
            int pc = idx / 9, sr = idx % 9;
            double2 acc = make_double2(0.0, 0.0);
            for (int x = F.cl_start[pc]; x < F.cl_start[pc + 1]; x++) {
                int c = F.cl_index[x];
                int4 at = F.atoms[c];
                int4 mk = F.mk[c];
                double2 kap = lattice_phase(S, n0, n1, n2, -mk.x, -mk.y, -mk.z);
                kap.x *= F.mu[c];
                kap.y *= F.mu[c];
                const double* ph = F.phi + (size_t)c * 27 + sr;
                double2 t1 = make_double2(0.0, 0.0);
#pragma unroll
                for (int t = 0; t < 3; t++) {
                    double2 e = ei[3 * at.x + t];
                    double f = ph[t * 9];
                    t1.x = fma(f, e.x, t1.x);
                    t1.y = fma(f, e.y, t1.y);
                }
                acc = cmac(acc, kap, t1);
            }
            Z[idx] = acc;
        }
    }
    __syncthreads();

    const long long total = (long long)nb * nptk * nb;
    long long running = 0;
    int qn = 0;
    Comp accP = {0.0, 0.0}, accR = {0.0, 0.0}, accW = {0.0, 0.0};
    const long long list_base = (MODE == 1 || MODE == 3) ? p.list_off[w][mm] : 0;
    const double twopi_sqrt = sqrt(3.141592653589793238);

    for (long long base = 0; base < total; base += blockDim.x) {
        long long x = base + threadIdx.x;
        bool ok = false;
        if (x < total) {
            int j = (int)(x / ((long long)nptk * nb));
            int rem = (int)(x % ((long long)nptk * nb));
            int ii = rem / nb, k = rem % nb;
            int a, b, c;
            q_coords(S, ii, a, b, c);
            int ss = q_index(S, pmod(n0 + sign * a, S.n[0]), pmod(n1 + sign * b, S.n[1]), pmod(n2 + sign * c, S.n[2]));
            double4 wp = S.wv[ii * nb + j];
            double4 wd = S.wv[ss * nb + k];
            if (wp.w != 0.0 && wd.w != 0.0) {
                double sigma = sigma_exact(S, wp, wd);
                double delta = (sign > 0) ? __dadd_rn(__dadd_rn(omega, wp.w), -wd.w)
                                          : __dadd_rn(__dadd_rn(omega, -wp.w), -wd.w);
                ok = fabs(delta) <= 2.0 * sigma;
            }
        }
        int cnt;
        int pos = block_exclusive_scan_flag(ok, reinterpret_cast<int*>(warp_tot), cnt);
        if (ok) {
            if (MODE == 1) {
                int j = (int)(x / ((long long)nptk * nb));
                int rem = (int)(x % ((long long)nptk * nb));
                int ii = rem / nb, k = rem % nb;
                int a, b, c;
                q_coords(S, ii, a, b, c);
                int ss = q_index(S, pmod(n0 + sign * a, S.n[0]), pmod(n1 + sign * b, S.n[1]),
                                 pmod(n2 + sign * c, S.n[2]));
                long long o = list_base + running + pos;
                if (running + pos < p.nlist_counts[w][mm]) {
                    p.ind2[w][o] = ii * nb + j + 1;
                    p.ind3[w][o] = ss * nb + k + 1;
                } else {
                    atomicOr(p.err, kErrQueue);
                }
            } else {
                queue[qn + pos] = (int)x;
                qpos[qn + pos] = (int)(running + pos);
            }
        }
        running += cnt;
        if (MODE != 1) qn += cnt;
        const bool last = (base + blockDim.x >= total);
        if (MODE != 1 && (qn > kQ3 - (int)blockDim.x || last)) {
            // process the queued survivors, one per thread
            for (int e = threadIdx.x; e < qn; e += blockDim.x) {
                int xx = queue[e];
                int j = xx / (nptk * nb);
                int rem = xx % (nptk * nb);
                int ii = rem / nb, k = rem % nb;
                int a, b, c;
                q_coords(S, ii, a, b, c);
                int ss = q_index(S, pmod(n0 + sign * a, S.n[0]), pmod(n1 + sign * b, S.n[1]),
                                 pmod(n2 + sign * c, S.n[2]));
                double4 wp = S.wv[ii * nb + j];
                double4 wd = S.wv[ss * nb + k];
                double sigma = sigma_exact(S, wp, wd);
                double delta = (sign > 0) ? __dadd_rn(__dadd_rn(omega, wp.w), -wd.w)
                                          : __dadd_rn(__dadd_rn(omega, -wp.w), -wd.w);
                double g = exp(-(delta * delta) / (sigma * sigma));
                if (MODE == 0) {
                    accP.add(g / (sigma * twopi_sqrt * (double)((long long)nptk * nptk) * (double)(nb * nb * nb)));
                    continue;
                }
                double fp = p.bose[ii * nb + j], fd = p.bose[ss * nb + k];
                double bose = (sign > 0) ? (fp - fd) : (fp + fd + 1.0);
                double wp3 = bose * g / sigma / twopi_sqrt / (omega * wp.w * wd.w);
                accW.add(wp3);
                if (!need_v) continue;
                // V = sum_p exp(+-2 pi i n'.D_p/N) e'_j[s] Z_p[s][r] conj(e''_k[r])
                double2 V = make_double2(0.0, 0.0);
                const double2* e1 = S.eig + (size_t)(ii * nb + j) * nb;
                const double2* e2 = S.eig + (size_t)(ss * nb + k) * nb;
                for (int blk = 0; blk < F.nblk; blk++) {
                    int p0 = F.blk_start[blk], p1 = F.blk_start[blk + 1];
                    if (p0 == p1) continue;
                    int a2 = blk / S.natoms, a3 = blk % S.natoms;
                    double2 u[3], v[3];
#pragma unroll
                    for (int s = 0; s < 3; s++) {
                        u[s] = e1[3 * a2 + s];
                        if (sign < 0) u[s] = cconj(u[s]);
                        v[s] = cconj(e2[3 * a3 + s]);
                    }
                    for (int pc = p0; pc < p1; pc++) {
                        int4 D = F.pi_d[pc];
                        double2 ph = lattice_phase(S, a, b, c, sign * D.x, sign * D.y, sign * D.z);
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
                double av2 = V.x * V.x + V.y * V.y;
                double gam = p.scale * wp3 * av2;
                if (MODE == 3) {
                    long long o = list_base + qpos[e];
                    p.ind2[w][o] = ii * nb + j + 1;
                    p.ind3[w][o] = ss * nb + k + 1;
                    p.gamma[w][o] = gam * p.unit / (double)nptk;
                } else {
                    accR.add(gam);
                }
            }
            __syncthreads();
            qn = 0;
        }
    }
    // per-mode outputs
    if (MODE == 0) {
        double P = block_sum(accP.val(), red);
        if (threadIdx.x == 0) {
            p.n_out[w][mm] = (int)running;
            p.p_out[w][mm] = P;
        }
    } else if (MODE >= 2) {
        double W = block_sum(accW.val(), red);
        double R = block_sum(accR.val(), red);
        if (threadIdx.x == 0) {
            W = (sign > 0) ? W / nptk : W * 5.e-1 / nptk;
            p.wp[w][mm] = W;
            if (MODE == 2) p.rate[w][mm] = R * p.unit / (double)nptk * (sign > 0 ? 1.0 : 5.e-1);
        }
    }
    if (MODE == 3) {
        // rate = sum of the mode's Gamma list in order (Ind_driver), minus channel halved
        __syncthreads();
        Comp acc = {0.0, 0.0};
        for (long long e = threadIdx.x; e < running; e += blockDim.x) acc.add(p.gamma[w][list_base + e]);
        double R = block_sum(acc.val(), red);
        if (threadIdx.x == 0) p.rate[w][mm] = (sign > 0) ? R : R * 5.e-1;
    }
    if (threadIdx.x == 0 && (MODE == 2 || MODE == 3)) {
        atomicAdd(&p.stats[0], (unsigned long long)running);
        if (need_v) atomicAdd(&p.stats[1], (unsigned long long)running);
    }
}

// ---------------------------------------------------------------------------
// Four-phonon work-item kernel
// ---------------------------------------------------------------------------
struct Smem4 {
    double* sval;   // nb*nb sorted sums
    int* sidx;      // nb*nb packed (i*nb+j)
    int* cnt;       // nb*nb queue counters
    int* ncount;    // nb per-branch survivor counts (NP)
    double* pacc;   // nb per-branch phase-space sums (NP)
    double* racc;   // nb*NT rate partials
    double* wacc;   // nb*NT weight partials
    double2* kap;   // ntri cluster prefactors of this work item
    void* Z;        // nb*npi*9 reciprocal cluster table (double2 or float2)
    double* red;    // 32
    int* misc;      // [0]=work id, [1]=ns, [2]=flush flag
};

template <bool MIXED>
__device__ __forceinline__ size_t z_elem() {
    return MIXED ? sizeof(float2) : sizeof(double2);
}

__device__ __forceinline__ int lower_bound_d(const double* a, int n, double x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Phase B: contract every queued process of the current work item.
template <int NT, bool MIXED>
__device__ void k4_flush(const P4Params& p, Smem4& sm, const unsigned long long* qbase, int ch, int ll, int ii,
                         int q0, int n0, int n1, int n2, int m0, int m1, int m2, unsigned long long& my_contr) {
    const DevSys& S = p.S;
    const DevIfc& F = p.F;
    const int nb = S.nb, nb2 = nb * nb, nptk = S.nptk, npi = F.npi;
    const double sqrtpi = sqrt(3.141592653589793238);
    const double floor_sigma = (double)0.001f;
    const int dsign = (ch == 0) ? 1 : -1;  // class displacement D = m_k - m_l (++), m_l - m_k (+-, --)
    for (int i = 0; i < nb; i++) {
        int tot = 0;
        for (int j = 0; j < nb; j++) tot += sm.cnt[i * nb + j];
        if (tot == 0) continue;
        if (threadIdx.x == 0) atomicAdd(&p.stats[4], 1ull);
        // reciprocal cluster table for branch i and every j
        const double2* ei = S.eig + (size_t)(q0 * nb + i) * nb;
        for (int idx = threadIdx.x; idx < nb * npi * 9; idx += blockDim.x) {
            int j = idx / (npi * 9), rem = idx % (npi * 9), pc = rem / 9, sr = rem % 9;
            const double2* ej = S.eig + (size_t)(ii * nb + j) * nb;
            double2 acc = make_double2(0.0, 0.0);
            for (int x = F.cl_start[pc]; x < F.cl_start[pc + 1]; x++) {
                int c = F.cl_index[x];
                int4 at = F.atoms[c];
                const double* ph = F.phi + (size_t)c * 81 + sr;
                double2 t1 = make_double2(0.0, 0.0);
#pragma unroll
                for (int u = 0; u < 3; u++) {
                    double2 eu = ei[3 * at.x + u];
#pragma unroll
                    for (int t = 0; t < 3; t++) {
                        double2 et = ej[3 * at.y + t];
                        if (ch == 2) et = cconj(et);
                        double2 pr = cmul(eu, et);
                        double f = ph[(u * 3 + t) * 9];
                        t1.x = fma(f, pr.x, t1.x);
                        t1.y = fma(f, pr.y, t1.y);
                    }
                }
                acc = cmac(acc, sm.kap[c], t1);
            }
            if (MIXED)
                reinterpret_cast<float2*>(sm.Z)[idx] = make_float2((float)acc.x, (float)acc.y);
            else
                reinterpret_cast<double2*>(sm.Z)[idx] = acc;
        }
        __syncthreads();
        Comp accr[NT], accw[NT];
#pragma unroll
        for (int t = 0; t < NT; t++) {
            accr[t] = {0.0, 0.0};
            accw[t] = {0.0, 0.0};
        }
        const double omega = S.wv[q0 * nb + i].w;
        for (int j = 0; j < nb; j++) {
            const int bin = i * nb + j, cntb = sm.cnt[bin];
            const double4 w1 = S.wv[ii * nb + j];
            for (int e = threadIdx.x; e < cntb; e += blockDim.x) {
                unsigned long long ent = qbase[(size_t)bin * p.subcap + e];
                int jj = (int)(ent >> 32), k = (int)((ent >> 8) & 0xff), l = (int)(ent & 0xff);
                int a, b, c;
                q_coords(S, jj, a, b, c);
                int t0, t1, t2;
                if (ch == 0) {
                    t0 = n0 + m0 + a; t1 = n1 + m1 + b; t2 = n2 + m2 + c;
                } else if (ch == 1) {
                    t0 = n0 + m0 - a; t1 = n1 + m1 - b; t2 = n2 + m2 - c;
                } else {
                    t0 = n0 - m0 - a; t1 = n1 - m1 - b; t2 = n2 - m2 - c;
                }
                int ss = q_index(S, pmod(t0, S.n[0]), pmod(t1, S.n[1]), pmod(t2, S.n[2]));
                double4 w2 = S.wv[jj * nb + k];
                double4 w3 = S.wv[ss * nb + l];
                double sigma = sigma_exact(S, w2, w3);
                double s = (ch == 2) ? __dadd_rn(omega, -w1.w) : __dadd_rn(omega, w1.w);
                double delta = (ch == 0) ? __dadd_rn(__dadd_rn(s, w2.w), -w3.w) : __dadd_rn(__dadd_rn(s, -w2.w), -w3.w);
                if (sigma <= floor_sigma) sigma = 1.0 / sqrtpi;
                double g = exp(-(delta * delta) / (sigma * sigma));
                double base = g / sigma / sqrtpi / (omega * w1.w * w2.w * w3.w);
                double v2;
                if (!S.onlyharmonic) {
                    if (MIXED) {
                        const float2* Zj = reinterpret_cast<const float2*>(sm.Z) + (size_t)j * npi * 9;
                        float2 V = make_float2(0.f, 0.f);
                        const float2* e2 = S.eigf + (size_t)(jj * nb + k) * nb;
                        const float2* e3 = S.eigf + (size_t)(ss * nb + l) * nb;
                        for (int blk = 0; blk < F.nblk; blk++) {
                            int p0 = F.blk_start[blk], p1 = F.blk_start[blk + 1];
                            if (p0 == p1) continue;
                            int a3 = blk / S.natoms, a4 = blk % S.natoms;
                            float2 u[3], v[3];
#pragma unroll
                            for (int x = 0; x < 3; x++) {
                                u[x] = e2[3 * a3 + x];
                                if (ch != 0) u[x] = cconjf(u[x]);
                                v[x] = cconjf(e3[3 * a4 + x]);
                            }
                            for (int pc = p0; pc < p1; pc++) {
                                int4 D = F.pi_d[pc];
                                float2 ph = lattice_phase_f(S, a, b, c, dsign * D.x, dsign * D.y, dsign * D.z);
                                const float2* z = Zj + pc * 9;
                                float2 tt = make_float2(0.f, 0.f);
#pragma unroll
                                for (int x = 0; x < 3; x++) {
                                    float2 h = make_float2(0.f, 0.f);
#pragma unroll
                                    for (int r = 0; r < 3; r++) h = cmacf(h, z[x * 3 + r], v[r]);
                                    tt = cmacf(tt, u[x], h);
                                }
                                V = cmacf(V, ph, tt);
                            }
                        }
                        v2 = (double)V.x * (double)V.x + (double)V.y * (double)V.y;
                    } else {
                        const double2* Zj = reinterpret_cast<const double2*>(sm.Z) + (size_t)j * npi * 9;
                        double2 V = make_double2(0.0, 0.0);
                        const double2* e2 = S.eig + (size_t)(jj * nb + k) * nb;
                        const double2* e3 = S.eig + (size_t)(ss * nb + l) * nb;
                        for (int blk = 0; blk < F.nblk; blk++) {
                            int p0 = F.blk_start[blk], p1 = F.blk_start[blk + 1];
                            if (p0 == p1) continue;
                            int a3 = blk / S.natoms, a4 = blk % S.natoms;
                            double2 u[3], v[3];
#pragma unroll
                            for (int x = 0; x < 3; x++) {
                                u[x] = e2[3 * a3 + x];
                                if (ch != 0) u[x] = cconj(u[x]);
                                v[x] = cconj(e3[3 * a4 + x]);
                            }
                            for (int pc = p0; pc < p1; pc++) {
                                int4 D = F.pi_d[pc];
                                double2 ph = lattice_phase(S, a, b, c, dsign * D.x, dsign * D.y, dsign * D.z);
                                const double2* z = Zj + pc * 9;
                                double2 tt = make_double2(0.0, 0.0);
#pragma unroll
                                for (int x = 0; x < 3; x++) {
                                    double2 h = make_double2(0.0, 0.0);
#pragma unroll
                                    for (int r = 0; r < 3; r++) h = cmac(h, z[x * 3 + r], v[r]);
                                    tt = cmac(tt, u[x], h);
                                }
                                V = cmac(V, ph, tt);
                            }
                        }
                        v2 = V.x * V.x + V.y * V.y;
                    }
                } else {
                    v2 = 0.0;
                }
                my_contr++;
                const size_t plane = (size_t)nptk * nb;
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    if (t < p.nT) {
                        const double* bz = p.bose + t * plane;
                        double f1 = bz[ii * nb + j], f2 = bz[jj * nb + k], f3 = bz[ss * nb + l];
                        double bc;
                        if (ch == 0)
                            bc = f1 * f2 * (1 + f3) - (1 + f1) * (1 + f2) * f3;
                        else if (ch == 1)
                            bc = f1 * (1 + f2) * (1 + f3) - (1 + f1) * f2 * f3;
                        else
                            bc = (1 + f1) * (1 + f2) * (1 + f3) - f1 * f2 * f3;
                        double wp4 = bc * base;
                        accr[t].add(wp4 * v2);
                        accw[t].add(wp4);
                    }
                }
            }
        }
#pragma unroll
        for (int t = 0; t < NT; t++) {
            if (t < p.nT) {
                double r = block_sum(accr[t].val(), sm.red);
                double w = block_sum(accw[t].val(), sm.red);
                if (threadIdx.x == 0) {
                    sm.racc[i * NT + t] += r;
                    sm.wacc[i * NT + t] += w;
                }
            }
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < nb2; idx += blockDim.x) sm.cnt[idx] = 0;
    __syncthreads();
}

template <int KIND, int NT, bool MIXED>  // KIND 0 = count (NP), 2 = rates (RTA)
__global__ void __launch_bounds__(256) k4_work(P4Params p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const DevSys& S = p.S;
    const DevIfc& F = p.F;
    const int nb = S.nb, nptk = S.nptk, nb2 = nb * nb;
    // carve shared memory
    unsigned char* sp = smem_raw;
    Smem4 sm;
    sm.Z = sp;
    sp += (KIND == 2) ? (size_t)nb * F.npi * 9 * z_elem<MIXED>() : 0;
    sm.kap = reinterpret_cast<double2*>(sp);
    sp += (KIND == 2) ? (size_t)F.ntri * sizeof(double2) : 0;
    sm.sval = reinterpret_cast<double*>(sp);
    sp += (size_t)nb2 * sizeof(double);
    sm.racc = reinterpret_cast<double*>(sp);
    sp += (size_t)nb * NT * sizeof(double);
    sm.wacc = reinterpret_cast<double*>(sp);
    sp += (size_t)nb * NT * sizeof(double);
    sm.pacc = reinterpret_cast<double*>(sp);
    sp += (size_t)nb * sizeof(double);
    sm.red = reinterpret_cast<double*>(sp);
    sp += 32 * sizeof(double);
    sm.sidx = reinterpret_cast<int*>(sp);
    sp += (size_t)nb2 * sizeof(int);
    sm.cnt = reinterpret_cast<int*>(sp);
    sp += (size_t)nb2 * sizeof(int);
    sm.ncount = reinterpret_cast<int*>(sp);
    sp += (size_t)nb * sizeof(int);
    sm.misc = reinterpret_cast<int*>(sp);

    unsigned long long* qbase = p.queue + (size_t)blockIdx.x * nb2 * p.subcap;
    unsigned long long my_surv = 0, my_contr = 0, my_sig = 0, my_cand = 0;
    const double sqrtpi = sqrt(3.141592653589793238);
    const double floor_sigma = (double)0.001f;

    for (;;) {
        if (threadIdx.x == 0) sm.misc[0] = atomicAdd(p.work_counter, 1);
        __syncthreads();
        const int wi = sm.misc[0];
        if (wi >= p.nwork) break;
        const int ch = wi % 3;
        const int rest = wi / 3;
        const int ii = rest % nptk, ll = rest / nptk;
        const int q0 = S.list0[ll];
        int n0, n1, n2, m0, m1, m2;
        q_coords(S, q0, n0, n1, n2);
        q_coords(S, ii, m0, m1, m2);
        // sums s_ij = w_i +- w'_j for the valid branch pairs, sorted by value
        for (int idx = threadIdx.x; idx < nb2; idx += blockDim.x) {
            int i = idx / nb, j = idx % nb;
            double wi_ = S.wv[q0 * nb + i].w, wj_ = S.wv[ii * nb + j].w;
            bool ok = (wi_ != 0.0) && (wi_ <= S.omega_max) && (wj_ != 0.0);
            double s = (ch == 2) ? __dadd_rn(wi_, -wj_) : __dadd_rn(wi_, wj_);
            int rank = 0, nvalid = 0;
            for (int y = 0; y < nb2; y++) {
                int iy = y / nb, jy = y % nb;
                double wiy = S.wv[q0 * nb + iy].w, wjy = S.wv[ii * nb + jy].w;
                bool oky = (wiy != 0.0) && (wiy <= S.omega_max) && (wjy != 0.0);
                if (!oky) continue;
                nvalid++;
                double sy = (ch == 2) ? __dadd_rn(wiy, -wjy) : __dadd_rn(wiy, wjy);
                if (sy < s || (sy == s && y < idx)) rank++;
            }
            if (ok) {
                sm.sval[rank] = s;
                sm.sidx[rank] = idx;
            }
            if (idx == 0) sm.misc[1] = nvalid;
            sm.cnt[idx] = 0;
        }
        for (int idx = threadIdx.x; idx < nb; idx += blockDim.x) {
            sm.ncount[idx] = 0;
            sm.pacc[idx] = 0.0;
        }
        for (int idx = threadIdx.x; idx < nb * NT; idx += blockDim.x) {
            sm.racc[idx] = 0.0;
            sm.wacc[idx] = 0.0;
        }
        if (KIND == 2) {
            // cluster prefactors kappa_c = mu_c exp(2 pi i (-n.m_l +- n'.(m_j - m_l))/N)
            for (int c = threadIdx.x; c < F.ntri; c += blockDim.x) {
                int4 mj = F.mj[c], ml = F.ml[c];
                double2 a = lattice_phase(S, n0, n1, n2, -ml.x, -ml.y, -ml.z);
                int sj = (ch == 2) ? -1 : 1;
                double2 b = lattice_phase(S, m0, m1, m2, sj * (mj.x - ml.x), sj * (mj.y - ml.y), sj * (mj.z - ml.z));
                double2 k = cmul(a, b);
                k.x *= F.mu[c];
                k.y *= F.mu[c];
                sm.kap[c] = k;
            }
        }
        __syncthreads();
        const int ns = sm.misc[1];
        if (ns > 0) {
            const int jj_lo = (ch == 1) ? 0 : ii;
            const long long total = (long long)(nptk - jj_lo) * nb2;
            double smax = 0.0;
            for (int x = 0; x < ns; x++) smax = fmax(smax, fabs(sm.sval[x]));
            for (long long base = 0; base < total; base += blockDim.x) {
                if (KIND == 2) {
                    // flush the queues before any of them could overflow
                    if (threadIdx.x == 0) {
                        int mx = 0;
                        for (int b = 0; b < nb2; b++) mx = max(mx, sm.cnt[b]);
                        sm.misc[2] = (mx > p.subcap - (int)blockDim.x);
                    }
                    __syncthreads();
                    if (sm.misc[2]) {
                        k4_flush<NT, MIXED>(p, sm, qbase, ch, ll, ii, q0, n0, n1, n2, m0, m1, m2, my_contr);
                    }
                }
                long long t = base + threadIdx.x;
                if (t < total) {
                    int jj = jj_lo + (int)(t / nb2);
                    int kl = (int)(t % nb2);
                    int k = kl / nb, l = kl % nb;
                    int a, b, c;
                    q_coords(S, jj, a, b, c);
                    int t0, t1, t2;
                    if (ch == 0) {
                        t0 = n0 + m0 + a; t1 = n1 + m1 + b; t2 = n2 + m2 + c;
                    } else if (ch == 1) {
                        t0 = n0 + m0 - a; t1 = n1 + m1 - b; t2 = n2 + m2 - c;
                    } else {
                        t0 = n0 - m0 - a; t1 = n1 - m1 - b; t2 = n2 - m2 - c;
                    }
                    int ss = q_index(S, pmod(t0, S.n[0]), pmod(t1, S.n[1]), pmod(t2, S.n[2]));
                    bool go = true;
                    if (ch != 0 && ss < jj) go = false;
                    if (ch != 0 && ss == jj && l < k) go = false;
                    double4 w2 = S.wv[jj * nb + k];
                    double4 w3 = S.wv[ss * nb + l];
                    if (go && w2.w != 0.0 && w3.w != 0.0) {
                        double sigma = sigma_exact(S, w2, w3);
                        my_sig++;
                        double cen = (ch == 0) ? (w3.w - w2.w) : (w2.w + w3.w);
                        double tol = 1e-12 * (1.0 + fabs(w2.w) + fabs(w3.w) + smax + sigma);
                        int x = lower_bound_d(sm.sval, ns, cen - sigma - tol);
                        for (; x < ns && sm.sval[x] <= cen + sigma + tol; x++) {
                            my_cand++;
                            double s = sm.sval[x];
                            double delta = (ch == 0) ? __dadd_rn(__dadd_rn(s, w2.w), -w3.w)
                                                     : __dadd_rn(__dadd_rn(s, -w2.w), -w3.w);
                            if (!(fabs(delta) <= sigma)) continue;
                            int idx = sm.sidx[x];
                            int i = idx / nb, j = idx % nb;
                            if (ch != 1 && jj == ii && k < j) continue;
                            if (ch == 1 && !((q0 != jj || i != k) && (q0 != ss || i != l) && (ii != jj || j != k) &&
                                             (ii != ss || j != l)))
                                continue;
                            my_surv++;
                            if (KIND == 0) {
                                atomicAdd(&sm.ncount[i], 1);
                                double sg = (sigma <= floor_sigma) ? 1.0 / sqrtpi : sigma;
                                double pc = exp(-(delta * delta) / (sg * sg)) /
                                            (sg * sqrtpi * ((double)nptk * (double)nptk * (double)nptk) *
                                             (double)(nb * nb * nb * nb));
                                atomicAdd(&sm.pacc[i], pc);
                                continue;
                            }
                            double w1 = S.wv[ii * nb + j].w;
                            if (w1 <= 1.25 || w2.w <= 1.25 || w3.w <= 1.25) continue;  // WP4 = 0
                            int pos = atomicAdd(&sm.cnt[idx], 1);
                            qbase[(size_t)idx * p.subcap + pos] = pack4(jj, j, k, l);
                        }
                    }
                }
            }
            if (KIND == 2) {
                __syncthreads();
                k4_flush<NT, MIXED>(p, sm, qbase, ch, ll, ii, q0, n0, n1, n2, m0, m1, m2, my_contr);
            }
        }
        __syncthreads();
        if (KIND == 0) {
            for (int i = threadIdx.x; i < nb; i += blockDim.x) {
                if (sm.ncount[i]) atomicAdd(&p.n_count[ch * S.nlist * nb + ll * nb + i], (unsigned long long)sm.ncount[i]);
                if (sm.pacc[i] != 0.0) atomicAdd(&p.p_sum[ch * S.nlist * nb + ll * nb + i], sm.pacc[i]);
            }
        } else {
            for (int idx = threadIdx.x; idx < nb * NT; idx += blockDim.x) {
                int i = idx / NT, t = idx % NT;
                if (t < p.nT) {
                    p.part_rate[((size_t)wi * p.nT + t) * nb + i] = sm.racc[idx];
                    p.part_wp[((size_t)wi * p.nT + t) * nb + i] = sm.wacc[idx];
                }
            }
        }
        __syncthreads();
    }
    // statistics
    double red_s = block_sum((double)my_surv, sm.red);
    double red_c = block_sum((double)my_contr, sm.red);
    double red_g = block_sum((double)my_sig, sm.red);
    double red_x = block_sum((double)my_cand, sm.red);
    if (threadIdx.x == 0) {
        atomicAdd(&p.stats[0], (unsigned long long)red_s);
        atomicAdd(&p.stats[1], (unsigned long long)red_c);
        atomicAdd(&p.stats[2], (unsigned long long)red_g);
        atomicAdd(&p.stats[3], (unsigned long long)red_x);
    }
}

}  // namespace fp4

namespace fp4 {

// ---------------------------------------------------------------------------
// Ordered four-phonon index lists (Ind_only_plusplus/plusminus/minusminus,
// processes.f90:2854-3074): one CTA per mode, candidates walked in the
// reference's loop order (q', q'', j, k, l) and compacted in order.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k4_order(P4OrderParams p) {
    __shared__ int warp_tot[34];
    const DevSys& S = p.S;
    const int nb = S.nb, nptk = S.nptk, ch = p.ch;
    const int mm = blockIdx.x, ll = mm / nb, i = mm % nb;
    const int q0 = S.list0[ll];
    int n0, n1, n2;
    q_coords(S, q0, n0, n1, n2);
    const double omega = S.wv[q0 * nb + i].w;
    if (!(omega != 0.0 && omega <= S.omega_max) || p.counts[mm] == 0) return;
    const long long nb3 = (long long)nb * nb * nb;
    const long long total = (long long)nptk * nptk * nb3;
    long long running = 0;
    const long long off = p.list_off[mm], cap = p.counts[mm];
    for (long long base = 0; base < total; base += blockDim.x) {
        long long x = base + threadIdx.x;
        bool ok = false;
        int ii = 0, jj = 0, j = 0, k = 0, l = 0, ss = 0;
        if (x < total) {
            long long pr = x / nb3;
            int br = (int)(x % nb3);
            ii = (int)(pr / nptk);
            jj = (int)(pr % nptk);
            j = br / (nb * nb);
            k = (br / nb) % nb;
            l = br % nb;
            bool go = (ch == 1) || (jj >= ii);
            int m0, m1, m2, a, b, c;
            q_coords(S, ii, m0, m1, m2);
            q_coords(S, jj, a, b, c);
            int t0, t1, t2;
            if (ch == 0) {
                t0 = n0 + m0 + a; t1 = n1 + m1 + b; t2 = n2 + m2 + c;
            } else if (ch == 1) {
                t0 = n0 + m0 - a; t1 = n1 + m1 - b; t2 = n2 + m2 - c;
            } else {
                t0 = n0 - m0 - a; t1 = n1 - m1 - b; t2 = n2 - m2 - c;
            }
            ss = q_index(S, pmod(t0, S.n[0]), pmod(t1, S.n[1]), pmod(t2, S.n[2]));
            if (ch != 0 && ss < jj) go = false;
            if (ch != 1 && jj == ii && k < j) go = false;
            if (ch != 0 && ss == jj && l < k) go = false;
            if (go) {
                double4 w1 = S.wv[ii * nb + j], w2 = S.wv[jj * nb + k], w3 = S.wv[ss * nb + l];
                if (w1.w != 0.0 && w2.w != 0.0 && w3.w != 0.0) {
                    bool excl = false;
                    if (ch == 1)
                        excl = !((q0 != jj || i != k) && (q0 != ss || i != l) && (ii != jj || j != k) &&
                                 (ii != ss || j != l));
                    if (!excl) {
                        double sigma = sigma_exact(S, w2, w3);
                        double s = (ch == 2) ? __dadd_rn(omega, -w1.w) : __dadd_rn(omega, w1.w);
                        double delta = (ch == 0) ? __dadd_rn(__dadd_rn(s, w2.w), -w3.w)
                                                 : __dadd_rn(__dadd_rn(s, -w2.w), -w3.w);
                        ok = fabs(delta) <= sigma;
                    }
                }
            }
        }
        int cnt;
        int pos = block_exclusive_scan_flag(ok, warp_tot, cnt);
        if (ok) {
            long long r = running + pos;
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
}

// Bose-Einstein occupations for every mode and temperature.
__global__ void k_bose(DevSys S, const double* T, int nT, double* bose) {
    const size_t plane = (size_t)S.nptk * S.nb;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < plane * nT; x += (size_t)gridDim.x * blockDim.x) {
        int t = (int)(x / plane);
        size_t qb = x % plane;
        bose[x] = bose_of(S.wv[qb].w, T[t]);
    }
}

// Fixed-order compensated reduction of the per-work-item partial sums.
__global__ void k4_reduce(P4Params p, double* r0, double* r1, double* r2, double* w0, double* w1, double* w2,
                          double rate_scale) {
    const DevSys& S = p.S;
    const int nb = S.nb, nptk = S.nptk, nl = S.nlist;
    const int total = 3 * nl * nb * p.nT;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < total; x += gridDim.x * blockDim.x) {
        int ch = x % 3;
        int rest = x / 3;
        int i = rest % nb;
        rest /= nb;
        int t = rest % p.nT;
        int ll = rest / p.nT;
        Comp ar = {0.0, 0.0}, aw = {0.0, 0.0};
        for (int ii = 0; ii < nptk; ii++) {
            size_t wi = ((size_t)ll * nptk + ii) * 3 + ch;
            ar.add(p.part_rate[(wi * p.nT + t) * nb + i]);
            aw.add(p.part_wp[(wi * p.nT + t) * nb + i]);
        }
        size_t o = ((size_t)t * nl + ll) * nb + i;
        double* R = ch == 0 ? r0 : (ch == 1 ? r1 : r2);
        double* W = ch == 0 ? w0 : (ch == 1 ? w1 : w2);
        R[o] = ar.val() * rate_scale / nptk / nptk;
        W[o] = aw.val() / nptk / nptk;
    }
}

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
size_t k3_smem(int mode, const DevIfc& F, bool onlyharmonic) {
    bool need_v = (mode == 3) || (mode == 2 && !onlyharmonic);
    size_t z = need_v ? (size_t)F.npi * 9 * sizeof(double2) : 0;
    return z + 2 * kQ3 * sizeof(int) + 34 * sizeof(int) + 32 * sizeof(double);
}

template <int MODE>
static cudaError_t launch_k3_t(const P3Params& p, int nmodes, cudaStream_t st) {
    size_t sm = k3_smem(MODE, p.F, p.S.onlyharmonic);
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

static int round_nt(int nT) { return nT <= 1 ? 1 : (nT <= 2 ? 2 : (nT <= 4 ? 4 : 8)); }

size_t k4_smem(int kind, int nT, bool mixed, const DevSys& S, const DevIfc& F) {
    const int NT = round_nt(nT);
    const size_t nb = S.nb, nb2 = nb * nb;
    size_t z = (kind == 2) ? nb * F.npi * 9 * (mixed ? sizeof(float2) : sizeof(double2)) : 0;
    size_t kap = (kind == 2) ? F.ntri * sizeof(double2) : 0;
    size_t s = z + kap + nb2 * sizeof(double) + 2 * nb * NT * sizeof(double) + nb * sizeof(double) +
               32 * sizeof(double) + nb2 * sizeof(int) * 2 + nb * sizeof(int) + 4 * sizeof(int);
    return (s + 15) & ~(size_t)15;
}

template <int KIND, int NT, bool MIXED>
static cudaError_t launch_k4_t(const P4Params& p, int nblocks, cudaStream_t st) {
    size_t sm = k4_smem(KIND, p.nT, MIXED, p.S, p.F);
    cudaError_t e = cudaFuncSetAttribute(k4_work<KIND, NT, MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k4_work<KIND, NT, MIXED><<<nblocks, 256, sm, st>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_k4(int kind, int nT, bool mixed, const P4Params& p, int nblocks, cudaStream_t st) {
    if (kind == 0) return launch_k4_t<0, 1, false>(p, nblocks, st);
    const int NT = round_nt(nT);
#define FP4_K4(NTV)                                                                                    \
    if (NT == NTV) return mixed ? launch_k4_t<2, NTV, true>(p, nblocks, st) : launch_k4_t<2, NTV, false>(p, nblocks, st);
    FP4_K4(1)
    FP4_K4(2)
    FP4_K4(4)
    FP4_K4(8)
#undef FP4_K4
    return cudaErrorInvalidValue;
}

cudaError_t launch_k4_reduce(const P4Params& p, double* r0, double* r1, double* r2, double* w0, double* w1, double* w2,
                             double rate_scale, cudaStream_t st) {
    int total = 3 * p.S.nlist * p.S.nb * p.nT;
    int threads = 128, blocks = (total + threads - 1) / threads;
    k4_reduce<<<blocks, threads, 0, st>>>(p, r0, r1, r2, w0, w1, w2, rate_scale);
    return cudaGetLastError();
}

cudaError_t launch_k4_order(const P4OrderParams& p, int nmodes, cudaStream_t st) {
    k4_order<<<nmodes, 256, 0, st>>>(p);
    return cudaGetLastError();
}

cudaError_t launch_bose(const DevSys& S, const double* T, int nT, double* bose, cudaStream_t st) {
    size_t n = (size_t)S.nptk * S.nb * nT;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    k_bose<<<blocks, 256, 0, st>>>(S, T, nT, bose);
    return cudaGetLastError();
}

}  // namespace fp4
