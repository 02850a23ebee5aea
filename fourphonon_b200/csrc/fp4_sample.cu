// Sampled four-phonon estimators on the device: NP_plusplus_sample ... and
// RTA_plusplus_sample ... (processes.f90:2480-2746, 4811-5172).
//
// For every mode and channel, `nsamples` uniform draws of (q', j, q'', k, l)
// are taken; a draw inside the channel's restricted set (the same restrictions
// as the full enumeration) that passes the 1-sigma energy test is a sampled
// process.  Its weight is the full driver's; the estimate is the sum scaled by
// total_process / nsamples, total_process = nb^3 nptk^2.  The draws come from a
// counter-based splitmix64 stream keyed by (seed, mode, channel, sample), so
// the CPU oracle draws exactly the same samples.
//
// One CTA takes a chunk of samples of one (mode, channel): its threads draw
// and filter, survivors go to a shared-memory list, and then each thread
// contracts one survivor's V(4) directly over the clusters (phases from the
// integer lattice coordinates, as in the rate kernel).  Per-chunk sums go to a
// buffer reduced afterwards in a fixed order with compensated sums.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "../../include/fourphonon_b200.h"
#include "fp4_ctx.h"
#include "fp4_device.cuh"
#include "fp4_internal.h"

using namespace fp4;

namespace {

constexpr int kSThreads = 256;
constexpr int kSChunk = 1024;  // samples per CTA item (= survivor list capacity)

struct PSParams {
    DevSys S;
    DevIfc F;
    int nT;
    const double* bose;  // [t][q*nb+b]
    long long nsamples;
    unsigned long long seed;
    int nchunk;  // chunks per (mode, channel)
    int mode;    // 0: counts and P4, 2: rates and WP4
    int nitems;
    int* work_counter;
    double* part;                // [item][2*nT] (mode 2: gamma_t, wp_t; mode 0: P)
    unsigned long long* part_n;  // [item] sampled processes
    unsigned long long* stats;
    int* err;
};

__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ int draw_k(unsigned long long base, int k, int range) {
    return (int)__umul64hi(mix64(base + (unsigned long long)k), (unsigned long long)range);
}

// V(4) of one process, summed over the clusters (Vp_pp/pm/mm, processes.f90:142-330):
//   sum_c mu_c exp(2 pi i (s_j n'.m_j + s_k n''.m_k - n'''.m_l)/N)
//         sum_{u,t,s,r} Psi_c[u][t][s][r] e_i[u] e~'_j[t] e~''_k[s] conj(e'''_l[r])
__device__ double2 vp4_direct(const DevSys& S, const DevIfc& F, int ch, const double2* ei, const double2* ej,
                              const double2* ek, const double2* el, int m0, int m1, int m2, int a0, int a1, int a2,
                              int t0, int t1, int t2) {
    const int sj = (ch == 2) ? -1 : 1, sk = (ch == 0) ? 1 : -1;
    double2 V = make_double2(0.0, 0.0);
    for (int c = 0; c < F.ntri; c++) {
        const int4 at = F.atoms[c];
        const int4 mj = F.mj[c], mk = F.mk[c], ml = F.ml[c];
        const double2 ph =
            cmul(cmul(S.root[0][pmod(sj * m0 * mj.x + sk * a0 * mk.x - t0 * ml.x, S.n[0])],
                      S.root[1][pmod(sj * m1 * mj.y + sk * a1 * mk.y - t1 * ml.y, S.n[1])]),
                 S.root[2][pmod(sj * m2 * mj.z + sk * a2 * mk.z - t2 * ml.z, S.n[2])]);
        double2 I[3], J[3], K[3], L[3];
#pragma unroll
        for (int x = 0; x < 3; x++) {
            I[x] = ei[3 * at.x + x];
            J[x] = ej[3 * at.y + x];
            if (ch == 2) J[x] = cconj(J[x]);
            K[x] = ek[3 * at.z + x];
            if (ch != 0) K[x] = cconj(K[x]);
            L[x] = cconj(el[3 * at.w + x]);
        }
        const double* psi = F.phi + (size_t)c * 81;
        double2 A = make_double2(0.0, 0.0);
#pragma unroll
        for (int u = 0; u < 3; u++) {
            double2 wu = make_double2(0.0, 0.0);
#pragma unroll
            for (int t = 0; t < 3; t++) {
                double2 y = make_double2(0.0, 0.0);
#pragma unroll
                for (int s = 0; s < 3; s++) {
                    const double* row = psi + ((u * 3 + t) * 3 + s) * 3;
                    double2 xs = make_double2(0.0, 0.0);
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        xs.x = fma(row[r], L[r].x, xs.x);
                        xs.y = fma(row[r], L[r].y, xs.y);
                    }
                    y = cmac(y, xs, K[s]);
                }
                wu = cmac(wu, y, J[t]);
            }
            A = cmac(A, wu, I[u]);
        }
        const double2 w = make_double2(F.mu[c] * ph.x, F.mu[c] * ph.y);
        V = cmac(V, w, A);
    }
    return V;
}

// The same sum in FP32 (mixed precision): FP32 eigenvectors and root tables,
// the cluster constants rounded to FP32 as they are read, FP32 accumulation.
__device__ float2 vp4_direct_f(const DevSys& S, const DevIfc& F, int ch, const float2* ei, const float2* ej,
                               const float2* ek, const float2* el, int m0, int m1, int m2, int a0, int a1, int a2,
                               int t0, int t1, int t2) {
    const int sj = (ch == 2) ? -1 : 1, sk = (ch == 0) ? 1 : -1;
    float2 V = make_float2(0.f, 0.f);
    for (int c = 0; c < F.ntri; c++) {
        const int4 at = F.atoms[c];
        const int4 mj = F.mj[c], mk = F.mk[c], ml = F.ml[c];
        const float2 ph =
            cmulf(cmulf(S.rootf[0][pmod(sj * m0 * mj.x + sk * a0 * mk.x - t0 * ml.x, S.n[0])],
                        S.rootf[1][pmod(sj * m1 * mj.y + sk * a1 * mk.y - t1 * ml.y, S.n[1])]),
                  S.rootf[2][pmod(sj * m2 * mj.z + sk * a2 * mk.z - t2 * ml.z, S.n[2])]);
        float2 I[3], J[3], K[3], L[3];
#pragma unroll
        for (int x = 0; x < 3; x++) {
            I[x] = ei[3 * at.x + x];
            J[x] = ej[3 * at.y + x];
            if (ch == 2) J[x] = cconjf(J[x]);
            K[x] = ek[3 * at.z + x];
            if (ch != 0) K[x] = cconjf(K[x]);
            L[x] = cconjf(el[3 * at.w + x]);
        }
        const double* psi = F.phi + (size_t)c * 81;
        float2 A = make_float2(0.f, 0.f);
#pragma unroll
        for (int u = 0; u < 3; u++) {
            float2 wu = make_float2(0.f, 0.f);
#pragma unroll
            for (int t = 0; t < 3; t++) {
                float2 y = make_float2(0.f, 0.f);
#pragma unroll
                for (int s = 0; s < 3; s++) {
                    const double* row = psi + ((u * 3 + t) * 3 + s) * 3;
                    float2 xs = make_float2(0.f, 0.f);
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        const float f = (float)row[r];
                        xs.x = fmaf(f, L[r].x, xs.x);
                        xs.y = fmaf(f, L[r].y, xs.y);
                    }
                    y = cmacf(y, xs, K[s]);
                }
                wu = cmacf(wu, y, J[t]);
            }
            A = cmacf(A, wu, I[u]);
        }
        const float mu = (float)F.mu[c];
        V = cmacf(V, make_float2(mu * ph.x, mu * ph.y), A);
    }
    return V;
}

struct SEntry {
    int ii, jj, ss, jkl;
    double sigma, delta;
};

template <int NT, bool MIXED>
__global__ void __launch_bounds__(kSThreads) k4_sample(PSParams p) {
    __shared__ SEntry q[kSChunk];
    __shared__ int s_cnt, s_item;
    __shared__ double red[32 * (2 * NT + 2)];
    const DevSys& S = p.S;
    const int nb = S.nb, nptk = S.nptk;
    const int N0 = S.n[0], N1 = S.n[1], N2 = S.n[2];
    const double sqrtpi = sqrt(3.141592653589793238);
    const double floor_sigma = (double)0.001f;
    for (;;) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(p.work_counter, 1);
            s_cnt = 0;
        }
        __syncthreads();
        const int item = s_item;
        if (item >= p.nitems) break;
        const int chunk = item % p.nchunk, rest = item / p.nchunk, ch = rest % 3, m0 = rest / 3;
        const int mm = m0 + 1, i = m0 % nb, ll = m0 / nb;
        const int q0 = S.list0[ll];
        int n0, n1, n2;
        q_coords_t(S, q0, n0, n1, n2);
        const double omega = S.wv[q0 * nb + i].w;
        const bool active = (omega != 0.0) && (omega <= S.omega_max);
        const long long c0 = (long long)chunk * kSChunk;
        const long long c1 = min(c0 + (long long)kSChunk, p.nsamples);
        unsigned long long my_n = 0;
        Comp accP = {0.0, 0.0};
        if (active) {
            for (long long it = c0 + threadIdx.x; it < c1; it += blockDim.x) {
                const unsigned long long c = ((unsigned long long)((mm - 1) * 3 + ch) << 32) | (unsigned long long)it;
                const unsigned long long base = mix64(p.seed ^ mix64(c));
                const int ii = draw_k(base, 0, nptk), j = draw_k(base, 1, nb);
                const int jj = draw_k(base, 2, nptk), k = draw_k(base, 3, nb), l = draw_k(base, 4, nb);
                int m0c, m1c, m2c, a, b, cc;
                q_coords_t(S, ii, m0c, m1c, m2c);
                q_coords_t(S, jj, a, b, cc);
                int t0, t1, t2;
                if (ch == 0) {
                    t0 = n0 + m0c + a; t1 = n1 + m1c + b; t2 = n2 + m2c + cc;
                } else if (ch == 1) {
                    t0 = n0 + m0c - a; t1 = n1 + m1c - b; t2 = n2 + m2c - cc;
                } else {
                    t0 = n0 - m0c - a; t1 = n1 - m1c - b; t2 = n2 - m2c - cc;
                }
                const int ss = q_index(S, wrapN(t0, N0), wrapN(t1, N1), wrapN(t2, N2));
                bool ok;
                if (ch == 0)
                    ok = jj >= ii && k >= ((jj == ii) ? j : 0);
                else if (ch == 1)
                    ok = ss >= jj && l >= ((ss == jj) ? k : 0);
                else
                    ok = jj >= ii && k >= ((jj == ii) ? j : 0) && ss >= jj && l >= ((ss == jj) ? k : 0);
                if (!ok) continue;
                const double w1 = S.wv[ii * nb + j].w;
                const double4 w2 = S.wv[jj * nb + k];
                const double4 w3 = S.wv[ss * nb + l];
                if (!(w1 != 0.0 && w2.w != 0.0 && w3.w != 0.0)) continue;
                const double sigma = sigma_exact(S, w2, w3);
                if (ch == 1 && !((q0 != jj || i != k) && (q0 != ss || i != l) && (ii != jj || j != k) &&
                                 (ii != ss || j != l)))
                    continue;
                const double sv = (ch == 2) ? __dadd_rn(omega, -w1) : __dadd_rn(omega, w1);
                const double delta = (ch == 0) ? __dadd_rn(__dadd_rn(sv, w2.w), -w3.w)
                                               : __dadd_rn(__dadd_rn(sv, -w2.w), -w3.w);
                if (!(fabs(delta) <= sigma)) continue;
                my_n++;
                const double sg = (sigma <= floor_sigma) ? 1.0 / sqrtpi : sigma;
                if (p.mode == 0) {
                    accP.add(exp(-(delta * delta) / (sg * sg)) /
                             (sg * sqrtpi * ((double)nptk * (double)nptk * (double)nptk) * (double)(nb * nb * nb * nb)));
                    continue;
                }
                const int pos = atomicAdd(&s_cnt, 1);  // one survivor at most per sample: pos < kSChunk
                SEntry e;
                e.ii = ii;
                e.jj = jj;
                e.ss = ss;
                e.jkl = j | (k << 8) | (l << 16);
                e.sigma = sg;
                e.delta = delta;
                q[pos] = e;
            }
        }
        __syncthreads();
        double acc[2 * NT];
#pragma unroll
        for (int x = 0; x < 2 * NT; x++) acc[x] = 0.0;
        if (p.mode == 2) {
            const int nq = s_cnt;
            const double2* ei = S.eig + (size_t)(q0 * nb + i) * nb;
            const size_t plane = (size_t)nptk * nb;
            for (int e = threadIdx.x; e < nq; e += blockDim.x) {
                const SEntry en = q[e];
                const int j = en.jkl & 0xff, k = (en.jkl >> 8) & 0xff, l = en.jkl >> 16;
                const double w1 = S.wv[en.ii * nb + j].w, w2 = S.wv[en.jj * nb + k].w, w3 = S.wv[en.ss * nb + l].w;
                double v2 = 0.0;
                if (!S.onlyharmonic) {
                    int m0c, m1c, m2c, a, b, cc, t0, t1, t2;
                    q_coords_t(S, en.ii, m0c, m1c, m2c);
                    q_coords_t(S, en.jj, a, b, cc);
                    q_coords_t(S, en.ss, t0, t1, t2);
                    if (MIXED) {
                        const float2* eif = S.eigf + (size_t)(q0 * nb + i) * nb;
                        const float2 V = vp4_direct_f(S, p.F, ch, eif, S.eigf + (size_t)(en.ii * nb + j) * nb,
                                                      S.eigf + (size_t)(en.jj * nb + k) * nb,
                                                      S.eigf + (size_t)(en.ss * nb + l) * nb, m0c, m1c, m2c, a, b,
                                                      cc, t0, t1, t2);
                        v2 = (double)V.x * (double)V.x + (double)V.y * (double)V.y;
                    } else {
                        const double2 V = vp4_direct(S, p.F, ch, ei, S.eig + (size_t)(en.ii * nb + j) * nb,
                                                     S.eig + (size_t)(en.jj * nb + k) * nb,
                                                     S.eig + (size_t)(en.ss * nb + l) * nb, m0c, m1c, m2c, a, b, cc,
                                                     t0, t1, t2);
                        v2 = V.x * V.x + V.y * V.y;
                    }
                }
                const double g = exp(-(en.delta * en.delta) / (en.sigma * en.sigma));
                const bool low = (w1 <= 1.25 || w2 <= 1.25 || w3 <= 1.25);
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    if (t < p.nT) {
                        const double* bz = p.bose + t * plane;
                        const double f1 = bz[en.ii * nb + j], f2 = bz[en.jj * nb + k], f3 = bz[en.ss * nb + l];
                        double bc;
                        if (ch == 0)
                            bc = f1 * f2 * (1 + f3) - (1 + f1) * (1 + f2) * f3;
                        else if (ch == 1)
                            bc = f1 * (1 + f2) * (1 + f3) - (1 + f1) * f2 * f3;
                        else
                            bc = (1 + f1) * (1 + f2) * (1 + f3) - f1 * f2 * f3;
                        const double wp4 = low ? 0.0 : bc * g / en.sigma / sqrtpi / (omega * w1 * w2 * w3);
                        acc[t] = fma(wp4, v2, acc[t]);
                        acc[NT + t] += wp4;
                    }
                }
            }
        } else {
            acc[0] = accP.val();
        }
        double v[2 * NT + 2];
#pragma unroll
        for (int x = 0; x < 2 * NT; x++) v[x] = acc[x];
        v[2 * NT] = (double)my_n;
        v[2 * NT + 1] = 0.0;
        block_sum_vec<2 * NT + 2>(v, red);
        if (threadIdx.x == 0) {
            for (int x = 0; x < 2 * p.nT; x++) {
                const int src = (x < p.nT) ? x : NT + (x - p.nT);
                p.part[(size_t)item * 2 * p.nT + x] = v[src];
            }
            p.part_n[item] = (unsigned long long)v[2 * NT];
            atomicAdd(&p.stats[0], (unsigned long long)v[2 * NT]);
            if (p.mode == 2 && !S.onlyharmonic) atomicAdd(&p.stats[1], (unsigned long long)v[2 * NT]);
        }
        __syncthreads();
    }
}

// Fixed-order compensated sums over the chunks of each (mode, channel), with the
// sampled drivers' scaling; outputs [t][ch][mode] for rates and WP4, [ch][mode] for
// the counts and P4.
__global__ void k4_sample_reduce(PSParams p, double rate_scale, double* rate, double* wp, long long* n_out,
                                 double* p_out) {
    const DevSys& S = p.S;
    const int nm = S.nb * S.nlist;
    const double nptk = (double)S.nptk;
    const double total = (double)S.nb * S.nptk * S.nb * S.nptk * S.nb;
    const double ns = (double)p.nsamples;
    const int nt = (p.mode == 2) ? p.nT : 1;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < 3 * nm * nt; x += gridDim.x * blockDim.x) {
        const int t = x / (3 * nm), rest = x - t * 3 * nm, ch = rest / nm, m0 = rest - ch * nm;
        Comp a = {0.0, 0.0}, b = {0.0, 0.0};
        unsigned long long n = 0;
        for (int c = 0; c < p.nchunk; c++) {
            const size_t item = ((size_t)m0 * 3 + ch) * p.nchunk + c;
            if (p.mode == 2) {
                a.add(p.part[item * 2 * p.nT + t]);
                b.add(p.part[item * 2 * p.nT + p.nT + t]);
            } else {
                a.add(p.part[item * 2 * p.nT]);
            }
            n += p.part_n[item];
        }
        const size_t o = (size_t)ch * nm + m0;
        if (p.mode == 2) {
            const double g = a.val() * rate_scale / nptk / nptk;
            rate[(size_t)t * 3 * nm + o] = g / ns * total;
            wp[(size_t)t * 3 * nm + o] = (b.val() / nptk / nptk) * total / ns;
        } else {
            n_out[o] = (long long)((double)n / ns * total);
            p_out[o] = a.val() * total / ns;
        }
    }
}


// ---------------------------------------------------------------------------
// Sampled three-phonon estimators: NP_plus/minus_sample (processes.f90:828-979)
// and RTA_plus/minus_sample (1474-1672).  One CTA per (mode, channel); its
// threads take the mode's `nsamples` draws in turn.  A draw is one integer of
// [0, nb*nptk*nb) decoded as the reference decodes rand_num: q' = r/(nb*nb),
// branch j = (r/nb) % nb, branch k = r % nb; q'' follows from the channel.  The
// 2-sigma test and the weights are the full drivers'; the sums are scaled by
// nb*nptk*nb/nsamples in the reference's operation order.  The draws come from
// the counter-based stream of the four-phonon estimators under keys of their
// own, so the CPU oracle draws exactly the same samples.
// ---------------------------------------------------------------------------
struct P3SParams {
    DevSys S;
    DevIfc F;
    const double* bose;  // [q*nb+b] at T (rates)
    long long nsamples;
    unsigned long long seed;
    double scale;  // hbarp*pi/4
    double unit;   // 5.60626442 (REAL) * 1e8
    int32_t* n_out[2];
    double* p_out[2];
    double* rate[2];
    double* wp[2];
    unsigned long long* stats;
};

template <int MODE>  // 0: counts and P3, 2: rates and WP3
__global__ void __launch_bounds__(256) k3_sample(P3SParams p) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red[32];
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
    const bool gate = omega <= S.omega_max;
    const bool need_v = (MODE == 2) && !S.onlyharmonic;
    double2* Z = reinterpret_cast<double2*>(smem_raw);  // npi*9 (rates)
    if (!(gate && omega != 0.0)) {
        if (threadIdx.x == 0) {
            if (MODE == 0) {
                p.n_out[w][mm] = 0;
                p.p_out[w][mm] = 0.0;
            } else {
                p.rate[w][mm] = 0.0;
                p.wp[w][mm] = 0.0;
            }
        }
        return;
    }
    if (need_v) {  // Z_p[s][r] = sum_{c in p} mu_c exp(-2 pi i n.m_k/N) sum_t Phi_c[t][s][r] e_i[t]
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
    const int total3 = nb * nptk * nb;
    const double sqrtpi = sqrt(3.141592653589793238);
    const unsigned long long key = (unsigned long long)((1u << 30) + (unsigned)(mm * 2 + w)) << 32;
    unsigned long long my_n = 0;
    Comp accP = {0.0, 0.0}, accR = {0.0, 0.0}, accW = {0.0, 0.0};
    for (long long it = threadIdx.x; it < p.nsamples; it += blockDim.x) {
        const unsigned long long base = mix64(p.seed ^ mix64(key | (unsigned long long)it));
        const int r = draw_k(base, 0, total3);
        const int k = r % nb, nn = r / nb, j = nn % nb, ii = nn / nb;
        int a, b, c;
        q_coords_t(S, ii, a, b, c);
        const int ss = q_index(S, wrapN(n0 + sign * a, N0), wrapN(n1 + sign * b, N1), wrapN(n2 + sign * c, N2));
        const double4 wp = S.wv[ii * nb + j];
        const double4 wd = S.wv[ss * nb + k];
        if (!(wp.w != 0.0 && wd.w != 0.0)) continue;
        const double sigma = sigma_exact(S, wp, wd);
        const double delta = (sign > 0) ? __dadd_rn(__dadd_rn(omega, wp.w), -wd.w)
                                        : __dadd_rn(__dadd_rn(omega, -wp.w), -wd.w);
        if (!(fabs(delta) <= 2.0 * sigma)) continue;
        my_n++;
        const double g = exp(-(delta * delta) / (sigma * sigma));
        if (MODE == 0) {
            accP.add(g / (sigma * sqrtpi * (double)((long long)nptk * nptk) * (double)(nb * nb * nb)));
            continue;
        }
        const double fp = p.bose[ii * nb + j], fd = p.bose[ss * nb + k];
        const double bose = (sign > 0) ? (fp - fd) : (fp + fd + 1.0);
        const double wp3 = bose * g / sigma / sqrtpi / (omega * wp.w * wd.w);
        accW.add(wp3);
        if (!need_v) continue;
        double2 V = make_double2(0.0, 0.0);
        const double2* e1 = S.eig + (size_t)(ii * nb + j) * nb;
        const double2* e2 = S.eig + (size_t)(ss * nb + k) * nb;
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
                    for (int q = 0; q < 3; q++) h = cmac(h, z[s * 3 + q], v[q]);
                    t = cmac(t, u[s], h);
                }
                V = cmac(V, ph, t);
            }
        }
        accR.add(p.scale * wp3 * (V.x * V.x + V.y * V.y));
    }
    const double n = block_sum((double)my_n, red);
    const double ns = (double)p.nsamples;
    if (MODE == 0) {
        const double P = block_sum(accP.val(), red);
        if (threadIdx.x == 0) {
            p.n_out[w][mm] = (int32_t)(n / ns * nb * nptk * nb);
            p.p_out[w][mm] = P * nb * nptk * nb / ns;
        }
    } else {
        double W = block_sum(accW.val(), red);
        double R = block_sum(accR.val(), red);
        if (threadIdx.x == 0) {
            W = (sign > 0) ? W / nptk : W * 5.e-1 / nptk;
            p.wp[w][mm] = W * nb * nptk * nb / ns;
            R = R * nb * nptk * nb / ns;
            R = R * p.unit / (double)nptk;
            p.rate[w][mm] = (sign > 0) ? R : R * 5.e-1;
            atomicAdd(&p.stats[0], (unsigned long long)n);
            if (need_v) atomicAdd(&p.stats[1], (unsigned long long)n);
        }
    }
}

}  // namespace

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return fp4_fail(c, FP4_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

int fp4_setup_ifc(fp4_ctx* c, const fp4_globals* g, int order, int32_t ntri, const double* phi, const double* rj,
                  const double* rk, const double* rl, const int32_t* ii, const int32_t* ij, const int32_t* ik,
                  const int32_t* il, IfcTables& T);

// Sampled estimators on the context's current system; results device-resident in
// c->b_out4: mode 2: rate[t][ch][mode] then wp[t][ch][mode]; mode 0: n (int64) then P.
static int run_sample(fp4_ctx* c, int mode, int nT, const double* temps, int64_t nsamples, uint64_t seed) {
    if (nsamples < 1) return fp4_fail(c, FP4_E_ARG, "nsamples must be >=1");
    if (nsamples >= ((int64_t)1 << 32)) return fp4_fail(c, FP4_E_ARG, "nsamples must be < 2^32");
    if (mode == 2 && (nT < 1 || nT > kMaxTemps)) return fp4_fail(c, FP4_E_ARG, "nT=%d outside [1,%d]", nT, kMaxTemps);
    const DevSys& S = c->S;
    const int nm = S.nb * S.nlist;
    const int64_t nchunk = (nsamples + kSChunk - 1) / kSChunk;
    const int64_t nitems = (int64_t)nm * 3 * nchunk;
    if (nitems > ((int64_t)1 << 30)) return fp4_fail(c, FP4_E_CAPACITY, "too many sample chunks (%lld)", (long long)nitems);
    const int nt = (mode == 2) ? nT : 1;
    int r;
    if (mode == 2) {
        if ((r = c->b_temps.upload(c, temps, nT * sizeof(double)))) return r;
        if ((r = c->b_bose.reserve(c, (size_t)S.nptk * S.nb * nT * sizeof(double)))) return r;
        CK(launch_bose(S, c->b_temps.as<double>(), nT, c->b_bose.as<double>(), c->stream));
        c->launches++;
    }
    if ((r = c->b_part.reserve(c, (size_t)nitems * (2 * nt * sizeof(double) + sizeof(unsigned long long)))) ||
        (r = c->b_work.reserve(c, 64)) || (r = c->b_out4.reserve(c, (size_t)3 * nm * nt * 2 * sizeof(double))))
        return r;
    CK(cudaMemsetAsync(c->b_work.ptr, 0, 64, c->stream));
    PSParams p{};
    p.S = S;
    p.F = c->ifc4.F;
    p.nT = nt;
    p.bose = mode == 2 ? c->b_bose.as<double>() : nullptr;
    p.nsamples = nsamples;
    p.seed = seed;
    p.nchunk = (int)nchunk;
    p.mode = mode;
    p.nitems = (int)nitems;
    p.work_counter = c->b_work.as<int>();
    p.part = c->b_part.as<double>();
    p.part_n = reinterpret_cast<unsigned long long*>(p.part + (size_t)nitems * 2 * nt);
    p.stats = c->b_stats.as<unsigned long long>();
    p.err = c->b_err.as<int>();
    const int nblocks = (int)std::min<int64_t>(nitems, (int64_t)c->sm_count * 8);
    CK(cudaEventRecord(c->evk0, c->stream));
    // mixed precision: the V(4) sums in FP32 (the draws, filter, weights and sums stay FP64)
    const bool mixed = mode == 2 && c->precision != FP4_PREC_FP64;
#define FP4_KS(NTV)                                                   \
    if (mixed)                                                        \
        k4_sample<NTV, true><<<nblocks, kSThreads, 0, c->stream>>>(p); \
    else                                                              \
        k4_sample<NTV, false><<<nblocks, kSThreads, 0, c->stream>>>(p);
    if (mode == 2 && nt > 4) {
        FP4_KS(8)
    } else if (mode == 2 && nt > 2) {
        FP4_KS(4)
    } else if (mode == 2 && nt > 1) {
        FP4_KS(2)
    } else {
        FP4_KS(1)
    }
#undef FP4_KS
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_timed = true;
    c->launches++;
    const double hbarp = 1.05457172647e-22 * (double)1e22f;
    const double rate_scale = hbarp * hbarp * 3.141592653589793238 / 8.0 * (double)3.37617087f * 1.e9;
    double* o = c->b_out4.as<double>();
    const int total = 3 * nm * nt;
    k4_sample_reduce<<<(total + 127) / 128, 128, 0, c->stream>>>(p, rate_scale, o, o + (size_t)3 * nm * nt,
                                                                reinterpret_cast<long long*>(o), o + 3 * nm);
    CK(cudaGetLastError());
    c->launches++;
    return FP4_OK;
}

extern "C" int fp4_np_driver_4ph_sample(fp4_ctx* c, const fp4_globals* g, const double* energy,
                                        const double* velocity, int32_t nlist, const int32_t* list,
                                        const int32_t* ijk, int64_t nsamples, uint64_t seed, int64_t* n_pp,
                                        double* p_pp, int64_t* n_pm, double* p_pm, int64_t* n_mm, double* p_mm) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!n_pp || !n_pm || !n_mm || !p_pp || !p_pm || !p_mm) return fp4_fail(c, FP4_E_ARG, "null output");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, nullptr, nlist, list, ijk))) return r;
    if ((r = run_sample(c, 0, 1, nullptr, nsamples, seed))) return r;
    const int nm = c->S.nb * nlist;
    std::vector<long long> hn((size_t)3 * nm);
    std::vector<double> hp((size_t)3 * nm);
    double* o = c->b_out4.as<double>();
    CK(cudaMemcpyAsync(hn.data(), o, hn.size() * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(hp.data(), o + 3 * nm, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((r = fp4_end(c))) return r;
    int64_t* N[3] = {n_pp, n_pm, n_mm};
    double* P[3] = {p_pp, p_pm, p_mm};
    for (int ch = 0; ch < 3; ch++)
        for (int m = 0; m < nm; m++) {
            N[ch][m] = hn[(size_t)ch * nm + m];
            P[ch][m] = hp[(size_t)ch * nm + m];
        }
    return FP4_OK;
}

extern "C" int fp4_rta_driver_4ph_sample_multi_t(fp4_ctx* c, const fp4_globals* g, int32_t nT,
                                                 const double* temperatures, const double* energy,
                                                 const double* velocity, const double* eigenvect, int32_t nlist,
                                                 const int32_t* list, const int32_t* ijk, int32_t ntri,
                                                 const double* psi, const double* r_j, const double* r_k,
                                                 const double* r_l, const int32_t* index_i, const int32_t* index_j,
                                                 const int32_t* index_k, const int32_t* index_l, int64_t nsamples,
                                                 uint64_t seed, double* rate_pp, double* rate_pm, double* rate_mm,
                                                 double* wp_pp, double* wp_pm, double* wp_mm) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!temperatures || !rate_pp || !rate_pm || !rate_mm || !wp_pp || !wp_pm || !wp_mm || !eigenvect)
        return fp4_fail(c, FP4_E_ARG, "null argument");
    for (int t = 0; t < nT; t++)
        if (!(temperatures[t] > 0.0)) return fp4_fail(c, FP4_E_ARG, "T must be >0 K");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, eigenvect, nlist, list, ijk))) return r;
    if ((r = fp4_setup_ifc(c, g, 4, ntri, psi, r_j, r_k, r_l, index_i, index_j, index_k, index_l, c->ifc4))) return r;
    if ((r = run_sample(c, 2, nT, temperatures, nsamples, seed))) return r;
    const int nm = c->S.nb * nlist;
    std::vector<double> h((size_t)3 * nm * nT * 2);
    CK(cudaMemcpyAsync(h.data(), c->b_out4.ptr, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((r = fp4_end(c))) return r;
    double* R[3] = {rate_pp, rate_pm, rate_mm};
    double* W[3] = {wp_pp, wp_pm, wp_mm};
    for (int t = 0; t < nT; t++)
        for (int ch = 0; ch < 3; ch++)
            for (int m = 0; m < nm; m++) {
                R[ch][(size_t)t * nm + m] = h[((size_t)t * 3 + ch) * nm + m];
                W[ch][(size_t)t * nm + m] = h[(size_t)3 * nm * nT + ((size_t)t * 3 + ch) * nm + m];
            }
    return FP4_OK;
}

extern "C" int fp4_rta_driver_4ph_sample(fp4_ctx* c, const fp4_globals* g, const double* energy,
                                         const double* velocity, const double* eigenvect, int32_t nlist,
                                         const int32_t* list, const int32_t* ijk, int32_t ntri, const double* psi,
                                         const double* r_j, const double* r_k, const double* r_l,
                                         const int32_t* index_i, const int32_t* index_j, const int32_t* index_k,
                                         const int32_t* index_l, int64_t nsamples, uint64_t seed, double* rate_4ph,
                                         double* rate_pp, double* rate_pm, double* rate_mm, double* wp_pp,
                                         double* wp_pm, double* wp_mm) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!g || !rate_4ph) return fp4_fail(c, FP4_E_ARG, "null argument");
    int r = fp4_rta_driver_4ph_sample_multi_t(c, g, 1, &g->T, energy, velocity, eigenvect, nlist, list, ijk, ntri, psi,
                                              r_j, r_k, r_l, index_i, index_j, index_k, index_l, nsamples, seed,
                                              rate_pp, rate_pm, rate_mm, wp_pp, wp_pm, wp_mm);
    if (r) return r;
    const int nm = g->nbands * nlist;
    for (int m = 0; m < nm; m++) rate_4ph[m] = rate_pp[m] + rate_pm[m] + rate_mm[m];
    return FP4_OK;
}

// Sampled three-phonon estimators on the context's current system.
static int run_sample3(fp4_ctx* c, int mode, const fp4_globals* g, int64_t nsamples, uint64_t seed, P3SParams& p) {
    if (nsamples < 1) return fp4_fail(c, FP4_E_ARG, "nsamples must be >=1");
    if (nsamples >= ((int64_t)1 << 32)) return fp4_fail(c, FP4_E_ARG, "nsamples must be < 2^32");
    const DevSys& S = c->S;
    if ((int64_t)S.nb * S.nptk * S.nb >= ((int64_t)1 << 31))
        return fp4_fail(c, FP4_E_CAPACITY, "nbands*nptk*nbands must be < 2^31");
    p.S = S;
    p.F = c->ifc3.F;
    p.nsamples = nsamples;
    p.seed = seed;
    p.scale = 1.05457172647e-22 * (double)1e22f * 3.141592653589793238 / 4.0;
    p.unit = (double)5.60626442f * 1.e8;
    p.stats = c->b_stats.as<unsigned long long>();
    size_t sm = 0;
    if (mode == 2) {
        int r;
        if ((r = c->b_temps.upload(c, &g->T, sizeof(double)))) return r;
        if ((r = c->b_bose.reserve(c, (size_t)S.nptk * S.nb * sizeof(double)))) return r;
        CK(launch_bose(S, c->b_temps.as<double>(), 1, c->b_bose.as<double>(), c->stream));
        c->launches++;
        p.bose = c->b_bose.as<double>();
        if (!S.onlyharmonic) sm = (size_t)p.F.npi * 9 * sizeof(double2);
        if (sm > 227 * 1024) return fp4_fail(c, FP4_E_CAPACITY, "3ph cluster table needs %zu B of shared memory", sm);
    }
    const dim3 grid(S.nb * S.nlist, 2);
    CK(cudaEventRecord(c->evk0, c->stream));
    if (mode == 2) {
        CK(cudaFuncSetAttribute(k3_sample<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k3_sample<2><<<grid, 256, sm, c->stream>>>(p);
    } else {
        k3_sample<0><<<grid, 256, 0, c->stream>>>(p);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_timed = true;
    c->launches++;
    return FP4_OK;
}

extern "C" int fp4_np_driver_sample(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                                    int32_t nlist, const int32_t* list, const int32_t* ijk, int64_t nsamples,
                                    uint64_t seed, int32_t* n_plus, double* p_plus, int32_t* n_minus,
                                    double* p_minus) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!n_plus || !p_plus || !n_minus || !p_minus) return fp4_fail(c, FP4_E_ARG, "null output");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, nullptr, nlist, list, ijk))) return r;
    const int nm = c->S.nb * nlist;
    if ((r = c->b_out.reserve(c, (size_t)nm * 4 * sizeof(double)))) return r;
    double* d = c->b_out.as<double>();
    P3SParams p{};
    p.p_out[0] = d;
    p.p_out[1] = d + nm;
    p.n_out[0] = reinterpret_cast<int32_t*>(d + 2 * nm);
    p.n_out[1] = p.n_out[0] + nm;
    if ((r = run_sample3(c, 0, g, nsamples, seed, p))) return r;
    std::vector<double> hp((size_t)2 * nm);
    std::vector<int32_t> hn((size_t)2 * nm);
    CK(cudaMemcpyAsync(hp.data(), d, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(hn.data(), p.n_out[0], hn.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    if ((r = fp4_end(c))) return r;
    for (int m = 0; m < nm; m++) {
        p_plus[m] = hp[m];
        p_minus[m] = hp[nm + m];
        n_plus[m] = hn[m];
        n_minus[m] = hn[nm + m];
    }
    return FP4_OK;
}

extern "C" int fp4_rta_driver_sample(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                                     const double* eigenvect, int32_t nlist, const int32_t* list, const int32_t* ijk,
                                     int32_t ntri, const double* phi, const double* r_j, const double* r_k,
                                     const int32_t* index_i, const int32_t* index_j, const int32_t* index_k,
                                     int64_t nsamples, uint64_t seed, double* rate, double* rate_plus,
                                     double* rate_minus, double* wp3_plus, double* wp3_minus) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!rate || !rate_plus || !rate_minus || !wp3_plus || !wp3_minus) return fp4_fail(c, FP4_E_ARG, "null output");
    if (!eigenvect) return fp4_fail(c, FP4_E_ARG, "null eigenvect");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, eigenvect, nlist, list, ijk))) return r;
    if ((r = fp4_setup_ifc(c, g, 3, ntri, phi, r_j, r_k, nullptr, index_i, index_j, index_k, nullptr, c->ifc3))) return r;
    const int nm = c->S.nb * nlist;
    if ((r = c->b_out.reserve(c, (size_t)nm * 4 * sizeof(double)))) return r;
    double* d = c->b_out.as<double>();
    P3SParams p{};
    p.rate[0] = d;
    p.rate[1] = d + nm;
    p.wp[0] = d + 2 * nm;
    p.wp[1] = d + 3 * nm;
    if ((r = run_sample3(c, 2, g, nsamples, seed, p))) return r;
    std::vector<double> h((size_t)nm * 4);
    CK(cudaMemcpyAsync(h.data(), d, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((r = fp4_end(c))) return r;
    for (int m = 0; m < nm; m++) {
        rate_plus[m] = h[m];
        rate_minus[m] = h[nm + m];
        wp3_plus[m] = h[2 * nm + m];
        wp3_minus[m] = h[3 * nm + m];
        rate[m] = rate_plus[m] + rate_minus[m];
    }
    return FP4_OK;
}
