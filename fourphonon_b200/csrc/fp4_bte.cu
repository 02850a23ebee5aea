// Linearised-BTE sweep and thermal conductivity on the device.
//
// iteration (Src/iterations.f90:34-92) and iteration_4ph (95-215, the same
// sweep with the ++, +- and -- lists added) are in-place Gauss-Seidel sweeps:
// modes are visited in the order (ll, i, kk) and each update reads F_n values
// already overwritten earlier in the same sweep.  The device sweep keeps that
// order exactly: one CTA walks the (ll, i, kk) steps in sequence and spreads
// each step's sum over the mode's processes across its threads (a tree
// reduction, so only the summation order inside one step differs from the
// reference's left-to-right loop).  F_n stays in the Fortran layout
// F_n(nbands,nptk,3).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/fourphonon_b200.h"
#include "fp4_ctx.h"
#include "fp4_internal.h"

using namespace fp4;

namespace {

struct BteParams {
    int nb, nptk, nlist, nsr;
    const int* nequi;
    const int* allequi;   // ALLEquiList(nsr, *) column-major
    const int* typeofsym; // TypeofSymmetry(nsr, *)
    const int* id_equi;   // ID_equi(nsr, nptk)
    const double* symm;   // symmetrizers(3,3,nptk)
    const int* n_plus;
    const int* n_minus;
    const long long* off_plus;
    const long long* off_minus;
    const int* i2p;
    const int* i3p;
    const int* i2m;
    const int* i3m;
    const double* gp;
    const double* gm;
    const double* energy;    // energy(nptk,nb)
    const double* velocity;  // velocity(nptk,nb,3)
    const double* tau_zero;  // tau_zero(nb,nlist)
    double* F;               // F_n(nb,nptk,3)
    // four-phonon lists of iteration_4ph (n4[0] == nullptr: three-phonon sweep)
    const long long* n4[3];
    const long long* off4[3];
    const long long* i2_4[3];
    const long long* i3_4[3];
    const long long* i4_4[3];
    const double* g4[3];
    int* err;
};

__device__ __forceinline__ double& Fat(const BteParams& p, int b, int q, int d) {
    return p.F[((size_t)d * p.nptk + q) * p.nb + b];
}

// This thread's share (x = t0, t0 + dt, ...) of one step's sum over the mode's
// processes, with the q-points mapped by symmetry operation `sym`, reading F.
__device__ __forceinline__ void step_sum(const BteParams& p, const double* F, int mm, int sym, long long t0,
                                         long long dt, double& a0, double& a1, double& a2) {
    const int nb = p.nb;
    auto Fv = [&](int b, int q, int d) { return F[((size_t)d * p.nptk + q) * nb + b]; };
    const int np_ = p.n_plus[mm], nm_ = p.n_minus[mm];
    const long long op = p.off_plus[mm], om = p.off_minus[mm];
    long long c4[3] = {0, 0, 0};
    if (p.n4[0])
        for (int ch = 0; ch < 3; ch++) c4[ch] = p.n4[ch][mm];
    const long long n3ph = (long long)np_ + nm_, ntot = n3ph + c4[0] + c4[1] + c4[2];
    const long long lim = (long long)p.nptk * nb;
    for (long long x = t0; x < ntot; x += dt) {
        if (x >= n3ph) {
            // iteration_4ph: ++ Gamma(F_l - F_j - F_k), +- Gamma(F_l - F_j + F_k),
            // -- Gamma(F_l + F_j + F_k), q-points mapped by the same symmetry
            long long y = x - n3ph;
            int ch = 0;
            while (ch < 2 && y >= c4[ch]) {
                y -= c4[ch];
                ch++;
            }
            const long long o = p.off4[ch][mm] + y;
            const long long y2 = p.i2_4[ch][o] - 1, y3 = p.i3_4[ch][o] - 1, y4 = p.i4_4[ch][o] - 1;
            if (y2 < 0 || y2 >= lim || y3 < 0 || y3 >= lim || y4 < 0 || y4 >= lim) {
                atomicOr(p.err, kErrList);
                continue;
            }
            const int j = (int)(y2 % nb), k = (int)(y3 % nb), l = (int)(y4 % nb);
            const int qj = p.id_equi[(y2 / nb) * p.nsr + sym] - 1;
            const int qk = p.id_equi[(y3 / nb) * p.nsr + sym] - 1;
            const int ql = p.id_equi[(y4 / nb) * p.nsr + sym] - 1;
            const double g = p.g4[ch][o];
            const double sj = (ch == 2) ? 1.0 : -1.0, sk = (ch == 0) ? -1.0 : 1.0;
            // F_l -+ F_j -+ F_k with the reference's left-to-right order
            a0 += g * ((Fv(l, ql, 0) + sj * Fv(j, qj, 0)) + sk * Fv(k, qk, 0));
            a1 += g * ((Fv(l, ql, 1) + sj * Fv(j, qj, 1)) + sk * Fv(k, qk, 1));
            a2 += g * ((Fv(l, ql, 2) + sj * Fv(j, qj, 2)) + sk * Fv(k, qk, 2));
            continue;
        }
        const bool plus = x < np_;
        const long long o = plus ? op + x : om + (x - np_);
        const int x2 = (plus ? p.i2p : p.i2m)[o] - 1, x3 = (plus ? p.i3p : p.i3m)[o] - 1;
        if (x2 < 0 || x2 >= lim || x3 < 0 || x3 >= lim) {
            atomicOr(p.err, kErrList);
            continue;
        }
        const int j = x2 % nb, m2 = x2 / nb, k = x3 % nb, n3 = x3 / nb;
        const int qa = p.id_equi[(size_t)n3 * p.nsr + sym] - 1;
        const int qb = p.id_equi[(size_t)m2 * p.nsr + sym] - 1;
        const double g = (plus ? p.gp : p.gm)[o];
        double t0_, t1_, t2_;
        if (plus) {
            t0_ = g * (Fv(k, qa, 0) - Fv(j, qb, 0));
            t1_ = g * (Fv(k, qa, 1) - Fv(j, qb, 1));
            t2_ = g * (Fv(k, qa, 2) - Fv(j, qb, 2));
        } else {
            t0_ = g * (Fv(k, qa, 0) + Fv(j, qb, 0)) * 5.e-1;
            t1_ = g * (Fv(k, qa, 1) + Fv(j, qb, 1)) * 5.e-1;
            t2_ = g * (Fv(k, qa, 2) + Fv(j, qb, 2)) * 5.e-1;
        }
        a0 += t0_;
        a1 += t1_;
        a2 += t2_;
    }
}

// Block sum of (a0, a1, a2) into thread 0 (red: 3 x 32 doubles of shared memory).
__device__ __forceinline__ void block_sum3(double& a0, double& a1, double& a2, double (*red)[32]) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_down_sync(0xffffffffu, a0, o);
        a1 += __shfl_down_sync(0xffffffffu, a1, o);
        a2 += __shfl_down_sync(0xffffffffu, a2, o);
    }
    if (lane == 0) {
        red[0][warp] = a0;
        red[1][warp] = a1;
        red[2][warp] = a2;
    }
    __syncthreads();
    if (warp == 0) {
        a0 = lane < nwarp ? red[0][lane] : 0.0;
        a1 = lane < nwarp ? red[1][lane] : 0.0;
        a2 = lane < nwarp ? red[2][lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_down_sync(0xffffffffu, a0, o);
            a1 += __shfl_down_sync(0xffffffffu, a1, o);
            a2 += __shfl_down_sync(0xffffffffu, a2, o);
        }
    }
}

// iteration / iteration_4ph (iterations.f90:34-215): one Gauss-Seidel sweep in the
// reference's order (ll, i, kk), updating F in place; one CTA.
__global__ void __launch_bounds__(1024) k_sweep(BteParams p) {
    __shared__ double red[3][32];
    const int nb = p.nb;
    for (int ll = 0; ll < p.nlist; ll++) {
        for (int i = 0; i < nb; i++) {
            const int mm = ll * nb + i;
            for (int kk = 0; kk < p.nequi[ll]; kk++) {
                const int qq = p.allequi[ll * p.nsr + kk] - 1;
                const int sym = p.typeofsym[ll * p.nsr + kk] - 1;
                double a0 = 0.0, a1 = 0.0, a2 = 0.0;
                step_sum(p, p.F, mm, sym, threadIdx.x, blockDim.x, a0, a1, a2);
                block_sum3(a0, a1, a2, red);
                if (threadIdx.x == 0) {
                    const double tz = p.tau_zero[ll * nb + i];
                    const size_t e = (size_t)i * p.nptk + qq, pl = (size_t)p.nptk * nb;
                    const double w = p.energy[e];
                    Fat(p, i, qq, 0) = tz * p.velocity[e] * w + tz * a0;
                    Fat(p, i, qq, 1) = tz * p.velocity[e + pl] * w + tz * a1;
                    Fat(p, i, qq, 2) = tz * p.velocity[e + 2 * pl] * w + tz * a2;
                }
                __syncthreads();
                // F_n(:,qq,:) = transpose(matmul(symmetrizers(:,:,qq), transpose(F_n(:,qq,:))))
                if (threadIdx.x < nb) {
                    const int b = threadIdx.x;
                    const double* Sq = p.symm + 9 * (size_t)qq;
                    double x0 = Fat(p, b, qq, 0), x1 = Fat(p, b, qq, 1), x2 = Fat(p, b, qq, 2);
                    double y[3];
#pragma unroll
                    for (int a = 0; a < 3; a++) y[a] = Sq[a] * x0 + Sq[a + 3] * x1 + Sq[a + 6] * x2;
                    Fat(p, b, qq, 0) = y[0];
                    Fat(p, b, qq, 1) = y[1];
                    Fat(p, b, qq, 2) = y[2];
                }
                __syncthreads();
            }
        }
    }
}

// The Jacobi form of the same update (no counterpart in the reference, whose
// sweep is Gauss-Seidel): every step reads the previous iterate F and writes
// Fout, so all steps run at once, one CTA per (mode, equivalent point).  The
// site symmetrizer is applied afterwards (k_symmetrize) to every point, which is
// what the in-place sweep's per-step projection does to the band it has just
// updated.  Converges to the same fixed point, in more sweeps.
__global__ void __launch_bounds__(256) k_jacobi_step(BteParams p, double* Fout) {
    __shared__ double red[3][32];
    const int nb = p.nb;
    const int mm = blockIdx.x, kk = blockIdx.y;
    const int ll = mm / nb, i = mm - ll * nb;
    if (kk >= p.nequi[ll]) return;
    const int qq = p.allequi[ll * p.nsr + kk] - 1;
    const int sym = p.typeofsym[ll * p.nsr + kk] - 1;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    step_sum(p, p.F, mm, sym, threadIdx.x, blockDim.x, a0, a1, a2);
    block_sum3(a0, a1, a2, red);
    if (threadIdx.x == 0) {
        const double tz = p.tau_zero[ll * nb + i];
        const size_t e = (size_t)i * p.nptk + qq, pl = (size_t)p.nptk * nb;
        const double w = p.energy[e];
        Fout[((size_t)0 * p.nptk + qq) * nb + i] = tz * p.velocity[e] * w + tz * a0;
        Fout[((size_t)1 * p.nptk + qq) * nb + i] = tz * p.velocity[e + pl] * w + tz * a1;
        Fout[((size_t)2 * p.nptk + qq) * nb + i] = tz * p.velocity[e + 2 * pl] * w + tz * a2;
    }
}

__global__ void k_iteration0(int nb, int nptk, int nlist, int nsr, const int* nequi, const int* allequi,
                             const double* energy, const double* velocity, const double* tau_zero, double* F) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nlist * nb * nsr; x += gridDim.x * blockDim.x) {
        int kk = x % nsr, rest = x / nsr, i = rest % nb, ll = rest / nb;
        if (kk >= nequi[ll]) continue;
        int qq = allequi[ll * nsr + kk] - 1;
        size_t e = (size_t)i * nptk + qq, pl = (size_t)nptk * nb;
        double tz = tau_zero[ll * nb + i], w = energy[e];
        for (int d = 0; d < 3; d++) F[((size_t)d * nptk + qq) * nb + i] = tz * velocity[e + d * pl] * w;
    }
}

__global__ void k_symmetrize(int nb, int nptk, const double* symm, double* F) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nb * nptk; x += gridDim.x * blockDim.x) {
        int b = x % nb, q = x / nb;
        const double* Sq = symm + 9 * (size_t)q;
        double v[3];
        for (int d = 0; d < 3; d++) v[d] = F[((size_t)d * nptk + q) * nb + b];
        for (int a = 0; a < 3; a++) F[((size_t)a * nptk + q) * nb + b] = Sq[a] * v[0] + Sq[a + 3] * v[1] + Sq[a + 6] * v[2];
    }
}

// TConduct (conductivity.f90:11-37): one CTA per branch, q >= 2, fixed-order tree sum.
__global__ void k_tconduct(int nb, int nptk, double T, double scale, const double* energy, const double* velocity,
                           const double* F, double* kappa, double* kmode) {
    __shared__ double red[9][32];
    const int jj = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const double hbar = 1.05457172647e-22, kb = 1.380648813e-23;
    double acc[9];
    for (int x = 0; x < 9; x++) acc[x] = 0.0;
    const size_t pl = (size_t)nptk * nb;
    for (int ii = 1 + threadIdx.x; ii < nptk; ii += blockDim.x) {
        size_t e = (size_t)jj * nptk + ii;
        double w = energy[e];
        double f = 1.0 / (exp(hbar * w / kb / T) - 1.0);
        double c = f * (f + 1) * w;
        for (int d2 = 0; d2 < 3; d2++) {
            double Fd = F[((size_t)d2 * nptk + ii) * nb + jj];
            for (int d1 = 0; d1 < 3; d1++) {
                double m = c * (velocity[e + d1 * pl] * Fd);
                acc[d2 * 3 + d1] += m;
                if (kmode) kmode[(((size_t)(d2 * 3 + d1)) * nb + jj) * nptk + ii] = scale * m;
            }
        }
    }
    for (int x = 0; x < 9; x++) {
        double v = acc[x];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[x][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        double t = 0.0;
        for (int w = 0; w < nwarp; w++) t += red[threadIdx.x][w];
        kappa[threadIdx.x * nb + jj] = scale * t;  // ThConductivity(jj,d1,d2): [(d2*3+d1)*nb + jj]
    }
}

// Euclidean norm of a 3-vector by the scaled sum of squares of reference BLAS
// dnrm2, unfused so that it rounds as the host evaluation does.
__device__ double nrm2_3(double x0, double x1, double x2) {
    double scale = 0.0, ssq = 1.0;
    const double x[3] = {x0, x1, x2};
    for (int i = 0; i < 3; i++) {
        if (x[i] != 0.0) {
            const double a = fabs(x[i]);
            if (scale < a) {
                const double q = scale / a;
                ssq = __dadd_rn(1.0, __dmul_rn(__dmul_rn(ssq, q), q));
                scale = a;
            } else {
                const double q = a / scale;
                ssq = __dadd_rn(ssq, __dmul_rn(q, q));
            }
        }
    }
    return __dmul_rn(scale, sqrt(ssq));
}

// CumulativeTConduct / CumulativeTConductOmega (conductivity.f90:64-148): one CTA
// per (tick, branch) sums the modes whose mean free path (or omega) is below
// the tick.  results(nb,3,3,nticks) as [((k*3 + d2)*3 + d1)*nb + b].
__global__ void k_cumulative(int nb, int nptk, int nticks, int omega_mode, double T, double scale,
                             const double* energy, const double* velocity, const double* F, const double* ticks,
                             double* results) {
    __shared__ double red[9][32];
    const int k = blockIdx.x, jj = blockIdx.y;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const double hbar = 1.05457172647e-22, kb = 1.380648813e-23;
    const double tick = ticks[k];
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const size_t pl = (size_t)nptk * nb;
    for (int ii = 1 + threadIdx.x; ii < nptk; ii += blockDim.x) {  // reference q index 2..nptk
        const size_t e = (size_t)jj * nptk + ii;
        const double w = energy[e];
        const double v[3] = {velocity[e], velocity[e + pl], velocity[e + 2 * pl]};
        const double f[3] = {F[(size_t)ii * nb + jj], F[((size_t)nptk + ii) * nb + jj], F[((size_t)2 * nptk + ii) * nb + jj]};
        double lambda;
        if (omega_mode) {
            lambda = w;
        } else {
            const double dot = __dadd_rn(__dadd_rn(__dmul_rn(f[0], v[0]), __dmul_rn(f[1], v[1])), __dmul_rn(f[2], v[2]));
            lambda = dot / __dmul_rn(__dadd_rn(w, 1e-12), nrm2_3(v[0], v[1], v[2]));
        }
        if (!(tick > lambda)) continue;
        const double fbe = 1.0 / (exp(hbar * w / kb / T) - 1.0);
        const double pre = fbe * (fbe + 1) * w;
        for (int d1 = 0; d1 < 3; d1++)
            for (int d2 = 0; d2 < 3; d2++) acc[d2 * 3 + d1] += pre * (v[d1] * f[d2]);
    }
    for (int x = 0; x < 9; x++) {
        double t = acc[x];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
        if (lane == 0) red[x][warp] = t;
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        double t = 0.0;
        for (int w = 0; w < nwarp; w++) t += red[threadIdx.x][w];
        results[((size_t)k * 9 + threadIdx.x) * nb + jj] = scale * t;
    }
}

}  // namespace

namespace fp4 {
cudaError_t launch_iteration0(int nb, int nptk, int nlist, int nsr, const int* nequi, const int* allequi,
                              const double* energy, const double* velocity, const double* tau_zero, double* F,
                              cudaStream_t st) {
    k_iteration0<<<256, 256, 0, st>>>(nb, nptk, nlist, nsr, nequi, allequi, energy, velocity, tau_zero, F);
    return cudaGetLastError();
}

cudaError_t launch_tconduct(int nb, int nptk, double T, double V, const double* energy, const double* velocity,
                            const double* F, double* kappa, cudaStream_t st) {
    const double hbar = 1.05457172647e-22, kb = 1.380648813e-23;
    const double scale = (double)1e21f * (hbar * hbar) / (kb * T * T * V * nptk);
    k_tconduct<<<nb, 256, 0, st>>>(nb, nptk, T, scale, energy, velocity, F, kappa, nullptr);
    return cudaGetLastError();
}
}  // namespace fp4

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return fp4_fail(c, FP4_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

static int check_g(fp4_ctx* c, const fp4_globals* g) {
    if (!g) return fp4_fail(c, FP4_E_ARG, "null globals");
    for (int d = 0; d < 3; d++)
        if (g->ngrid[d] < 1) return fp4_fail(c, FP4_E_ARG, "ngrid must be >0");
    if (g->nbands < 3) return fp4_fail(c, FP4_E_ARG, "nbands must be >=3");
    return FP4_OK;
}

extern "C" int fp4_iteration0(fp4_ctx* c, const fp4_globals* g, int32_t nlist, const int32_t* nequi,
                              const int32_t* allequi, int32_t nsr, const double* omega, const double* velocity,
                              const double* tau_zero, double* f_n) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    int r;
    if ((r = check_g(c, g))) return r;
    if (!nequi || !allequi || !omega || !velocity || !tau_zero || !f_n || nlist < 1 || nsr < 1)
        return fp4_fail(c, FP4_E_ARG, "bad argument");
    if ((r = fp4_begin(c))) return r;
    const int nb = g->nbands, nptk = g->ngrid[0] * g->ngrid[1] * g->ngrid[2];
    DevBuffer* B = c->b_bte;
    if ((r = B[0].upload(c, nequi, nlist * sizeof(int))) || (r = B[1].upload(c, allequi, (size_t)nlist * nsr * sizeof(int))) ||
        (r = B[2].upload(c, omega, (size_t)nptk * nb * sizeof(double))) ||
        (r = B[3].upload(c, velocity, (size_t)nptk * nb * 3 * sizeof(double))) ||
        (r = B[4].upload(c, tau_zero, (size_t)nlist * nb * sizeof(double))) ||
        (r = B[5].reserve(c, (size_t)nptk * nb * 3 * sizeof(double))))
        return r;
    CK(cudaMemsetAsync(B[5].ptr, 0, (size_t)nptk * nb * 3 * sizeof(double), c->stream));
    k_iteration0<<<256, 256, 0, c->stream>>>(nb, nptk, nlist, nsr, B[0].as<int>(), B[1].as<int>(), B[2].as<double>(),
                                            B[3].as<double>(), B[4].as<double>(), B[5].as<double>());
    CK(cudaGetLastError());
    c->launches++;
    CK(cudaMemcpyAsync(f_n, B[5].ptr, (size_t)nptk * nb * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return fp4_end(c);
}

namespace {
// The four-phonon arguments of iteration_4ph (all null for the three-phonon sweep).
struct Lists4 {
    const int64_t* n[3];
    int64_t ntotal[3];
    const int64_t* i2[3];
    const int64_t* i3[3];
    const int64_t* i4[3];
    const double* g[3];
};
}  // namespace

static int run_sweep(fp4_ctx* c, const fp4_globals* g, int32_t nlist, const int32_t* nequi, const int32_t* allequi,
                     const int32_t* typeofsym, int32_t nsr, const int32_t* id_equi, const double* symmetrizers,
                     const int32_t* n_plus, const int32_t* n_minus, int32_t ntotal_plus, int32_t ntotal_minus,
                     const int32_t* i2p, const int32_t* i3p, const int32_t* i2m, const int32_t* i3m,
                     const double* omega, const double* velocity, const double* gp, const double* gm,
                     const double* tau_zero, double* f_n, const Lists4* l4, bool jacobi = false) {
    if (!c) return FP4_E_ARG;
    int r;
    if ((r = check_g(c, g))) return r;
    if (!nequi || !allequi || !typeofsym || !id_equi || !symmetrizers || !n_plus || !n_minus || !omega || !velocity ||
        !tau_zero || !f_n || nlist < 1 || nsr < 1 || ntotal_plus < 0 || ntotal_minus < 0)
        return fp4_fail(c, FP4_E_ARG, "bad argument");
    if ((ntotal_plus && (!i2p || !i3p || !gp)) || (ntotal_minus && (!i2m || !i3m || !gm)))
        return fp4_fail(c, FP4_E_ARG, "null process list");
    const int nb = g->nbands, nptk = g->ngrid[0] * g->ngrid[1] * g->ngrid[2], nm = nb * nlist;
    std::vector<long long> op(nm + 1, 0), om(nm + 1, 0);
    for (int m = 0; m < nm; m++) {
        if (n_plus[m] < 0 || n_minus[m] < 0) return fp4_fail(c, FP4_E_ARG, "negative count");
        op[m + 1] = op[m] + n_plus[m];
        om[m + 1] = om[m] + n_minus[m];
    }
    if (op[nm] != ntotal_plus || om[nm] != ntotal_minus)
        return fp4_fail(c, FP4_E_ARG, "sum(N_plus)/sum(N_minus) differ from Ntotal_plus/Ntotal_minus");
    for (int q = 0; q < nptk * nsr; q++)
        if (id_equi[q] < 1 || id_equi[q] > nptk) return fp4_fail(c, FP4_E_ARG, "ID_equi entry outside [1,nptk]");
    for (int ll = 0; ll < nlist; ll++) {
        if (nequi[ll] < 0 || nequi[ll] > nsr) return fp4_fail(c, FP4_E_ARG, "Nequi entry outside [0,nsymm_rot]");
        for (int kk = 0; kk < nequi[ll]; kk++) {
            const int q = ll * nsr + kk;
            if (typeofsym[q] < 1 || typeofsym[q] > nsr || allequi[q] < 1 || allequi[q] > nptk)
                return fp4_fail(c, FP4_E_ARG, "TypeofSymmetry/ALLEquiList entry out of range");
        }
    }
    std::vector<long long> off4;
    if (l4) {
        off4.assign((size_t)3 * (nm + 1), 0);
        for (int ch = 0; ch < 3; ch++) {
            if (!l4->n[ch]) return fp4_fail(c, FP4_E_ARG, "null 4-phonon counts");
            long long* o = off4.data() + (size_t)ch * (nm + 1);
            for (int m = 0; m < nm; m++) {
                if (l4->n[ch][m] < 0) return fp4_fail(c, FP4_E_ARG, "negative count");
                o[m + 1] = o[m] + l4->n[ch][m];
            }
            if (o[nm] != l4->ntotal[ch])
                return fp4_fail(c, FP4_E_ARG, "sum(N_plusplus/plusminus/minusminus) differs from its Ntotal");
            if (o[nm] && (!l4->i2[ch] || !l4->i3[ch] || !l4->i4[ch] || !l4->g[ch]))
                return fp4_fail(c, FP4_E_ARG, "null 4-phonon process list");
        }
    }
    if ((r = fp4_begin(c))) return r;
    DevBuffer* B = c->b_bte;
    if ((r = B[0].upload(c, nequi, nlist * sizeof(int))) || (r = B[1].upload(c, allequi, (size_t)nlist * nsr * sizeof(int))) ||
        (r = B[2].upload(c, omega, (size_t)nptk * nb * sizeof(double))) ||
        (r = B[3].upload(c, velocity, (size_t)nptk * nb * 3 * sizeof(double))) ||
        (r = B[4].upload(c, tau_zero, (size_t)nlist * nb * sizeof(double))) ||
        (r = B[5].upload(c, f_n, (size_t)nptk * nb * 3 * sizeof(double))) ||
        (r = B[6].upload(c, typeofsym, (size_t)nlist * nsr * sizeof(int))) ||
        (r = B[7].upload(c, id_equi, (size_t)nptk * nsr * sizeof(int))) ||
        (r = B[8].upload(c, symmetrizers, (size_t)nptk * 9 * sizeof(double))))
        return r;
    // process lists: [n_plus|n_minus|off_plus|off_minus] and [i2p|i3p|i2m|i3m] and [gp|gm]
    std::vector<unsigned char> meta((size_t)nm * 2 * sizeof(int) + (size_t)(nm + 1) * 2 * sizeof(long long));
    memcpy(meta.data(), n_plus, nm * sizeof(int));
    memcpy(meta.data() + nm * sizeof(int), n_minus, nm * sizeof(int));
    memcpy(meta.data() + 2 * nm * sizeof(int), op.data(), (nm + 1) * sizeof(long long));
    memcpy(meta.data() + 2 * nm * sizeof(int) + (nm + 1) * sizeof(long long), om.data(), (nm + 1) * sizeof(long long));
    if ((r = B[9].upload(c, meta.data(), meta.size()))) return r;
    const size_t tp = ntotal_plus, tm = ntotal_minus;
    if ((r = B[10].reserve(c, (2 * tp + 2 * tm) * sizeof(int) + 64)) || (r = B[11].reserve(c, (tp + tm) * sizeof(double) + 64)))
        return r;
    int* L = B[10].as<int>();
    double* G = B[11].as<double>();
    if (tp) {
        CK(cudaMemcpyAsync(L, i2p, tp * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(L + tp, i3p, tp * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(G, gp, tp * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    if (tm) {
        CK(cudaMemcpyAsync(L + 2 * tp, i2m, tm * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(L + 2 * tp + tm, i3m, tm * sizeof(int), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(G + tp, gm, tm * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    BteParams p{};
    p.nb = nb;
    p.nptk = nptk;
    p.nlist = nlist;
    p.nsr = nsr;
    p.nequi = B[0].as<int>();
    p.allequi = B[1].as<int>();
    p.energy = B[2].as<double>();
    p.velocity = B[3].as<double>();
    p.tau_zero = B[4].as<double>();
    p.F = B[5].as<double>();
    p.typeofsym = B[6].as<int>();
    p.id_equi = B[7].as<int>();
    p.symm = B[8].as<double>();
    const unsigned char* mb = static_cast<const unsigned char*>(B[9].ptr);
    p.n_plus = reinterpret_cast<const int*>(mb);
    p.n_minus = p.n_plus + nm;
    p.off_plus = reinterpret_cast<const long long*>(mb + 2 * nm * sizeof(int));
    p.off_minus = p.off_plus + nm + 1;
    p.i2p = L;
    p.i3p = L + tp;
    p.i2m = L + 2 * tp;
    p.i3m = L + 2 * tp + tm;
    p.gp = G;
    p.gm = G + tp;
    p.err = c->b_err.as<int>();
    if (l4) {
        // [n4 (3 x nm) | off4 (3 x (nm+1))] and [i2|i3|i4 per channel] and [gamma per channel]
        const size_t t4 = (size_t)(l4->ntotal[0] + l4->ntotal[1] + l4->ntotal[2]);
        if ((r = c->b_counts.reserve(c, ((size_t)3 * nm + off4.size()) * sizeof(long long))) ||
            (r = c->b_lists.reserve(c, t4 * 3 * sizeof(long long) + 64)) ||
            (r = c->b_gamma.reserve(c, t4 * sizeof(double) + 64)))
            return r;
        long long* dn = c->b_counts.as<long long>();
        long long* doff = dn + 3 * nm;
        long long* L4 = c->b_lists.as<long long>();
        double* G4 = c->b_gamma.as<double>();
        CK(cudaMemcpyAsync(doff, off4.data(), off4.size() * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
        size_t base = 0;
        for (int ch = 0; ch < 3; ch++) {
            const size_t t = (size_t)l4->ntotal[ch];
            CK(cudaMemcpyAsync(dn + (size_t)ch * nm, l4->n[ch], nm * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
            long long* l = L4 + 3 * base;
            if (t) {
                CK(cudaMemcpyAsync(l, l4->i2[ch], t * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
                CK(cudaMemcpyAsync(l + t, l4->i3[ch], t * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
                CK(cudaMemcpyAsync(l + 2 * t, l4->i4[ch], t * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
                CK(cudaMemcpyAsync(G4 + base, l4->g[ch], t * sizeof(double), cudaMemcpyHostToDevice, c->stream));
            }
            p.n4[ch] = dn + (size_t)ch * nm;
            p.off4[ch] = doff + (size_t)ch * (nm + 1);
            p.i2_4[ch] = l;
            p.i3_4[ch] = l + t;
            p.i4_4[ch] = l + 2 * t;
            p.g4[ch] = G4 + base;
            base += t;
        }
    }
    if (jacobi) {
        if ((r = B[12].reserve(c, (size_t)nptk * nb * 3 * sizeof(double)))) return r;
        double* Fout = B[12].as<double>();
        CK(cudaEventRecord(c->evk0, c->stream));
        k_jacobi_step<<<dim3((unsigned)nm, (unsigned)nsr), 256, 0, c->stream>>>(p, Fout);
        CK(cudaGetLastError());
        k_symmetrize<<<256, 256, 0, c->stream>>>(nb, nptk, B[8].as<double>(), Fout);
        CK(cudaGetLastError());
        CK(cudaEventRecord(c->evk1, c->stream));
        c->kernel_timed = true;
        c->launches += 2;
        CK(cudaMemcpyAsync(f_n, Fout, (size_t)nptk * nb * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        return fp4_end(c);
    }
    CK(cudaEventRecord(c->evk0, c->stream));
    k_sweep<<<1, 1024, 0, c->stream>>>(p);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_timed = true;
    c->launches++;
    CK(cudaMemcpyAsync(f_n, B[5].ptr, (size_t)nptk * nb * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    B[5].key = 0;  // device copy now differs from the caller's previous F_n
    return fp4_end(c);
}

extern "C" int fp4_iteration(fp4_ctx* c, const fp4_globals* g, int32_t nlist, const int32_t* nequi,
                             const int32_t* allequi, const int32_t* typeofsym, int32_t nsr, const int32_t* id_equi,
                             const double* symmetrizers, const int32_t* n_plus, const int32_t* n_minus,
                             int32_t ntotal_plus, int32_t ntotal_minus, const int32_t* i2p, const int32_t* i3p,
                             const int32_t* i2m, const int32_t* i3m, const double* omega, const double* velocity,
                             const double* gp, const double* gm, const double* tau_zero, double* f_n) {
    FP4_TRACE();
    return run_sweep(c, g, nlist, nequi, allequi, typeofsym, nsr, id_equi, symmetrizers, n_plus, n_minus, ntotal_plus,
                     ntotal_minus, i2p, i3p, i2m, i3m, omega, velocity, gp, gm, tau_zero, f_n, nullptr);
}

extern "C" int fp4_iteration_jacobi(fp4_ctx* c, const fp4_globals* g, int32_t nlist, const int32_t* nequi,
                                    const int32_t* allequi, const int32_t* typeofsym, int32_t nsr,
                                    const int32_t* id_equi, const double* symmetrizers, const int32_t* n_plus,
                                    const int32_t* n_minus, int32_t ntotal_plus, int32_t ntotal_minus,
                                    const int32_t* i2p, const int32_t* i3p, const int32_t* i2m, const int32_t* i3m,
                                    const double* omega, const double* velocity, const double* gp, const double* gm,
                                    const double* tau_zero, double* f_n) {
    FP4_TRACE();
    return run_sweep(c, g, nlist, nequi, allequi, typeofsym, nsr, id_equi, symmetrizers, n_plus, n_minus, ntotal_plus,
                     ntotal_minus, i2p, i3p, i2m, i3m, omega, velocity, gp, gm, tau_zero, f_n, nullptr, true);
}

extern "C" int fp4_iteration_4ph(fp4_ctx* c, const fp4_globals* g, int32_t nlist, const int32_t* nequi,
                                 const int32_t* allequi, const int32_t* typeofsym, int32_t nsr,
                                 const int32_t* id_equi, const double* symmetrizers, const int32_t* n_plus,
                                 const int32_t* n_minus, int32_t ntotal_plus, int32_t ntotal_minus,
                                 const int64_t* n_pp, const int64_t* n_pm, const int64_t* n_mm, int64_t ntotal_pp,
                                 int64_t ntotal_pm, int64_t ntotal_mm, const int32_t* i2p, const int32_t* i3p,
                                 const int32_t* i2m, const int32_t* i3m, const int64_t* i2pp, const int64_t* i3pp,
                                 const int64_t* i4pp, const int64_t* i2pm, const int64_t* i3pm, const int64_t* i4pm,
                                 const int64_t* i2mm, const int64_t* i3mm, const int64_t* i4mm, const double* omega,
                                 const double* velocity, const double* gp, const double* gm, const double* gpp,
                                 const double* gpm, const double* gmm, const double* tau_zero, double* f_n) {
    FP4_TRACE();
    Lists4 l4{{n_pp, n_pm, n_mm}, {ntotal_pp, ntotal_pm, ntotal_mm}, {i2pp, i2pm, i2mm}, {i3pp, i3pm, i3mm},
              {i4pp, i4pm, i4mm}, {gpp, gpm, gmm}};
    return run_sweep(c, g, nlist, nequi, allequi, typeofsym, nsr, id_equi, symmetrizers, n_plus, n_minus, ntotal_plus,
                     ntotal_minus, i2p, i3p, i2m, i3m, omega, velocity, gp, gm, tau_zero, f_n, &l4);
}

extern "C" int fp4_symmetrize_fn(fp4_ctx* c, const fp4_globals* g, const double* symmetrizers, double* f_n) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    int r;
    if ((r = check_g(c, g))) return r;
    if (!symmetrizers || !f_n) return fp4_fail(c, FP4_E_ARG, "null argument");
    const int nb = g->nbands, nptk = g->ngrid[0] * g->ngrid[1] * g->ngrid[2];
    if ((r = fp4_begin(c))) return r;
    DevBuffer* B = c->b_bte;
    if ((r = B[8].upload(c, symmetrizers, (size_t)nptk * 9 * sizeof(double))) ||
        (r = B[5].upload(c, f_n, (size_t)nptk * nb * 3 * sizeof(double))))
        return r;
    k_symmetrize<<<256, 256, 0, c->stream>>>(nb, nptk, B[8].as<double>(), B[5].as<double>());
    CK(cudaGetLastError());
    c->launches++;
    CK(cudaMemcpyAsync(f_n, B[5].ptr, (size_t)nptk * nb * 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    B[5].key = 0;
    return fp4_end(c);
}

extern "C" int fp4_tconduct(fp4_ctx* c, const fp4_globals* g, double V, const double* omega, const double* velocity,
                            const double* f_n, double* kappa, double* kmode) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    int r;
    if ((r = check_g(c, g))) return r;
    if (!omega || !velocity || !f_n || !kappa || !(V > 0.0) || !(g->T > 0.0)) return fp4_fail(c, FP4_E_ARG, "bad argument");
    const int nb = g->nbands, nptk = g->ngrid[0] * g->ngrid[1] * g->ngrid[2];
    if ((r = fp4_begin(c))) return r;
    DevBuffer* B = c->b_bte;
    if ((r = B[2].upload(c, omega, (size_t)nptk * nb * sizeof(double))) ||
        (r = B[3].upload(c, velocity, (size_t)nptk * nb * 3 * sizeof(double))) ||
        (r = B[5].upload(c, f_n, (size_t)nptk * nb * 3 * sizeof(double))) || (r = c->b_out.reserve(c, nb * 9 * sizeof(double))))
        return r;
    double* km = nullptr;
    if (kmode) {
        if ((r = B[10].reserve(c, (size_t)nptk * nb * 9 * sizeof(double)))) return r;
        km = B[10].as<double>();
        CK(cudaMemsetAsync(km, 0, (size_t)nptk * nb * 9 * sizeof(double), c->stream));
        B[10].key = 0;
    }
    const double hbar = 1.05457172647e-22, kb = 1.380648813e-23;
    // 1e21*hbar**2*ThConductivity/(kB*T*T*V*nptk), 1e21 a default-REAL literal
    const double scale = (double)1e21f * (hbar * hbar) / (kb * g->T * g->T * V * nptk);
    k_tconduct<<<nb, 256, 0, c->stream>>>(nb, nptk, g->T, scale, B[2].as<double>(), B[3].as<double>(),
                                          B[5].as<double>(), c->b_out.as<double>(), km);
    CK(cudaGetLastError());
    c->launches++;
    CK(cudaMemcpyAsync(kappa, c->b_out.ptr, nb * 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (kmode) CK(cudaMemcpyAsync(kmode, km, (size_t)nptk * nb * 9 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return fp4_end(c);
}

// CumulativeTConduct (omega_mode 0) and CumulativeTConductOmega (1).
static int run_cumulative(fp4_ctx* c, const fp4_globals* g, double V, const double* omega, const double* velocity,
                          const double* f_n, int32_t nticks, double* ticks, double* results, int omega_mode) {
    if (!c) return FP4_E_ARG;
    int r;
    if ((r = check_g(c, g))) return r;
    if (!omega || !velocity || !f_n || !ticks || !results || !(V > 0.0) || !(g->T > 0.0) || nticks < 2)
        return fp4_fail(c, FP4_E_ARG, "bad argument");
    const int nb = g->nbands, nptk = g->ngrid[0] * g->ngrid[1] * g->ngrid[2];
    // the thresholds, computed on the host as the reference computes them
    if (omega_mode == 0) {
        for (int ii = 1; ii <= nticks; ii++)  // 10.**(8.*(ii-1.)/(nticks-1.)-2.) in default REAL
            ticks[ii - 1] = (double)powf(10.0f, 8.0f * ((float)ii - 1.0f) / ((float)nticks - 1.0f) - 2.0f);
    } else {
        double emin = 1.e10, emax = -1.e10;
        for (size_t x = 0; x < (size_t)nptk * nb; x++) {
            emin = std::min(emin, omega[x]);
            emax = std::max(emax, omega[x]);
        }
        emax = emax * 1.1;
        for (int ii = 1; ii <= nticks; ii++) ticks[ii - 1] = emin + (emax - emin) * ii / nticks;
    }
    if ((r = fp4_begin(c))) return r;
    DevBuffer* B = c->b_bte;
    if ((r = B[2].upload(c, omega, (size_t)nptk * nb * sizeof(double))) ||
        (r = B[3].upload(c, velocity, (size_t)nptk * nb * 3 * sizeof(double))) ||
        (r = B[5].upload(c, f_n, (size_t)nptk * nb * 3 * sizeof(double))) ||
        (r = B[9].upload(c, ticks, (size_t)nticks * sizeof(double))) ||
        (r = c->b_out.reserve(c, (size_t)nb * 9 * nticks * sizeof(double))))
        return r;
    const double hbar = 1.05457172647e-22, kb = 1.380648813e-23;
    const double scale = (double)1e21f * (hbar * hbar) / (kb * g->T * g->T * V * nptk);
    k_cumulative<<<dim3(nticks, nb), 128, 0, c->stream>>>(nb, nptk, nticks, omega_mode, g->T, scale,
                                                          B[2].as<double>(), B[3].as<double>(), B[5].as<double>(),
                                                          B[9].as<double>(), c->b_out.as<double>());
    CK(cudaGetLastError());
    c->launches++;
    CK(cudaMemcpyAsync(results, c->b_out.ptr, (size_t)nb * 9 * nticks * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    B[9].key = 0;
    return fp4_end(c);
}

extern "C" int fp4_cumulative_tconduct(fp4_ctx* c, const fp4_globals* g, double V, const double* omega,
                                       const double* velocity, const double* f_n, int32_t nticks, double* ticks,
                                       double* results) {
    FP4_TRACE();
    return run_cumulative(c, g, V, omega, velocity, f_n, nticks, ticks, results, 0);
}

extern "C" int fp4_cumulative_tconduct_omega(fp4_ctx* c, const fp4_globals* g, double V, const double* omega,
                                             const double* velocity, const double* f_n, int32_t nticks,
                                             double* ticks, double* results) {
    FP4_TRACE();
    return run_cumulative(c, g, V, omega, velocity, f_n, nticks, ticks, results, 1);
}
