// Device-side data layout and arithmetic shared by the rate kernels.
//
// Layout in HBM (built once per system by the C-ABI layer):
//   wv[q*nb + b]            double4 {vx, vy, vz, omega}: one 32-byte load per mode
//   eig[(q*nb + b)*nb + c]  double2 eigenvector component c of mode (q,b)
//   eigf[...]               float2 copy for the mixed-precision contraction
//   bose[t*nptk*nb + q*nb + b]  Bose-Einstein occupation at temperature t
//   root_d[x]               exp(2*pi*i*x/N_d), x in [0,N_d), per grid axis d
// Clusters carry integer lattice coordinates of their cells, so every Bloch
// phase exp(i q.R) is exp(2*pi*i*sum_d n_d m_d / N_d), looked up exactly in
// the root tables instead of evaluating cos/sin of a rounded dot product.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace fp4 {

constexpr int kMaxNb = 32;       // nbands <= 32 (natoms <= 10)
constexpr int kMaxTemps = 8;     // temperatures fused in one rate call
constexpr int kMaxGrid = 64;     // ngrid(d) <= 64

struct DevSys {
    int n[3];
    int nptk, nb, nlist, natoms;
    double rl[9];  // rlattvec(3,3) column-major
    double ngd[3], rinv[3];  // ngrid(d) as double and RN(1/ngrid(d))
    double scalebroad, omega_max;
    int onlyharmonic;
    const double4* wv;
    const double2* eig;
    const float2* eigf;
    const int* list0;  // 0-based q of irreducible point ll
    const int* qc;     // grid coordinates of q packed as a | b<<8 | c<<16 (Id2ind)
    const double2* root[3];
    const float2* rootf[3];
};

struct DevIfc {
    int order, ntri, npi, nblk;  // nblk = natoms^2 atom-pair blocks of the class table
    const double* phi;           // per cluster 27 (3ph: [t][s][r]) or 81 (4ph: [u][t][s][r]) entries
    const int4* atoms;           // 0-based (a1,a2,a3,a4)
    const int4* mj;              // lattice coordinates of the 2nd atom's cell
    const int4* mk;              // ... 3rd
    const int4* ml;              // ... 4th (4ph)
    const double* mu;            // 1/sqrt(product of masses)
    const int* cl_start;         // clusters sorted by class: class p owns [cl_start[p], cl_start[p+1])
    const int* cl_index;         // cluster ids in class order
    const int4* pi_d;            // class displacement D (x,y,z) and packed atom pair in .w
    const int* blk_start;        // classes sorted by atom-pair block: block b owns [blk_start[b], blk_start[b+1])
};

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cmac(double2 acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmacf(float2 acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ float2 cconjf(float2 a) { return make_float2(a.x, -a.y); }

__device__ __forceinline__ int pmod(int a, int n) {
    int r = a % n;
    return r < 0 ? r + n : r;
}

// exp(2*pi*i * sum_d n_d*m_d/N_d): three table lookups, two complex products
__device__ __forceinline__ double2 lattice_phase(const DevSys& S, int n0, int n1, int n2, int m0, int m1, int m2) {
    double2 a = S.root[0][pmod(n0 * m0, S.n[0])];
    double2 b = S.root[1][pmod(n1 * m1, S.n[1])];
    double2 c = S.root[2][pmod(n2 * m2, S.n[2])];
    return cmul(cmul(a, b), c);
}
__device__ __forceinline__ float2 lattice_phase_f(const DevSys& S, int n0, int n1, int n2, int m0, int m1, int m2) {
    float2 a = S.rootf[0][pmod(n0 * m0, S.n[0])];
    float2 b = S.rootf[1][pmod(n1 * m1, S.n[1])];
    float2 c = S.rootf[2][pmod(n2 * m2, S.n[2])];
    return cmulf(cmulf(a, b), c);
}

// q index <-> grid coordinates (Id2ind, config.f90:458-468; Index_N of processes.f90)
__device__ __forceinline__ void q_coords(const DevSys& S, int q, int& a, int& b, int& c) {
    a = q % S.n[0];
    int t = q / S.n[0];
    b = t % S.n[1];
    c = t / S.n[1];
}
__device__ __forceinline__ int q_index(const DevSys& S, int a, int b, int c) { return (c * S.n[1] + b) * S.n[0] + a; }
// table form of q_coords: one load instead of integer divisions
__device__ __forceinline__ void q_coords_t(const DevSys& S, int q, int& a, int& b, int& c) {
    int v = __ldg(S.qc + q);
    a = v & 0xff;
    b = (v >> 8) & 0xff;
    c = v >> 16;
}
// (t mod N) for t in (-2N, 3N), without a division
__device__ __forceinline__ int wrapN(int t, int N) {
    t = (t >= N) ? t - N : t;
    t = (t >= N) ? t - N : t;
    t = (t < 0) ? t + N : t;
    t = (t < 0) ? t + N : t;
    return t;
}

// ---------------------------------------------------------------------------
// block-wide helpers
// ---------------------------------------------------------------------------
// exclusive prefix of a per-thread flag, in thread order; total in `total`
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

// fixed-order block sum; result valid in thread 0
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
    return t;
}

// fixed-order block sum of NV values at once; results valid in thread 0 (red holds 32*NV)
template <int NV>
__device__ __forceinline__ void block_sum_vec(double (&v)[NV], double* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int x = 0; x < NV; x++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[x] += __shfl_down_sync(0xffffffffu, v[x], o);
        if (lane == 0) red[x * 32 + warp] = v[x];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int x = 0; x < NV; x++) {
            double t = 0.0;
            for (int w = 0; w < nwarp; w++) t += red[x * 32 + w];
            v[x] = t;
        }
    }
    __syncthreads();
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

// First index i with a[i] >= x in a sorted a[0..n-1], by a descent over powers of two
// from the largest one <= n: the step count depends only on n, so the lanes of a warp
// stay together.
__device__ __forceinline__ int lower_bound_desc(const double* a, int n, double x) {
    int i = 0;
    if (n <= 0) return 0;
    for (int step = 1 << (31 - __clz(n)); step > 0; step >>= 1) {
        const int y = i + step;
        if (y <= n && a[y - 1] < x) i = y;
    }
    return i;
}
// First index i with a[i] > x (the count of entries <= x), by the same descent.
__device__ __forceinline__ int upper_bound_desc(const double* a, int n, double x) {
    int i = 0;
    if (n <= 0) return 0;
    for (int step = 1 << (31 - __clz(n)); step > 0; step >>= 1) {
        const int y = i + step;
        if (y <= n && a[y - 1] <= x) i = y;
    }
    return i;
}

// ---------------------------------------------------------------------------
// Energy-conservation filter, bit-exact with the reference's source order.
// base_sigma (config.f90:481-499):  max over nu of
//   ((rl(1,nu)*v1 + rl(2,nu)*v2) + rl(3,nu)*v3) / ngrid(nu), squared;
// then sqrt(x/2) and the scalebroad factor.  Every product and sum is
// rounded separately (no fused multiply-add), exactly as written.
// ---------------------------------------------------------------------------
// x/N for a grid size N (a small positive integer), correctly rounded.
// Reciprocal multiplication followed by two residual corrections
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34 (1990)): with r = RN(1/N) the
// residual e = x - q*N is exact in one fused multiply-add, and q + e*r rounds
// to RN(x/N).  tests/cuda/div_check.cu compares it with __ddiv_rn.
__device__ __forceinline__ double div_by_grid(double x, double N, double r) {
    double q = __dmul_rn(x, r);
    double e = __fma_rn(-q, N, x);
    q = __fma_rn(e, r, q);
    e = __fma_rn(-q, N, x);
    return __fma_rn(e, r, q);
}

// On a cubic grid all three quotients share N: correct rounding is monotone and
// symmetric, so RN(RN(dp/N)^2) grows with |dp| and the largest of the three is the
// one of the largest |dp| -- one division gives the reference's maximum exactly.
__device__ __forceinline__ double sigma_exact(const DevSys& S, double4 a, double4 b) {
    double v0 = __dadd_rn(a.x, -b.x);
    double v1 = __dadd_rn(a.y, -b.y);
    double v2 = __dadd_rn(a.z, -b.z);
    if (S.n[0] == S.n[1] && S.n[1] == S.n[2]) {
        double dmax = 0.0;
#pragma unroll
        for (int nu = 0; nu < 3; nu++) {
            const double* r = S.rl + 3 * nu;
            const double dp = __dadd_rn(__dadd_rn(__dmul_rn(r[0], v0), __dmul_rn(r[1], v1)), __dmul_rn(r[2], v2));
            dmax = fmax(dmax, fabs(dp));
        }
        const double x = div_by_grid(dmax, S.ngd[0], S.rinv[0]);
        return __dmul_rn(S.scalebroad, __dsqrt_rn(__dmul_rn(__dmul_rn(x, x), 0.5)));
    }
    double m = 0.0;
#pragma unroll
    for (int nu = 0; nu < 3; nu++) {
        const double* r = S.rl + 3 * nu;
        double dp = __dadd_rn(__dadd_rn(__dmul_rn(r[0], v0), __dmul_rn(r[1], v1)), __dmul_rn(r[2], v2));
        double x = div_by_grid(dp, S.ngd[nu], S.rinv[nu]);
        double x2 = __dmul_rn(x, x);
        m = (nu == 0 || x2 > m) ? x2 : m;
    }
    return __dmul_rn(S.scalebroad, __dsqrt_rn(__dmul_rn(m, 0.5)));
}

// Occupation 1/(exp(hbar*w/kB/T)-1), with the reference's operation order.
__device__ __forceinline__ double bose_of(double w, double T) {
    const double hbar = 1.05457172647e-22, kb = 1.380648813e-23;
    return 1.0 / (exp(hbar * w / kb / T) - 1.0);
}

// A queued four-phonon process in a 64-bit word: the grid coordinates (a,b,c) of
// q'' (6 bits each, ngrid <= 64), the index of q''' (18 bits, nptk <= 64^3) and
// the branches k, l (8 bits each).  j is the bin's.
__device__ __forceinline__ unsigned long long pack_proc(int a, int b, int c, int ss, int k, int l) {
    return ((unsigned long long)(unsigned)c << 46) | ((unsigned long long)(unsigned)b << 40) |
           ((unsigned long long)(unsigned)a << 34) | ((unsigned long long)(unsigned)ss << 16) |
           ((unsigned)k << 8) | (unsigned)l;
}
__device__ __forceinline__ void unpack_proc(unsigned long long e, int& a, int& b, int& c, int& ss, int& k, int& l) {
    l = (int)(e & 0xff);
    k = (int)((e >> 8) & 0xff);
    ss = (int)((e >> 16) & 0x3ffff);
    a = (int)((e >> 34) & 0x3f);
    b = (int)((e >> 40) & 0x3f);
    c = (int)((e >> 46) & 0x3f);
}

// Error flags raised by kernels (read back by the host after each call)
// kErrTimeout: a bounded wait for the tensor core gave up (the kernel stopped early).
enum : int { kErrQueue = 1, kErrTable = 2, kErrList = 4, kErrTimeout = 8 };

}  // namespace fp4
