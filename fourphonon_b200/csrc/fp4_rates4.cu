// Four-phonon scattering-rate kernel for sm_100a.
//
// Persistent CTAs pull work items (q = List(ll), q', channel) from an atomic
// counter.  For each work item:
//   * the valid sums s_ij = w_i +- w'_j are rank-sorted in shared memory;
//   * phase A walks every (q'', k, l) once: q''' from integer grid
//     arithmetic, the channel's restrictions, sigma(v''-v''') in base_sigma's
//     exact operation order (computed once for all (i,j)), a binary search for
//     the window of s_ij that can pass the 1-sigma test, and the exact test in
//     the reference's operation order.  Survivors are queued per (i,j);
//   * phase B builds, per branch i, the reciprocal cluster table
//         Z_p^{(ij)}[s][r] = sum_{c in p} kappa_c sum_{u,t} Psi_c[u][t][s][r] e_i[u] e~'_j[t]
//     and contracts each queued process as
//         V = sum_p w_p(q'') e~''_k[s] Z_p[s][r] conj(e'''_l[r]),
//     with w_p(q'') = exp(+-2 pi i n''.D_p/N) read from per-class phase tables
//     in shared memory.  This is Vp_pp/Vp_pm/Vp_mm (processes.f90:142-330)
//     with the cluster phases factored through integer lattice coordinates.
//   * weights (Bose factors, Gaussian, sigma floor) are FP64 for every
//     temperature of the call; |V|^2 is formed once for all of them.
// Per-(work item, branch, temperature) partial sums are reduced afterwards in
// a fixed order with compensated summation (k4_reduce).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fp4_device.cuh"
#include "fp4_internal.h"
#include "fp4_tc.cuh"

namespace fp4 {

namespace {

constexpr int kThreads = 256;
constexpr int kCheckEvery = 8;  // list mode: passes between queue-capacity checks; also the most passes
                                 // in a phase-A stage (the queues are drained at stage boundaries)
// Resident persistent CTAs per SM, which sets the register budget.  Three CTAs
// (80 registers) suit the FP32 contraction of one or two temperatures (1.21x
// faster than two CTAs on the 16^3 diamond workload) and the counting kernel.
// The FP64 contraction keeps two CTAs (128 registers): at 80 it spills, and the
// spill traffic cancels the extra warps.
// The multi-solve kernel keeps more state per thread (the slot, its layout) and runs
// two CTAs per SM in both precisions: at three the FP32 form spills.
constexpr int kMultiCtasPerSm = 2;

template <int KIND, int NT, bool MIXED>
constexpr int ctas_per_sm() {
    return (KIND == 0 || (MIXED && NT <= 2)) ? 3 : 2;
}

template <bool MIXED>
struct CT;
template <>
struct CT<false> {
    using T = double2;
    __device__ static T zero() { return make_double2(0.0, 0.0); }
    __device__ static T conj(T a) { return cconj(a); }
    __device__ static T mul(T a, T b) { return cmul(a, b); }
    __device__ static T mac(T acc, T a, T b) { return cmac(acc, a, b); }
    __device__ static T from(double2 a) { return a; }
    __device__ static double norm(T a) { return a.x * a.x + a.y * a.y; }
};
template <>
struct CT<true> {
    using T = float2;
    __device__ static T zero() { return make_float2(0.f, 0.f); }
    __device__ static T conj(T a) { return cconjf(a); }
    __device__ static T mul(T a, T b) { return cmulf(a, b); }
    __device__ static T mac(T acc, T a, T b) { return cmacf(acc, a, b); }
    __device__ static T from(double2 a) { return make_float2((float)a.x, (float)a.y); }
    __device__ static double norm(T a) { return (double)a.x * (double)a.x + (double)a.y * (double)a.y; }
};

struct Layout {
    size_t z, kap, pt, sval, swj, racc, wacc, pacc, red, sidx, cnt, ncnt, klt, pre, blk, seg, jjl, stg, stgi, misc,
        total;
    int allz;  // 1: the reciprocal cluster tables of all (i,j) at once, 0: one branch i at a time
    int njjl;  // capacity of the list of q'' that the channel's restriction keeps (0: no list)
    int stgp;  // phase-A passes per stage of (v, omega) records
};

// Phase A stages the (v, omega) records of the third phonon's grid points of the
// next stgp passes, and those of the matching fourth-phonon points, in shared
// memory (at most kStageSlots points per stage), so that a candidate reads them
// there instead of from global memory.  The queues are drained only at a stage
// boundary, so a stage never straddles a flush; stgp <= kCheckEvery keeps the
// queue headroom within the capacity the host reserves.
constexpr int kStageSlots = 32;
__host__ __device__ inline int stage_passes(int nb2) {
    int P = 8;
    while (P > 1 && (P * 256 - 1) / nb2 + 2 > kStageSlots) P >>= 1;
    return P;
}
__host__ __device__ inline int stage_slots(int nb2) { return (stage_passes(nb2) * 256 - 1) / nb2 + 2; }

// The +- and -- channels keep a q'' only when q''' >= q''; phase A then walks a list of
// those q'' (16-bit indices, built per work item) instead of testing every q''.
constexpr int kMaxJJList = 16384;

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

// Shared memory per CTA below which the tables of all branches are kept at once
// (three CTAs per SM still fit).
constexpr size_t kAllZCap = 72 * 1024;

__host__ __device__ inline Layout k4_layout_z(int kind, int NT, bool mixed, int nb, int npi, int ntri, int lsum,
                                              int allz, int njjl, bool noz = false) {
    Layout L;
    L.allz = allz;
    L.njjl = njjl;
    const size_t cs = mixed ? 8 : 16;  // complex size
    const size_t nb2 = (size_t)nb * nb;
    size_t o = 0;
    L.z = o;
    o = al16(o + ((kind >= 2 && !noz) ? (allz ? nb2 : (size_t)nb) * npi * 9 * cs : 0));
    L.kap = o;
    o = al16(o + ((kind >= 2) ? (size_t)ntri * 16 : 0));
    L.pt = o;
    o = al16(o + ((kind >= 2) ? (size_t)npi * lsum * cs : 0));
    L.sval = o;
    o = al16(o + nb2 * 8);
    L.swj = o;  // omega'_j of each sorted pair
    o = al16(o + nb2 * 8);
    L.racc = o;
    o = al16(o + (size_t)nb * NT * 8);
    L.wacc = o;
    o = al16(o + (size_t)nb * NT * 8);
    // counting: one copy of the per-branch count and phase-space sum per warp, so that
    // the shared-memory atomics of a survivor contend within its warp only
    const size_t ncopy = (kind == 0) ? kThreads / 32 : 1;
    L.pacc = o;
    o = al16(o + (size_t)nb * ncopy * 8);
    L.red = o;  // block_sum_vec of 2*NT values (phase B) or 4 (work counters)
    o = al16(o + (size_t)32 * (2 * NT > 4 ? 2 * NT : 4) * 8);
    L.sidx = o;
    o = al16(o + nb2 * 4);
    L.cnt = o;
    o = al16(o + nb2 * 4);
    L.ncnt = o;
    o = al16(o + (size_t)nb * ncopy * 4);
    L.klt = o;
    o = al16(o + nb2 * 4);
    L.pre = o;
    o = al16(o + (nb2 + 1) * 4);
    L.blk = o;  // non-empty atom-pair blocks of the class table: (first class, end, atom k, atom l)
    o = al16(o + (size_t)(kMaxNb / 3) * (kMaxNb / 3) * 16);
    L.seg = o;  // kind 3: first list position of each branch's q' segment, then the segments' prefix
    o = al16(o + (size_t)(2 * nb + 1) * 8);
    L.jjl = o;
    o = al16(o + (size_t)njjl * 2 + 32 * 4);  // the list, then per-warp counts of the compaction
    L.stgp = stage_passes((int)nb2);
    L.stg = o;  // per staged point: the records (v, omega) of its nb branches, then those of its partner
    o = al16(o + (size_t)stage_slots((int)nb2) * 2 * nb * 32);
    L.stgi = o;  // per staged point: (its index, its grid coordinates packed, the partner's index)
    o = al16(o + (size_t)stage_slots((int)nb2) * 16);
    L.misc = o;
    o = al16(o + 8 * 4);
    L.total = o;
    return L;
}

// nptk_list: the grid size when the kernel may use the q'' list (0: never).  The list
// is kept only where it costs no other choice: the all-branch tables come first.
// The all-branch tables are used while the whole layout keeps the kernel's CTAs
// per SM resident: kAllZCap for three, kAllZCap2 for two.
constexpr size_t kAllZCap2 = 110 * 1024;
__host__ __device__ inline Layout k4_layout(int kind, int NT, bool mixed, int nb, int npi, int ntri, int lsum,
                                            int nptk_list, size_t cap_override = 0) {
    const int nl = (kind == 0 || kind == 2) && nptk_list <= kMaxJJList ? nptk_list : 0;
    const size_t cap = cap_override ? cap_override : ((kind == 0 || (mixed && NT <= 2)) ? kAllZCap : kAllZCap2);
    if (kind >= 2) {
        Layout A = k4_layout_z(kind, NT, mixed, nb, npi, ntri, lsum, 1, nl);
        if (A.total <= cap) return A;
        A = k4_layout_z(kind, NT, mixed, nb, npi, ntri, lsum, 1, 0);
        if (A.total <= cap) return A;
    }
    Layout B = k4_layout_z(kind, NT, mixed, nb, npi, ntri, lsum, 0, nl);
    if (nl && B.total > cap) B = k4_layout_z(kind, NT, mixed, nb, npi, ntri, lsum, 0, 0);
    return B;
}

// Shared memory of the tensor-core contraction, after the common layout (no Z
// tables): the A tiles of the two warpgroups, the B tables and FP64 Z entries
// of one group of bins, two mbarriers, the TMEM address and the parities of the
// two mbarriers, the group's bins and its chunk list.
struct TcLayout {
    size_t a, b, zs, eig, plan, bar, slot, gbin, chunk, total;
};

__host__ __device__ inline Layout k4_layout_tcbase(int NT, int nb, int npi, int ntri, int lsum, int nptk) {
    const int nl = nptk <= kMaxJJList ? nptk : 0;
    return k4_layout_z(2, NT, true, nb, npi, ntri, lsum, 0, nl, true);
}

__host__ __device__ inline TcLayout k4_tc_layout(size_t base, int ksteps, int bin_bytes, int zbins, int npi,
                                                 int chunk_cap, int nb) {
    TcLayout T;
    size_t o = (base + 127) & ~(size_t)127;
    T.a = o;
    o += 2 * (size_t)ksteps * kTcRows * 32;
    T.b = o;
    o += (size_t)zbins * bin_bytes;
    T.zs = o;
    o += (size_t)zbins * npi * 9 * 16;
    T.eig = o;  // per warpgroup and row: the two eigenvector rows of its process
    o += (size_t)2 * kTcRows * (2 * nb + 1) * 8;
    T.plan = o;  // a copy of the plan
    o = al16(o + sizeof(TcPlan));
    T.bar = o;
    o += 16;
    T.slot = o;
    o += 16;
    T.gbin = o;
    o = al16(o + (size_t)zbins * 4);
    T.chunk = o;
    o = al16(o + (size_t)chunk_cap * 4);
    T.total = o;
    return T;
}

template <bool MIXED>
__device__ __forceinline__ const typename CT<MIXED>::T* eig_table(const DevSys& S);
template <>
__device__ __forceinline__ const double2* eig_table<false>(const DevSys& S) {
    return S.eig;
}
template <>
__device__ __forceinline__ const float2* eig_table<true>(const DevSys& S) {
    return S.eigf;
}

// One entry of the reciprocal cluster table of branches (i, j):
//   Z_p[s][r] = sum_{c in p} kappa_c sum_{u,t} Psi_c[u][t][s][r] e_i[u] e~'_j[t]
__device__ __forceinline__ double2 k4_z_entry(const DevSys& S, const DevIfc& F, const double2* kap, int ch, int q0,
                                              int ii, int i, int j, int pc, int sr) {
    const int nb = S.nb;
    const double2* ei = S.eig + (size_t)(q0 * nb + i) * nb;
    const double2* ej = S.eig + (size_t)(ii * nb + j) * nb;
    double2 acc = make_double2(0.0, 0.0);
    for (int x = F.cl_start[pc]; x < F.cl_start[pc + 1]; x++) {
        const int c = F.cl_index[x];
        const int4 at = F.atoms[c];
        const double* ph = F.phi + (size_t)c * 81 + sr;
        double2 t1 = make_double2(0.0, 0.0);
#pragma unroll
        for (int u = 0; u < 3; u++) {
            const double2 eu = ei[3 * at.x + u];
#pragma unroll
            for (int t = 0; t < 3; t++) {
                double2 et = ej[3 * at.y + t];
                if (ch == 2) et = cconj(et);
                const double2 pr = cmul(eu, et);
                const double f = ph[(u * 3 + t) * 9];
                t1.x = fma(f, pr.x, t1.x);
                t1.y = fma(f, pr.y, t1.y);
            }
        }
        acc = cmac(acc, kap[c], t1);
    }
    return acc;
}

// Contract one queued process of branches (i, j) against the table Zj and add
// its weights for every temperature to accr/accw (LIST: also store its Gamma).
template <int NT, bool MIXED, bool LIST>
__device__ __forceinline__ void k4_entry(const P4Params& p, const typename CT<MIXED>::T* Zj,
                                         const typename CT<MIXED>::T* PT, const int4* blkinfo, int nbk,
                                         unsigned long long ent, double sigma, long long pos, int ch, int ii, int i,
                                         int j, double omega, int m0, int m1, int m2, int n0, int n1, int n2,
                                         double (&accr)[NT], double (&accw)[NT]) {
    using C = CT<MIXED>;
    using cx = typename C::T;
    const DevSys& S = p.S;
    const int nb = S.nb;
    const int N0 = S.n[0], N1 = S.n[1], lsum = N0 + N1 + S.n[2];
    const double sqrtpi = sqrt(3.141592653589793238);
    const double floor_sigma = (double)0.001f;
    const bool neg = (ch != 0);  // class displacement D = m_k - m_l (++) or m_l - m_k (+-, --)
    const cx* etab = eig_table<MIXED>(S);
    int a, b, c, ss, k, l;
    unpack_proc(ent, a, b, c, ss, k, l);
    const int jj = q_index(S, a, b, c);
    // (omega, Bose factors) records of the three other modes: omega now, the factors
    // (same cache line) after the contraction, so that they are not live across it
    constexpr int WS = wb_stride(NT);
    const double* x1 = p.wb + (size_t)(ii * nb + j) * WS;
    const double* x2 = p.wb + (size_t)(jj * nb + k) * WS;
    const double* x3 = p.wb + (size_t)(ss * nb + l) * WS;
    const double w1 = x1[0], w2 = x2[0], w3 = x3[0];
    const double sv = (ch == 2) ? __dadd_rn(omega, -w1) : __dadd_rn(omega, w1);
    const double delta = (ch == 0) ? __dadd_rn(__dadd_rn(sv, w2), -w3) : __dadd_rn(__dadd_rn(sv, -w2), -w3);
    if (sigma <= floor_sigma) sigma = 1.0 / sqrtpi;
    const double g = exp(-(delta * delta) / (sigma * sigma));
    const double base = g / (sigma * sqrtpi * (omega * w1 * w2 * w3));
    double v2 = 0.0;
    if (LIST || !S.onlyharmonic) {
        const cx* e2 = etab + (size_t)(jj * nb + k) * nb;
        const cx* e3 = etab + (size_t)(ss * nb + l) * nb;
        cx V = C::zero();
        for (int bb = 0; bb < nbk; bb++) {
            const int4 bi = blkinfo[bb];
            const int p0 = bi.x, p1 = bi.y, a3 = bi.z, a4 = bi.w;
            cx u[3], v[3];
#pragma unroll
            for (int x = 0; x < 3; x++) {
                u[x] = e2[3 * a3 + x];
                if (ch != 0) u[x] = C::conj(u[x]);
                v[x] = C::conj(e3[3 * a4 + x]);
            }
            for (int pc = p0; pc < p1; pc++) {
                const cx* pt = PT + pc * lsum;
                cx w = C::mul(C::mul(pt[a], pt[N0 + b]), pt[N0 + N1 + c]);
                if (neg) w = C::conj(w);
                const cx* z = Zj + pc * 9;
                cx tt = C::zero();
#pragma unroll
                for (int x = 0; x < 3; x++) {
                    cx h = C::zero();
#pragma unroll
                    for (int r = 0; r < 3; r++) h = C::mac(h, z[x * 3 + r], v[r]);
                    tt = C::mac(tt, u[x], h);
                }
                V = C::mac(V, w, tt);
            }
        }
        v2 = C::norm(V);
    }
#pragma unroll
    for (int t = 0; t < NT; t++) {
        if (t < p.nT) {
            const double f1 = x1[1 + t], f2 = x2[1 + t], f3 = x3[1 + t];
            double bc;
            if (ch == 0)
                bc = f1 * f2 * (1 + f3) - (1 + f1) * (1 + f2) * f3;
            else if (ch == 1)
                bc = f1 * (1 + f2) * (1 + f3) - (1 + f1) * f2 * f3;
            else
                bc = (1 + f1) * (1 + f2) * (1 + f3) - f1 * f2 * f3;
            const double wp4 = bc * base;
            accr[t] = fma(wp4, v2, accr[t]);
            accw[t] += wp4;
            if (LIST) p.gamma_out[ch][pos] = wp4 * v2 * p.gamma_scale;
        }
    }
}

// Phase B: contract every queued process of the current work item, branch by branch.
// LIST: also store each process's own Gamma at its list position (Ind_plusplus etc.).
template <int NT, bool MIXED, bool LIST>
__device__ void k4_phase_b(const P4Params& p, unsigned char* smem, const Layout& L, const unsigned long long* qbase,
                           const double* qsig, const long long* qpos, int ch, int ii, int q0, int m0, int m1, int m2,
                           int n0, int n1, int n2, unsigned long long& my_contr) {
    using C = CT<MIXED>;
    using cx = typename C::T;
    const DevSys& S = p.S;
    const DevIfc& F = p.F;
    const int nb = S.nb, nb2 = nb * nb, npi = F.npi;
    cx* Z = reinterpret_cast<cx*>(smem + L.z);
    const double2* kap = reinterpret_cast<const double2*>(smem + L.kap);
    const cx* PT = reinterpret_cast<const cx*>(smem + L.pt);
    double* racc = reinterpret_cast<double*>(smem + L.racc);
    double* wacc = reinterpret_cast<double*>(smem + L.wacc);
    double* red = reinterpret_cast<double*>(smem + L.red);
    int* cnt = reinterpret_cast<int*>(smem + L.cnt);
    int* pre = reinterpret_cast<int*>(smem + L.pre);
    const int4* blkinfo = reinterpret_cast<const int4*>(smem + L.blk);
    const int nbk = reinterpret_cast<const int*>(smem + L.misc)[3];
    const double* wvw = reinterpret_cast<const double*>(S.wv) + 3;
    for (int i = 0; i < nb; i++) {
        if (threadIdx.x == 0) {
            int acc = 0;
            for (int j = 0; j < nb; j++) {
                pre[j] = acc;
                acc += min(cnt[i * nb + j], p.subcap);
            }
            pre[nb] = acc;
        }
        __syncthreads();
        const int tot = pre[nb];
        if (tot == 0) {
            __syncthreads();
            continue;
        }
        if (threadIdx.x == 0) atomicAdd(&p.stats[4], 1ull);
        for (int idx = threadIdx.x; idx < nb * npi * 9; idx += blockDim.x) {
            const int j = idx / (npi * 9), rem = idx - j * (npi * 9), pc = rem / 9, sr = rem - pc * 9;
            Z[idx] = C::from(k4_z_entry(S, F, kap, ch, q0, ii, i, j, pc, sr));
        }
        __syncthreads();
        // plain per-thread partial sums (a few tens of terms each); the cross-work-item
        // reduction (k4_reduce) is the compensated one
        double accr[NT], accw[NT];
#pragma unroll
        for (int t = 0; t < NT; t++) {
            accr[t] = 0.0;
            accw[t] = 0.0;
        }
        const double omega = wvw[4 * (q0 * nb + i)];
        for (int e = threadIdx.x; e < tot; e += blockDim.x) {
            int j = 0;
            while (j + 1 < nb && pre[j + 1] <= e) j++;
            const size_t qi = (size_t)(i * nb + j) * p.subcap + (e - pre[j]);
            k4_entry<NT, MIXED, LIST>(p, Z + (size_t)j * npi * 9, PT, blkinfo, nbk, qbase[qi], qsig[qi],
                                      LIST ? qpos[qi] : 0, ch, ii, i, j, omega, m0, m1, m2, n0, n1, n2, accr, accw);
            my_contr++;
        }
        double v[2 * NT];
#pragma unroll
        for (int t = 0; t < NT; t++) {
            v[t] = accr[t];
            v[NT + t] = accw[t];
        }
        block_sum_vec<2 * NT>(v, red);
        if (threadIdx.x == 0) {
            for (int t = 0; t < p.nT; t++) {
                racc[i * NT + t] += v[t];
                wacc[i * NT + t] += v[NT + t];
            }
        }
        __syncthreads();
    }
    for (int x = threadIdx.x; x < nb2; x += blockDim.x) cnt[x] = 0;
    __syncthreads();
}

// Phase B with the tables of all (i,j) in shared memory at once: one table build
// and one pass over every queued process of the work item.  A thread's entries
// run in (i,j) order; its sums for one branch go to shared memory when its
// branch changes.
template <int NT, bool MIXED, bool LIST>
__device__ void k4_phase_b_all(const P4Params& p, unsigned char* smem, const Layout& L,
                               const unsigned long long* qbase, const double* qsig, const long long* qpos, int ch,
                               int ii, int q0, int m0, int m1, int m2, int n0, int n1, int n2,
                               unsigned long long& my_contr) {
    using C = CT<MIXED>;
    using cx = typename C::T;
    const DevSys& S = p.S;
    const DevIfc& F = p.F;
    const int nb = S.nb, nb2 = nb * nb, npi = F.npi;
    cx* Z = reinterpret_cast<cx*>(smem + L.z);
    const double2* kap = reinterpret_cast<const double2*>(smem + L.kap);
    const cx* PT = reinterpret_cast<const cx*>(smem + L.pt);
    double* racc = reinterpret_cast<double*>(smem + L.racc);
    double* wacc = reinterpret_cast<double*>(smem + L.wacc);
    int* cnt = reinterpret_cast<int*>(smem + L.cnt);
    int* pre = reinterpret_cast<int*>(smem + L.pre);
    const int4* blkinfo = reinterpret_cast<const int4*>(smem + L.blk);
    const int nbk = reinterpret_cast<const int*>(smem + L.misc)[3];
    const double* wvw = reinterpret_cast<const double*>(S.wv) + 3;
    if (threadIdx.x == 0) {
        int acc = 0, built = 0;
        for (int i = 0; i < nb; i++) {
            int bi = 0;
            for (int j = 0; j < nb; j++) {
                pre[i * nb + j] = acc;
                const int n = min(cnt[i * nb + j], p.subcap);
                acc += n;
                bi += n;
            }
            built += (bi > 0);
        }
        pre[nb2] = acc;
        if (built) atomicAdd(&p.stats[4], (unsigned long long)built);
    }
    __syncthreads();
    const int tot = pre[nb2];
    if (tot > 0) {
        for (int idx = threadIdx.x; idx < nb2 * npi * 9; idx += blockDim.x) {
            const int bin = idx / (npi * 9);
            if (cnt[bin] == 0) continue;
            const int rem = idx - bin * (npi * 9), pc = rem / 9, sr = rem - pc * 9;
            const int i = bin / nb, j = bin - i * nb;
            Z[idx] = C::from(k4_z_entry(S, F, kap, ch, q0, ii, i, j, pc, sr));
        }
        __syncthreads();
        double accr[NT], accw[NT];
#pragma unroll
        for (int t = 0; t < NT; t++) {
            accr[t] = 0.0;
            accw[t] = 0.0;
        }
        // each thread loads its next queue entry one iteration ahead
        int bin_n = 0, cur_i = -1;
        double omega = 0.0;
        unsigned long long ent_n = 0;
        double sig_n = 0.0;
        if ((int)threadIdx.x < tot) {
            while (pre[bin_n + 1] <= (int)threadIdx.x) bin_n++;
            const size_t q1 = (size_t)bin_n * p.subcap + (threadIdx.x - pre[bin_n]);
            ent_n = qbase[q1];
            sig_n = qsig[q1];
        }
        for (int e = threadIdx.x; e < tot; e += blockDim.x) {
            const int bin = bin_n;
            const unsigned long long ent_c = ent_n;
            const double sig_c = sig_n;
            const int e2 = e + blockDim.x;
            if (e2 < tot) {
                while (pre[bin_n + 1] <= e2) bin_n++;
                const size_t q2 = (size_t)bin_n * p.subcap + (e2 - pre[bin_n]);
                ent_n = qbase[q2];
                sig_n = qsig[q2];
            }
            const int i = bin / nb, j = bin - i * nb;
            if (i != cur_i) {
                if (cur_i >= 0) {
#pragma unroll
                    for (int t = 0; t < NT; t++) {
                        if (t < p.nT) {
                            atomicAdd(&racc[cur_i * NT + t], accr[t]);
                            atomicAdd(&wacc[cur_i * NT + t], accw[t]);
                        }
                        accr[t] = 0.0;
                        accw[t] = 0.0;
                    }
                }
                cur_i = i;
                omega = wvw[4 * (q0 * nb + i)];
            }
            const size_t qi = (size_t)bin * p.subcap + (e - pre[bin]);
            k4_entry<NT, MIXED, LIST>(p, Z + (size_t)bin * npi * 9, PT, blkinfo, nbk, ent_c, sig_c,
                                      LIST ? qpos[qi] : 0, ch, ii, i, j, omega, m0, m1, m2, n0, n1, n2, accr, accw);
            my_contr++;
        }
        if (cur_i >= 0) {
#pragma unroll
            for (int t = 0; t < NT; t++)
                if (t < p.nT) {
                    atomicAdd(&racc[cur_i * NT + t], accr[t]);
                    atomicAdd(&wacc[cur_i * NT + t], accw[t]);
                }
        }
    }
    __syncthreads();
    for (int x = threadIdx.x; x < nb2; x += blockDim.x) cnt[x] = 0;
    __syncthreads();
}

// ---------------------------------------------------------------------------- tensor-core phase B
// 16 bytes (8 bf16 values, k = kb..kb+7) of row n of pass `pass` of a bin's B
// table: n runs over the pass's blocks (32 columns each: re(Z[sr]) at sr,
// im(Z[sr]) at 9+sr) and k over its classes (6 values each, see TcPlan); zero
// outside the class's own block.
__device__ __forceinline__ uint4 tc_b_chunk(const TcPlan* P, const double2* Zs, int npi, int slot, int pass, int n,
                                            int kb) {
    const int lb = n >> 5, nn = n & 31;
    const int4 bk = P->blk[P->pass_blk0[pass] + lb];
    const int c0 = P->pass_cls0[pass];
    const int cls_lo = c0 + kb / 6, cls_hi = c0 + (kb + 7) / 6;
    uint32_t w4[4] = {0, 0, 0, 0};
    if (nn < 18 && cls_hi >= bk.x && cls_lo < bk.y) {
        const int ro = nn >= 9, sr = nn - 9 * ro;
#pragma unroll
        for (int y = 0; y < 8; y++) {
            const int k = kb + y, cls = c0 + k / 6;
            if (cls < bk.x || cls >= bk.y) continue;
            const int r6 = k - (k / 6) * 6, split = r6 >> 1, ri = r6 & 1;
            const double2 z = Zs[((size_t)slot * npi + cls) * 9 + sr];
            // the product's real (ro = 0) or imaginary (ro = 1) part takes, from A's
            // (re, im) pair of w: (Z.re, -Z.im) or (Z.im, Z.re)
            const double v = (ri == 0) ? (ro == 0 ? z.x : z.y) : (ro == 0 ? -z.y : z.x);
            uint16_t hi, lo;
            tc::split_bf16(v, hi, lo);
            w4[y >> 1] |= (uint32_t)(split == 1 ? lo : hi) << (16 * (y & 1));
        }
    }
    return make_uint4(w4[0], w4[1], w4[2], w4[3]);
}

// Phase B on the tensor cores (mixed precision, RTA): the queued processes of
// each (i,j) bin are contracted 128 at a time.  Row m of the A tile holds the
// bf16 hi/lo Bloch phases w_p(q'') of process m (a copy of its q'' row of the
// phase table); the bin's B table holds the bf16 hi/lo split of
// Z_p^{(ij)}[s][r], block-diagonal over the atom-pair blocks.  One product per
// pass gives, in TMEM, T_b[s][r] = sum_{p in b} w_p Z_p[s][r] for every block b
// of the pass, and the epilogue forms V = sum_b u_b^T T_b v_b with u_b the
// eigenvector of the third phonon on atom a3 of block b (conjugated for the +-
// and -- channels) and v_b the conjugated eigenvector of the fourth on atom a4.
// Each warpgroup owns one A tile, one eigenvector stage, one mbarrier and one
// 128-column TMEM region and takes every other chunk of the group's bins.  A
// chunk first issues all its global loads (the phase rows into the A tile, the
// two eigenvector rows into the stage, the (omega, Bose) records) and forms
// the FP64 weights; the entry of the warpgroup's next chunk is loaded while
// the current one runs.  Rate sums stay in registers until the branch i of
// the chunks changes.
template <int NT>
__device__ void k4_phase_b_tc(const P4Params& p, unsigned char* smem, const Layout& L, const TcLayout& TL,
                              const unsigned long long* qbase, const double* qsig, int ch, int ii, int q0,
                              unsigned long long& my_contr) {
    const DevSys& S = p.S;
    const DevIfc& F = p.F;
    const TcPlan* P = reinterpret_cast<const TcPlan*>(smem + TL.plan);
    const int nb = S.nb, nb2 = nb * nb, npi = F.npi;
    const double2* kap = reinterpret_cast<const double2*>(smem + L.kap);
    double* racc = reinterpret_cast<double*>(smem + L.racc);
    double* wacc = reinterpret_cast<double*>(smem + L.wacc);
    int* cnt = reinterpret_cast<int*>(smem + L.cnt);
    int* misc = reinterpret_cast<int*>(smem + L.misc);
    unsigned char* Abuf = smem + TL.a;
    unsigned char* Bbuf = smem + TL.b;
    double2* Zs = reinterpret_cast<double2*>(smem + TL.zs);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TL.bar);
    uint32_t* slotw = reinterpret_cast<uint32_t*>(smem + TL.slot);  // [0] TMEM base, [1+g] parity of mbarrier g
    int* gbin = reinterpret_cast<int*>(smem + TL.gbin);
    int* chunks = reinterpret_cast<int*>(smem + TL.chunk);
    const int zbins = P->zbins, npass = P->npass, ksteps = P->ksteps, bin_bytes = P->bin_bytes;
    const int wg = threadIdx.x >> 7, m = threadIdx.x & 127, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t tbase = slotw[0];
    const uint32_t tregion = tbase + (uint32_t)(wg * kTcRegionCols) + ((uint32_t)((warp & 3) * 32) << 16);
    uint32_t par = slotw[1 + wg];
    const double* wvw = reinterpret_cast<const double*>(S.wv) + 3;
    const uint4* wrows = reinterpret_cast<const uint4*>(p.wtab + (size_t)(ch != 0) * S.nptk * ksteps * 16);
    unsigned char* Aw = Abuf + (size_t)wg * ksteps * kTcRows * 32;
    // this thread's two eigenvector rows: e''_k then e'''_l (nb components each)
    // (rows 2*nb+1 float2 apart: an odd stride in 8-byte words keeps the warp's accesses on distinct banks)
    float2* est = reinterpret_cast<float2*>(smem + TL.eig) + ((size_t)wg * kTcRows + m) * (2 * nb + 1);
    const double sqrtpi = sqrt(3.141592653589793238);
    const double floor_sigma = (double)0.001f;
    constexpr int WS = wb_stride(NT);
    // the warpgroup's running rate sums of branch cur_i
    int cur_i = -1;
    double accr[NT], accw[NT];
#pragma unroll
    for (int t = 0; t < NT; t++) {
        accr[t] = 0.0;
        accw[t] = 0.0;
    }
    auto flush_acc = [&]() {  // warp-uniform: every thread of the warpgroup calls it at the same chunk
#pragma unroll
        for (int t = 0; t < NT; t++) {
            double r = accr[t], w = accw[t];
            for (int o = 16; o > 0; o >>= 1) {
                r += __shfl_down_sync(0xffffffffu, r, o);
                w += __shfl_down_sync(0xffffffffu, w, o);
            }
            if (lane == 0 && t < p.nT && cur_i >= 0) {
                atomicAdd(&racc[cur_i * NT + t], r);
                atomicAdd(&wacc[cur_i * NT + t], w);
            }
            accr[t] = 0.0;
            accw[t] = 0.0;
        }
    };
    if (threadIdx.x == 0) misc[4] = 0;
    __syncthreads();
    for (;;) {
        // the next group: up to zbins non-empty bins and their chunks of kTcRows processes
        if (threadIdx.x == 0) {
            int b = misc[4], ng = 0, nc = 0;
            while (b < nb2 && ng < zbins) {
                const int n = min(cnt[b], p.subcap);
                if (n > 0) {
                    gbin[ng] = b;
                    for (int e = 0; e < n; e += kTcRows) chunks[nc++] = (ng << 16) | (e / kTcRows);
                    ng++;
                }
                b++;
            }
            misc[4] = b;
            misc[5] = ng;
            misc[6] = nc;
            if (ng) atomicAdd(&p.stats[5], (unsigned long long)ng);
        }
        __syncthreads();
        const int ng = misc[5], nc = misc[6];
        if (ng == 0 || misc[7]) break;
        const long long tg0 = clock64();
        // FP64 reciprocal cluster entries of the group's bins
        for (int idx = threadIdx.x; idx < ng * npi * 9; idx += blockDim.x) {
            const int slot = idx / (npi * 9), rem = idx - slot * (npi * 9), pc = rem / 9, sr = rem - pc * 9;
            const int bin = gbin[slot], i = bin / nb, j = bin - i * nb;
            Zs[idx] = k4_z_entry(S, F, kap, ch, q0, ii, i, j, pc, sr);
        }
        __syncthreads();
        // their B tables, 16 bytes (8 values of one row n) per store
        const int chunks16 = bin_bytes >> 4;
        for (int idx = threadIdx.x; idx < ng * chunks16; idx += blockDim.x) {
            const int slot = idx / chunks16;
            const int off = (idx - slot * chunks16) << 4;
            int pass = 0;
            while (pass + 1 < npass && P->pass_boff[pass + 1] <= off) pass++;
            const int rel = off - P->pass_boff[pass];
            const int N = 32 * (P->pass_blk0[pass + 1] - P->pass_blk0[pass]);
            const int s = rel / (N * 32), within = rel - s * (N * 32);
            const int n = (within >> 8) * 8 + ((within >> 4) & 7);
            const int kb = s * 16 + ((within >> 7) & 1) * 8;
            *reinterpret_cast<uint4*>(Bbuf + (size_t)slot * bin_bytes + off) = tc_b_chunk(P, Zs, npi, slot, pass, n, kb);
        }
        tc::fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) atomicAdd(&p.stats[10], (unsigned long long)(clock64() - tg0));
        // the chunks: warpgroup wg takes chunks wg, wg+2, ...
        unsigned long long ent_n = 0;
        double sig_n = 0.0;
        auto load_entry = [&](int c) {
            if (c < nc) {
                const int code = chunks[c];
                const int bin = gbin[code >> 16], e0 = (code & 0xffff) * kTcRows;
                if (m < min(cnt[bin], p.subcap) - e0) {
                    const size_t qi = (size_t)bin * p.subcap + e0 + m;
                    ent_n = qbase[qi];
                    sig_n = qsig[qi];
                }
            }
        };
        load_entry(wg);
        for (int c = wg; c < nc; c += 2) {
            const long long tc0 = clock64();
            const int code = chunks[c];
            const int slot = code >> 16, e0 = (code & 0xffff) * kTcRows;
            const int bin = gbin[slot], i = bin / nb, j = bin - i * nb;
            const int n = min(cnt[bin], p.subcap) - e0;
            const bool valid = m < n;
            const unsigned long long ent = ent_n;
            double sig = sig_n;
            load_entry(c + 2);
            if (i != cur_i) {
                flush_acc();
                cur_i = i;
            }
            int a = 0, b = 0, cc = 0, ss = 0, k = 0, l = 0, jj = 0;
            double wts[NT];
#pragma unroll
            for (int t = 0; t < NT; t++) wts[t] = 0.0;
            if (valid) {
                unpack_proc(ent, a, b, cc, ss, k, l);
                jj = q_index(S, a, b, cc);
                // A row m: the phase row of q''; the two eigenvector rows into the stage.
                // Asynchronous copies: all in flight at once while the weights are formed.
                const uint4* src = wrows + (size_t)jj * ksteps * 2;
                for (int x = 0; x < 2 * ksteps; x++)
                    tc::cp_async16(Aw + (size_t)(x >> 1) * (kTcRows * 32) + tc::kmajor_offset(m, (x & 1) * 8), src + x);
                const float2* e2 = S.eigf + (size_t)(jj * nb + k) * nb;
                const float2* e3 = S.eigf + (size_t)(ss * nb + l) * nb;
                for (int x = 0; x < nb; x++) {
                    tc::cp_async8(est + x, e2 + x);
                    tc::cp_async8(est + nb + x, e3 + x);
                }
                // FP64 weights of every temperature
                const double* x1 = p.wb + (size_t)(ii * nb + j) * WS;
                const double* x2 = p.wb + (size_t)(jj * nb + k) * WS;
                const double* x3 = p.wb + (size_t)(ss * nb + l) * WS;
                const double omega = wvw[4 * (q0 * nb + i)];
                const double w1 = x1[0], w2 = x2[0], w3 = x3[0];
                const double sv = (ch == 2) ? __dadd_rn(omega, -w1) : __dadd_rn(omega, w1);
                const double delta =
                    (ch == 0) ? __dadd_rn(__dadd_rn(sv, w2), -w3) : __dadd_rn(__dadd_rn(sv, -w2), -w3);
                if (sig <= floor_sigma) sig = 1.0 / sqrtpi;
                const double g = exp(-(delta * delta) / (sig * sig));
                const double base = g / (sig * sqrtpi * (omega * w1 * w2 * w3));
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    if (t < p.nT) {
                        const double f1 = x1[1 + t], f2 = x2[1 + t], f3 = x3[1 + t];
                        double bc;
                        if (ch == 0)
                            bc = f1 * f2 * (1 + f3) - (1 + f1) * (1 + f2) * f3;
                        else if (ch == 1)
                            bc = f1 * (1 + f2) * (1 + f3) - (1 + f1) * f2 * f3;
                        else
                            bc = (1 + f1) * (1 + f2) * (1 + f3) - f1 * f2 * f3;
                        wts[t] = bc * base;
                    }
                }
                tc::cp_async_wait_all();
            }
            tc::fence_async_smem();
            tc::fence_before_sync();
            tc::named_sync(1 + wg, kTcRows);
            const long long tc1 = clock64();
            long long tc2 = tc1;
            float2 V = make_float2(0.f, 0.f);
            bool ok = true;
            for (int pass = 0; pass < npass; pass++) {
                if (m == 0) {
                    tc::fence_after_sync();
                    const int N = 32 * (P->pass_blk0[pass + 1] - P->pass_blk0[pass]);
                    const uint32_t idesc = tc::idesc_bf16_f32(N);
                    const int ks0 = P->pass_kstep0[pass], ksn = P->pass_kstep0[pass + 1] - ks0;
                    const uint32_t aaddr = tc::smem_u32(Aw) + (uint32_t)ks0 * (kTcRows * 32);
                    const uint32_t baddr = tc::smem_u32(Bbuf + (size_t)slot * bin_bytes + P->pass_boff[pass]);
                    for (int x = 0; x < ksn; x++)
                        tc::mma_bf16(tbase + (uint32_t)(wg * kTcRegionCols), tc::smem_desc(aaddr + x * (kTcRows * 32)),
                                     tc::smem_desc(baddr + x * N * 32), idesc, x > 0);
                    tc::commit(tc::smem_u32(&bars[wg]));
                    atomicAdd(&p.stats[6], (unsigned long long)(ksn * (N / 16)));
                }
                const bool done = tc::mbar_wait(tc::smem_u32(&bars[wg]), par);
                ok = tc::named_all(1 + wg, kTcRows, done);
                if (!ok) break;  // par stays the parity of the product still pending
                par ^= 1u;
                if (pass == 0) tc2 = clock64();
                tc::fence_after_sync();
                for (int bl = P->pass_blk0[pass]; bl < P->pass_blk0[pass + 1]; bl++) {
                    const uint32_t col = (uint32_t)((bl - P->pass_blk0[pass]) * 32);
                    float T0[16], T1[16];
                    tc::ld16(tregion + col, T0);
                    tc::ld16(tregion + col + 16, T1);
                    tc::ld_wait();
                    if (valid) {
                        const int4 bk = P->blk[bl];
                        float2 u[3], v[3];
#pragma unroll
                        for (int x = 0; x < 3; x++) {
                            u[x] = est[3 * bk.z + x];
                            if (ch != 0) u[x] = cconjf(u[x]);
                            v[x] = cconjf(est[nb + 3 * bk.w + x]);
                        }
                        float2 tt = make_float2(0.f, 0.f);
#pragma unroll
                        for (int x = 0; x < 3; x++) {
                            float2 h = make_float2(0.f, 0.f);
#pragma unroll
                            for (int r = 0; r < 3; r++) {
                                const int sr = x * 3 + r;
                                const float im = (sr < 7) ? T0[9 + sr] : T1[sr - 7];
                                h = cmacf(h, make_float2(T0[sr], im), v[r]);
                            }
                            tt = cmacf(tt, u[x], h);
                        }
                        V.x += tt.x;
                        V.y += tt.y;
                    }
                }
                tc::fence_before_sync();
                if (pass + 1 < npass) tc::named_sync(1 + wg, kTcRows);
            }
            if (!ok) {
                if (m == 0) {
                    atomicOr(p.err, kErrTimeout);
                    misc[7] = 1;
                }
                break;
            }
            if (valid) {
                const double v2 = (double)V.x * (double)V.x + (double)V.y * (double)V.y;
#pragma unroll
                for (int t = 0; t < NT; t++) {
                    accr[t] = fma(wts[t], v2, accr[t]);
                    accw[t] += wts[t];
                }
                my_contr++;
            }
            if (m == 0) {  // cycles of this chunk: gather and weights, product, epilogue
                const long long tc3 = clock64();
                atomicAdd(&p.stats[11], (unsigned long long)(tc1 - tc0));
                atomicAdd(&p.stats[12], (unsigned long long)(tc2 - tc1));
                atomicAdd(&p.stats[13], (unsigned long long)(tc3 - tc2));
            }
        }
        if (m == 0) slotw[1 + wg] = par;
        __syncthreads();
    }
    flush_acc();
    for (int x = threadIdx.x; x < nb2; x += blockDim.x) cnt[x] = 0;
    __syncthreads();
}

template <int NT, bool MIXED, bool LIST, bool TC>
__device__ __forceinline__ void k4_flush_body(const P4Params& p, unsigned char* smem, const Layout& L,
                                              const unsigned long long* qbase, const double* qsig, const long long* qpos,
                                              int ch, int ii, int q0, int m0, int m1, int m2, int n0, int n1, int n2,
                                              unsigned long long& my_contr) {
    if constexpr (TC) {
        const TcPlan* P = p.tc;
        const Layout Lb = k4_layout_tcbase(NT, p.S.nb, p.F.npi, p.F.ntri, p.S.n[0] + p.S.n[1] + p.S.n[2], p.S.nptk);
        const TcLayout TL = k4_tc_layout(Lb.total, P->ksteps, P->bin_bytes, P->zbins, p.F.npi, P->chunk_cap, p.S.nb);
        k4_phase_b_tc<NT>(p, smem, L, TL, qbase, qsig, ch, ii, q0, my_contr);
    } else if (L.allz) {
        k4_phase_b_all<NT, MIXED, LIST>(p, smem, L, qbase, qsig, qpos, ch, ii, q0, m0, m1, m2, n0, n1, n2, my_contr);
    } else {
        k4_phase_b<NT, MIXED, LIST>(p, smem, L, qbase, qsig, qpos, ch, ii, q0, m0, m1, m2, n0, n1, n2, my_contr);
    }
}

template <int NT, bool MIXED, bool LIST, bool TC>
__device__ __forceinline__ void k4_flush(const P4Params& p, unsigned char* smem, const Layout& L,
                                         const unsigned long long* qbase, const double* qsig, const long long* qpos,
                                         int ch, int ii, int q0, int m0, int m1, int m2, int n0, int n1, int n2,
                                         unsigned long long& my_contr) {
    const long long t0 = clock64();  // thread 0 adds the CTA's cycles in phase B to stats[9]
    k4_flush_body<NT, MIXED, LIST, TC>(p, smem, L, qbase, qsig, qpos, ch, ii, q0, m0, m1, m2, n0, n1, n2, my_contr);
    if (threadIdx.x == 0) atomicAdd(&p.stats[9], (unsigned long long)(clock64() - t0));
}

// True (for the whole CTA) when some (i,j) queue could overflow within the next
// kCheckEvery passes of at most one new entry per thread.  The barrier first
// makes every thread's earlier appends visible: between checks the warps of the
// CTA drift apart by up to kCheckEvery passes, so without it the counts read
// here could be short by that many passes and a queue could overflow.
__device__ __forceinline__ bool queue_nearly_full(const P4Params& p, const int* cnt, int nb2, int* misc) {
    __syncthreads();
    if (threadIdx.x < 32) {  // the largest bin count, over the lanes of warp 0
        int mx = 0;
        for (int b = threadIdx.x; b < nb2; b += 32) mx = max(mx, cnt[b]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (threadIdx.x == 0) misc[2] = (mx > p.subcap - kCheckEvery * (int)blockDim.x);
    }
    __syncthreads();
    return misc[2] != 0;
}

// Ind_driver_4ph work item: instead of enumerating, read the processes of q' = ii
// from the channel's ordered lists (one contiguous segment per branch i, found by
// bisection: the lists are ordered by q' within each mode) and queue them with
// their list positions; phase B then stores each Gamma in place.  Entries that are
// out of range or break momentum conservation raise kErrList and are skipped.
template <int NT, bool MIXED>
__device__ void k4_list_segment(const P4Params& p, unsigned char* smem, const Layout& L, unsigned long long* qbase,
                                double* qsig, long long* qpos, int ch, int ii, int ll, int q0, int m0, int m1, int m2,
                                int n0, int n1, int n2, unsigned long long& my_surv, unsigned long long& my_contr) {
    const DevSys& S = p.S;
    const int nb = S.nb, nb2 = nb * nb, nptk = S.nptk;
    const int N0 = S.n[0], N1 = S.n[1], N2 = S.n[2];
    long long* seglo = reinterpret_cast<long long*>(smem + L.seg);
    long long* segpre = seglo + nb;
    int* cnt = reinterpret_cast<int*>(smem + L.cnt);
    int* misc = reinterpret_cast<int*>(smem + L.misc);
    const long long* I2 = p.lind2[ch];
    const long long* I3 = p.lind3[ch];
    const long long* I4 = p.lind4[ch];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        const int mm = ll * nb + i;
        const long long o = p.list_off[ch][mm], n = p.list_n[ch][mm];
        long long lo = o, hi = o + n;
        while (lo < hi) {  // first entry with q' >= ii
            const long long mid = (lo + hi) >> 1;
            if ((I2[mid] - 1) / nb < ii) lo = mid + 1; else hi = mid;
        }
        const long long a = lo;
        hi = o + n;
        while (lo < hi) {  // first entry with q' > ii
            const long long mid = (lo + hi) >> 1;
            if ((I2[mid] - 1) / nb <= ii) lo = mid + 1; else hi = mid;
        }
        seglo[i] = a;
        segpre[i + 1] = lo - a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        segpre[0] = 0;
        for (int i = 0; i < nb; i++) segpre[i + 1] += segpre[i];
    }
    __syncthreads();
    const long long total = segpre[nb];
    const long long lim = (long long)nptk * nb;
    int iter = 0;
    for (long long base = 0; base < total; base += blockDim.x, iter++) {
        if ((iter % kCheckEvery) == 0 && queue_nearly_full(p, cnt, nb2, misc))
            k4_flush<NT, MIXED, true, false>(p, smem, L, qbase, qsig, qpos, ch, ii, q0, m0, m1, m2, n0, n1, n2, my_contr);
        const long long e = base + threadIdx.x;
        if (e >= total) continue;
        int i = 0;
        while (i + 1 < nb && segpre[i + 1] <= e) i++;
        const long long pos = seglo[i] + (e - segpre[i]);
        const long long x2 = I2[pos] - 1, x3 = I3[pos] - 1, x4 = I4[pos] - 1;
        bool ok = x2 >= 0 && x2 < lim && x3 >= 0 && x3 < lim && x4 >= 0 && x4 < lim && x2 / nb == ii;
        const int j = (int)(x2 % nb), jj = (int)(x3 / nb), k = (int)(x3 % nb), ss = (int)(x4 / nb), l = (int)(x4 % nb);
        int a = 0, b = 0, c = 0;
        if (ok) {
            q_coords_t(S, jj, a, b, c);
            int t0, t1, t2;
            if (ch == 0) {
                t0 = n0 + m0 + a; t1 = n1 + m1 + b; t2 = n2 + m2 + c;
            } else if (ch == 1) {
                t0 = n0 + m0 - a; t1 = n1 + m1 - b; t2 = n2 + m2 - c;
            } else {
                t0 = n0 - m0 - a; t1 = n1 - m1 - b; t2 = n2 - m2 - c;
            }
            ok = q_index(S, wrapN(t0, N0), wrapN(t1, N1), wrapN(t2, N2)) == ss;
        }
        if (!ok) {
            atomicOr(p.err, kErrList);
            continue;
        }
        my_surv++;
        const double w1 = S.wv[ii * nb + j].w;
        const double4 w2 = S.wv[jj * nb + k];
        const double4 w3 = S.wv[ss * nb + l];
        if (w1 <= 1.25 || w2.w <= 1.25 || w3.w <= 1.25) continue;  // WP4 = 0, Gamma = 0 (output pre-zeroed)
        const int idx = i * nb + j;
        const int qp = atomicAdd(&cnt[idx], 1);
        if (qp >= p.subcap) {  // cannot happen with the capacity checks; never write past the bin
            atomicOr(p.err, kErrQueue);
            continue;
        }
        const size_t qi = (size_t)idx * p.subcap + qp;
        qbase[qi] = pack_proc(a, b, c, ss, k, l);
        qsig[qi] = sigma_exact(S, w2, w3);
        qpos[qi] = pos;
    }
    __syncthreads();
    k4_flush<NT, MIXED, true, false>(p, smem, L, qbase, qsig, qpos, ch, ii, q0, m0, m1, m2, n0, n1, n2, my_contr);
}

// Per-thread work counters of one kernel, flushed into a P4Params::stats array.
struct K4Stats {
    unsigned long long surv, contr, sig, cand;
};

__device__ __forceinline__ void k4_flush_stats(unsigned long long* stats, K4Stats& st, double* red) {
    double v[4] = {(double)st.surv, (double)st.contr, (double)st.sig, (double)st.cand};
    block_sum_vec<4>(v, red);
    if (threadIdx.x == 0) {
        atomicAdd(&stats[0], (unsigned long long)v[0]);
        atomicAdd(&stats[1], (unsigned long long)v[1]);
        atomicAdd(&stats[2], (unsigned long long)v[2]);
        atomicAdd(&stats[3], (unsigned long long)v[3]);
    }
    st = K4Stats{0, 0, 0, 0};
}

// The q'' >= jj_lo (in order) whose q''' = q +- q' - q'' (channel ch) is >= q'': an
// ordered block-wide compaction into list; returns the count (the same in every thread).
__device__ int k4_jj_list(const DevSys& S, int ch, int jj_lo, int n0, int n1, int n2, int m0, int m1, int m2,
                          unsigned short* list, int* wcnt) {
    const int n = S.nptk - jj_lo;
    const int chunk = (n + blockDim.x - 1) / blockDim.x;
    const int x0 = min(n, (int)threadIdx.x * chunk), x1 = min(n, x0 + chunk);
    auto keep = [&](int x) {
        const int jj = jj_lo + x;
        int a, b, c;
        q_coords_t(S, jj, a, b, c);
        const int t0 = (ch == 1) ? n0 + m0 - a : n0 - m0 - a;
        const int t1 = (ch == 1) ? n1 + m1 - b : n1 - m1 - b;
        const int t2 = (ch == 1) ? n2 + m2 - c : n2 - m2 - c;
        return q_index(S, wrapN(t0, S.n[0]), wrapN(t1, S.n[1]), wrapN(t2, S.n[2])) >= jj;
    };
    int cnt = 0;
    for (int x = x0; x < x1; x++) cnt += keep(x);
    // exclusive prefix of the per-thread counts over the block, in thread order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = cnt;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wcnt[warp] = inc;
    __syncthreads();
    int off = inc - cnt, total = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
        if (w < warp) off += wcnt[w];
        total += wcnt[w];
    }
    for (int x = x0; x < x1; x++)
        if (keep(x)) list[off++] = (unsigned short)(jj_lo + x);
    __syncthreads();
    return total;
}

// Per-CTA tables of one solve: (k,l) decode table, non-empty class blocks and
// per-class phase tables.
template <int KIND, bool MIXED>
__device__ void k4_cta_init(const P4Params& p, unsigned char* smem, const Layout& L) {
    using C = CT<MIXED>;
    using cx = typename C::T;
    const DevSys& S = p.S;
    const DevIfc& F = p.F;
    const int nb = S.nb, nb2 = nb * nb, npi = F.npi;
    const int N0 = S.n[0], N1 = S.n[1], N2 = S.n[2], lsum = N0 + N1 + N2;
    cx* PT = reinterpret_cast<cx*>(smem + L.pt);
    int* klt = reinterpret_cast<int*>(smem + L.klt);
    int* misc = reinterpret_cast<int*>(smem + L.misc);
    for (int x = threadIdx.x; x < nb2; x += blockDim.x) klt[x] = ((x / nb) << 8) | (x % nb);
    if (threadIdx.x == 0) {
        int4* blkinfo = reinterpret_cast<int4*>(smem + L.blk);
        int nbk = 0;
        if (KIND >= 2)
            for (int b = 0; b < F.nblk; b++)
                if (F.blk_start[b] < F.blk_start[b + 1])
                    blkinfo[nbk++] = make_int4(F.blk_start[b], F.blk_start[b + 1], b / S.natoms, b % S.natoms);
        misc[3] = nbk;
    }
    if (KIND >= 2) {
        for (int x = threadIdx.x; x < npi * lsum; x += blockDim.x) {
            int pc = x / lsum, r = x % lsum;
            int d = (r < N0) ? 0 : (r < N0 + N1 ? 1 : 2);
            int xi = r - (d == 0 ? 0 : (d == 1 ? N0 : N0 + N1));
            int4 D = F.pi_d[pc];
            int Dd = (d == 0) ? D.x : (d == 1 ? D.y : D.z);
            PT[x] = C::from(S.root[d][pmod(xi * Dd, S.n[d])]);
        }
    }
    __syncthreads();

}

// One work item (q = List(ll), q', channel) of one solve.  TC: phase B on the
// tensor cores (RTA, mixed precision).
template <int KIND, int NT, bool MIXED, bool TC = false>
__device__ __forceinline__ void k4_item(const P4Params& p, unsigned char* smem, const Layout& L, int wi,
                                        unsigned long long* qbase, double* qsig, long long* qpos, K4Stats& st) {
    const DevSys& S = p.S;
    const DevIfc& F = p.F;
    const int nb = S.nb, nptk = S.nptk, nb2 = nb * nb;
    const int N0 = S.n[0], N1 = S.n[1], N2 = S.n[2];
    double2* kap = reinterpret_cast<double2*>(smem + L.kap);
    double* sval = reinterpret_cast<double*>(smem + L.sval);
    double* swj = reinterpret_cast<double*>(smem + L.swj);
    double* racc = reinterpret_cast<double*>(smem + L.racc);
    double* wacc = reinterpret_cast<double*>(smem + L.wacc);
    double* pacc = reinterpret_cast<double*>(smem + L.pacc);
    int* sidx = reinterpret_cast<int*>(smem + L.sidx);
    int* cnt = reinterpret_cast<int*>(smem + L.cnt);
    int* ncnt = reinterpret_cast<int*>(smem + L.ncnt);
    int* klt = reinterpret_cast<int*>(smem + L.klt);
    int* misc = reinterpret_cast<int*>(smem + L.misc);
    constexpr bool LIST = (KIND == 3);
    const double sqrtpi = sqrt(3.141592653589793238);
    const double floor_sigma = (double)0.001f;
    unsigned long long& my_surv = st.surv;
    unsigned long long& my_contr = st.contr;
    unsigned long long& my_sig = st.sig;
    unsigned long long& my_cand = st.cand;
    const long long t_item = clock64();  // thread 0 adds the CTA's cycles per work item to stats[8]
    const int ch = wi % 3;
    const int rest = wi / 3;
    const int ii = rest % nptk, ll = rest / nptk;
    const int q0 = S.list0[ll];
    int n0, n1, n2, m0, m1, m2;
    q_coords_t(S, q0, n0, n1, n2);
    q_coords_t(S, ii, m0, m1, m2);
    // sorted branch sums s_ij = w_i +- w'_j over the valid pairs
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
            sval[rank] = s;
            swj[rank] = wj_;
            sidx[rank] = (i << 16) | j;  // the pair itself: no division by nb in the window loop
        }
        if (idx == 0) {
            misc[1] = nvalid;
            misc[2] = 0;  // no bin near its capacity
        }
        cnt[idx] = 0;
    }
    for (int x = threadIdx.x; x < nb * (KIND == 0 ? kThreads / 32 : 1); x += blockDim.x) {
        ncnt[x] = 0;
        pacc[x] = 0.0;
    }
    for (int x = threadIdx.x; x < nb * NT; x += blockDim.x) {
        racc[x] = 0.0;
        wacc[x] = 0.0;
    }
    if (KIND >= 2) {
        // kappa_c = mu_c exp(2 pi i (-n.m_l +- n'.(m_j - m_l))/N)
        for (int c = threadIdx.x; c < F.ntri; c += blockDim.x) {
            int4 mj = F.mj[c], ml = F.ml[c];
            double2 a = lattice_phase(S, n0, n1, n2, -ml.x, -ml.y, -ml.z);
            int sj = (ch == 2) ? -1 : 1;
            double2 b = lattice_phase(S, m0, m1, m2, sj * (mj.x - ml.x), sj * (mj.y - ml.y), sj * (mj.z - ml.z));
            double2 k = cmul(a, b);
            k.x *= F.mu[c];
            k.y *= F.mu[c];
            kap[c] = k;
        }
    }
    __syncthreads();
    const int ns = misc[1];
    if (KIND == 3) {
        k4_list_segment<NT, MIXED>(p, smem, L, qbase, qsig, qpos, ch, ii, ll, q0, m0, m1, m2, n0, n1, n2, my_surv,
                                   my_contr);
    } else if (ns > 0) {
        double smax = 0.0;
        for (int x = 0; x < ns; x++) smax = fmax(smax, fabs(sval[x]));
        const int jj_lo = (ch == 1) ? 0 : ii;
        // the +- and -- channels walk only the q'' whose q''' is not smaller
        const bool use_list = (ch != 0) && L.njjl >= nptk;
        const unsigned short* jjl = reinterpret_cast<const unsigned short*>(smem + L.jjl);
        const int nq = use_list ? k4_jj_list(S, ch, jj_lo, n0, n1, n2, m0, m1, m2,
                                             reinterpret_cast<unsigned short*>(smem + L.jjl),
                                             reinterpret_cast<int*>(smem + L.jjl + al16((size_t)L.njjl * 2)))
                                : nptk - jj_lo;
        const int total = nq * nb2;
        // thread t covers index base+t; keep (jj, kl) of it incrementally
        const int Bq = blockDim.x / nb2, Br = blockDim.x % nb2;
        int cj = threadIdx.x / nb2, ckl = threadIdx.x % nb2;
        int iter = 0;
        double4* stg = reinterpret_cast<double4*>(smem + L.stg);
        int4* stgi = reinterpret_cast<int4*>(smem + L.stgi);
        int stage_first = 0;
        for (int base = 0; base < total; base += blockDim.x, iter++) {
            if ((iter % L.stgp) == 0) {
                __syncthreads();
                // Queue capacity: an append that leaves a bin with fewer than stgp passes
                // of room (one entry per thread and pass) raises misc[2]; at this barrier
                // every thread sees the flag, and the queues are drained before the next
                // stgp passes, which cannot then overflow them.
                if (KIND == 2 && misc[2]) {
                    k4_flush<NT, MIXED, LIST, TC>(p, smem, L, qbase, qsig, qpos, ch, ii, q0, m0, m1, m2, n0, n1, n2,
                                                my_contr);
                    __syncthreads();  // every thread has read the flag
                    if (threadIdx.x == 0) misc[2] = 0;
                }
                // stage the points of the next stgp passes: their records, their partners and theirs
                stage_first = base / nb2;
                const int nslot = (min(total, base + L.stgp * (int)blockDim.x) - 1) / nb2 - stage_first + 1;
                for (int x = threadIdx.x; x < nslot * 2 * nb; x += blockDim.x) {
                    const int slot = x / (2 * nb), r = x - slot * 2 * nb;
                    const int cjs = stage_first + slot;
                    const int jj = use_list ? (int)jjl[cjs] : jj_lo + cjs;
                    int a, b, c;
                    q_coords_t(S, jj, a, b, c);
                    int t0, t1, t2;
                    if (ch == 0) {
                        t0 = n0 + m0 + a; t1 = n1 + m1 + b; t2 = n2 + m2 + c;
                    } else if (ch == 1) {
                        t0 = n0 + m0 - a; t1 = n1 + m1 - b; t2 = n2 + m2 - c;
                    } else {
                        t0 = n0 - m0 - a; t1 = n1 - m1 - b; t2 = n2 - m2 - c;
                    }
                    const int ss = q_index(S, wrapN(t0, N0), wrapN(t1, N1), wrapN(t2, N2));
                    stg[x] = (r < nb) ? S.wv[jj * nb + r] : S.wv[ss * nb + (r - nb)];
                    if (r == 0) stgi[slot] = make_int4(jj, a | (b << 8) | (c << 16), ss, 0);
                }
                __syncthreads();
            }
            // This lane's candidate (q'', k, l): sigma, and the window [lo, lo + n) of the
            // sorted sums that can pass the 1-sigma test.
            int n = 0, lo = 0, jj = 0;
            double w2w = 0.0, w3w = 0.0, sigma = 0.0;
            unsigned long long pk = 0;
            if (base + (int)threadIdx.x < total) {
                const int slot = cj - stage_first;
                const int4 si = stgi[slot];
                jj = si.x;
                const int ss = si.z;
                const int kl = klt[ckl];
                const int k = kl >> 8, l = kl & 0xff;
                bool go = true;
                if (ch != 0 && ss < jj) go = false;
                if (ch != 0 && ss == jj && l < k) go = false;
                if (go) {
                    const double4 w2 = stg[slot * 2 * nb + k];
                    const double4 w3 = stg[slot * 2 * nb + nb + l];
                    if (w2.w != 0.0 && w3.w != 0.0) {
                        sigma = sigma_exact(S, w2, w3);
                        my_sig++;
                        const double cen = (ch == 0) ? (w3.w - w2.w) : (w2.w + w3.w);
                        const double tol = 1e-12 * (1.0 + fabs(w2.w) + fabs(w3.w) + smax + sigma);
                        lo = lower_bound_desc(sval, ns, cen - sigma - tol);
                        n = max(0, upper_bound_desc(sval, ns, cen + sigma + tol) - lo);
                        w2w = w2.w;
                        w3w = w3.w;
                        pk = pack_proc(si.y & 0xff, (si.y >> 8) & 0xff, si.y >> 16, ss, k, l);
                    }
                }
            }
            // The windows differ in length from lane to lane.  Their entries are dealt
            // out over the warp's lanes (an inclusive scan of the lengths; entry e
            // belongs to the first lane whose prefix exceeds e), so the exact test and
            // the queue append run with every lane busy instead of for as many
            // iterations as the longest window.
            const int lane = threadIdx.x & 31;
            int incl = n;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += y;
            }
            const int wtot = __shfl_sync(0xffffffffu, incl, 31);
            for (int r0 = 0; r0 < wtot; r0 += 32) {
                const int e = r0 + lane;
                int src = 0;
#pragma unroll
                for (int step = 16; step > 0; step >>= 1)
                    if (__shfl_sync(0xffffffffu, incl, src + step - 1) <= e) src += step;
                const int x = __shfl_sync(0xffffffffu, lo - (incl - n), src) + e;
                const double ew2 = __shfl_sync(0xffffffffu, w2w, src);
                const double ew3 = __shfl_sync(0xffffffffu, w3w, src);
                const double esg = __shfl_sync(0xffffffffu, sigma, src);
                const unsigned long long epk = __shfl_sync(0xffffffffu, pk, src);
                const int ejj = __shfl_sync(0xffffffffu, jj, src);
                if (e >= wtot) continue;
                my_cand++;
                const double s = sval[x];
                const double delta = (ch == 0) ? __dadd_rn(__dadd_rn(s, ew2), -ew3)
                                               : __dadd_rn(__dadd_rn(s, -ew2), -ew3);
                if (!(fabs(delta) <= esg)) continue;
                const int ij = sidx[x];
                const int i = ij >> 16, j = ij & 0xffff;
                const int idx = i * nb + j;
                const int k = (int)((epk >> 8) & 0xff), l = (int)(epk & 0xff);
                const int ss = (int)((epk >> 16) & 0x3ffff);
                if (ch != 1 && ejj == ii && k < j) continue;
                if (ch == 1 && !((q0 != ejj || i != k) && (q0 != ss || i != l) && (ii != ejj || j != k) &&
                                 (ii != ss || j != l)))
                    continue;
                my_surv++;
                if (KIND == 0) {
                    const double sg = (esg <= floor_sigma) ? 1.0 / sqrtpi : esg;
                    const double pc = exp(-(delta * delta) / (sg * sg)) /
                                      (sg * sqrtpi * ((double)nptk * (double)nptk * (double)nptk) *
                                       (double)(nb * nb * nb * nb));
                    const int o = (threadIdx.x >> 5) * nb + i;
                    atomicAdd(&ncnt[o], 1);
                    atomicAdd(&pacc[o], pc);
                    continue;
                }
                const double w1 = swj[x];
                if (w1 <= 1.25 || ew2 <= 1.25 || ew3 <= 1.25) continue;  // WP4 = 0 exactly
                const int pos = atomicAdd(&cnt[idx], 1);
                if (pos >= p.subcap - L.stgp * (int)blockDim.x) misc[2] = 1;
                if (pos >= p.subcap) {  // cannot happen with the capacity checks
                    atomicOr(p.err, kErrQueue);
                    continue;
                }
                qbase[(size_t)idx * p.subcap + pos] = epk;
                qsig[(size_t)idx * p.subcap + pos] = esg;
            }
            ckl += Br;
            cj += Bq;
            if (ckl >= nb2) {
                ckl -= nb2;
                cj += 1;
            }
        }
        if (KIND == 2) {
            __syncthreads();
            k4_flush<NT, MIXED, LIST, TC>(p, smem, L, qbase, qsig, qpos, ch, ii, q0, m0, m1, m2, n0, n1, n2,
                                        my_contr);
        }
    }
    __syncthreads();
    if (KIND == 0) {
        for (int i = threadIdx.x; i < nb; i += blockDim.x) {
            unsigned long long n = 0;
            double ps = 0.0;
            for (int w = 0; w < kThreads / 32; w++) {  // fixed order over the warp copies
                n += (unsigned long long)ncnt[w * nb + i];
                ps += pacc[w * nb + i];
            }
            if (n) atomicAdd(&p.n_count[ch * S.nlist * nb + ll * nb + i], n);
            if (ps != 0.0) atomicAdd(&p.p_sum[ch * S.nlist * nb + ll * nb + i], ps);
        }
    } else {
        for (int idx = threadIdx.x; idx < nb * NT; idx += blockDim.x) {
            int i = idx / NT, t = idx % NT;
            if (t < p.nT) {
                p.part_rate[((size_t)wi * p.nT + t) * nb + i] = racc[idx];
                p.part_wp[((size_t)wi * p.nT + t) * nb + i] = wacc[idx];
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&p.stats[8], (unsigned long long)(clock64() - t_item));
}

template <int KIND, int NT, bool MIXED>
__global__ void __launch_bounds__(kThreads, (ctas_per_sm<KIND, NT, MIXED>())) k4_work(P4Params p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int nb2 = p.S.nb * p.S.nb;
    const Layout L = k4_layout(KIND, NT, MIXED, p.S.nb, p.F.npi, p.F.ntri, p.S.n[0] + p.S.n[1] + p.S.n[2], p.S.nptk);
    int* misc = reinterpret_cast<int*>(smem + L.misc);
    k4_cta_init<KIND, MIXED>(p, smem, L);
    unsigned long long* qbase = p.queue + (size_t)blockIdx.x * nb2 * p.subcap;
    double* qsig = p.queue_sigma + (size_t)blockIdx.x * nb2 * p.subcap;
    long long* qpos = (KIND == 3) ? p.queue_pos + (size_t)blockIdx.x * nb2 * p.subcap : nullptr;
    K4Stats st{0, 0, 0, 0};
    for (;;) {
        if (threadIdx.x == 0) misc[0] = atomicAdd(p.work_counter, 1);
        __syncthreads();
        const int wi = misc[0];
        if (wi >= p.nwork) break;
        k4_item<KIND, NT, MIXED>(p, smem, L, wi, qbase, qsig, qpos, st);
    }
    k4_flush_stats(p.stats, st, reinterpret_cast<double*>(smem + L.red));
}

// The four-phonon RTA work kernel with phase B on the tensor cores (mixed
// precision): phase A as in k4_work, then k4_phase_b_tc.  Each CTA holds 256
// TMEM columns (two warpgroup regions) for its lifetime; two CTAs per SM use
// the whole TMEM.  A bounded wait that gives up raises kErrTimeout and stops
// the CTA, which waits (bounded) for its outstanding products before it frees
// its TMEM.
template <int NT>
__global__ void __launch_bounds__(kThreads, 2) k4_work_tc(P4Params p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int nb2 = p.S.nb * p.S.nb;
    const TcPlan* P = p.tc;
    const Layout L = k4_layout_tcbase(NT, p.S.nb, p.F.npi, p.F.ntri, p.S.n[0] + p.S.n[1] + p.S.n[2], p.S.nptk);
    const TcLayout TL = k4_tc_layout(L.total, P->ksteps, P->bin_bytes, P->zbins, p.F.npi, P->chunk_cap, p.S.nb);
    int* misc = reinterpret_cast<int*>(smem + L.misc);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + TL.bar);
    uint32_t* slotw = reinterpret_cast<uint32_t*>(smem + TL.slot);
    k4_cta_init<2, true>(p, smem, L);
    {  // the plan, copied into shared memory
        const int* src = reinterpret_cast<const int*>(P);
        int* dst = reinterpret_cast<int*>(smem + TL.plan);
        for (int x = threadIdx.x; x < (int)(sizeof(TcPlan) / sizeof(int)); x += blockDim.x) dst[x] = src[x];
    }
    if (threadIdx.x == 0) {
        tc::mbar_init(tc::smem_u32(&bars[0]), 1);
        tc::mbar_init(tc::smem_u32(&bars[1]), 1);
        tc::mbar_fence_init();
        slotw[1] = 0;
        slotw[2] = 0;
        misc[7] = 0;
    }
    if (threadIdx.x < 32) {
        tc::tmem_alloc(tc::smem_u32(&slotw[0]), 2 * kTcRegionCols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    unsigned long long* qbase = p.queue + (size_t)blockIdx.x * nb2 * p.subcap;
    double* qsig = p.queue_sigma + (size_t)blockIdx.x * nb2 * p.subcap;
    K4Stats st{0, 0, 0, 0};
    for (;;) {
        if (threadIdx.x == 0) misc[0] = atomicAdd(p.work_counter, 1);
        __syncthreads();
        const int wi = misc[0];
        if (wi >= p.nwork || misc[7]) break;
        k4_item<2, NT, true, true>(p, smem, L, wi, qbase, qsig, nullptr, st);
    }
    k4_flush_stats(p.stats, st, reinterpret_cast<double*>(smem + L.red));
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (threadIdx.x == 0 && misc[7]) {
        // after a wait that gave up: give the products still in flight a bounded time
        tc::mbar_wait(tc::smem_u32(&bars[0]), slotw[1]);
        tc::mbar_wait(tc::smem_u32(&bars[1]), slotw[2]);
    }
    __syncthreads();
    if (threadIdx.x < 32) tc::tmem_dealloc(slotw[0], 2 * kTcRegionCols);
}

// A rows of the tensor-core contraction for every q'' and both channel signs:
// 16-byte words of 8 bf16 values, the K layout of TcPlan with the Bloch phases
// w_p(q'') = exp(+-2 pi i n''.D_p / N) formed in FP64 from the exact root tables.
__global__ void k4_wtab(DevSys S, DevIfc F, const TcPlan* P, int ksteps, uint16_t* wtab) {
    const int words = 2 * ksteps;  // 16-byte words per row
    const size_t total = (size_t)2 * S.nptk * words;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < total; x += (size_t)gridDim.x * blockDim.x) {
        const int word = (int)(x % words);
        const size_t row = x / words;
        const int q = (int)(row % S.nptk), sgn = (int)(row / S.nptk);
        int a, b, c;
        q_coords(S, q, a, b, c);
        const int k0 = word * 8;
        int pass = 0;
        while (pass + 1 < P->npass && P->pass_kstep0[pass + 1] * 16 <= k0) pass++;
        uint32_t w4[4] = {0, 0, 0, 0};
        for (int y = 0; y < 8; y++) {
            const int kk = k0 + y - P->pass_kstep0[pass] * 16;
            const int cls = P->pass_cls0[pass] + kk / 6;
            if (cls >= P->pass_cls0[pass + 1]) continue;
            const int r6 = kk - (kk / 6) * 6, split = r6 >> 1, ri = r6 & 1;
            const int4 D = F.pi_d[cls];
            double2 w = lattice_phase(S, a, b, c, D.x, D.y, D.z);
            if (sgn) w = cconj(w);
            uint16_t hi, lo;
            tc::split_bf16(ri ? w.y : w.x, hi, lo);
            const uint32_t v = (split == 2) ? lo : hi;
            w4[y >> 1] |= v << (16 * (y & 1));
        }
        reinterpret_cast<uint4*>(wtab)[x] = make_uint4(w4[0], w4[1], w4[2], w4[3]);
    }
}

// Several solves in one persistent launch (the serving path).  The tick lists
// ranges of work items, each of one solve slot; a CTA that moves to another
// slot flushes its counters, loads that slot's parameters into shared memory
// and rebuilds its per-CTA tables.  The queue is per CTA, sized for the largest
// branch count the server admits.
template <int NT, bool MIXED>
__global__ void __launch_bounds__(kThreads, kMultiCtasPerSm) k4_work_multi(const P4Params* slots, const K4Tick* tick,
                                                                                int* counter, unsigned long long* queue,
                                                                                double* queue_sigma, int cta_bins,
                                                                                int subcap) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ P4Params sp;
    __shared__ int s_slot, s_wi;
    unsigned long long* qbase = queue + (size_t)blockIdx.x * cta_bins * subcap;
    double* qsig = queue_sigma + (size_t)blockIdx.x * cta_bins * subcap;
    K4Stats st{0, 0, 0, 0};
    int cur = -1;
    Layout L{};
    const int total = tick->prefix[tick->nranges];
    for (;;) {
        if (threadIdx.x == 0) {
            const int g = atomicAdd(counter, 1);
            int slot = -1, wi = 0;
            if (g < total) {
                int r = 0;
                while (r + 1 < tick->nranges && tick->prefix[r + 1] <= g) r++;
                slot = tick->slot[r];
                wi = tick->begin[r] + (g - tick->prefix[r]);
            }
            s_slot = slot;
            s_wi = wi;
        }
        __syncthreads();
        const int slot = s_slot, wi = s_wi;
        if (slot < 0) break;
        if (slot != cur) {
            if (cur >= 0) k4_flush_stats(sp.stats, st, reinterpret_cast<double*>(smem + L.red));
            __syncthreads();
            const int* src = reinterpret_cast<const int*>(slots + slot);
            int* dst = reinterpret_cast<int*>(&sp);
            for (int x = threadIdx.x; x < (int)(sizeof(P4Params) / sizeof(int)); x += blockDim.x) dst[x] = src[x];
            __syncthreads();
            L = k4_layout(2, NT, MIXED, sp.S.nb, sp.F.npi, sp.F.ntri, sp.S.n[0] + sp.S.n[1] + sp.S.n[2], 0, kAllZCap2);
            k4_cta_init<2, MIXED>(sp, smem, L);
            cur = slot;
        }
        k4_item<2, NT, MIXED>(sp, smem, L, wi, qbase, qsig, nullptr, st);
    }
    if (cur >= 0) k4_flush_stats(sp.stats, st, reinterpret_cast<double*>(smem + L.red));
}

}  // namespace
}  // namespace fp4

namespace fp4 {
namespace {

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

int round_nt(int nT) { return nT <= 1 ? 1 : (nT <= 2 ? 2 : (nT <= 4 ? 4 : 8)); }

template <int KIND, int NT, bool MIXED>
cudaError_t launch_k4_t(const P4Params& p, int nblocks, cudaStream_t st) {
    size_t sm = k4_smem(KIND, p.nT, MIXED, p.S, p.F);
    cudaError_t e = cudaFuncSetAttribute(k4_work<KIND, NT, MIXED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k4_work<KIND, NT, MIXED><<<nblocks, kThreads, sm, st>>>(p);
    return cudaGetLastError();
}

}  // namespace

size_t k4_smem(int kind, int nT, bool mixed, const DevSys& S, const DevIfc& F) {
    Layout L = k4_layout(kind, round_nt(nT), mixed, S.nb, F.npi, F.ntri, S.n[0] + S.n[1] + S.n[2], S.nptk);
    return L.total;
}

int k4_threads() { return kThreads; }

int k4_tc_plan(int nb, int natoms, int npi, const int* blk_start, int subcap, TcPlan& P) {
    P = TcPlan{};
    const int nat2 = natoms * natoms;
    for (int b = 0; b < nat2; b++)
        if (blk_start[b] < blk_start[b + 1]) {
            if (P.nblk >= kTcMaxBlocks) return -1;
            P.blk[P.nblk++] = make_int4(blk_start[b], blk_start[b + 1], b / natoms, b % natoms);
        }
    if (P.nblk == 0 || blk_start[nat2] != npi) return -1;
    int ks = 0, boff = 0;
    for (int b0 = 0; b0 < P.nblk; b0 += kTcPassBlocks) {
        const int b1 = std::min(P.nblk, b0 + kTcPassBlocks);
        const int x = P.npass++;
        P.pass_blk0[x] = b0;
        P.pass_cls0[x] = P.blk[b0].x;
        P.pass_kstep0[x] = ks;
        P.pass_boff[x] = boff;
        const int C = P.blk[b1 - 1].y - P.blk[b0].x;
        const int k = (6 * C + 15) / 16;
        ks += k;
        boff += k * 32 * (b1 - b0) * 32;  // K-steps x N rows x 32 bytes
    }
    P.pass_blk0[P.npass] = P.nblk;
    P.pass_cls0[P.npass] = npi;
    P.pass_kstep0[P.npass] = ks;
    P.pass_boff[P.npass] = boff;
    P.ksteps = ks;
    P.bin_bytes = boff;
    P.zbins = 1;
    P.chunk_cap = (subcap + kTcRows - 1) / kTcRows;
    (void)nb;
    return 0;
}

// Shared memory of k4_work_tc for the plan's zbins (the plan's chunk_cap must match).
size_t k4_tc_smem(int nT, const DevSys& S, const DevIfc& F, const TcPlan& P) {
    const Layout L = k4_layout_tcbase(round_nt(nT), S.nb, F.npi, F.ntri, S.n[0] + S.n[1] + S.n[2], S.nptk);
    return k4_tc_layout(L.total, P.ksteps, P.bin_bytes, P.zbins, F.npi, P.chunk_cap, S.nb).total;
}

int k4_tc_ctas_per_sm() { return 2; }

cudaError_t launch_k4_tc(int nT, const P4Params& p, size_t smem, int nblocks, cudaStream_t st) {
    const int NT = round_nt(nT);
#define FP4_K4TC(NTV)                                                                                            \
    if (NT == NTV) {                                                                                             \
        cudaError_t e = cudaFuncSetAttribute(k4_work_tc<NTV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        if (e != cudaSuccess) return e;                                                                          \
        k4_work_tc<NTV><<<nblocks, kThreads, smem, st>>>(p);                                                     \
        return cudaGetLastError();                                                                               \
    }
    FP4_K4TC(1)
    FP4_K4TC(2)
    FP4_K4TC(4)
    FP4_K4TC(8)
#undef FP4_K4TC
    return cudaErrorInvalidValue;
}

cudaError_t launch_k4_wtab(const DevSys& S, const DevIfc& F, const TcPlan* plan_dev, int ksteps, uint16_t* wtab,
                           cudaStream_t st) {
    const size_t total = (size_t)2 * S.nptk * 2 * ksteps;
    const int threads = 256;
    const int blocks = (int)std::min<size_t>((total + threads - 1) / threads, 148 * 16);
    k4_wtab<<<blocks, threads, 0, st>>>(S, F, plan_dev, ksteps, wtab);
    return cudaGetLastError();
}
int k4_round_nt(int nT) { return round_nt(nT); }
int k4_multi_ctas_per_sm() { return kMultiCtasPerSm; }

int k4_ctas_per_sm(int kind, int nT, bool mixed) {
    if (kind == 0) return ctas_per_sm<0, 1, false>();
    const int NT = round_nt(nT);
    if (mixed) return NT >= 4 ? ctas_per_sm<2, 4, true>() : ctas_per_sm<2, 1, true>();
    return ctas_per_sm<2, 1, false>();
}

cudaError_t launch_k4(int kind, int nT, bool mixed, const P4Params& p, int nblocks, cudaStream_t st) {
    if (kind == 0) return launch_k4_t<0, 1, false>(p, nblocks, st);
    if (kind == 3) {
        if (nT != 1) return cudaErrorInvalidValue;
        return mixed ? launch_k4_t<3, 1, true>(p, nblocks, st) : launch_k4_t<3, 1, false>(p, nblocks, st);
    }
    const int NT = round_nt(nT);
#define FP4_K4(NTV)                                                                                   \
    if (NT == NTV) return mixed ? launch_k4_t<2, NTV, true>(p, nblocks, st) : launch_k4_t<2, NTV, false>(p, nblocks, st);
    FP4_K4(1)
    FP4_K4(2)
    FP4_K4(4)
    FP4_K4(8)
#undef FP4_K4
    return cudaErrorInvalidValue;
}

size_t k4_multi_smem(bool mixed, const DevSys& S, const DevIfc& F) {
    return k4_layout(2, 1, mixed, S.nb, F.npi, F.ntri, S.n[0] + S.n[1] + S.n[2], 0, kAllZCap2).total;
}

cudaError_t prepare_k4_multi(bool mixed, size_t smem) {
    return mixed ? cudaFuncSetAttribute(k4_work_multi<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                 : cudaFuncSetAttribute(k4_work_multi<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

// The caller sets the dynamic shared-memory limit once with prepare_k4_multi (so the
// launch can be captured into a graph).
cudaError_t launch_k4_multi(bool mixed, const P4Params* slots, const K4Tick* tick, int* counter,
                            unsigned long long* queue, double* queue_sigma, int cta_bins, int subcap, size_t smem,
                            int nblocks, cudaStream_t st) {
    if (mixed)
        k4_work_multi<1, true><<<nblocks, kThreads, smem, st>>>(slots, tick, counter, queue, queue_sigma, cta_bins, subcap);
    else
        k4_work_multi<1, false><<<nblocks, kThreads, smem, st>>>(slots, tick, counter, queue, queue_sigma, cta_bins, subcap);
    return cudaGetLastError();
}

cudaError_t launch_k4_reduce(const P4Params& p, double* r0, double* r1, double* r2, double* w0, double* w1, double* w2,
                             double rate_scale, cudaStream_t st) {
    int total = 3 * p.S.nlist * p.S.nb * p.nT;
    int threads = 128, blocks = (total + threads - 1) / threads;
    k4_reduce<<<blocks, threads, 0, st>>>(p, r0, r1, r2, w0, w1, w2, rate_scale);
    return cudaGetLastError();
}

}  // namespace fp4
