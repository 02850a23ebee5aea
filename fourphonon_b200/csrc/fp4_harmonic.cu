// Harmonic stage on the device: eigenDM with phonon_phonopy
// (Src/phonon_routines.f90:12-81, 84-307), the dielectric correction included.
//
// For every q of the Gamma-centred grid one warp builds the dynamical matrix
// D(q) and its q-derivative from the Phonopy force constants with the
// Wigner-Seitz image weights, adds the dielectric correction (Born charges,
// epsilon) through the first-zone image of q, diagonalises D(q) with cyclic
// complex Jacobi rotations, sorts the eigenvalues ascending as zheev does, and
// forms omega = sign(w2) sqrt(|w2|), the eigenvectors and the group velocities
// Re(e^+ dD e)/(2 omega), symmetrised with the grid point's symmetrizer.  The
// acoustic branches at Gamma are set to zero as eigenDM does.  Eigenvectors
// carry an arbitrary phase (and an arbitrary basis inside a degenerate set),
// exactly as LAPACK's do; every quantity of the rate path is invariant under
// the phase, and sums over a degenerate set are invariant under its basis.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <vector>

#include "../../include/fourphonon_b200.h"
#include "fp4_ctx.h"
#include "fp4_device.cuh"
#include "fp4_internal.h"

using namespace fp4;

namespace {

constexpr int kMaxSweeps = 40;  // cyclic Jacobi converges quadratically: ~6-10 sweeps at nb <= 30

struct HTerm {
    double blk[9];  // blk[i*3+j] = fc(a2, j, cell, a1, i)
    int img0, nimg;
};

struct HParams {
    int nb, natoms, nptk, n0, n1, n2;
    int nac, ncell;               // dielectric correction on; supercell size
    double rl[9];                 // rlattvec(3,3) column-major
    double eps[9];                // epsilon(3,3) column-major
    double pref_v[2];             // prefactor (default REAL), V (nm^3)
    const int* pair_start;        // [a1*natoms + a2] .. [+1]: terms of the atom pair
    const HTerm* terms;
    const double* img;            // [3*x]: image vectors rl + rcell (nm)
    const double* born_mm;        // born(3,3,natoms), then mm(natoms,natoms)
    const double* symm;           // symmetrizers(3,3,nptk)
    double* omega;                // omega(nptk,nb)
    double* velocity;             // velocity(nptk,nb,3)
    double2* eig;                 // eigenvect(nptk,nb,nb)
};

// |r|, correctly rounded: the squares and their rounding errors are summed
// in double-double before the square root.  The first-zone search compares
// images of equal length, and the reference's dnrm2 sums squares in extended
// precision; a plain double sum breaks some of those ties the other way.
__device__ double norm3_rn(double x, double y, double z) {
    const double px = __dmul_rn(x, x), py = __dmul_rn(y, y), pz = __dmul_rn(z, z);
    const double ex = fma(x, x, -px), ey = fma(y, y, -py), ez = fma(z, z, -pz);
    double s = __dadd_rn(px, py);
    double bb = __dsub_rn(s, px);
    double c = __dadd_rn(__dsub_rn(px, __dsub_rn(s, bb)), __dsub_rn(py, bb));
    const double s2 = __dadd_rn(s, pz);
    bb = __dsub_rn(s2, s);
    c = __dadd_rn(c, __dadd_rn(__dsub_rn(s, __dsub_rn(s2, bb)), __dsub_rn(pz, bb)));
    c = __dadd_rn(c, __dadd_rn(__dadd_rn(ex, ey), ez));
    const double hi = __dadd_rn(s2, c), lo = __dsub_rn(c, __dsub_rn(hi, s2));
    if (!(hi > 0.0)) return 0.0;
    const double r = sqrt(hi);
    const double res = __dadd_rn(fma(-r, r, hi), lo);
    return __dadd_rn(r, __ddiv_rn(res, __dmul_rn(2.0, r)));
}

__global__ void __launch_bounds__(32) k_eigen_dm(HParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int nb = p.nb, nb2 = nb * nb;
    double2* A = reinterpret_cast<double2*>(smem);
    double2* V = A + nb2;
    double2* dD = V + nb2;  // 3 x nb2
    double* w2 = reinterpret_cast<double*>(dD + 3 * nb2);
    int* perm = reinterpret_cast<int*>(w2 + nb);
    const int lane = threadIdx.x;
    const double* born = p.born_mm;
    const double* mm = p.born_mm + 9 * p.natoms;
    for (int q = blockIdx.x; q < p.nptk; q += gridDim.x) {
        const int i0 = q % p.n0, i1 = (q / p.n0) % p.n1, i2 = q / (p.n0 * p.n1);
        // kspace(q,:) = rlattvec(:,1)*i0/n0 + rlattvec(:,2)*i1/n1 + rlattvec(:,3)*i2/n2
        double kv[3];
        for (int d = 0; d < 3; d++)
            kv[d] = __dadd_rn(__dadd_rn(__ddiv_rn(__dmul_rn(p.rl[d], (double)i0), (double)p.n0),
                                        __ddiv_rn(__dmul_rn(p.rl[3 + d], (double)i1), (double)p.n1)),
                              __ddiv_rn(__dmul_rn(p.rl[6 + d], (double)i2), (double)p.n2));
        const bool k_zero = (i0 == 0 && i1 == 0 && i2 == 0);
        // first-zone image of q: the first strictly shorter one, q itself first,
        // then the (-2..2)^3 scan (phonon_routines.f90:140-156)
        double qs[3] = {kv[0], kv[1], kv[2]};
        bool nac = false;
        if (p.nac) {
            double best = lane == 0 ? norm3_rn(kv[0], kv[1], kv[2]) : HUGE_VAL;
            int bidx = lane == 0 ? -1 : 1 << 20;
            for (int x = lane; x < 125; x += 32) {
                const double ix = x / 25 - 2, iy = (x / 5) % 5 - 2, iz = x % 5 - 2;
                double r[3];
                for (int d = 0; d < 3; d++)
                    r[d] = __dadd_rn(__dadd_rn(__dadd_rn(kv[d], __dmul_rn(ix, p.rl[d])), __dmul_rn(iy, p.rl[3 + d])),
                                     __dmul_rn(iz, p.rl[6 + d]));
                const double n = norm3_rn(r[0], r[1], r[2]);
                if (n < best) {
                    best = n;
                    bidx = x;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bidx, o);
                if (ob < best || (ob == best && oi < bidx)) {
                    best = ob;
                    bidx = oi;
                }
            }
            if (bidx >= 0) {
                const double ix = bidx / 25 - 2, iy = (bidx / 5) % 5 - 2, iz = bidx % 5 - 2;
                for (int d = 0; d < 3; d++)
                    qs[d] = __dadd_rn(__dadd_rn(__dadd_rn(kv[d], __dmul_rn(ix, p.rl[d])), __dmul_rn(iy, p.rl[3 + d])),
                                      __dmul_rn(iz, p.rl[6 + d]));
            }
            nac = !(qs[0] == 0.0 && qs[1] == 0.0 && qs[2] == 0.0);
        }
        double tmp3 = 1.0, eq[3] = {0.0, 0.0, 0.0};
        if (nac) {  // tmp3 = q . (epsilon q); eq(ip) = epsilon(ip,:) . q
            tmp3 = 0.0;
            for (int a = 0; a < 3; a++) {
                eq[a] = p.eps[a] * qs[0] + p.eps[a + 3] * qs[1] + p.eps[a + 6] * qs[2];
                tmp3 += qs[a] * eq[a];
            }
        }
        // D(q) and dD/dq: contributions in the reference's order (cells, then images)
        for (int e = lane; e < nb2; e += 32) {
            const int row = e / nb, col = e - row * nb;
            const int a1 = row / 3, i = row - 3 * a1, a2 = col / 3, j = col - 3 * a2;
            double fd = 0.0, dn[3] = {0.0, 0.0, 0.0};  // fc_diel and ddyn_nac/ncell of this element
            if (nac) {
                const double* b1 = born + 3 * (i + 3 * a1);
                const double* b2 = born + 3 * (j + 3 * a2);
                const double t1 = qs[0] * b1[0] + qs[1] * b1[1] + qs[2] * b1[2];
                const double t2 = qs[0] * b2[0] + qs[1] * b2[1] + qs[2] * b2[2];
                const double m = mm[a1 + p.natoms * a2];
                fd = p.pref_v[0] * (t1 * t2 / m) / tmp3 / p.pref_v[1] / p.ncell;
                for (int ip = 0; ip < 3; ip++) {
                    const double dd = (t1 * born[ip + 3 * (j + 3 * a2)] + t2 * born[ip + 3 * (i + 3 * a1)] -
                                       2.0 * t1 * t2 * eq[ip] / tmp3) / m;
                    dn[ip] = k_zero ? 0.0 : p.pref_v[0] * dd / tmp3 / p.pref_v[1] / p.ncell;
                }
            }
            double2 d = make_double2(0.0, 0.0), g0 = d, g1 = d, g2 = d;
            for (int t = p.pair_start[a1 * p.natoms + a2]; t < p.pair_start[a1 * p.natoms + a2 + 1]; t++) {
                const HTerm& T = p.terms[t];
                const double f = T.blk[i * 3 + j] + fd;
                double2 star = make_double2(0.0, 0.0);
                for (int x = T.img0; x < T.img0 + T.nimg; x++) {
                    const double* r = p.img + 3 * x;
                    const double qr = (kv[0] * r[0] + kv[1] * r[1]) + kv[2] * r[2];
                    double sn, cs;
                    sincos(-qr, &sn, &cs);
                    const double2 z = make_double2(cs / T.nimg, sn / T.nimg);
                    star.x += z.x;
                    star.y += z.y;
                    d.x += z.x * f;
                    d.y += z.y * f;
                    const double2 iz = make_double2(-z.y, z.x);  // i*z
                    g0.x -= (iz.x * r[0]) * f; g0.y -= (iz.y * r[0]) * f;
                    g1.x -= (iz.x * r[1]) * f; g1.y -= (iz.y * r[1]) * f;
                    g2.x -= (iz.x * r[2]) * f; g2.y -= (iz.y * r[2]) * f;
                }
                if (nac) {
                    g0.x += star.x * dn[0]; g0.y += star.y * dn[0];
                    g1.x += star.x * dn[1]; g1.y += star.y * dn[1];
                    g2.x += star.x * dn[2]; g2.y += star.y * dn[2];
                }
            }
            A[e] = d;
            dD[e] = g0;
            dD[nb2 + e] = g1;
            dD[2 * nb2 + e] = g2;
            V[e] = make_double2(row == col ? 1.0 : 0.0, 0.0);
        }
        __syncwarp();
        // the upper triangle defines the matrix (zheev "U")
        for (int e = lane; e < nb2; e += 32) {
            const int row = e / nb, col = e - row * nb;
            if (row > col) A[e] = cconj(A[col * nb + row]);
            if (row == col) A[e].y = 0.0;
        }
        __syncwarp();
        double norm2 = 0.0;
        for (int e = lane; e < nb2; e += 32) norm2 += A[e].x * A[e].x + A[e].y * A[e].y;
        for (int o = 16; o > 0; o >>= 1) norm2 += __shfl_xor_sync(0xffffffffu, norm2, o);
        for (int sweep = 0; sweep < kMaxSweeps; sweep++) {
            double off = 0.0;
            for (int e = lane; e < nb2; e += 32) {
                const int row = e / nb, col = e - row * nb;
                if (row < col) off += A[e].x * A[e].x + A[e].y * A[e].y;
            }
            for (int o = 16; o > 0; o >>= 1) off += __shfl_xor_sync(0xffffffffu, off, o);
            // stop at the rounding floor: every off-diagonal element near eps * |A|
            if (!(off > 1e-30 * (double)nb2 * norm2)) break;
            for (int pp = 0; pp < nb - 1; pp++) {
                for (int qq = pp + 1; qq < nb; qq++) {
                    const double2 c = A[pp * nb + qq];
                    const double ac = sqrt(c.x * c.x + c.y * c.y);
                    if (!(ac > 1e-300)) continue;
                    const double a = A[pp * nb + pp].x, b = A[qq * nb + qq].x;
                    const double tau = (b - a) / (2.0 * ac);
                    const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
                    const double cs = 1.0 / sqrt(1.0 + t * t), sn = t * cs;
                    const double2 ph = make_double2(c.x / ac, c.y / ac);  // e = c/|c|
                    const double2 sph = make_double2(sn * ph.x, sn * ph.y), sphc = make_double2(sn * ph.x, -sn * ph.y);
                    __syncwarp();
                    if (lane < nb) {  // columns: A <- A U, V <- V U
                        const double2 akp = A[lane * nb + pp], akq = A[lane * nb + qq];
                        const double2 u = cmul(sphc, akq), w = cmul(sph, akp);
                        A[lane * nb + pp] = make_double2(cs * akp.x - u.x, cs * akp.y - u.y);
                        A[lane * nb + qq] = make_double2(w.x + cs * akq.x, w.y + cs * akq.y);
                        const double2 vkp = V[lane * nb + pp], vkq = V[lane * nb + qq];
                        const double2 uv = cmul(sphc, vkq), wv = cmul(sph, vkp);
                        V[lane * nb + pp] = make_double2(cs * vkp.x - uv.x, cs * vkp.y - uv.y);
                        V[lane * nb + qq] = make_double2(wv.x + cs * vkq.x, wv.y + cs * vkq.y);
                    }
                    __syncwarp();
                    if (lane < nb) {  // rows: A <- U^+ A
                        const double2 apk = A[pp * nb + lane], aqk = A[qq * nb + lane];
                        const double2 u = cmul(sph, aqk), w = cmul(sphc, apk);
                        A[pp * nb + lane] = make_double2(cs * apk.x - u.x, cs * apk.y - u.y);
                        A[qq * nb + lane] = make_double2(w.x + cs * aqk.x, w.y + cs * aqk.y);
                    }
                    __syncwarp();
                    if (lane == 0) {
                        A[pp * nb + qq] = make_double2(0.0, 0.0);
                        A[qq * nb + pp] = make_double2(0.0, 0.0);
                        A[pp * nb + pp].y = 0.0;
                        A[qq * nb + qq].y = 0.0;
                    }
                    __syncwarp();
                }
            }
        }
        // ascending eigenvalues (ties by index; a NaN sorts last, so the ranks
        // stay a permutation of 0..nb-1 whatever the input)
        if (lane < nb) w2[lane] = A[lane * nb + lane].x;
        __syncwarp();
        if (lane < nb) {
            auto key = [](double w) { return isnan(w) ? HUGE_VAL : w; };
            const double wl = key(w2[lane]);
            int rank = 0;
            for (int m = 0; m < nb; m++) {
                const double wm = key(w2[m]);
                if (wm < wl || (wm == wl && m < lane)) rank++;
            }
            perm[rank] = lane;
        }
        __syncwarp();
        const size_t np = (size_t)p.nptk;
        for (int e = lane; e < nb2; e += 32) {  // eigenvect(q, band r, comp c) = V[c][perm[r]]
            const int r = e / nb, c = e - r * nb;
            p.eig[((size_t)c * nb + r) * np + q] = V[c * nb + perm[r]];
        }
        if (lane < nb) {
            const int r = lane, n = perm[r];
            const double wv = w2[n];
            const double om = (wv >= 0.0 ? 1.0 : -1.0) * sqrt(fabs(wv));
            double v[3];
            for (int d = 0; d < 3; d++) {
                double acc = 0.0;
                for (int a = 0; a < nb; a++) {
                    double2 h = make_double2(0.0, 0.0);
                    for (int b = 0; b < nb; b++) h = cmac(h, dD[d * nb2 + a * nb + b], V[b * nb + n]);
                    const double2 za = V[a * nb + n];
                    acc += za.x * h.x + za.y * h.y;  // Re(conj(z_a) h_a)
                }
                v[d] = acc / (2.0 * om);
                if (!isfinite(v[d])) v[d] = 0.0;  // omega == 0 away from the Gamma acoustic branches
            }
            const double* S = p.symm + 9 * (size_t)q;  // velocity = symmetrizer . velocity
            double y[3];
            for (int a = 0; a < 3; a++) y[a] = S[a] * v[0] + S[a + 3] * v[1] + S[a + 6] * v[2];
            const bool gamma_ac = (q == 0 && r < 3);
            p.omega[(size_t)r * np + q] = gamma_ac ? 0.0 : om;
            for (int d = 0; d < 3; d++) p.velocity[((size_t)d * nb + r) * np + q] = gamma_ac ? 0.0 : y[d];
        }
        __syncwarp();
    }
}

}  // namespace

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return fp4_fail(c, FP4_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

extern "C" int fp4_eigen_dm(fp4_ctx* c, const fp4_globals* g, const double* lattvec, const double* cartesian,
                            const int32_t scell[3], const double* fc, int32_t nonanalytic, const double* epsilon,
                            const double* born, double V, const double* symmetrizers, double* omega,
                            double* velocity, double* eigenvect) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!g || !lattvec || !cartesian || !scell || !fc || !symmetrizers || !omega || !velocity || !eigenvect)
        return fp4_fail(c, FP4_E_ARG, "null argument");
    if (nonanalytic && (!epsilon || !born || !(V > 0.0)))
        return fp4_fail(c, FP4_E_ARG, "nonanalytic needs epsilon, born and V > 0");
    const int nat = g->natoms, nb = g->nbands;
    if (nat < 1 || nb != 3 * nat || nb > kMaxNb) return fp4_fail(c, FP4_E_ARG, "nbands=%d natoms=%d", nb, nat);
    if (!g->masses || !g->types) return fp4_fail(c, FP4_E_ARG, "masses and types are needed");
    for (int a = 0; a < nat; a++)
        if (g->types[a] < 1 || g->types[a] > g->nelements)
            return fp4_fail(c, FP4_E_ARG, "types(%d)=%d outside [1,%d]", a + 1, g->types[a], g->nelements);
    for (int d = 0; d < 3; d++) {
        if (scell[d] < 1 || scell[d] > 64) return fp4_fail(c, FP4_E_ARG, "scell(%d)=%d outside [1,64]", d + 1, scell[d]);
        if (g->ngrid[d] < 1 || g->ngrid[d] > kMaxGrid) return fp4_fail(c, FP4_E_ARG, "ngrid outside [1,%d]", kMaxGrid);
    }
    const int sx = scell[0], sy = scell[1], sz = scell[2];
    const int nptk = g->ngrid[0] * g->ngrid[1] * g->ngrid[2];
    // Wigner-Seitz images of every (a1, a2, cell) (phonon_routines.f90:224-251)
    auto L = [&](int d, int col) { return lattvec[col * 3 + d]; };
    std::vector<HTerm> terms;
    std::vector<double> img;
    std::vector<int> pair_start(nat * nat + 1, 0);
    for (int a1 = 0; a1 < nat; a1++)
        for (int a2 = 0; a2 < nat; a2++) {
            pair_start[a1 * nat + a2] = (int)terms.size();
            for (int ix = 0; ix < sx; ix++)
                for (int iy = 0; iy < sy; iy++)
                    for (int iz = 0; iz < sz; iz++) {
                        double rcell[3], r[3];
                        for (int d = 0; d < 3; d++) {
                            rcell[d] = L(d, 0) * ix + L(d, 1) * iy + L(d, 2) * iz;
                            r[d] = cartesian[3 * a1 + d] - cartesian[3 * a2 + d] + rcell[d];
                        }
                        HTerm T;
                        T.img0 = (int)(img.size() / 3);
                        T.nimg = 0;
                        double dmin = HUGE_VAL;
                        for (int jx = -2; jx <= 2; jx++)
                            for (int jy = -2; jy <= 2; jy++)
                                for (int jz = -2; jz <= 2; jz++) {
                                    double rl[3], s2 = 0.0;
                                    for (int d = 0; d < 3; d++) {
                                        rl[d] = (jx * sx) * L(d, 0) + (jy * sy) * L(d, 1) + (jz * sz) * L(d, 2);
                                        const double x = rl[d] + r[d];
                                        s2 += x * x;
                                    }
                                    const double rn = std::sqrt(s2);
                                    if (std::fabs(rn - dmin) > 1e-5) {
                                        if (rn < dmin) {
                                            dmin = rn;
                                            img.resize((size_t)T.img0 * 3);
                                            T.nimg = 0;
                                        } else {
                                            continue;
                                        }
                                    }
                                    for (int d = 0; d < 3; d++) img.push_back(rl[d] + rcell[d]);
                                    T.nimg++;
                                }
                        // fc(a2, j, ix, iy, iz, a1, i), column-major (natoms,3,sx,sy,sz,natoms,3)
                        for (int i = 0; i < 3; i++)
                            for (int j = 0; j < 3; j++) {
                                const size_t o =
                                    a2 + (size_t)nat * (j + 3 * (ix + (size_t)sx * (iy + (size_t)sy * (iz + (size_t)sz * (a1 + (size_t)nat * i)))));
                                T.blk[i * 3 + j] = fc[o];
                            }
                        terms.push_back(T);
                    }
        }
    pair_start[nat * nat] = (int)terms.size();
    // born(3,3,natoms) and the mass products mm(natoms,natoms) of phonon_phonopy (lines 122-128)
    std::vector<double> born_mm(9 * (size_t)nat + (size_t)nat * nat, 0.0);
    if (nonanalytic)
        for (int x = 0; x < 9 * nat; x++) born_mm[x] = born[x];
    for (int a = 0; a < nat; a++)
        for (int b = 0; b < nat; b++) {
            const double ma = g->masses[g->types[a] - 1], mb = g->masses[g->types[b] - 1];
            born_mm[9 * nat + a + (size_t)nat * b] = a == b ? ma : std::sqrt(ma * mb);
        }
    int r;
    if ((r = fp4_begin(c))) return r;
    DevBuffer* B = c->b_harm;
    const size_t plane = (size_t)nptk * nb;
    if ((r = B[0].upload(c, pair_start.data(), pair_start.size() * sizeof(int))) ||
        (r = B[1].upload(c, terms.data(), terms.size() * sizeof(HTerm))) ||
        (r = B[2].upload(c, img.data(), img.size() * sizeof(double))) ||
        (r = B[3].upload(c, symmetrizers, (size_t)nptk * 9 * sizeof(double))) ||
        (r = B[4].reserve(c, plane * (1 + 3) * sizeof(double) + plane * nb * sizeof(double2))) ||
        (r = B[5].upload(c, born_mm.data(), born_mm.size() * sizeof(double))))
        return r;
    HParams p{};
    p.nb = nb;
    p.natoms = nat;
    p.nptk = nptk;
    p.n0 = g->ngrid[0];
    p.n1 = g->ngrid[1];
    p.n2 = g->ngrid[2];
    p.nac = nonanalytic ? 1 : 0;
    p.ncell = sx * sy * sz;
    for (int x = 0; x < 9; x++) {
        p.rl[x] = g->rlattvec[x];
        p.eps[x] = nonanalytic ? epsilon[x] : (x % 4 == 0 ? 1.0 : 0.0);
    }
    p.pref_v[0] = (double)1745.91429109f;  // prefactor, THz^2 amu nm^3 (a default REAL literal)
    p.pref_v[1] = nonanalytic ? V : 1.0;
    p.born_mm = B[5].as<double>();
    p.pair_start = B[0].as<int>();
    p.terms = B[1].as<HTerm>();
    p.img = B[2].as<double>();
    p.symm = B[3].as<double>();
    p.omega = B[4].as<double>();
    p.velocity = p.omega + plane;
    p.eig = reinterpret_cast<double2*>(p.velocity + 3 * plane);
    const size_t sm = (size_t)5 * nb * nb * sizeof(double2) + nb * sizeof(double) + nb * sizeof(int) + 16;
    CK(cudaFuncSetAttribute(k_eigen_dm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int blocks = std::min(nptk, c->sm_count * 32);
    CK(cudaEventRecord(c->evk0, c->stream));
    k_eigen_dm<<<blocks, 32, sm, c->stream>>>(p);
    CK(cudaGetLastError());
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_timed = true;
    c->launches++;
    CK(cudaMemcpyAsync(omega, p.omega, plane * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(velocity, p.velocity, 3 * plane * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(eigenvect, p.eig, plane * nb * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    return fp4_end(c);
}
