// C-ABI entry points of the B200 scattering-rate path (include/fourphonon_b200.h).
//
// Every call validates its arguments on the host, uploads the caller's
// column-major Fortran arrays (skipping uploads whose bytes did not change
// since the previous call on the context), repacks them on the device into
// the kernel layout, runs the kernels on the context's stream and copies the
// results back into the caller's arrays.  Failures return a negative code
// and leave a message for fp4_last_error(); nothing falls back to the CPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fourphonon_b200.h"
#include "fp4_ctx.h"
#include "fp4_internal.h"

using namespace fp4;

// ---------------------------------------------------------------------------
// context plumbing
// ---------------------------------------------------------------------------
int fp4_fail(fp4_ctx* c, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CK(call)                                                                                      \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) return fp4_fail(c, FP4_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

uint64_t fp4_hash(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    uint64_t h = 1469598103934665603ull;
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t v;
        memcpy(&v, b + i, 8);
        h = (h ^ v) * 1099511628211ull;
        h ^= h >> 29;
    }
    for (; i < n; i++) h = (h ^ b[i]) * 1099511628211ull;
    return h ^ n;
}

int DevBuffer::reserve(fp4_ctx* c, size_t bytes) {
    if (bytes <= cap) return FP4_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    key = 0;
    size_t want = std::max<size_t>(bytes, 256);
    cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) return fp4_fail(c, FP4_E_CUDA, "cudaMalloc(%zu): %s", want, cudaGetErrorString(e));
    cap = want;
    return FP4_OK;
}

int DevBuffer::upload(fp4_ctx* c, const void* host, size_t bytes) {
    uint64_t h = c->upload_cache ? fp4_hash(host, bytes) : 0;
    if (c->upload_cache && ptr && cap >= bytes && key == h && bytes > 0) return FP4_OK;
    int r = reserve(c, bytes);
    if (r) return r;
    if (bytes) {
        cudaError_t e = cudaMemcpyAsync(ptr, host, bytes, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) return fp4_fail(c, FP4_E_CUDA, "upload: %s", cudaGetErrorString(e));
    }
    key = h;
    return FP4_OK;
}

void DevBuffer::release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    key = 0;
}

extern "C" int fp4_create(fp4_ctx** out, int device) {
    if (!out) return FP4_E_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FP4_E_CUDA;
    if (device >= ndev) return FP4_E_ARG;
    fp4_ctx* c = new fp4_ctx();
    if (device < 0) cudaGetDevice(&device);
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev0) != cudaSuccess || cudaEventCreate(&c->ev1) != cudaSuccess ||
        cudaEventCreate(&c->evk0) != cudaSuccess || cudaEventCreate(&c->evk1) != cudaSuccess) {
        delete c;
        return FP4_E_CUDA;
    }
    c->stream = c->own_stream;
    cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device);
    *out = c;
    return FP4_OK;
}

extern "C" int fp4_destroy(fp4_ctx* c) {
    if (!c) return FP4_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (DevBuffer* b : c->all_buffers()) b->release();
    cudaEventDestroy(c->ev0);
    cudaEventDestroy(c->ev1);
    cudaEventDestroy(c->evk0);
    cudaEventDestroy(c->evk1);
    cudaStreamDestroy(c->own_stream);
    delete c;
    return FP4_OK;
}

extern "C" const char* fp4_last_error(const fp4_ctx* c) { return c ? c->err.c_str() : "null context"; }

extern "C" int fp4_set_precision(fp4_ctx* c, int precision) {
    if (!c) return FP4_E_ARG;
    if (precision != FP4_PREC_FP64 && precision != FP4_PREC_MIXED && precision != FP4_PREC_MIXED_SIMT)
        return fp4_fail(c, FP4_E_ARG, "unknown precision %d", precision);
    c->precision = precision;
    return FP4_OK;
}

extern "C" int fp4_last_stats(const fp4_ctx* c, int64_t* n_proc, int64_t* n_contr, double* ms, double* kms,
                              int64_t* launches) {
    if (!c) return FP4_E_ARG;
    if (n_proc) *n_proc = c->last_nproc;
    if (n_contr) *n_contr = c->last_ncontr;
    if (ms) *ms = c->last_ms;
    if (kms) *kms = c->last_kernel_ms;
    if (launches) *launches = c->last_launches;
    return FP4_OK;
}

extern "C" int fp4_last_counters(const fp4_ctx* c, int64_t counters[8]) {
    if (!c || !counters) return FP4_E_ARG;
    for (int x = 0; x < 8; x++) counters[x] = c->last_counters[x];
    return FP4_OK;
}

extern "C" int fp4_last_phase_cycles(const fp4_ctx* c, int64_t cycles[8]) {
    if (!c || !cycles) return FP4_E_ARG;
    for (int x = 0; x < 8; x++) cycles[x] = c->last_counters[8 + x];
    return FP4_OK;
}

extern "C" int fp4_set_stream(fp4_ctx* c, void* stream) {
    if (!c) return FP4_E_ARG;
    cudaStreamSynchronize(c->stream);
    c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream;
    return FP4_OK;
}

extern "C" int fp4_set_upload_cache(fp4_ctx* c, int enable) {
    if (!c) return FP4_E_ARG;
    c->upload_cache = enable != 0;
    if (!c->upload_cache) {
        for (DevBuffer* b : c->all_buffers()) b->key = 0;
        c->eig_packed = false;
        c->wv_packed = false;
    }
    return FP4_OK;
}

// ---------------------------------------------------------------------------
// system upload: globals, harmonic arrays, wedge list
// ---------------------------------------------------------------------------
__global__ void k_pack_wv(int nptk, int nb, const double* energy, const double* velocity, double4* wv) {
    int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= nptk * nb) return;
    int q = x / nb, b = x % nb;
    size_t o = (size_t)b * nptk + q;  // energy(q,b)
    size_t pl = (size_t)nptk * nb;
    wv[x] = make_double4(velocity[o], velocity[o + pl], velocity[o + 2 * pl], energy[o]);
}

__global__ void k_pack_eig(int nptk, int nb, const double2* eigF, double2* eig, float2* eigf) {
    size_t n = (size_t)nptk * nb * nb;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < n; x += (size_t)gridDim.x * blockDim.x) {
        int comp = (int)(x % nb);
        size_t qb = x / nb;
        int q = (int)(qb / nb), b = (int)(qb % nb);
        double2 v = eigF[((size_t)comp * nb + b) * nptk + q];  // eigenvect(q,b,comp)
        eig[x] = v;
        eigf[x] = make_float2((float)v.x, (float)v.y);
    }
}

int fp4_setup_system(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                     const double* eigenvect, int32_t nlist, const int32_t* list, const int32_t* ijk) {
    if (!g || !energy || !velocity || !list || !ijk) return fp4_fail(c, FP4_E_ARG, "null argument");
    for (int d = 0; d < 3; d++)
        if (g->ngrid[d] < 1 || g->ngrid[d] > kMaxGrid)
            return fp4_fail(c, FP4_E_ARG, "ngrid(%d)=%d outside [1,%d]", d + 1, g->ngrid[d], kMaxGrid);
    if (g->natoms < 1 || g->nbands != 3 * g->natoms)
        return fp4_fail(c, FP4_E_ARG, "nbands=%d must equal 3*natoms=%d", g->nbands, 3 * g->natoms);
    if (g->nbands > kMaxNb) return fp4_fail(c, FP4_E_ARG, "nbands=%d exceeds %d", g->nbands, kMaxNb);
    if (g->nelements < 1 || !g->masses || !g->types) return fp4_fail(c, FP4_E_ARG, "masses/types missing");
    for (int a = 0; a < g->natoms; a++)
        if (g->types[a] < 1 || g->types[a] > g->nelements)
            return fp4_fail(c, FP4_E_ARG, "types(%d)=%d outside [1,%d]", a + 1, g->types[a], g->nelements);
    if (!(g->T > 0.0)) return fp4_fail(c, FP4_E_ARG, "T must be >0 K");
    const int nptk = g->ngrid[0] * g->ngrid[1] * g->ngrid[2], nb = g->nbands;
    if (nlist < 1 || nlist > nptk) return fp4_fail(c, FP4_E_ARG, "nlist=%d outside [1,nptk=%d]", nlist, nptk);
    // IJK must be Id2ind's table (config.f90:458-468): the kernels derive grid coordinates from q.
    for (int q = 0; q < nptk; q++) {
        int a = q % g->ngrid[0], b = (q / g->ngrid[0]) % g->ngrid[1], cc = q / (g->ngrid[0] * g->ngrid[1]);
        if (ijk[3 * q] != a || ijk[3 * q + 1] != b || ijk[3 * q + 2] != cc)
            return fp4_fail(c, FP4_E_ARG, "IJK(:,%d) is not the Id2ind table", q + 1);
    }
    std::vector<int> l0(nlist);
    for (int l = 0; l < nlist; l++) {
        if (list[l] < 1 || list[l] > nptk) return fp4_fail(c, FP4_E_ARG, "List(%d)=%d outside [1,nptk]", l + 1, list[l]);
        l0[l] = list[l] - 1;
    }
    DevSys& S = c->S;
    for (int d = 0; d < 3; d++) S.n[d] = g->ngrid[d];
    S.nptk = nptk;
    S.nb = nb;
    S.nlist = nlist;
    S.natoms = g->natoms;
    for (int x = 0; x < 9; x++) S.rl[x] = g->rlattvec[x];
    for (int d = 0; d < 3; d++) {
        S.ngd[d] = (double)g->ngrid[d];
        S.rinv[d] = 1.0 / (double)g->ngrid[d];
    }
    S.scalebroad = g->scalebroad;
    S.omega_max = g->omega_max;
    S.onlyharmonic = g->onlyharmonic ? 1 : 0;
    int r;
    const size_t plane = (size_t)nptk * nb;
    if ((r = c->b_energy.upload(c, energy, plane * sizeof(double)))) return r;
    if ((r = c->b_velocity.upload(c, velocity, 3 * plane * sizeof(double)))) return r;
    const uint64_t wkey = c->b_energy.key ^ (c->b_velocity.key * 31u) ^ (uint64_t)plane;
    if (!c->upload_cache || !c->wv_packed || wkey != c->wv_key) {
        if ((r = c->b_wv.reserve(c, plane * sizeof(double4)))) return r;
        k_pack_wv<<<(int)((plane + 255) / 256), 256, 0, c->stream>>>(nptk, nb, c->b_energy.as<double>(),
                                                                      c->b_velocity.as<double>(), c->b_wv.as<double4>());
        CK(cudaGetLastError());
        c->launches++;
        c->wv_packed = true;
        c->wv_key = wkey;
    }
    if (eigenvect) {
        uint64_t before = c->b_eigraw.key;
        if ((r = c->b_eigraw.upload(c, eigenvect, plane * nb * sizeof(double2)))) return r;
        if (c->b_eigraw.key != before || !c->eig_packed || !c->upload_cache) {
            if ((r = c->b_eig.reserve(c, plane * nb * sizeof(double2)))) return r;
            if ((r = c->b_eigf.reserve(c, plane * nb * sizeof(float2)))) return r;
            k_pack_eig<<<1024, 256, 0, c->stream>>>(nptk, nb, c->b_eigraw.as<double2>(), c->b_eig.as<double2>(),
                                                    c->b_eigf.as<float2>());
            CK(cudaGetLastError());
            c->launches++;
            c->eig_packed = true;
        }
        S.eig = c->b_eig.as<double2>();
        S.eigf = c->b_eigf.as<float2>();
    } else {
        S.eig = nullptr;
        S.eigf = nullptr;
    }
    if ((r = c->b_list.upload(c, l0.data(), nlist * sizeof(int)))) return r;
    std::vector<int> qc(nptk);
    for (int q = 0; q < nptk; q++) qc[q] = ijk[3 * q] | (ijk[3 * q + 1] << 8) | (ijk[3 * q + 2] << 16);
    if ((r = c->b_qc.upload(c, qc.data(), nptk * sizeof(int)))) return r;
    S.qc = c->b_qc.as<int>();
    S.wv = c->b_wv.as<double4>();
    S.list0 = c->b_list.as<int>();
    // root tables exp(2 pi i x / N_d)
    for (int d = 0; d < 3; d++) {
        int N = g->ngrid[d];
        std::vector<double2> rt(N);
        std::vector<float2> rf(N);
        for (int x = 0; x < N; x++) {
            long double ang = 2.0L * 3.141592653589793238462643383279502884L * (long double)x / (long double)N;
            rt[x] = make_double2((double)cosl(ang), (double)sinl(ang));
            rf[x] = make_float2((float)cosl(ang), (float)sinl(ang));
        }
        if ((r = c->b_root[d].upload(c, rt.data(), N * sizeof(double2)))) return r;
        if ((r = c->b_rootf[d].upload(c, rf.data(), N * sizeof(float2)))) return r;
        S.root[d] = c->b_root[d].as<double2>();
        S.rootf[d] = c->b_rootf[d].as<float2>();
    }
    // masses per atom for the cluster prefactors
    c->atom_mass.assign(g->natoms, 0.0);
    for (int a = 0; a < g->natoms; a++) c->atom_mass[a] = g->masses[g->types[a] - 1];
    return FP4_OK;
}

// ---------------------------------------------------------------------------
// cluster tables: integer cells, displacement classes, device layout
// ---------------------------------------------------------------------------
int fp4_setup_ifc(fp4_ctx* c, const fp4_globals* g, int order, int32_t ntri, const double* phi, const double* rj,
                  const double* rk, const double* rl, const int32_t* ii, const int32_t* ij, const int32_t* ik,
                  const int32_t* il, IfcTables& T) {
    if (ntri < 1 || !phi || !rj || !rk || !ii || !ij || !ik || (order == 4 && (!rl || !il)))
        return fp4_fail(c, FP4_E_ARG, "IFC arrays missing (Ntri=%d)", ntri);
    const int nat = g->natoms;
    const int K = order == 3 ? 27 : 81;
    // integer lattice coordinates m = rlattvec^T R / (2 pi) (R was rounded to a lattice vector by read3fc/read4fc)
    auto cell = [&](const double* R, int cidx, int4& m) -> bool {
        double x[3];
        for (int d = 0; d < 3; d++) {
            const double* b = g->rlattvec + 3 * d;
            x[d] = (b[0] * R[3 * cidx] + b[1] * R[3 * cidx + 1] + b[2] * R[3 * cidx + 2]) / (2.0 * M_PI);
        }
        int v[3];
        for (int d = 0; d < 3; d++) {
            v[d] = (int)std::lround(x[d]);
            if (std::fabs(x[d] - v[d]) > 1e-6) return false;
        }
        m = make_int4(v[0], v[1], v[2], 0);
        return true;
    };
    std::vector<int4> atoms(ntri), mj(ntri), mk(ntri), ml(ntri, make_int4(0, 0, 0, 0));
    std::vector<double> mu(ntri), ph((size_t)ntri * K);
    for (int t = 0; t < ntri; t++) {
        int a[4] = {ii[t], ij[t], ik[t], order == 4 ? il[t] : 1};
        for (int x = 0; x < order; x++)
            if (a[x] < 1 || a[x] > nat) return fp4_fail(c, FP4_E_ARG, "cluster %d: atom index %d outside [1,%d]", t + 1, a[x], nat);
        atoms[t] = make_int4(a[0] - 1, a[1] - 1, a[2] - 1, a[3] - 1);
        if (!cell(rj, t, mj[t]) || !cell(rk, t, mk[t]) || (order == 4 && !cell(rl, t, ml[t])))
            return fp4_fail(c, FP4_E_ARG, "cluster %d: cell vector is not a lattice vector", t + 1);
        double m = c->atom_mass[a[0] - 1] * c->atom_mass[a[1] - 1] * c->atom_mass[a[2] - 1];
        if (order == 4) m = m * c->atom_mass[a[3] - 1];
        mu[t] = 1.0 / std::sqrt(m);
        // device layout [first][second][third]([fourth]) from Fortran Phi(t,s,r,c) / Psi(u,t,s,r,c)
        for (int e = 0; e < K; e++) {
            int i0 = e % 3, i1 = (e / 3) % 3, i2 = (e / 9) % 3, i3 = e / 27;
            int dst = (order == 3) ? ((i0 * 3 + i1) * 3 + i2) : (((i0 * 3 + i1) * 3 + i2) * 3 + i3);
            ph[(size_t)t * K + dst] = phi[(size_t)t * K + e];
        }
    }
    // displacement classes: 3ph (m_j-m_k, a2, a3), 4ph (m_k-m_l, a3, a4)
    std::map<std::tuple<int, int, int, int, int, int>, std::vector<int>> cls;  // (block, Dx, Dy, Dz) -> clusters
    for (int t = 0; t < ntri; t++) {
        int4 A = order == 3 ? mj[t] : mk[t];
        int4 B = order == 3 ? mk[t] : ml[t];
        int aa = order == 3 ? atoms[t].y : atoms[t].z;
        int ab = order == 3 ? atoms[t].z : atoms[t].w;
        int blk = aa * nat + ab;
        cls[std::make_tuple(blk, A.x - B.x, A.y - B.y, A.z - B.z, aa, ab)].push_back(t);
    }
    const int npi = (int)cls.size();
    std::vector<int> cl_start(npi + 1), cl_index, blk_start(nat * nat + 1, 0);
    std::vector<int4> pi_d(npi);
    int p = 0;
    for (auto& kv : cls) {
        cl_start[p] = (int)cl_index.size();
        for (int t : kv.second) cl_index.push_back(t);
        pi_d[p] = make_int4(std::get<1>(kv.first), std::get<2>(kv.first), std::get<3>(kv.first),
                            std::get<4>(kv.first) * 256 + std::get<5>(kv.first));
        blk_start[std::get<0>(kv.first) + 1]++;
        p++;
    }
    cl_start[npi] = (int)cl_index.size();
    for (int b = 0; b < nat * nat; b++) blk_start[b + 1] += blk_start[b];
    int r;
    if ((r = T.phi.upload(c, ph.data(), ph.size() * sizeof(double)))) return r;
    if ((r = T.atoms.upload(c, atoms.data(), ntri * sizeof(int4)))) return r;
    if ((r = T.mj.upload(c, mj.data(), ntri * sizeof(int4)))) return r;
    if ((r = T.mk.upload(c, mk.data(), ntri * sizeof(int4)))) return r;
    if ((r = T.ml.upload(c, ml.data(), ntri * sizeof(int4)))) return r;
    if ((r = T.mu.upload(c, mu.data(), ntri * sizeof(double)))) return r;
    if ((r = T.cl_start.upload(c, cl_start.data(), (npi + 1) * sizeof(int)))) return r;
    if ((r = T.cl_index.upload(c, cl_index.data(), ntri * sizeof(int)))) return r;
    if ((r = T.pi_d.upload(c, pi_d.data(), npi * sizeof(int4)))) return r;
    if ((r = T.blk_start.upload(c, blk_start.data(), (nat * nat + 1) * sizeof(int)))) return r;
    T.h_blk_start = blk_start;
    DevIfc& F = T.F;
    F.order = order;
    F.ntri = ntri;
    F.npi = npi;
    F.nblk = nat * nat;
    F.phi = T.phi.as<double>();
    F.atoms = T.atoms.as<int4>();
    F.mj = T.mj.as<int4>();
    F.mk = T.mk.as<int4>();
    F.ml = T.ml.as<int4>();
    F.mu = T.mu.as<double>();
    F.cl_start = T.cl_start.as<int>();
    F.cl_index = T.cl_index.as<int>();
    F.pi_d = T.pi_d.as<int4>();
    F.blk_start = T.blk_start.as<int>();
    return FP4_OK;
}

// ---------------------------------------------------------------------------
// helpers for kernels' error flag and timing
// ---------------------------------------------------------------------------
int fp4_begin(fp4_ctx* c) {
    cudaError_t e = cudaSetDevice(c->device);
    if (e != cudaSuccess) return fp4_fail(c, FP4_E_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    int r;
    if ((r = c->b_err.reserve(c, 64))) return r;
    if ((r = c->b_stats.reserve(c, 128))) return r;
    c->launches = 0;
    c->kernel_timed = false;
    c->last_tc = false;
    CK(cudaEventRecord(c->ev0, c->stream));
    CK(cudaMemsetAsync(c->b_err.ptr, 0, 64, c->stream));
    CK(cudaMemsetAsync(c->b_stats.ptr, 0, 128, c->stream));
    return FP4_OK;
}

int fp4_end(fp4_ctx* c) {
    CK(cudaEventRecord(c->ev1, c->stream));
    int flags = 0;
    unsigned long long st[16] = {0};
    CK(cudaMemcpyAsync(&flags, c->b_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(st, c->b_stats.ptr, sizeof st, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    c->last_ms = ms;
    c->last_kernel_ms = 0.0;
    if (c->kernel_timed) {
        float kms = 0.f;
        cudaEventElapsedTime(&kms, c->evk0, c->evk1);
        c->last_kernel_ms = kms;
    }
    c->last_launches = c->launches;
    c->last_nproc = (int64_t)st[0];
    c->last_ncontr = (int64_t)st[1];
    for (int x = 0; x < 16; x++) c->last_counters[x] = (int64_t)st[x];
    c->last_counters[7] = c->last_tc ? 1 : 0;
    if (flags & kErrQueue) return fp4_fail(c, FP4_E_CAPACITY, "an output list or work queue was smaller than the process count");
    if (flags & kErrTable) return fp4_fail(c, FP4_E_CAPACITY, "a device table limit was exceeded");
    if (flags & kErrList) return fp4_fail(c, FP4_E_ARG, "a process list entry is out of range or breaks momentum conservation");
    if (flags & kErrTimeout) return fp4_fail(c, FP4_E_TIMEOUT, "a bounded wait for the tensor core gave up");
    return FP4_OK;
}

static const double kPi = 3.141592653589793238;
static double hbarp() { return 1.05457172647e-22 * (double)1e22f; }  // processes.f90:20, REAL 1e22

// ---------------------------------------------------------------------------
// three-phonon drivers
// ---------------------------------------------------------------------------
static int run_k3(fp4_ctx* c, int mode, const fp4_globals* g, P3Params& p) {
    p.S = c->S;
    p.F = c->ifc3.F;
    p.stats = c->b_stats.as<unsigned long long>();
    p.err = c->b_err.as<int>();
    p.scale = hbarp() * kPi / 4.0;
    p.unit = (double)5.60626442f * 1.e8;
    if (mode >= 2) {
        int r;
        if ((r = c->b_temps.upload(c, &g->T, sizeof(double)))) return r;
        if ((r = c->b_bose.reserve(c, (size_t)c->S.nptk * c->S.nb * sizeof(double)))) return r;
        CK(launch_bose(c->S, c->b_temps.as<double>(), 1, c->b_bose.as<double>(), c->stream));
        c->launches++;
        p.bose = c->b_bose.as<double>();
    }
    size_t sm = k3_smem(mode, p.F, c->S.onlyharmonic);
    if (sm > 227 * 1024) return fp4_fail(c, FP4_E_CAPACITY, "3ph cluster table needs %zu B of shared memory", sm);
    CK(cudaEventRecord(c->evk0, c->stream));
    CK(launch_k3(mode, p, c->S.nb * c->S.nlist, c->stream));
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_timed = true;
    c->launches++;
    return FP4_OK;
}

// 3-phonon RTA of the context's current system into device memory d_out:
// rate_plus, rate_minus (with the factor 1/2), WP3_plus, WP3_minus, each nbands*nlist.
int fp4_launch_rta3(fp4_ctx* c, const fp4_globals* g, double* d_out) {
    const int nm = c->S.nb * c->S.nlist;
    P3Params p{};
    p.rate[0] = d_out;
    p.rate[1] = d_out + nm;
    p.wp[0] = d_out + 2 * nm;
    p.wp[1] = d_out + 3 * nm;
    return run_k3(c, 2, g, p);
}

extern "C" int fp4_np_driver(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                             int32_t nlist, const int32_t* list, const int32_t* ijk, int32_t* n_plus,
                             double* p_plus, int32_t* n_minus, double* p_minus) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!n_plus || !n_minus || !p_plus || !p_minus) return fp4_fail(c, FP4_E_ARG, "null output");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, nullptr, nlist, list, ijk))) return r;
    const int nm = c->S.nb * nlist;
    if ((r = c->b_out.reserve(c, (size_t)nm * 2 * (sizeof(int32_t) + sizeof(double))))) return r;
    int32_t* dn = c->b_out.as<int32_t>();
    double* dp = reinterpret_cast<double*>(dn + 2 * nm + (2 * nm & 1));
    P3Params p{};
    p.n_out[0] = dn;
    p.n_out[1] = dn + nm;
    p.p_out[0] = dp;
    p.p_out[1] = dp + nm;
    c->ifc3.F.npi = 0;
    if ((r = run_k3(c, 0, g, p))) return r;
    CK(cudaMemcpyAsync(n_plus, dn, nm * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(n_minus, dn + nm, nm * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(p_plus, dp, nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(p_minus, dp + nm, nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return fp4_end(c);
}

static int offsets_of(const int32_t* n, int nm, std::vector<long long>& off) {
    off.assign(nm + 1, 0);
    for (int m = 0; m < nm; m++) off[m + 1] = off[m] + n[m];
    return FP4_OK;
}

extern "C" int fp4_ind_only_driver(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                                   int32_t nlist, const int32_t* list, const int32_t* ijk, const int32_t* n_plus,
                                   const int32_t* n_minus, int32_t* ind2_plus, int32_t* ind3_plus, int32_t* ind2_minus,
                                   int32_t* ind3_minus) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!n_plus || !n_minus) return fp4_fail(c, FP4_E_ARG, "null N_plus/N_minus");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, nullptr, nlist, list, ijk))) return r;
    const int nm = c->S.nb * nlist;
    std::vector<long long> op, om;
    offsets_of(n_plus, nm, op);
    offsets_of(n_minus, nm, om);
    const long long tp = op[nm], tm = om[nm];
    if ((tp && (!ind2_plus || !ind3_plus)) || (tm && (!ind2_minus || !ind3_minus)))
        return fp4_fail(c, FP4_E_ARG, "null index list");
    if ((r = c->b_lists.reserve(c, (size_t)(tp + tm) * 2 * sizeof(int32_t) + 64))) return r;
    if ((r = c->b_off.reserve(c, (size_t)(nm + 1) * 2 * sizeof(long long)))) return r;
    if ((r = c->b_counts.reserve(c, (size_t)nm * 2 * sizeof(int32_t)))) return r;
    long long* doff = c->b_off.as<long long>();
    int32_t* dcnt = c->b_counts.as<int32_t>();
    CK(cudaMemcpyAsync(doff, op.data(), (nm + 1) * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(doff + nm + 1, om.data(), (nm + 1) * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dcnt, n_plus, nm * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dcnt + nm, n_minus, nm * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    int32_t* L = c->b_lists.as<int32_t>();
    P3Params p{};
    p.list_off[0] = doff;
    p.list_off[1] = doff + nm + 1;
    p.nlist_counts[0] = dcnt;
    p.nlist_counts[1] = dcnt + nm;
    p.ind2[0] = L;
    p.ind3[0] = L + tp;
    p.ind2[1] = L + 2 * tp;
    p.ind3[1] = L + 2 * tp + tm;
    c->ifc3.F.npi = 0;
    if ((r = run_k3(c, 1, g, p))) return r;
    if (tp) {
        CK(cudaMemcpyAsync(ind2_plus, L, tp * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(ind3_plus, L + tp, tp * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    }
    if (tm) {
        CK(cudaMemcpyAsync(ind2_minus, L + 2 * tp, tm * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(ind3_minus, L + 2 * tp + tm, tm * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
    }
    return fp4_end(c);
}

extern "C" int fp4_rta_driver(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                              const double* eigenvect, int32_t nlist, const int32_t* list, const int32_t* ijk,
                              int32_t ntri, const double* phi, const double* r_j, const double* r_k,
                              const int32_t* index_i, const int32_t* index_j, const int32_t* index_k, double* rate,
                              double* rate_plus, double* rate_minus, double* wp3_plus, double* wp3_minus) {
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
    P3Params p{};
    p.rate[0] = d;
    p.rate[1] = d + nm;
    p.wp[0] = d + 2 * nm;
    p.wp[1] = d + 3 * nm;
    if ((r = run_k3(c, 2, g, p))) return r;
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

extern "C" int fp4_ind_driver(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                              const double* eigenvect, int32_t nlist, const int32_t* list, const int32_t* ijk,
                              const int32_t* n_plus, const int32_t* n_minus, int32_t ntri, const double* phi,
                              const double* r_j, const double* r_k, const int32_t* index_i, const int32_t* index_j,
                              const int32_t* index_k, int32_t* ind2_plus, int32_t* ind3_plus, double* gamma_plus,
                              int32_t* ind2_minus, int32_t* ind3_minus, double* gamma_minus, double* rate,
                              double* rate_plus, double* rate_minus, double* wp3_plus, double* wp3_minus) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!n_plus || !n_minus || !rate || !rate_plus || !rate_minus || !wp3_plus || !wp3_minus || !eigenvect)
        return fp4_fail(c, FP4_E_ARG, "null argument");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, eigenvect, nlist, list, ijk))) return r;
    if ((r = fp4_setup_ifc(c, g, 3, ntri, phi, r_j, r_k, nullptr, index_i, index_j, index_k, nullptr, c->ifc3))) return r;
    const int nm = c->S.nb * nlist;
    std::vector<long long> op, om;
    offsets_of(n_plus, nm, op);
    offsets_of(n_minus, nm, om);
    const long long tp = op[nm], tm = om[nm];
    if ((tp && (!ind2_plus || !ind3_plus || !gamma_plus)) || (tm && (!ind2_minus || !ind3_minus || !gamma_minus)))
        return fp4_fail(c, FP4_E_ARG, "null list output");
    if ((r = c->b_lists.reserve(c, (size_t)(tp + tm) * 2 * sizeof(int32_t) + 64))) return r;
    if ((r = c->b_gamma.reserve(c, (size_t)(tp + tm) * sizeof(double) + 64))) return r;
    if ((r = c->b_off.reserve(c, (size_t)(nm + 1) * 2 * sizeof(long long)))) return r;
    if ((r = c->b_counts.reserve(c, (size_t)nm * 2 * sizeof(int32_t)))) return r;
    if ((r = c->b_out.reserve(c, (size_t)nm * 4 * sizeof(double)))) return r;
    long long* doff = c->b_off.as<long long>();
    int32_t* dcnt = c->b_counts.as<int32_t>();
    CK(cudaMemcpyAsync(doff, op.data(), (nm + 1) * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(doff + nm + 1, om.data(), (nm + 1) * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dcnt, n_plus, nm * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dcnt + nm, n_minus, nm * sizeof(int32_t), cudaMemcpyHostToDevice, c->stream));
    int32_t* L = c->b_lists.as<int32_t>();
    double* G = c->b_gamma.as<double>();
    double* d = c->b_out.as<double>();
    P3Params p{};
    p.list_off[0] = doff;
    p.list_off[1] = doff + nm + 1;
    p.nlist_counts[0] = dcnt;
    p.nlist_counts[1] = dcnt + nm;
    p.ind2[0] = L;
    p.ind3[0] = L + tp;
    p.ind2[1] = L + 2 * tp;
    p.ind3[1] = L + 2 * tp + tm;
    p.gamma[0] = G;
    p.gamma[1] = G + tp;
    p.rate[0] = d;
    p.rate[1] = d + nm;
    p.wp[0] = d + 2 * nm;
    p.wp[1] = d + 3 * nm;
    if ((r = run_k3(c, 3, g, p))) return r;
    if (tp) {
        CK(cudaMemcpyAsync(ind2_plus, L, tp * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(ind3_plus, L + tp, tp * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(gamma_plus, G, tp * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    if (tm) {
        CK(cudaMemcpyAsync(ind2_minus, L + 2 * tp, tm * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(ind3_minus, L + 2 * tp + tm, tm * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(gamma_minus, G + tp, tm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
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

// ---------------------------------------------------------------------------
// four-phonon drivers
// ---------------------------------------------------------------------------
static int k4_blocks(fp4_ctx* c, int nwork, int kind, int nT) {
    int nbk = c->sm_count * k4_ctas_per_sm(kind, nT, c->precision != FP4_PREC_FP64);
    return std::max(1, std::min(nbk, nwork));
}

// The four-phonon work items of the context's system, or FP4_E_CAPACITY when
// there are more than the kernels' 32-bit work counter can hand out.
static int k4_nwork(fp4_ctx* c, int& nwork) {
    const long long n = k4_work_items(c->S.nlist, c->S.nptk);
    if (n > kMaxWorkItems)
        return fp4_fail(c, FP4_E_CAPACITY, "3*nlist*nptk = %lld four-phonon work items, above the limit of %lld", n,
                        kMaxWorkItems);
    nwork = (int)n;
    return FP4_OK;
}

static int run_np4(fp4_ctx* c, int64_t* n_out[3], double* p_out[3]) {
    const int nm = c->S.nb * c->S.nlist;
    int r, nwork = 0;
    if ((r = k4_nwork(c, nwork))) return r;
    if ((r = c->b_out.reserve(c, (size_t)nm * 3 * (sizeof(unsigned long long) + sizeof(double))))) return r;
    if ((r = c->b_work.reserve(c, 64))) return r;
    unsigned long long* dn = c->b_out.as<unsigned long long>();
    double* dp = reinterpret_cast<double*>(dn + 3 * nm);
    CK(cudaMemsetAsync(dn, 0, (size_t)nm * 3 * (sizeof(unsigned long long) + sizeof(double)), c->stream));
    CK(cudaMemsetAsync(c->b_work.ptr, 0, 64, c->stream));
    P4Params p{};
    p.S = c->S;
    p.F = DevIfc{};
    p.nT = 1;
    p.nwork = nwork;
    p.work_counter = c->b_work.as<int>();
    p.n_count = dn;
    p.p_sum = dp;
    p.stats = c->b_stats.as<unsigned long long>();
    p.err = c->b_err.as<int>();
    CK(cudaEventRecord(c->evk0, c->stream));
    CK(launch_k4(0, 1, false, p, k4_blocks(c, p.nwork, 0, 1), c->stream));
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_timed = true;
    c->launches++;
    std::vector<unsigned long long> hn((size_t)nm * 3);
    std::vector<double> hp((size_t)nm * 3);
    CK(cudaMemcpyAsync(hn.data(), dn, hn.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(hp.data(), dp, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((r = fp4_end(c))) return r;
    for (int ch = 0; ch < 3; ch++)
        for (int m = 0; m < nm; m++) {
            n_out[ch][m] = (int64_t)hn[(size_t)ch * nm + m];
            p_out[ch][m] = hp[(size_t)ch * nm + m];
        }
    return FP4_OK;
}

extern "C" int fp4_np_driver_4ph(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                                 int32_t nlist, const int32_t* list, const int32_t* ijk, int64_t* n_pp, double* p_pp,
                                 int64_t* n_pm, double* p_pm, int64_t* n_mm, double* p_mm) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!n_pp || !n_pm || !n_mm || !p_pp || !p_pm || !p_mm) return fp4_fail(c, FP4_E_ARG, "null output");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, nullptr, nlist, list, ijk))) return r;
    int64_t* n_out[3] = {n_pp, n_pm, n_mm};
    double* p_out[3] = {p_pp, p_pm, p_mm};
    return run_np4(c, n_out, p_out);
}

extern "C" int fp4_ind_only_driver_4ph(fp4_ctx* c, const fp4_globals* g, const double* energy,
                                       const double* velocity, int32_t nlist, const int32_t* list, const int32_t* ijk,
                                       const int64_t* n_pp, const int64_t* n_pm, const int64_t* n_mm, int64_t* i2pp,
                                       int64_t* i3pp, int64_t* i4pp, int64_t* i2pm, int64_t* i3pm, int64_t* i4pm,
                                       int64_t* i2mm, int64_t* i3mm, int64_t* i4mm) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!n_pp || !n_pm || !n_mm) return fp4_fail(c, FP4_E_ARG, "null counts");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, nullptr, nlist, list, ijk))) return r;
    const int nm = c->S.nb * nlist;
    const int64_t* N[3] = {n_pp, n_pm, n_mm};
    int64_t* O[3][3] = {{i2pp, i3pp, i4pp}, {i2pm, i3pm, i4pm}, {i2mm, i3mm, i4mm}};
    for (int ch = 0; ch < 3; ch++) {
        std::vector<long long> off(nm + 1, 0);
        for (int m = 0; m < nm; m++) {
            if (N[ch][m] < 0) return fp4_fail(c, FP4_E_ARG, "negative count");
            off[m + 1] = off[m] + N[ch][m];
        }
        const long long tot = off[nm];
        if (tot == 0) continue;
        if (!O[ch][0] || !O[ch][1] || !O[ch][2]) return fp4_fail(c, FP4_E_ARG, "null index list");
        if ((r = c->b_lists.reserve(c, (size_t)tot * 3 * sizeof(long long)))) return r;
        if ((r = c->b_off.reserve(c, (size_t)(nm + 1) * sizeof(long long)))) return r;
        if ((r = c->b_counts.reserve(c, (size_t)nm * sizeof(long long)))) return r;
        CK(cudaMemcpyAsync(c->b_off.ptr, off.data(), (nm + 1) * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
        CK(cudaMemcpyAsync(c->b_counts.ptr, N[ch], nm * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
        long long* L = c->b_lists.as<long long>();
        P4OrderParams p{};
        p.S = c->S;
        p.ch = ch;
        p.list_off = c->b_off.as<long long>();
        p.counts = c->b_counts.as<long long>();
        p.ind2 = L;
        p.ind3 = L + tot;
        p.ind4 = L + 2 * tot;
        p.err = c->b_err.as<int>();
        CK(launch_k4_order(p, nm, c->stream));
        c->launches++;
        for (int x = 0; x < 3; x++)
            CK(cudaMemcpyAsync(O[ch][x], L + x * tot, tot * sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return fp4_end(c);
}

// Queue of the four-phonon work kernel: per CTA nb*nb bins of `subcap` entries of
// (packed indices, sigma[, list position]).  The kernel flushes when a bin could
// exceed subcap within the next capacity check (8 passes of one entry per thread),
// so subcap must exceed 8*threads.
static int k4_queue(fp4_ctx* c, int nblocks, bool with_pos, P4Params& p) {
    const DevSys& S = c->S;
    const size_t bins = (size_t)nblocks * S.nb * S.nb;
    const int min_cap = 16 * k4_threads();
    int subcap = 2 * min_cap;
    const size_t entry = sizeof(unsigned long long) + sizeof(double) + (with_pos ? sizeof(long long) : 0);
    while (subcap > min_cap && bins * subcap * entry > ((size_t)4 << 30)) subcap /= 2;
    int r;
    if ((r = c->b_queue.reserve(c, bins * subcap * entry))) return r;
    p.queue = c->b_queue.as<unsigned long long>();
    p.queue_sigma = reinterpret_cast<double*>(p.queue + bins * subcap);
    p.queue_pos = with_pos ? reinterpret_cast<long long*>(p.queue_sigma + bins * subcap) : nullptr;
    p.subcap = subcap;
    return FP4_OK;
}

// Four-phonon RTA at nT temperatures; outputs device-resident in c->b_out4 as (nb,nlist,nT) x 6.
// The tensor-core plan of the four-phonon RTA call, if the mixed precision asks for
// it and its tables fit in shared memory: zbins as large as keeps two CTAs per SM
// (else one); returns false when the CUDA-core FP32 contraction has to run instead.
static bool k4_tc_setup(fp4_ctx* c, int nT, int subcap, TcPlan& plan, size_t& smem, int& ctas) {
    const DevSys& S = c->S;
    const DevIfc& F = c->ifc4.F;
    if (c->precision != FP4_PREC_MIXED || S.onlyharmonic) return false;
    if (k4_tc_plan(S.nb, S.natoms, F.npi, c->ifc4.h_blk_start.data(), subcap, plan) != 0) return false;
    const size_t per_sm = 228 * 1024, per_cta_max = 227 * 1024;
    const int base_cap = plan.chunk_cap;
    for (int zb = 8; zb >= 1; zb--) {
        TcPlan q = plan;
        q.zbins = zb;
        q.chunk_cap = zb * base_cap;
        const size_t need = k4_tc_smem(nT, S, F, q);
        if (2 * (need + 1024) <= per_sm || (zb == 1 && need <= per_cta_max)) {
            plan = q;
            smem = need;
            ctas = (2 * (need + 1024) <= per_sm) ? 2 : 1;
            return true;
        }
    }
    return false;
}

int fp4_run_rta4(fp4_ctx* c, int nT, const double* temps) {
    if (nT < 1 || nT > kMaxTemps) return fp4_fail(c, FP4_E_ARG, "nT=%d outside [1,%d]", nT, kMaxTemps);
    for (int t = 0; t < nT; t++)
        if (!(temps[t] > 0.0)) return fp4_fail(c, FP4_E_ARG, "T must be >0 K");
    const DevSys& S = c->S;
    const int nm = S.nb * S.nlist;
    const bool mixed = (c->precision != FP4_PREC_FP64);
    size_t sm = k4_smem(2, nT, mixed, S, c->ifc4.F);
    int r, nwork = 0;
    if ((r = k4_nwork(c, nwork))) return r;
    // the queue is sized for the larger of the two grids; the tensor-core plan needs its capacity
    int nblocks = k4_blocks(c, nwork, 2, nT);
    P4Params p{};
    if ((r = k4_queue(c, std::max(nblocks, c->sm_count * k4_tc_ctas_per_sm()), false, p))) return r;
    TcPlan plan{};
    size_t tc_smem = 0;
    int tc_ctas = 0;
    const bool use_tc = k4_tc_setup(c, nT, p.subcap, plan, tc_smem, tc_ctas);
    if (!use_tc && sm > 227 * 1024)
        return fp4_fail(c, FP4_E_CAPACITY, "4ph reciprocal cluster table needs %zu B of shared memory (limit 227 KB)", sm);
    if (use_tc) nblocks = std::max(1, std::min(nwork, c->sm_count * tc_ctas));
    c->last_tc = use_tc;
    if ((r = c->b_temps.upload(c, temps, nT * sizeof(double)))) return r;
    const int wbs = wb_stride(k4_round_nt(nT));
    if ((r = c->b_wb.reserve(c, (size_t)S.nptk * S.nb * wbs * sizeof(double)))) return r;
    CK(launch_wbose(S, c->b_temps.as<double>(), nT, wbs, c->b_wb.as<double>(), c->stream));
    c->launches++;
    if (use_tc) {
        if ((r = c->b_tcplan.reserve(c, sizeof(TcPlan)))) return r;
        CK(cudaMemcpyAsync(c->b_tcplan.ptr, &plan, sizeof(TcPlan), cudaMemcpyHostToDevice, c->stream));
        if ((r = c->b_wtab.reserve(c, (size_t)2 * S.nptk * plan.ksteps * 16 * sizeof(uint16_t)))) return r;
        CK(launch_k4_wtab(S, c->ifc4.F, c->b_tcplan.as<TcPlan>(), plan.ksteps, c->b_wtab.as<uint16_t>(), c->stream));
        c->launches++;
        p.tc = c->b_tcplan.as<TcPlan>();
        p.wtab = c->b_wtab.as<uint16_t>();
    }
    if ((r = c->b_part.reserve(c, (size_t)nwork * nT * S.nb * 2 * sizeof(double)))) return r;
    if ((r = c->b_work.reserve(c, 64))) return r;
    if ((r = c->b_out4.reserve(c, (size_t)nm * nT * 6 * sizeof(double)))) return r;
    CK(cudaMemsetAsync(c->b_work.ptr, 0, 64, c->stream));
    p.S = S;
    p.F = c->ifc4.F;
    p.nT = nT;
    p.wb = c->b_wb.as<double>();
    p.nwork = nwork;
    p.work_counter = c->b_work.as<int>();
    p.part_rate = c->b_part.as<double>();
    p.part_wp = p.part_rate + (size_t)nwork * nT * S.nb;
    p.stats = c->b_stats.as<unsigned long long>();
    p.err = c->b_err.as<int>();
    CK(cudaEventRecord(c->evk0, c->stream));
    if (use_tc)
        CK(launch_k4_tc(nT, p, tc_smem, nblocks, c->stream));
    else
        CK(launch_k4(2, nT, mixed, p, nblocks, c->stream));
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_timed = true;
    c->launches++;
    c->last_rta4_nT = nT;
    double* o = c->b_out4.as<double>();
    const size_t blk = (size_t)nm * nT;
    const double rate_scale = hbarp() * hbarp() * kPi / 8.0 * (double)3.37617087f * 1.e9;
    CK(launch_k4_reduce(p, o, o + blk, o + 2 * blk, o + 3 * blk, o + 4 * blk, o + 5 * blk, rate_scale, c->stream));
    c->launches++;
    return FP4_OK;
}

extern "C" int fp4_rta_driver_4ph_multi_t(fp4_ctx* c, const fp4_globals* g, int32_t nT, const double* temperatures,
                                          const double* energy, const double* velocity, const double* eigenvect,
                                          int32_t nlist, const int32_t* list, const int32_t* ijk, int32_t ntri,
                                          const double* psi, const double* r_j, const double* r_k, const double* r_l,
                                          const int32_t* index_i, const int32_t* index_j, const int32_t* index_k,
                                          const int32_t* index_l, double* rate_pp, double* rate_pm, double* rate_mm,
                                          double* wp_pp, double* wp_pm, double* wp_mm) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!temperatures || !rate_pp || !rate_pm || !rate_mm || !wp_pp || !wp_pm || !wp_mm || !eigenvect)
        return fp4_fail(c, FP4_E_ARG, "null argument");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, eigenvect, nlist, list, ijk))) return r;
    if ((r = fp4_setup_ifc(c, g, 4, ntri, psi, r_j, r_k, r_l, index_i, index_j, index_k, index_l, c->ifc4))) return r;
    if ((r = fp4_run_rta4(c, nT, temperatures))) return r;
    const size_t blk = (size_t)c->S.nb * nlist * nT;
    double* o = c->b_out4.as<double>();
    double* outs[6] = {rate_pp, rate_pm, rate_mm, wp_pp, wp_pm, wp_mm};
    for (int x = 0; x < 6; x++) CK(cudaMemcpyAsync(outs[x], o + x * blk, blk * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return fp4_end(c);
}

// Per-q' parts of the last four-phonon RTA call: the rates and WP4 of list point ll
// (0-based) at temperature t from the processes whose second phonon q' lies in
// [ii0, ii1), normalised as the full driver normalises them.  The per-work-item
// partial sums stay on the device until the next four-phonon call.
extern "C" int fp4_rta4_partials(fp4_ctx* c, int32_t ll, int32_t ii0, int32_t ii1, int32_t t, double* rate_pp,
                                 double* rate_pm, double* rate_mm, double* wp_pp, double* wp_pm, double* wp_mm) {
    if (!c) return FP4_E_ARG;
    const DevSys& S = c->S;
    const int nT = c->last_rta4_nT;
    if (nT < 1) return fp4_fail(c, FP4_E_STATE, "no four-phonon RTA call to inspect");
    if (ll < 0 || ll >= S.nlist || ii0 < 0 || ii1 > S.nptk || ii0 >= ii1 || t < 0 || t >= nT)
        return fp4_fail(c, FP4_E_ARG, "partials: ll=%d q' [%d,%d) t=%d outside the last call", ll, ii0, ii1, t);
    if (!rate_pp || !rate_pm || !rate_mm || !wp_pp || !wp_pm || !wp_mm) return fp4_fail(c, FP4_E_ARG, "null output");
    const int nb = S.nb;
    const size_t nwork = (size_t)3 * S.nlist * S.nptk;
    const size_t per_q = (size_t)3 * nT * nb;  // the three channels' records of one q'
    const size_t first = ((size_t)ll * S.nptk + ii0) * 3;
    const size_t n = (size_t)(ii1 - ii0) * per_q;
    std::vector<double> hr(n), hw(n);
    const double* part = c->b_part.as<double>();
    CK(cudaMemcpyAsync(hr.data(), part + first * nT * nb, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(hw.data(), part + nwork * nT * nb + first * nT * nb, n * sizeof(double), cudaMemcpyDeviceToHost,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double* R[3] = {rate_pp, rate_pm, rate_mm};
    double* W[3] = {wp_pp, wp_pm, wp_mm};
    const double rate_scale = hbarp() * hbarp() * kPi / 8.0 * (double)3.37617087f * 1.e9;
    for (int ch = 0; ch < 3; ch++)
        for (int i = 0; i < nb; i++) {
            double r = 0.0, w = 0.0;
            for (int q = 0; q < ii1 - ii0; q++) {
                const size_t o = (((size_t)q * 3 + ch) * nT + t) * nb + i;
                r += hr[o];
                w += hw[o];
            }
            R[ch][i] = r * rate_scale / S.nptk / S.nptk;
            W[ch][i] = w / S.nptk / S.nptk;
        }
    return FP4_OK;
}

// Ind_driver_4ph (processes.f90:3551-3822): the ordered index lists of the three
// channels (the Ind_only enumeration), each process's Gamma stored at its list
// position, and the per-mode rates and WP4 (fixed-order compensated sums).
extern "C" int fp4_ind_driver_4ph(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                                  const double* eigenvect, int32_t nlist, const int32_t* list, const int32_t* ijk,
                                  const int64_t* n_pp, const int64_t* n_pm, const int64_t* n_mm, int32_t ntri,
                                  const double* psi, const double* r_j, const double* r_k, const double* r_l,
                                  const int32_t* index_i, const int32_t* index_j, const int32_t* index_k,
                                  const int32_t* index_l, int64_t* i2pp, int64_t* i3pp, int64_t* i4pp,
                                  double* gamma_pp, int64_t* i2pm, int64_t* i3pm, int64_t* i4pm, double* gamma_pm,
                                  int64_t* i2mm, int64_t* i3mm, int64_t* i4mm, double* gamma_mm, double* rate_4ph,
                                  double* rate_pp, double* rate_pm, double* rate_mm, double* wp_pp, double* wp_pm,
                                  double* wp_mm) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!g || !n_pp || !n_pm || !n_mm || !rate_4ph || !rate_pp || !rate_pm || !rate_mm || !wp_pp || !wp_pm ||
        !wp_mm || !eigenvect)
        return fp4_fail(c, FP4_E_ARG, "null argument");
    int r;
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, eigenvect, nlist, list, ijk))) return r;
    if ((r = fp4_setup_ifc(c, g, 4, ntri, psi, r_j, r_k, r_l, index_i, index_j, index_k, index_l, c->ifc4))) return r;
    const DevSys& S = c->S;
    const int nm = S.nb * nlist;
    const bool mixed = (c->precision != FP4_PREC_FP64);
    size_t sm = k4_smem(3, 1, mixed, S, c->ifc4.F);
    if (sm > 227 * 1024)
        return fp4_fail(c, FP4_E_CAPACITY, "4ph reciprocal cluster table needs %zu B of shared memory (limit 227 KB)", sm);
    int nwork = 0;
    if ((r = k4_nwork(c, nwork))) return r;
    const int64_t* N[3] = {n_pp, n_pm, n_mm};
    int64_t* O[3][3] = {{i2pp, i3pp, i4pp}, {i2pm, i3pm, i4pm}, {i2mm, i3mm, i4mm}};
    double* GO[3] = {gamma_pp, gamma_pm, gamma_mm};
    std::vector<long long> off((size_t)3 * (nm + 1), 0);
    long long tot[3], base[4] = {0, 0, 0, 0};
    for (int ch = 0; ch < 3; ch++) {
        long long* o = off.data() + (size_t)ch * (nm + 1);
        for (int m = 0; m < nm; m++) {
            if (N[ch][m] < 0) return fp4_fail(c, FP4_E_ARG, "negative count");
            o[m + 1] = o[m] + N[ch][m];
        }
        tot[ch] = o[nm];
        if (tot[ch] && (!O[ch][0] || !O[ch][1] || !O[ch][2] || !GO[ch]))
            return fp4_fail(c, FP4_E_ARG, "null process list output");
        base[ch + 1] = base[ch] + tot[ch];
    }
    const size_t T = (size_t)base[3];
    if ((r = c->b_lists.reserve(c, T * 3 * sizeof(long long) + 64)) || (r = c->b_gamma.reserve(c, T * sizeof(double) + 64)) ||
        (r = c->b_off.reserve(c, off.size() * sizeof(long long))) ||
        (r = c->b_counts.reserve(c, (size_t)3 * nm * sizeof(long long))))
        return r;
    long long* doff = c->b_off.as<long long>();
    long long* dcnt = c->b_counts.as<long long>();
    CK(cudaMemcpyAsync(doff, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    for (int ch = 0; ch < 3; ch++)
        CK(cudaMemcpyAsync(dcnt + (size_t)ch * nm, N[ch], nm * sizeof(long long), cudaMemcpyHostToDevice, c->stream));
    long long* Lb = c->b_lists.as<long long>();
    double* Gb = c->b_gamma.as<double>();
    if (T) CK(cudaMemsetAsync(Gb, 0, T * sizeof(double), c->stream));
    P4Params p{};
    for (int ch = 0; ch < 3; ch++) {
        long long* l2 = Lb + 3 * base[ch];
        p.list_off[ch] = doff + (size_t)ch * (nm + 1);
        p.list_n[ch] = dcnt + (size_t)ch * nm;
        p.lind2[ch] = l2;
        p.lind3[ch] = l2 + tot[ch];
        p.lind4[ch] = l2 + 2 * tot[ch];
        p.gamma_out[ch] = Gb + base[ch];
        if (tot[ch] == 0) continue;
        P4OrderParams q{};
        q.S = S;
        q.ch = ch;
        q.list_off = p.list_off[ch];
        q.counts = p.list_n[ch];
        q.ind2 = l2;
        q.ind3 = l2 + tot[ch];
        q.ind4 = l2 + 2 * tot[ch];
        q.err = c->b_err.as<int>();
        CK(launch_k4_order(q, nm, c->stream));
        c->launches++;
    }
    if ((r = c->b_temps.upload(c, &g->T, sizeof(double)))) return r;
    if ((r = c->b_wb.reserve(c, (size_t)S.nptk * S.nb * wb_stride(1) * sizeof(double)))) return r;
    CK(launch_wbose(S, c->b_temps.as<double>(), 1, wb_stride(1), c->b_wb.as<double>(), c->stream));
    c->launches++;
    const int nblocks = k4_blocks(c, nwork, 3, 1);
    if ((r = k4_queue(c, nblocks, true, p))) return r;
    if ((r = c->b_part.reserve(c, (size_t)nwork * S.nb * 2 * sizeof(double)))) return r;
    if ((r = c->b_work.reserve(c, 64))) return r;
    if ((r = c->b_out4.reserve(c, (size_t)nm * 6 * sizeof(double)))) return r;
    CK(cudaMemsetAsync(c->b_work.ptr, 0, 64, c->stream));
    p.S = S;
    p.F = c->ifc4.F;
    p.nT = 1;
    p.wb = c->b_wb.as<double>();
    p.nwork = nwork;
    p.work_counter = c->b_work.as<int>();
    p.part_rate = c->b_part.as<double>();
    p.part_wp = p.part_rate + (size_t)nwork * S.nb;
    p.stats = c->b_stats.as<unsigned long long>();
    p.err = c->b_err.as<int>();
    const double rate_scale = hbarp() * hbarp() * kPi / 8.0 * (double)3.37617087f * 1.e9;
    p.gamma_scale = rate_scale / S.nptk / S.nptk;
    CK(cudaEventRecord(c->evk0, c->stream));
    CK(launch_k4(3, 1, mixed, p, nblocks, c->stream));
    CK(cudaEventRecord(c->evk1, c->stream));
    c->kernel_timed = true;
    c->launches++;
    double* o = c->b_out4.as<double>();
    CK(launch_k4_reduce(p, o, o + nm, o + 2 * nm, o + 3 * nm, o + 4 * nm, o + 5 * nm, rate_scale, c->stream));
    c->launches++;
    for (int ch = 0; ch < 3; ch++) {
        if (tot[ch] == 0) continue;
        for (int x = 0; x < 3; x++)
            CK(cudaMemcpyAsync(O[ch][x], Lb + 3 * base[ch] + x * tot[ch], tot[ch] * sizeof(long long),
                               cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(GO[ch], Gb + base[ch], tot[ch] * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    double* outs[6] = {rate_pp, rate_pm, rate_mm, wp_pp, wp_pm, wp_mm};
    for (int x = 0; x < 6; x++)
        CK(cudaMemcpyAsync(outs[x], o + (size_t)x * nm, nm * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if ((r = fp4_end(c))) return r;
    for (int m = 0; m < nm; m++) rate_4ph[m] = rate_pp[m] + rate_pm[m] + rate_mm[m];
    return FP4_OK;
}

extern "C" int fp4_rta_driver_4ph(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                                  const double* eigenvect, int32_t nlist, const int32_t* list, const int32_t* ijk,
                                  int32_t ntri, const double* psi, const double* r_j, const double* r_k,
                                  const double* r_l, const int32_t* index_i, const int32_t* index_j,
                                  const int32_t* index_k, const int32_t* index_l, double* rate_4ph, double* rate_pp,
                                  double* rate_pm, double* rate_mm, double* wp_pp, double* wp_pm, double* wp_mm) {
    FP4_TRACE();
    if (!c) return FP4_E_ARG;
    if (!g || !rate_4ph) return fp4_fail(c, FP4_E_ARG, "null argument");
    int r = fp4_rta_driver_4ph_multi_t(c, g, 1, &g->T, energy, velocity, eigenvect, nlist, list, ijk, ntri, psi, r_j,
                                       r_k, r_l, index_i, index_j, index_k, index_l, rate_pp, rate_pm, rate_mm, wp_pp,
                                       wp_pm, wp_mm);
    if (r) return r;
    const int nm = g->nbands * nlist;
    for (int m = 0; m < nm; m++) rate_4ph[m] = rate_pp[m] + rate_pm[m] + rate_mm[m];
    return FP4_OK;
}
