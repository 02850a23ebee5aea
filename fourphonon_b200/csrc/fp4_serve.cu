// Serving: many solves resident on one GPU, their four-phonon work packed into
// one persistent kernel per tick.
//
// A solve is admitted into a free slot when its device footprint fits the HBM
// budget.  Its inputs (harmonic arrays, cluster tables, Bose factors, symmetry
// of the wedge) stay on the device in the slot's own context until its result
// is collected.  Each tick hands every active slot a share of its remaining
// work items (q = List(ll), q', channel) and runs them in one launch of
// k4_work_multi, replayed from a CUDA graph: a copy of the tick descriptor from
// pinned host memory, a reset of the work counter and the kernel.  A solve
// whose last items ran in the tick is finished on the same stream: the
// compensated reduction of its partial sums, the 3-phonon RTA, tau_zero,
// iteration0, TConduct and the symmetrised kappa tensor.  Requests that arrive
// while others run are admitted between ticks and share the next launches.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fourphonon_b200.h"
#include "fp4_ctx.h"
#include "fp4_internal.h"

using namespace fp4;

int fp4_setup_ifc(fp4_ctx* c, const fp4_globals* g, int order, int32_t ntri, const double* phi, const double* rj,
                  const double* rk, const double* rl, const int32_t* ii, const int32_t* ij, const int32_t* ik,
                  const int32_t* il, IfcTables& T);

namespace {

constexpr size_t kSmemCap = 110 * 1024;  // dynamic shared memory of the multi-solve kernel (2 CTAs per SM)

struct Slot {
    fp4_ctx* ctx = nullptr;
    enum { FREE, RUNNING, DONE } state = FREE;
    int64_t footprint = 0;
    int nwork = 0, next = 0;
    int nb = 0, nlist = 0, nptk = 0, nsr = 0;
    double T = 0.0, volume = 0.0;
    fp4_globals g{};
    P4Params p{};
    DevBuffer crot, result;  // crotations(3,3,nsr); [kappa per branch (9 nb) | kappa total (9)]
};

// tau_zero = 1/(rate3 + rate4) per irreducible mode (0 where the rate is 0), with
// rate3 = rate_plus + rate_minus and rate4 = (pp + pm) + mm as the driver sums them
__global__ void k_tau(int nm, const double* r3, const double* r4, double* tau) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < nm; m += gridDim.x * blockDim.x) {
        const double rate3 = r3[m] + r3[nm + m];
        const double rate4 = (r4[m] + r4[nm + m]) + r4[2 * nm + m];
        const double rate = rate3 + rate4;
        tau[m] = (rate != 0.0) ? 1.0 / rate : 0.0;
    }
}

// symmetrize_tensor (config.f90:503-518) of each branch's kappa and of the sum
// over branches; kappa in: ThConductivity(nb,3,3) as [(d2*3+d1)*nb + b]
__global__ void k_kappa_sym(int nb, int nsr, const double* crot, const double* kappa, double* out) {
    const int b = threadIdx.x;
    if (b > nb) return;
    double t[9];  // t(d1,d2) column-major: t[d2*3+d1]
    for (int x = 0; x < 9; x++) {
        double v = 0.0;
        if (b < nb) {
            v = kappa[x * nb + b];
        } else {
            for (int bb = 0; bb < nb; bb++) v += kappa[x * nb + bb];
        }
        t[x] = v;
    }
    // sum_r R t R^T / nsr with R = crotations(:,:,r) column-major
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int r = 0; r < nsr; r++) {
        const double* R = crot + 9 * r;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                double s = 0.0;
                for (int k = 0; k < 3; k++)
                    for (int l = 0; l < 3; l++) s += R[k * 3 + i] * t[l * 3 + k] * R[l * 3 + j];
                acc[j * 3 + i] += s;
            }
    }
    for (int x = 0; x < 9; x++) out[b * 9 + x] = acc[x] / nsr;
}

}  // namespace

struct fp4_server {
    int device = 0, precision = 0, max_slots = 0, max_bands = 0, sm_count = 148;
    int64_t budget = 0, in_use = 0, fixed = 0;
    cudaStream_t stream = nullptr;
    std::vector<Slot> slots;
    P4Params* d_params = nullptr;
    K4Tick* h_tick = nullptr;
    K4Tick* d_tick = nullptr;
    int* d_counter = nullptr;
    unsigned long long* queue = nullptr;
    double* queue_sigma = nullptr;
    int subcap = 0, cta_bins = 0, nblocks = 0;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    double last_tick_ms = 0.0;
    int64_t ticks = 0;
    std::string err;
};

static int sfail(fp4_server* s, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (s) s->err = buf;
    return code;
}

#define SCK(call)                                                                                          \
    do {                                                                                                   \
        cudaError_t e_ = (call);                                                                           \
        if (e_ != cudaSuccess) return sfail(srv, FP4_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_));     \
    } while (0)

static int64_t footprint_of(int nb, int nlist, const int32_t ngrid[3], int ntri3, int ntri4, int nsr) {
    const int64_t nptk = (int64_t)ngrid[0] * ngrid[1] * ngrid[2];
    const int64_t nm = (int64_t)nb * nlist;
    int64_t b = 0;
    b += nptk * nb * (8 + 24 + 32 + 8 + 16);   // energy, velocity (raw and packed), Bose factors, (omega, Bose) records
    b += nptk * nb * nb * (16 + 16 + 8);       // eigenvectors raw, packed FP64, packed FP32
    b += 3 * nlist * nptk * nb * 2 * 8;        // per-work-item partial sums
    b += (int64_t)ntri3 * (27 * 8 + 64) + (int64_t)ntri4 * (81 * 8 + 80);
    b += nm * 16 * 8 + nptk * nb * 3 * 8;      // outputs, tau, F_n
    b += (int64_t)nlist * nsr * 4 + nptk * 16 + 4096;
    return b;
}

extern "C" int64_t fp4_server_footprint(int32_t nbands, int32_t nlist, const int32_t ngrid[3], int32_t ntri3,
                                        int32_t ntri4, int32_t nsymm_rot) {
    if (nbands < 3 || nlist < 1 || !ngrid || ngrid[0] < 1 || ngrid[1] < 1 || ngrid[2] < 1) return -1;
    return footprint_of(nbands, nlist, ngrid, ntri3, ntri4, nsymm_rot);
}

extern "C" const char* fp4_server_last_error(const fp4_server* s) { return s ? s->err.c_str() : "null server"; }

extern "C" int fp4_server_destroy(fp4_server* srv) {
    if (!srv) return FP4_E_ARG;
    cudaSetDevice(srv->device);
    if (srv->stream) cudaStreamSynchronize(srv->stream);
    if (srv->exec) cudaGraphExecDestroy(srv->exec);
    for (auto& sl : srv->slots) {
        sl.crot.release();
        sl.result.release();
        if (sl.ctx) fp4_destroy(sl.ctx);
    }
    if (srv->d_params) cudaFree(srv->d_params);
    if (srv->d_tick) cudaFree(srv->d_tick);
    if (srv->h_tick) cudaFreeHost(srv->h_tick);
    if (srv->d_counter) cudaFree(srv->d_counter);
    if (srv->queue) cudaFree(srv->queue);
    if (srv->e0) cudaEventDestroy(srv->e0);
    if (srv->e1) cudaEventDestroy(srv->e1);
    if (srv->stream) cudaStreamDestroy(srv->stream);
    delete srv;
    return FP4_OK;
}

static int server_init(fp4_server* srv) {
    if (cudaSetDevice(srv->device) != cudaSuccess) return sfail(srv, FP4_E_CUDA, "cudaSetDevice failed");
    cudaDeviceGetAttribute(&srv->sm_count, cudaDevAttrMultiProcessorCount, srv->device);
    SCK(cudaStreamCreateWithFlags(&srv->stream, cudaStreamNonBlocking));
    SCK(cudaEventCreate(&srv->e0));
    SCK(cudaEventCreate(&srv->e1));
    srv->nblocks = srv->sm_count * k4_multi_ctas_per_sm();
    srv->cta_bins = srv->max_bands * srv->max_bands;
    srv->subcap = 16 * k4_threads();
    const size_t qbytes = (size_t)srv->nblocks * srv->cta_bins * srv->subcap * (sizeof(unsigned long long) + sizeof(double));
    srv->fixed = (int64_t)qbytes;
    if (srv->fixed >= srv->budget)
        return sfail(srv, FP4_E_CAPACITY, "the work queues alone need %zu B, above the HBM budget", qbytes);
    SCK(cudaMalloc(&srv->queue, qbytes));
    srv->queue_sigma = reinterpret_cast<double*>(srv->queue + (size_t)srv->nblocks * srv->cta_bins * srv->subcap);
    SCK(cudaMalloc(&srv->d_params, sizeof(P4Params) * srv->max_slots));
    SCK(cudaMalloc(&srv->d_tick, sizeof(K4Tick)));
    SCK(cudaMallocHost(&srv->h_tick, sizeof(K4Tick)));
    SCK(cudaMalloc(&srv->d_counter, 64));
    memset(srv->h_tick, 0, sizeof(K4Tick));
    const bool mixed = srv->precision == FP4_PREC_MIXED;
    SCK(prepare_k4_multi(mixed, kSmemCap));
    // the tick as a graph: descriptor copy, counter reset, multi-solve kernel
    cudaGraph_t graph = nullptr;
    SCK(cudaStreamBeginCapture(srv->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(srv->d_tick, srv->h_tick, sizeof(K4Tick), cudaMemcpyHostToDevice, srv->stream);
    cudaMemsetAsync(srv->d_counter, 0, 64, srv->stream);
    launch_k4_multi(mixed, srv->d_params, srv->d_tick, srv->d_counter, srv->queue, srv->queue_sigma, srv->cta_bins,
                    srv->subcap, kSmemCap, srv->nblocks, srv->stream);
    SCK(cudaStreamEndCapture(srv->stream, &graph));
    cudaError_t e = cudaGraphInstantiate(&srv->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return sfail(srv, FP4_E_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
    return FP4_OK;
}

extern "C" int fp4_server_create(fp4_server** out, int device, int precision, int32_t max_slots, int32_t max_bands,
                                 int64_t hbm_budget_bytes) {
    if (!out) return FP4_E_ARG;
    *out = nullptr;
    if (max_slots < 1 || max_slots > kMaxTickRanges || max_bands < 3 || max_bands > kMaxNb || hbm_budget_bytes <= 0 ||
        (precision != FP4_PREC_FP64 && precision != FP4_PREC_MIXED))
        return FP4_E_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FP4_E_CUDA;
    if (device < 0 || device >= ndev) return FP4_E_ARG;
    fp4_server* srv = new fp4_server();
    srv->device = device;
    srv->precision = precision;
    srv->max_slots = max_slots;
    srv->max_bands = max_bands;
    srv->budget = hbm_budget_bytes;
    srv->slots.resize(max_slots);
    *out = srv;  // also on failure, so that fp4_server_last_error can explain it before fp4_server_destroy
    return server_init(srv);
}

extern "C" int fp4_server_admit(fp4_server* srv, const fp4_globals* g, const double* energy, const double* velocity,
                                const double* eigenvect, int32_t nlist, const int32_t* list, const int32_t* ijk,
                                int32_t ntri3, const double* phi, const double* r_j3, const double* r_k3,
                                const int32_t* index_i3, const int32_t* index_j3, const int32_t* index_k3,
                                int32_t ntri4, const double* psi, const double* r_j4, const double* r_k4,
                                const double* r_l4, const int32_t* index_i4, const int32_t* index_j4,
                                const int32_t* index_k4, const int32_t* index_l4, int32_t nsymm_rot,
                                const int32_t* nequi, const int32_t* allequilist, const double* crotations,
                                double volume, int32_t* slot_out) {
    FP4_TRACE();
    if (!srv) return FP4_E_ARG;
    if (!g || !slot_out || !nequi || !allequilist || !crotations || !energy || !velocity || !eigenvect || nsymm_rot < 1)
        return sfail(srv, FP4_E_ARG, "null argument");
    if (g->nbands > srv->max_bands)
        return sfail(srv, FP4_E_CAPACITY, "nbands=%d above the server's max_bands=%d", g->nbands, srv->max_bands);
    if (!(volume > 0.0) || !(g->T > 0.0)) return sfail(srv, FP4_E_ARG, "volume and T must be >0");
    const int64_t fp = footprint_of(g->nbands, nlist, g->ngrid, ntri3, ntri4, nsymm_rot);
    if (srv->fixed + fp > srv->budget)
        return sfail(srv, FP4_E_CAPACITY, "solve needs %lld B, above the HBM budget", (long long)fp);
    int si = -1;
    for (int x = 0; x < srv->max_slots; x++)
        if (srv->slots[x].state == Slot::FREE) {
            si = x;
            break;
        }
    if (si < 0) return sfail(srv, FP4_E_STATE, "no free slot");
    if (srv->fixed + srv->in_use + fp > srv->budget) return sfail(srv, FP4_E_STATE, "HBM budget in use; retry later");
    Slot& sl = srv->slots[si];
    if (!sl.ctx) {
        int r = fp4_create(&sl.ctx, srv->device);
        if (r) return sfail(srv, r, "fp4_create failed");
    }
    fp4_ctx* c = sl.ctx;
    fp4_set_precision(c, srv->precision);
    c->stream = srv->stream;
    int r;
    auto pass = [&](int code) { return sfail(srv, code, "%s", c->err.c_str()); };
    if ((r = fp4_begin(c)) || (r = fp4_setup_system(c, g, energy, velocity, eigenvect, nlist, list, ijk))) return pass(r);
    if ((r = fp4_setup_ifc(c, g, 3, ntri3, phi, r_j3, r_k3, nullptr, index_i3, index_j3, index_k3, nullptr, c->ifc3)))
        return pass(r);
    if ((r = fp4_setup_ifc(c, g, 4, ntri4, psi, r_j4, r_k4, r_l4, index_i4, index_j4, index_k4, index_l4, c->ifc4)))
        return pass(r);
    const DevSys& S = c->S;
    const bool mixed = srv->precision == FP4_PREC_MIXED;
    if (k4_multi_smem(mixed, S, c->ifc4.F) > kSmemCap)
        return sfail(srv, FP4_E_CAPACITY, "4ph tables need %zu B of shared memory, above the serving kernel's %zu B",
                     k4_multi_smem(mixed, S, c->ifc4.F), kSmemCap);
    const int nm = S.nb * nlist;
    for (int ll = 0; ll < nlist; ll++) {
        if (nequi[ll] < 1 || nequi[ll] > nsymm_rot) return sfail(srv, FP4_E_ARG, "Nequi entry outside [1,nsymm_rot]");
        for (int kk = 0; kk < nequi[ll]; kk++) {
            const int q = allequilist[ll * nsymm_rot + kk];
            if (q < 1 || q > S.nptk) return sfail(srv, FP4_E_ARG, "ALLEquiList entry outside [1,nptk]");
        }
    }
    // BTE inputs: Nequi, ALLEquiList, energy, velocity; F_n and tau in b_bte[5], b_bte[4]
    DevBuffer* B = c->b_bte;
    if ((r = B[0].upload(c, nequi, nlist * sizeof(int))) ||
        (r = B[1].upload(c, allequilist, (size_t)nlist * nsymm_rot * sizeof(int))) ||
        (r = B[2].upload(c, energy, (size_t)S.nptk * S.nb * sizeof(double))) ||
        (r = B[3].upload(c, velocity, (size_t)S.nptk * S.nb * 3 * sizeof(double))) ||
        (r = B[4].reserve(c, (size_t)nm * sizeof(double))) ||
        (r = B[5].reserve(c, (size_t)S.nptk * S.nb * 3 * sizeof(double))) ||
        (r = sl.crot.upload(c, crotations, (size_t)nsymm_rot * 9 * sizeof(double))) ||
        (r = sl.result.reserve(c, (size_t)(S.nb + 1) * 9 * sizeof(double))))
        return pass(r);
    // Bose factors at T, partial sums, outputs
    if (k4_work_items(nlist, S.nptk) > kMaxWorkItems)
        return sfail(srv, FP4_E_CAPACITY, "3*nlist*nptk = %lld four-phonon work items, above the limit of %lld",
                     k4_work_items(nlist, S.nptk), kMaxWorkItems);
    const int nwork = (int)k4_work_items(nlist, S.nptk);
    if ((r = c->b_temps.upload(c, &g->T, sizeof(double))) ||
        (r = c->b_wb.reserve(c, (size_t)S.nptk * S.nb * wb_stride(1) * sizeof(double))) ||
        (r = c->b_part.reserve(c, (size_t)nwork * S.nb * 2 * sizeof(double))) ||
        (r = c->b_out4.reserve(c, (size_t)nm * 6 * sizeof(double))) ||
        (r = c->b_out.reserve(c, (size_t)nm * 4 * sizeof(double) + (size_t)S.nb * 9 * sizeof(double))))
        return pass(r);
    if (launch_wbose(S, c->b_temps.as<double>(), 1, wb_stride(1), c->b_wb.as<double>(), c->stream) != cudaSuccess)
        return sfail(srv, FP4_E_CUDA, "launch_wbose failed");
    P4Params& p = sl.p;
    p = P4Params{};
    p.S = S;
    p.F = c->ifc4.F;
    p.nT = 1;
    p.wb = c->b_wb.as<double>();
    p.nwork = nwork;
    p.subcap = srv->subcap;
    p.part_rate = c->b_part.as<double>();
    p.part_wp = p.part_rate + (size_t)nwork * S.nb;
    p.stats = c->b_stats.as<unsigned long long>();
    p.err = c->b_err.as<int>();
    if (cudaMemcpyAsync(srv->d_params + si, &p, sizeof(P4Params), cudaMemcpyHostToDevice, srv->stream) != cudaSuccess)
        return sfail(srv, FP4_E_CUDA, "parameter upload failed");
    if ((r = fp4_end(c))) return pass(r);
    sl.state = Slot::RUNNING;
    sl.footprint = fp;
    sl.nwork = nwork;
    sl.next = 0;
    sl.nb = S.nb;
    sl.nlist = nlist;
    sl.nptk = S.nptk;
    sl.nsr = nsymm_rot;
    sl.T = g->T;
    sl.volume = volume;
    sl.g = *g;
    sl.g.masses = nullptr;
    sl.g.types = nullptr;
    srv->in_use += fp;
    *slot_out = si;
    return FP4_OK;
}

// Rates, tau, iteration0, TConduct and the symmetrised kappa of a slot whose
// work items have all run (enqueued on the server stream).
static int finish_slot(fp4_server* srv, Slot& sl) {
    fp4_ctx* c = sl.ctx;
    const int nm = sl.nb * sl.nlist;
    const double rate_scale = 1.05457172647e-22 * (double)1e22f;
    const double hp2 = rate_scale * rate_scale * 3.141592653589793238 / 8.0 * (double)3.37617087f * 1.e9;
    double* o4 = c->b_out4.as<double>();
    SCK(launch_k4_reduce(sl.p, o4, o4 + nm, o4 + 2 * nm, o4 + 3 * nm, o4 + 4 * nm, o4 + 5 * nm, hp2, srv->stream));
    double* o3 = c->b_out.as<double>();
    int r = fp4_launch_rta3(c, &sl.g, o3);
    if (r) return sfail(srv, r, "%s", c->err.c_str());
    DevBuffer* B = c->b_bte;
    k_tau<<<(nm + 255) / 256, 256, 0, srv->stream>>>(nm, o3, o4, B[4].as<double>());
    SCK(cudaGetLastError());
    SCK(cudaMemsetAsync(B[5].ptr, 0, (size_t)sl.nptk * sl.nb * 3 * sizeof(double), srv->stream));
    SCK(launch_iteration0(sl.nb, sl.nptk, sl.nlist, sl.nsr, B[0].as<int>(), B[1].as<int>(), B[2].as<double>(),
                          B[3].as<double>(), B[4].as<double>(), B[5].as<double>(), srv->stream));
    double* kap = o3 + 4 * nm;
    SCK(launch_tconduct(sl.nb, sl.nptk, sl.T, sl.volume, B[2].as<double>(), B[3].as<double>(), B[5].as<double>(), kap,
                        srv->stream));
    k_kappa_sym<<<1, 64, 0, srv->stream>>>(sl.nb, sl.nsr, sl.crot.as<double>(), kap, sl.result.as<double>());
    SCK(cudaGetLastError());
    return FP4_OK;
}

extern "C" int fp4_server_tick(fp4_server* srv, int64_t max_items, int32_t* finished, int32_t* nfinished) {
    FP4_TRACE();
    if (!srv) return FP4_E_ARG;
    if (!finished || !nfinished || max_items < 1) return sfail(srv, FP4_E_ARG, "bad argument");
    *nfinished = 0;
    SCK(cudaSetDevice(srv->device));
    std::vector<int> active;
    for (int x = 0; x < srv->max_slots; x++)
        if (srv->slots[x].state == Slot::RUNNING && srv->slots[x].next < srv->slots[x].nwork) active.push_back(x);
    if (active.empty()) return FP4_OK;
    // equal shares of max_items; what a short slot leaves goes to the others
    K4Tick& t = *srv->h_tick;
    t.nranges = 0;
    int64_t left = max_items;
    std::vector<int> take(active.size(), 0);
    for (size_t pass = 0; pass < 2 && left > 0; pass++) {
        int nopen = 0;
        for (size_t a = 0; a < active.size(); a++)
            if (srv->slots[active[a]].next + take[a] < srv->slots[active[a]].nwork) nopen++;
        if (!nopen) break;
        const int64_t share = std::max<int64_t>(1, left / nopen);
        for (size_t a = 0; a < active.size() && left > 0; a++) {
            Slot& sl = srv->slots[active[a]];
            const int64_t rem = sl.nwork - sl.next - take[a];
            const int64_t n = std::min<int64_t>(std::min(rem, share), left);
            take[a] += (int)n;
            left -= n;
        }
    }
    t.prefix[0] = 0;
    std::vector<int> done;
    for (size_t a = 0; a < active.size(); a++) {
        if (take[a] == 0) continue;
        Slot& sl = srv->slots[active[a]];
        const int r = t.nranges++;
        t.slot[r] = active[a];
        t.begin[r] = sl.next;
        t.prefix[r + 1] = t.prefix[r] + take[a];
        sl.next += take[a];
        if (sl.next == sl.nwork) done.push_back(active[a]);
    }
    SCK(cudaEventRecord(srv->e0, srv->stream));
    SCK(cudaGraphLaunch(srv->exec, srv->stream));
    SCK(cudaEventRecord(srv->e1, srv->stream));
    for (int si : done) {
        int r = finish_slot(srv, srv->slots[si]);
        if (r) return r;
    }
    SCK(cudaStreamSynchronize(srv->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, srv->e0, srv->e1);
    srv->last_tick_ms = ms;
    srv->ticks++;
    for (int si : done) {
        Slot& sl = srv->slots[si];
        int flags = 0;
        SCK(cudaMemcpy(&flags, sl.ctx->b_err.ptr, sizeof(int), cudaMemcpyDeviceToHost));
        if (flags) return sfail(srv, FP4_E_CAPACITY, "slot %d: kernel error flags 0x%x", si, flags);
        sl.state = Slot::DONE;
        finished[(*nfinished)++] = si;
    }
    return FP4_OK;
}

extern "C" int fp4_server_collect(fp4_server* srv, int32_t slot, double* rate3_plus, double* rate3_minus,
                                  double* rate4_pp, double* rate4_pm, double* rate4_mm, double* kappa_branch,
                                  double* kappa, int64_t* n_processes) {
    FP4_TRACE();
    if (!srv) return FP4_E_ARG;
    if (slot < 0 || slot >= srv->max_slots || srv->slots[slot].state != Slot::DONE)
        return sfail(srv, FP4_E_STATE, "slot %d holds no finished solve", slot);
    Slot& sl = srv->slots[slot];
    fp4_ctx* c = sl.ctx;
    const int nm = sl.nb * sl.nlist;
    const double* o3 = c->b_out.as<double>();
    const double* o4 = c->b_out4.as<double>();
    double* dst[5] = {rate3_plus, rate3_minus, rate4_pp, rate4_pm, rate4_mm};
    const double* src[5] = {o3, o3 + nm, o4, o4 + nm, o4 + 2 * nm};
    for (int x = 0; x < 5; x++)
        if (dst[x]) SCK(cudaMemcpyAsync(dst[x], src[x], nm * sizeof(double), cudaMemcpyDeviceToHost, srv->stream));
    const double* res = sl.result.as<double>();
    if (kappa_branch)
        SCK(cudaMemcpyAsync(kappa_branch, res, (size_t)sl.nb * 9 * sizeof(double), cudaMemcpyDeviceToHost, srv->stream));
    if (kappa) SCK(cudaMemcpyAsync(kappa, res + (size_t)sl.nb * 9, 9 * sizeof(double), cudaMemcpyDeviceToHost, srv->stream));
    unsigned long long st[2] = {0, 0};
    SCK(cudaMemcpyAsync(st, c->b_stats.ptr, sizeof st, cudaMemcpyDeviceToHost, srv->stream));
    SCK(cudaStreamSynchronize(srv->stream));
    if (n_processes) *n_processes = (int64_t)st[0];
    sl.state = Slot::FREE;
    srv->in_use -= sl.footprint;
    sl.footprint = 0;
    return FP4_OK;
}

extern "C" int fp4_server_status(const fp4_server* srv, int32_t* running, int32_t* done, int64_t* bytes_in_use,
                                 double* last_tick_ms, int64_t* ticks) {
    if (!srv) return FP4_E_ARG;
    int nr = 0, nd = 0;
    for (const auto& sl : srv->slots) {
        nr += sl.state == Slot::RUNNING;
        nd += sl.state == Slot::DONE;
    }
    if (running) *running = nr;
    if (done) *done = nd;
    if (bytes_in_use) *bytes_in_use = srv->fixed + srv->in_use;
    if (last_tick_ms) *last_tick_ms = srv->last_tick_ms;
    if (ticks) *ticks = srv->ticks;
    return FP4_OK;
}
