// Allocation-free four-phonon process counting: fp4_np_driver_4ph_noalloc.
//
// Some callers cannot allocate device memory: a host that manages all device
// memory through its own pool, or code that must not change the allocator
// state of a process it is embedded in.  This entry point runs the same
// counting kernel as fp4_np_driver_4ph but allocates nothing: the caller
// passes device arrays for its inputs and outputs, and the scratch the kernel
// needs (the packed mode table, grid and List tables, the work counter, the
// statistics and error words, the staged results) lives in one file-scope
// __device__ array of fixed size, which every GPU that loads the library
// keeps until the process exits.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "../../include/fourphonon_b200.h"
#include "fp4_device.cuh"
#include "fp4_internal.h"

using namespace fp4;

namespace {

// 12 MiB.  A call needs nptk*nbands*32 B (the packed (v, w) table), nptk*4 B (grid
// coordinates), nlist*4 B (List), nlist*nbands*48 B (staged counts and phase spaces of
// the three channels) and 256 B of counters, each part rounded up to 256 B.
constexpr size_t kScratchBytes = 12u << 20;
__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

// The array has one copy per CUDA context, so its device address is looked up once per
// context, keyed by the context's unique id (cuCtxGetId ids are never reused, unlike
// CUcontext handles): a host that creates its own context, or resets the device between
// calls, gets the address that belongs to its current context.
typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);
constexpr int kMaxContexts = 64;
std::mutex g_setup_mutex;
bool g_entry_points_done = false;
PfnCtxGetCurrent g_ctx_get_current = nullptr;
PfnCtxGetId g_ctx_get_id = nullptr;
unsigned long long g_ctx_ids[kMaxContexts] = {0};
unsigned char* g_ctx_addr[kMaxContexts] = {nullptr};
int g_nctx = 0;

// Unique id of the calling thread's current context; false if there is none yet or the
// driver does not offer the query.  Called with g_setup_mutex held.
bool current_context_id(unsigned long long* id) {
    if (!g_entry_points_done) {
        g_entry_points_done = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_current = reinterpret_cast<PfnCtxGetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            g_ctx_get_id = reinterpret_cast<PfnCtxGetId>(f);
    }
    if (!g_ctx_get_current || !g_ctx_get_id) return false;
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return g_ctx_get_id(ctx, id) == CUDA_SUCCESS;
}

// Device address of g_scratch in the current context (set-up on the first call in each
// context; the runtime creates the device's context here if it does not exist yet).
cudaError_t scratch_address(unsigned char** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    unsigned long long id = 0;
    const bool have_id = current_context_id(&id);
    if (have_id)
        for (int x = 0; x < g_nctx; x++)
            if (g_ctx_ids[x] == id) {
                *out = g_ctx_addr[x];
                return cudaSuccess;
            }
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
    if (e != cudaSuccess) return e;
    if (!ptr) return cudaErrorInvalidSymbol;
    *out = static_cast<unsigned char*>(ptr);
    unsigned long long id2 = 0;  // the context may have been created by the lookup itself
    if (current_context_id(&id2)) {
        const int slot = (g_nctx < kMaxContexts) ? g_nctx++ : (int)(id2 % kMaxContexts);
        g_ctx_ids[slot] = id2;
        g_ctx_addr[slot] = *out;
    }
    return cudaSuccess;
}

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

__global__ void k_noalloc_pack(int nptk, int nb, int n0, int n1, int nlist, const double* energy,
                               const double* velocity, const int* list, double4* wv, int* qc, int* list0, int* err) {
    const size_t plane = (size_t)nptk * nb;
    for (size_t x = blockIdx.x * (size_t)blockDim.x + threadIdx.x; x < plane; x += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(x / nb), b = (int)(x % nb);
        const size_t o = (size_t)b * nptk + q;  // energy(q,b), velocity(q,b,d)
        wv[x] = make_double4(velocity[o], velocity[o + plane], velocity[o + 2 * plane], energy[o]);
        if (b == 0) {
            const int a = q % n0, t = q / n0;
            qc[q] = a | ((t % n1) << 8) | ((t / n1) << 16);
        }
        if (x < (size_t)nlist) {
            const int v = list[x];
            if (v < 1 || v > nptk) {
                atomicOr(err, 1);
                list0[x] = 0;
            } else {
                list0[x] = v - 1;
            }
        }
    }
}

// (counts, phase spaces) staged in scratch as [ch][mode] are copied into the caller's arrays
__global__ void k_noalloc_unpack(int nm, const unsigned long long* cnt, const double* ps, int64_t* n0, int64_t* n1,
                                 int64_t* n2, double* p0, double* p1, double* p2) {
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < nm; x += gridDim.x * blockDim.x) {
        n0[x] = (int64_t)cnt[x];
        n1[x] = (int64_t)cnt[nm + x];
        n2[x] = (int64_t)cnt[2 * nm + x];
        p0[x] = ps[x];
        p1[x] = ps[nm + x];
        p2[x] = ps[2 * nm + x];
    }
}

}  // namespace

extern "C" int fp4_np_driver_4ph_noalloc(const fp4_globals* g, const double* energy, const double* velocity,
                                         int32_t nlist, const int32_t* list, int64_t* n_plusplus,
                                         double* pspace_plusplus, int64_t* n_plusminus, double* pspace_plusminus,
                                         int64_t* n_minusminus, double* pspace_minusminus, void* stream) {
    if (!g || !energy || !velocity || !list || !n_plusplus || !pspace_plusplus || !n_plusminus ||
        !pspace_plusminus || !n_minusminus || !pspace_minusminus)
        return FP4_E_ARG;
    for (int d = 0; d < 3; d++)
        if (g->ngrid[d] < 1 || g->ngrid[d] > kMaxGrid) return FP4_E_ARG;
    if (g->natoms < 1 || g->nbands != 3 * g->natoms || g->nbands > kMaxNb) return FP4_E_ARG;
    const int nptk = g->ngrid[0] * g->ngrid[1] * g->ngrid[2], nb = g->nbands;
    if (nlist < 1 || nlist > nptk) return FP4_E_ARG;
    if (k4_work_items(nlist, nptk) > kMaxWorkItems) return FP4_E_CAPACITY;
    const int nm = nb * nlist;
    // scratch layout
    const size_t o_wv = 0;
    const size_t o_qc = al256(o_wv + (size_t)nptk * nb * sizeof(double4));
    const size_t o_list = al256(o_qc + (size_t)nptk * sizeof(int));
    const size_t o_cnt = al256(o_list + (size_t)nlist * sizeof(int));
    const size_t o_ps = al256(o_cnt + (size_t)3 * nm * sizeof(unsigned long long));
    const size_t o_misc = al256(o_ps + (size_t)3 * nm * sizeof(double));
    const size_t need = o_misc + 256;
    if (need > kScratchBytes) return FP4_E_CAPACITY;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return FP4_E_CUDA;
    unsigned char* base = nullptr;
    if (scratch_address(&base) != cudaSuccess) return FP4_E_CUDA;
    int sm_count = 148;
    cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, dev);
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    double4* wv = reinterpret_cast<double4*>(base + o_wv);
    int* qc = reinterpret_cast<int*>(base + o_qc);
    int* list0 = reinterpret_cast<int*>(base + o_list);
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(base + o_cnt);
    double* ps = reinterpret_cast<double*>(base + o_ps);
    int* misc = reinterpret_cast<int*>(base + o_misc);  // [0] work counter, [1] error, [2..] statistics
    unsigned long long* stats = reinterpret_cast<unsigned long long*>(base + o_misc + 64);

    // what must start at zero: the work counter, error word, statistics and the staged results
    if (cudaMemsetAsync(base + o_cnt, 0, need - o_cnt, st) != cudaSuccess) return FP4_E_CUDA;
    const size_t plane = (size_t)nptk * nb;
    int blocks = (int)((plane + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    k_noalloc_pack<<<blocks, 256, 0, st>>>(nptk, nb, g->ngrid[0], g->ngrid[1], nlist, energy, velocity, list, wv, qc,
                                          list0, misc + 1);
    if (cudaGetLastError() != cudaSuccess) return FP4_E_CUDA;

    P4Params p{};
    DevSys& S = p.S;
    for (int d = 0; d < 3; d++) {
        S.n[d] = g->ngrid[d];
        S.ngd[d] = (double)g->ngrid[d];
        S.rinv[d] = 1.0 / (double)g->ngrid[d];
    }
    S.nptk = nptk;
    S.nb = nb;
    S.nlist = nlist;
    S.natoms = g->natoms;
    for (int x = 0; x < 9; x++) S.rl[x] = g->rlattvec[x];
    S.scalebroad = g->scalebroad;
    S.omega_max = g->omega_max;
    S.onlyharmonic = g->onlyharmonic ? 1 : 0;
    S.wv = wv;
    S.qc = qc;
    S.list0 = list0;
    p.F = DevIfc{};
    p.nT = 1;
    p.nwork = (int)k4_work_items(nlist, nptk);
    p.work_counter = misc;
    p.n_count = cnt;
    p.p_sum = ps;
    p.stats = stats;
    p.err = misc + 1;
    const int nblocks = std::min(k4_ctas_per_sm(0, 1, false) * sm_count, p.nwork);
    if (launch_k4(0, 1, false, p, nblocks, st) != cudaSuccess) return FP4_E_CUDA;
    k_noalloc_unpack<<<(nm + 255) / 256, 256, 0, st>>>(nm, cnt, ps, n_plusplus, n_plusminus, n_minusminus,
                                                        pspace_plusplus, pspace_plusminus, pspace_minusminus);
    if (cudaGetLastError() != cudaSuccess) return FP4_E_CUDA;
    int err = 0;
    if (cudaMemcpyAsync(&err, misc + 1, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess) return FP4_E_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return FP4_E_CUDA;
    return err ? FP4_E_ARG : FP4_OK;
}
