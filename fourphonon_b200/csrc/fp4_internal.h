// Kernel parameter blocks and launch helpers shared by the .cu files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp4_device.cuh"

namespace fp4 {

constexpr int kQ3 = 2048;  // 3-phonon survivor queue (shared memory entries)

struct P3Params {
    DevSys S;
    DevIfc F;
    const double* bose;  // [q*nb+b] at T
    double scale;        // hbarp*pi/4
    double unit;         // 5.60626442 (REAL) * 1e8
    // outputs, index 0 = absorption (+), 1 = emission (-)
    int32_t* n_out[2];
    double* p_out[2];
    double* rate[2];
    double* wp[2];
    const int32_t* nlist_counts[2];  // N_plus/N_minus (Ind_only, Ind)
    const long long* list_off[2];    // Naccum offsets
    int32_t* ind2[2];
    int32_t* ind3[2];
    double* gamma[2];
    unsigned long long* stats;
    int* err;
};

struct P4Params {
    DevSys S;
    DevIfc F;
    int nT;
    const double* bose;  // [t][q*nb+b]
    const double* wb;    // [q*nb+b][wb_stride(NT)]: omega, the Bose factor at each T, padding
    int nwork;
    int* work_counter;
    int ch_of_work[3];
    unsigned long long* queue;  // per CTA nb*nb bins of subcap entries
    double* queue_sigma;        // broadening of each queued process, same indexing as queue
    int subcap;
    double* part_rate;  // [work][t][i]
    double* part_wp;
    unsigned long long* n_count;  // NP: [ch][mode]
    double* p_sum;                // NP: [ch][mode]
    unsigned long long* stats;    // [0] surviving processes, [1] contracted
    int* err;
    // kind 3 (Ind_driver_4ph): the ordered lists of each channel and its Gamma output
    const long long* list_off[3];  // Naccum(mm)
    const long long* list_n[3];    // N(mm)
    const long long* lind2[3];
    const long long* lind3[3];
    const long long* lind4[3];
    double* gamma_out[3];
    double gamma_scale;     // hbarp^2 pi/8 * 3.37617087 * 1e9 / nptk^2
    long long* queue_pos;   // list position of each queued process, same indexing as queue
};

// One launch of the multi-solve kernel: ranges of work items, each of one solve slot.
constexpr int kMaxTickRanges = 64;
struct K4Tick {
    int nranges;
    int slot[kMaxTickRanges];
    int begin[kMaxTickRanges];
    int prefix[kMaxTickRanges + 1];  // prefix[r]: work items in ranges before r; prefix[nranges] = total
};

struct P4OrderParams {
    DevSys S;
    int ch;
    const long long* list_off;  // Naccum per mode
    const long long* counts;    // N per mode
    long long* ind2;
    long long* ind3;
    long long* ind4;
    int* err;
};

// launchers (fp4_rates.cu / fp4_order.cu)
cudaError_t launch_k3(int mode, const P3Params& p, int nmodes, cudaStream_t st);
size_t k3_smem(int mode, const DevIfc& F, bool onlyharmonic);
cudaError_t launch_k4(int kind, int nT, bool mixed, const P4Params& p, int nblocks, cudaStream_t st);
size_t k4_smem(int kind, int nT, bool mixed, const DevSys& S, const DevIfc& F);
int k4_threads();
int k4_ctas_per_sm(int kind, int nT, bool mixed);
int k4_multi_ctas_per_sm();
cudaError_t launch_k4_multi(bool mixed, const P4Params* slots, const K4Tick* tick, int* counter,
                            unsigned long long* queue, double* queue_sigma, int cta_bins, int subcap, size_t smem,
                            int nblocks, cudaStream_t st);
size_t k4_multi_smem(bool mixed, const DevSys& S, const DevIfc& F);
cudaError_t launch_k4_reduce(const P4Params& p, double* rate_pp, double* rate_pm, double* rate_mm, double* wp_pp,
                             double* wp_pm, double* wp_mm, double rate_scale, cudaStream_t st);
cudaError_t launch_k4_order(const P4OrderParams& p, int nmodes, cudaStream_t st);
cudaError_t launch_bose(const DevSys& S, const double* T, int nT, double* bose, cudaStream_t st);
// Per-mode records of the four-phonon contraction: omega and its Bose factors,
// (NT + 1) doubles padded to an even count so that a record is whole 16-byte words.
__host__ __device__ constexpr int wb_stride(int NT) { return (NT + 2) & ~1; }
int k4_round_nt(int nT);  // the temperature count the four-phonon kernels are instantiated for (1, 2, 4, 8)
cudaError_t launch_wbose(const DevSys& S, const double* T, int nT, int stride, double* wb, cudaStream_t st);
cudaError_t prepare_k4_multi(bool mixed, size_t smem);
// fp4_bte.cu: iteration0 and TConduct on device-resident arrays (reference layouts)
cudaError_t launch_iteration0(int nb, int nptk, int nlist, int nsr, const int* nequi, const int* allequi,
                              const double* energy, const double* velocity, const double* tau_zero, double* F,
                              cudaStream_t st);
cudaError_t launch_tconduct(int nb, int nptk, double T, double V, const double* energy, const double* velocity,
                            const double* F, double* kappa, cudaStream_t st);

}  // namespace fp4
