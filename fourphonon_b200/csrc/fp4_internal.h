// Kernel parameter blocks and launch helpers shared by the .cu files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fp4_device.cuh"

namespace fp4 {

constexpr int kQ3 = 2048;  // 3-phonon survivor queue (shared memory entries)

// Four-phonon work items (q, q', channel) of one solve: 3*nlist*nptk.  The kernels
// index them and hand them out with 32-bit integers, and every CTA fetches once
// past the last item, so calls with more than kMaxWorkItems are refused.
constexpr long long kMaxWorkItems = (1LL << 31) - (1LL << 20);
inline long long k4_work_items(int nlist, int nptk) { return 3LL * nlist * nptk; }

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

// Plan of the tensor-core contraction (mixed precision, RTA): how the
// displacement classes are laid out along K and the atom-pair blocks along N.
// Classes run in block order; consecutive non-empty blocks are grouped into
// passes of at most kTcPassBlocks blocks (32 accumulator columns each: 9 real
// parts, 9 imaginary parts, padding).  A pass's K range holds 6 values per
// class, (w_hi.re, w_hi.im, w_hi.re, w_hi.im, w_lo.re, w_lo.im), padded to a
// multiple of 16, so that one product over K gives
//   sum_p (w_hi Z_hi + w_hi Z_lo + w_lo Z_hi) ~ sum_p w_p Z_p.
constexpr int kTcPassBlocks = 4;
constexpr int kTcMaxBlocks = (kMaxNb / 3) * (kMaxNb / 3);
constexpr int kTcMaxPass = kTcMaxBlocks;
constexpr int kTcRows = 128;      // processes per product (the M of one tcgen05.mma)
constexpr int kTcRegionCols = 128;  // accumulator columns of one warpgroup's TMEM region
struct TcPlan {
    int npass;      // passes
    int ksteps;     // K-steps (16 values each) of one A row over all passes
    int bin_bytes;  // bytes of one (i,j) bin's B table (all passes)
    int zbins;      // bins whose tables are built together
    int nblk;       // non-empty atom-pair blocks
    int chunk_cap;  // capacity of the chunk list of one group of bins
    int pass_blk0[kTcMaxPass + 1];    // non-empty blocks [pass_blk0[x], pass_blk0[x+1]) form pass x
    int pass_cls0[kTcMaxPass + 1];    // first class of each pass
    int pass_kstep0[kTcMaxPass + 1];  // first K-step of each pass inside an A row
    int pass_boff[kTcMaxPass + 1];    // byte offset of each pass inside a bin's B table
    int4 blk[kTcMaxBlocks];           // (first class, end class, atom of the 3rd phonon, atom of the 4th)
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
    // tensor-core contraction: its plan and the A rows (bf16 hi/lo phases) of every q''
    // for the two channel signs, [sign][q''][ksteps*16]
    const TcPlan* tc;
    const uint16_t* wtab;
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
// tensor-core contraction (mixed precision, RTA)
int k4_tc_plan(int nb, int natoms, int npi, const int* blk_start_host, int subcap, TcPlan& plan);
size_t k4_tc_smem(int nT, const DevSys& S, const DevIfc& F, const TcPlan& plan);
int k4_tc_ctas_per_sm();
cudaError_t launch_k4_tc(int nT, const P4Params& p, size_t smem, int nblocks, cudaStream_t st);
cudaError_t launch_k4_wtab(const DevSys& S, const DevIfc& F, const TcPlan* plan_dev, int ksteps, uint16_t* wtab,
                           cudaStream_t st);
// fp4_bte.cu: iteration0 and TConduct on device-resident arrays (reference layouts)
cudaError_t launch_iteration0(int nb, int nptk, int nlist, int nsr, const int* nequi, const int* allequi,
                              const double* energy, const double* velocity, const double* tau_zero, double* F,
                              cudaStream_t st);
cudaError_t launch_tconduct(int nb, int nptk, double T, double V, const double* energy, const double* velocity,
                            const double* F, double* kappa, cudaStream_t st);

}  // namespace fp4
