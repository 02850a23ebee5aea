// The opaque fp4_ctx of the C-ABI: one CUDA stream and the device-resident
// copies of a solve (harmonic arrays, cluster tables, queues, outputs).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/fourphonon_b200.h"
#include "fp4_device.cuh"

struct fp4_ctx;

// An NVTX range over one C-ABI call, named after the entry point: a CUDA
// profiler's timeline then shows which call launched which kernels.  Without a
// profiler attached the push and pop do nothing.
struct Fp4Trace {
    explicit Fp4Trace(const char* name) { nvtxRangePushA(name); }
    ~Fp4Trace() { nvtxRangePop(); }
    Fp4Trace(const Fp4Trace&) = delete;
    Fp4Trace& operator=(const Fp4Trace&) = delete;
};
#define FP4_TRACE() Fp4Trace fp4_trace_range_(__func__)

// Grow-only device buffer that remembers a hash of the bytes last uploaded,
// so repeated calls with unchanged inputs skip the host-to-device copy.
struct DevBuffer {
    void* ptr = nullptr;
    size_t cap = 0;
    uint64_t key = 0;
    int reserve(fp4_ctx* c, size_t bytes);
    int upload(fp4_ctx* c, const void* host, size_t bytes);
    void release();
    template <class T>
    T* as() const {
        return static_cast<T*>(ptr);
    }
};

struct IfcTables {
    DevBuffer phi, atoms, mj, mk, ml, mu, cl_start, cl_index, pi_d, blk_start;
    fp4::DevIfc F{};
    std::vector<int> h_blk_start;  // host copy of the classes' block ranges
    std::vector<DevBuffer*> list() { return {&phi, &atoms, &mj, &mk, &ml, &mu, &cl_start, &cl_index, &pi_d, &blk_start}; }
};

struct fp4_ctx {
    int device = 0;
    int sm_count = 148;
    int precision = 0;
    cudaStream_t stream = nullptr;      // stream in use (own or caller's)
    cudaStream_t own_stream = nullptr;  // created with the context
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evk0 = nullptr, evk1 = nullptr;
    bool upload_cache = true;
    bool kernel_timed = false;
    bool wv_packed = false;
    uint64_t wv_key = 0;
    int64_t launches = 0;
    std::string err;
    fp4::DevSys S{};
    std::vector<double> atom_mass;
    bool eig_packed = false;
    DevBuffer b_energy, b_velocity, b_wv, b_eigraw, b_eig, b_eigf, b_list, b_qc, b_root[3], b_rootf[3];
    DevBuffer b_temps, b_bose, b_wb, b_out, b_out4, b_lists, b_gamma, b_off, b_counts;
    DevBuffer b_queue, b_part, b_work, b_err, b_stats;
    DevBuffer b_tcplan, b_wtab;  // tensor-core contraction: its plan and phase rows
    bool last_tc = false;        // the last four-phonon RTA call ran its contraction on the tensor cores
    DevBuffer b_bte[13];  // [12]: the new iterate of a Jacobi sweep
    DevBuffer b_harm[6];  // harmonic stage: pair ranges, terms, images, symmetrizers, outputs, born/masses
    IfcTables ifc3, ifc4;
    int64_t last_nproc = 0, last_ncontr = 0, last_launches = 0;
    int last_rta4_nT = 0;  // temperatures of the last four-phonon RTA call (0: none; its partials are in b_part)
    int64_t last_counters[16] = {0};  // [0..7] work counters, [8..9] phase cycles
    double last_ms = 0.0, last_kernel_ms = 0.0;
    std::vector<DevBuffer*> all_buffers() {
        std::vector<DevBuffer*> v = {&b_qc, &b_energy, &b_velocity, &b_wv,  &b_eigraw, &b_eig,   &b_eigf,  &b_list,
                                     &b_temps,  &b_bose,     &b_wb, &b_out, &b_out4,   &b_lists, &b_gamma, &b_off,
                                     &b_counts, &b_queue,    &b_part, &b_work,  &b_err,   &b_stats,
                                     &b_tcplan, &b_wtab};
        for (int d = 0; d < 3; d++) {
            v.push_back(&b_root[d]);
            v.push_back(&b_rootf[d]);
        }
        for (auto& b : b_bte) v.push_back(&b);
        for (auto& b : b_harm) v.push_back(&b);
        for (auto* b : ifc3.list()) v.push_back(b);
        for (auto* b : ifc4.list()) v.push_back(b);
        return v;
    }
};

int fp4_fail(fp4_ctx* c, int code, const char* fmt, ...);
int fp4_begin(fp4_ctx* c);
int fp4_end(fp4_ctx* c);
int fp4_setup_system(fp4_ctx* c, const fp4_globals* g, const double* energy, const double* velocity,
                     const double* eigenvect, int32_t nlist, const int32_t* list, const int32_t* ijk);
int fp4_launch_rta3(fp4_ctx* c, const fp4_globals* g, double* d_out);
