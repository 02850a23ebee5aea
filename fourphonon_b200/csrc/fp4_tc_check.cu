// Self-check of the tensor-core primitives that the mixed-precision
// contraction uses (fp4_tc.cuh): one CTA of 128 threads stages a 128 x K bf16
// A and an N x K bf16 B in the canonical K-major shared-memory layout, runs
// K/16 tcgen05.mma K-steps into TMEM, waits on the commit mbarrier (bounded)
// and reads D = A B^T back with tcgen05.ld.  The host compares D with an FP64
// product of the same bf16 values.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fourphonon_b200.h"
#include "fp4_tc.cuh"

namespace {

using namespace fp4;

__global__ void __launch_bounds__(128, 1) k_tc_selftest(int K, int N, const uint16_t* A, const uint16_t* B, float* D,
                                                        int* err) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int ks = K / 16;
    unsigned char* sa = smem;
    unsigned char* sb = smem + (size_t)ks * 128 * 32;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sb + (size_t)ks * N * 32);
    uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
    const int m = threadIdx.x, warp = m >> 5;
    // row m of A and (for m < N) row m of B, 8 values per 16-byte store
    for (int x = 0; x < 2 * ks; x++) {
        const uint4 v = *reinterpret_cast<const uint4*>(A + (size_t)m * K + 8 * x);
        *reinterpret_cast<uint4*>(sa + (size_t)(x >> 1) * 128 * 32 + tc::kmajor_offset(m, (x & 1) * 8)) = v;
    }
    for (int n = m; n < N; n += 128)
        for (int x = 0; x < 2 * ks; x++) {
            const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)n * K + 8 * x);
            *reinterpret_cast<uint4*>(sb + (size_t)(x >> 1) * N * 32 + tc::kmajor_offset(n, (x & 1) * 8)) = v;
        }
    if (m == 0) {
        tc::mbar_init(tc::smem_u32(bar), 1);
        tc::mbar_fence_init();
    }
    uint32_t ncols = 32;
    while ((int)ncols < N) ncols <<= 1;
    if (warp == 0) {
        tc::tmem_alloc(tc::smem_u32(slot), ncols);
        tc::tmem_relinquish();
    }
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *slot;
    if (m == 0) {
        const uint32_t idesc = tc::idesc_bf16_f32(N);
        for (int x = 0; x < ks; x++)
            tc::mma_bf16(tbase, tc::smem_desc(tc::smem_u32(sa) + x * 128 * 32), tc::smem_desc(tc::smem_u32(sb) + x * N * 32),
                         idesc, x > 0);
        tc::commit(tc::smem_u32(bar));
    }
    const bool done = tc::mbar_wait(tc::smem_u32(bar), 0);
    if (!done) atomicOr(err, 1);
    tc::fence_after_sync();
    if (__syncthreads_and(done)) {
        const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
        for (int c = 0; c < N; c += 16) {
            float v[16];
            tc::ld16(tbase + lane_base + (uint32_t)c, v);
            tc::ld_wait();
            for (int x = 0; x < 16; x++) D[(size_t)m * N + c + x] = v[x];
        }
    } else if (m == 0) {
        tc::mbar_wait(tc::smem_u32(bar), 0);  // bounded: the product may still be in flight
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc(tbase, ncols);
}

}  // namespace

extern "C" int fp4_tc_selftest(int32_t K, int32_t N, const uint16_t* A, const uint16_t* B, float* D) {
    if (!A || !B || !D || K < 16 || K % 16 || K > 1024 || N < 16 || N > 256 || N % 16) return FP4_E_ARG;
    const size_t smem = (size_t)(K / 16) * (128 + N) * 32 + 16;
    if (smem > 227 * 1024) return FP4_E_CAPACITY;
    uint16_t *dA = nullptr, *dB = nullptr;
    float* dD = nullptr;
    int* dErr = nullptr;
    int rc = FP4_OK, herr = 0;
    if (cudaMalloc(&dA, (size_t)128 * K * 2) != cudaSuccess || cudaMalloc(&dB, (size_t)N * K * 2) != cudaSuccess ||
        cudaMalloc(&dD, (size_t)128 * N * 4) != cudaSuccess || cudaMalloc(&dErr, sizeof(int)) != cudaSuccess) {
        rc = FP4_E_CUDA;
    } else if (cudaMemcpy(dA, A, (size_t)128 * K * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(dB, B, (size_t)N * K * 2, cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemset(dErr, 0, sizeof(int)) != cudaSuccess ||
               cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
                   cudaSuccess) {
        rc = FP4_E_CUDA;
    } else {
        k_tc_selftest<<<1, 128, smem>>>(K, N, dA, dB, dD, dErr);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(&herr, dErr, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(D, dD, (size_t)128 * N * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = FP4_E_CUDA;
        else if (herr)
            rc = FP4_E_TIMEOUT;
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(dErr);
    return rc;
}
