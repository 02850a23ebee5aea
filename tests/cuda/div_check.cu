// Bit-for-bit check of div_by_grid (fp4_device.cuh) against the correctly
// rounded __ddiv_rn for every grid size 1..64 and 2^26 pseudo-random
// dividends per size spread over 2^-60..2^60 in magnitude, both signs.
// Prints the number of mismatches; exit status 0 when it is zero.
#include <cstdio>
#include <cstdint>

#include "../../fourphonon_b200/csrc/fp4_device.cuh"

__device__ __forceinline__ uint64_t mix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void check(int N, uint64_t n, unsigned long long* bad) {
    const double dN = (double)N, r = 1.0 / dN;
    unsigned long long local = 0;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < n; x += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t h = mix(x * 131u + (uint64_t)N);
        // random mantissa, exponent in [-60, 60], random sign
        int ex = (int)((h >> 52) % 121) - 60;
        uint64_t bits = ((uint64_t)(1023 + ex) << 52) | (h & 0x000fffffffffffffull);
        double v = __longlong_as_double((long long)bits);
        if (h & 1) v = -v;
        double a = fp4::div_by_grid(v, dN, r);
        double b = __ddiv_rn(v, dN);
        if (__double_as_longlong(a) != __double_as_longlong(b)) local++;
    }
    if (local) atomicAdd(bad, local);
}

int main() {
    unsigned long long* d;
    cudaMalloc(&d, sizeof(unsigned long long));
    unsigned long long total = 0;
    for (int N = 1; N <= 64; N++) {
        cudaMemset(d, 0, sizeof(unsigned long long));
        check<<<1184, 256>>>(N, 1ull << 26, d);
        unsigned long long h = 0;
        cudaMemcpy(&h, d, sizeof h, cudaMemcpyDeviceToHost);
        if (h) printf("N=%d mismatches=%llu\n", N, h);
        total += h;
    }
    cudaError_t e = cudaGetLastError();
    printf("div_by_grid vs __ddiv_rn: %llu mismatches in %llu quotients (%s)\n", total, 64ull << 26,
           cudaGetErrorString(e));
    cudaFree(d);
    return (total == 0 && e == cudaSuccess) ? 0 : 1;
}
