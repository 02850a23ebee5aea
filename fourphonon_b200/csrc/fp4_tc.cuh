// Fifth-generation tensor-core primitives for sm_100a (tcgen05), in inline PTX.
//
// The mixed-precision four-phonon contraction issues its products through
// these: operands in shared memory in the canonical K-major layout without
// swizzling, accumulators in tensor memory (TMEM), completion signalled on an
// mbarrier by tcgen05.commit, and the accumulators read back with tcgen05.ld.
//
// K-major operand layout (no swizzle) for one MMA K-step of 16 bf16 values:
// rows come in groups of 8; the 8 rows x 8 K-values of a "core matrix" are
// 128 contiguous bytes (16 bytes per row).  The two core matrices of a row
// group (K 0-7 and K 8-15) are kLBO bytes apart and consecutive row groups
// are kSBO bytes apart:
//     byte(row, k) = (row / 8) * kSBO + (k / 8) * kLBO + (row % 8) * 16 + (k % 8) * 2
// One K-step of an operand with R rows therefore takes R * 32 bytes.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace fp4 {
namespace tc {

constexpr uint32_t kLBO = 128;  // bytes between the two K-halves of a row group
constexpr uint32_t kSBO = 256;  // bytes between consecutive groups of 8 rows

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Byte offset of element (row, k) inside one K-step block of a K-major operand.
__host__ __device__ __forceinline__ uint32_t kmajor_offset(int row, int k) {
    return (uint32_t)(row >> 3) * kSBO + (uint32_t)(k >> 3) * kLBO + (uint32_t)(row & 7) * 16u + (uint32_t)(k & 7) * 2u;
}

// Shared-memory matrix descriptor: start address, leading and stride byte
// offsets (all >> 4), descriptor version 1 (sm_100), no swizzle, base offset 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((kLBO >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((kSBO >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // version
    return d;                // layout type 0 (no swizzle) in bits 61-63
}

// Instruction descriptor of kind::f16 with bf16 A and B, f32 accumulation,
// both operands K-major, dense, M = 128.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int N) {
    return (1u << 4)                        // D format f32
           | (1u << 7)                      // A format bf16
           | (1u << 10)                     // B format bf16
           | ((uint32_t)(N >> 3) << 17)     // N / 8
           | ((uint32_t)(128 >> 4) << 24);  // M / 16
}

// D[tmem] (+)= A[smem] * B[smem]^T for one K-step of 16; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((uint32_t)accumulate));
}

// The mbarrier at `bar` (shared memory) gets one arrival when every tcgen05
// operation this thread issued before has completed.
__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMEM allocation: one full warp executes these.  `ncols` is a power of two >= 32.
__device__ __forceinline__ void tmem_alloc(uint32_t dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 lanes x 32 bits, 16 consecutive columns per thread (thread t of the warp
// reads lane base+t).  Wait with ld_wait() before using the values.
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
#pragma unroll
    for (int x = 0; x < 16; x++) v[x] = __uint_as_float(r[x]);
}
__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---------------------------------------------------------------------------- mbarriers
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity to complete.  Returns false
// (and leaves the caller to raise its error flag) after `limit` polls; every
// poll already suspends the thread for a hardware-chosen time.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint32_t limit = 1u << 24) {
    for (uint32_t n = 0; n < limit; n++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Named barrier over `nthreads` threads (a multiple of 32) with id 1..15.
__device__ __forceinline__ void named_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
// Named barrier that also returns whether `pred` held in every participating thread.
__device__ __forceinline__ bool named_all(int id, int nthreads, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// ---------------------------------------------------------------------------- asynchronous copies
// Global -> shared copies that need no registers (cp.async): 16 bytes (L2 only)
// or 8 bytes; both addresses aligned to the size.  Wait with cp_async_wait_all().
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem_dst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// ---------------------------------------------------------------------------- bf16 splitting
// x = hi + lo + O(2^-16 |x|): hi = RN_bf16(x), lo = RN_bf16(x - hi).
__device__ __forceinline__ void split_bf16(float x, uint16_t& hi, uint16_t& lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    const float r = x - __bfloat162float(h);
    const __nv_bfloat16 l = __float2bfloat16_rn(r);
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

// The same split of a double: hi = RN_bf16(x), lo = RN_bf16(x - hi) with the
// remainder formed in double.
__device__ __forceinline__ void split_bf16(double x, uint16_t& hi, uint16_t& lo) {
    const __nv_bfloat16 h = __float2bfloat16_rn((float)x);
    const __nv_bfloat16 l = __float2bfloat16_rn((float)(x - (double)__bfloat162float(h)));
    hi = __bfloat16_as_ushort(h);
    lo = __bfloat16_as_ushort(l);
}

}  // namespace tc
}  // namespace fp4
