// tcgen05 (5th-generation tensor core) helpers for sm_100a: tensor-memory allocation, shared-memory
// matrix descriptors, the BF16 MMA with FP32 accumulation in tensor memory, its completion on an
// mbarrier, and loads of the accumulator back into registers. Single-CTA form (cta_group::1), no
// clusters and no multicast.
//
// Operand layout used here (both operands K-major, no swizzle): an operand of R rows and K
// columns (BF16) is stored as 8 x 8 "core matrices" of 128 contiguous bytes (8 rows of 16 bytes,
// each row 8 consecutive K elements). Element (r, k) sits at
//     (r / 8) * SBO + (k / 8) * LBO + (r % 8) * 16 + (k % 8) * 2
// bytes from the operand's start: LBO is the distance between core matrices adjacent along K,
// SBO between core matrices adjacent along the rows. One MMA consumes K = 16 (two core matrices
// along K); the next K step starts 2 * LBO bytes further.
//
// Accumulator (M = 128): row m of D is tensor-memory lane m, column n is column n (32-bit). Warp w
// of the CTA reads lanes 32 (w % 4) .. 32 (w % 4) + 31.
#pragma once

#include <stdint.h>

namespace wfd_umma {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, LBO, SBO (bytes, multiples of 16), no swizzle,
// descriptor version 1 (bits 46-47), base offset 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((start >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1u << 46;
    return d;  // layout type (bits 61-63) 0: no swizzle
}

// Instruction descriptor of kind::f16: BF16 A and B (both K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
    return (1u << 4)                       // D format: F32
           | (1u << 7)                     // A format: BF16
           | (1u << 10)                    // B format: BF16
           | ((uint32_t)(N >> 3) << 17)    // N / 8
           | ((uint32_t)(M >> 4) << 24);   // M / 16
}

// Allocation by one whole warp: ncols (a power of two, >= 32) columns; the tensor-memory address
// is written to *slot (shared memory). The permit is given up at once so that other CTAs on the
// SM can allocate.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D (tensor memory) = A B^T (+ D when accumulate): issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         bool accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)accumulate)
        : "memory");
}

// Arrive once on the mbarrier when every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Generic-proxy shared-memory writes made visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive 32-bit columns of this thread's lane (32x32b shape). The wait is in the same asm
// statement, so that no use of the destination registers can be scheduled before it.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace wfd_umma
