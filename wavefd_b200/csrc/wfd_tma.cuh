// TMA (cp.async.bulk.tensor) and mbarrier helpers for the fused step kernels (sm_100a).
//
// Loads are tiled 3D tensor copies global -> shared, completed on an mbarrier with a transaction
// count; no multicast. Every wait is bounded by the global timer: on timeout the caller records
// an error in a device status word and leaves its loop instead of spinning forever.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace wfd {

// Host: encode a 3D FP32 tensor map over a (nz, ny, nx) array (z fastest) with the given box.
// Returns false when the driver rejects it (e.g. nz*4 not a multiple of 16).
bool make_tensor_map_3d(CUtensorMap *map, const float *base, long nx, long ny, long nz, unsigned box_z,
                        unsigned box_y, unsigned box_x);

}  // namespace wfd

namespace wfd_dev {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Limit of the waits for tile loads (2 s), per translation unit. A test hook shortens it
// (WFD_Debug_SetPipelineWait) so that a wait runs out while its copy is still in flight; the drain
// waits at the end of a kernel pass their own limit and are not affected.
static __device__ uint64_t d_pipeline_wait_ns = 2000000000ull;

// Bounded wait for the phase with the given parity to complete; false on timeout. Without an
// explicit limit the pipeline limit applies (read only once the first poll has failed). The first
// poll does not block (test_wait); the later ones let the hardware suspend the thread (try_wait).
// A limit of 1 ns (the test hook) gives up at the first poll that finds the copy still in flight:
// a blocking poll would sleep until the copy lands, and the timer may not advance within 1 ns.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, uint64_t limit_ns = 0) {
    const uint32_t addr = smem_u32(bar);
    uint32_t ok = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
    const uint64_t t0 = globaltimer_ns();
    if (limit_ns == 0) limit_ns = *(volatile uint64_t *)&d_pipeline_wait_ns;
    if (limit_ns <= 1) return false;
    for (;;) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}

// 3D tiled bulk tensor load of one box at element coordinates (c0 = z, c1 = y, c2 = x).
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0, int c1,
                                            int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void prefetch_tensor_map(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

}  // namespace wfd_dev
