// Grid-wide barrier of the persistent 2D time loops.
#pragma once

#include <stdint.h>

namespace wfd {

// Grid-wide barrier of the persistent run (all CTAs co-resident: cooperative launch). One counter
// that only grows: barrier number gen + 1 is passed once it reaches (gen + 1) x the CTA count. Each
// CTA adds its arrival with release semantics and polls the counter with acquire loads (no reset and
// no separate publication: one hop fewer than a sense-reversing barrier). Every wait is bounded
// (2 s): a CTA that gives up, or sees that another gave up, sets the status word and returns false,
// and so does every CTA after it, so the kernel always ends.
__device__ __forceinline__ bool grid_barrier(unsigned *words, unsigned &gen, int *ok_flag) {
    unsigned *count = words, *status = words + 2;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned target = (gen + 1) * gridDim.x;
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(count) : "memory");
        uint64_t t0;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
        for (unsigned spin = 1;; spin++) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(count) : "memory");
            if ((int)(v - target) >= 0) break;  // wrap-safe
            if ((spin & 63) == 0) {
                if (*(volatile unsigned *)status) {
                    ok = 0;
                    break;
                }
                uint64_t t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                if (t - t0 > 2000000000ull) {
                    atomicOr(status, 1u);
                    ok = 0;
                    break;
                }
            }
        }
        gen++;
        *ok_flag = ok;
    }
    __syncthreads();
    return *ok_flag != 0;
}

}  // namespace wfd
