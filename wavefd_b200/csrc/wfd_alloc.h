// Device, managed and pinned allocations of the library go through these wrappers, which carry a
// host-side fault injector for the failure paths: with WAVEFD_B200_FAIL_ALLOC=N in the environment the
// Nth allocation of the process (counted from 1, every wrapper together) fails with
// cudaErrorMemoryAllocation without calling CUDA, and later ones proceed. The caller's ordinary
// failure handling then runs (status codes, messages, partial objects released).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace wfd {

// true when this allocation is the one to fail; the message of the last injected failure is kept
bool alloc_should_fail();
// "" or a note naming the injected failure, for error messages
const char *alloc_injected_note();

template <class T>
inline cudaError_t dMalloc(T **p, size_t bytes) {
    if (alloc_should_fail()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(reinterpret_cast<void **>(p), bytes);
}

template <class T>
inline cudaError_t dMallocManaged(T **p, size_t bytes, unsigned flags = cudaMemAttachGlobal) {
    if (alloc_should_fail()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMallocManaged(reinterpret_cast<void **>(p), bytes, flags);
}

template <class T>
inline cudaError_t dMallocAsync(T **p, size_t bytes, cudaStream_t s) {
    if (alloc_should_fail()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMallocAsync(reinterpret_cast<void **>(p), bytes, s);
}

template <class T>
inline cudaError_t dMallocHost(T **p, size_t bytes) {
    if (alloc_should_fail()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMallocHost(reinterpret_cast<void **>(p), bytes);
}

}  // namespace wfd
