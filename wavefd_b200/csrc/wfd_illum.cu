// Source illumination (src/illumination.c:3-53, bound by src/illumination.jl:1-15): the square of
// a wavefield, or its running sum over time steps, used for preconditioning. On the GPU with a
// separate IEEE multiply and add per cell (the reference's arithmetic, bit for bit).
//
// The drop-in exports take the arrays the reference does (host, device or managed memory);
// WFD_IllumAccumulate is the device add-on for the time loop (asynchronous, one launch per step:
// reads the field and the sum, writes the sum, 12 B/cell for FP32).
#include <string>

#include "wavefd_b200.h"
#include "wfd_alloc.h"
#include "wfd_prop.h"

namespace wfd {
namespace {

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// accum = nullptr: field[i] = field[i]^2 (srcillum_helper); else accum[i] += field[i]^2
template <class T>
__global__ void k_illum(T *__restrict__ accum, T *__restrict__ field, long n) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const T f = field[i];
        if (accum) accum[i] = add_rn(accum[i], mul_rn(f, f));
        else field[i] = mul_rn(f, f);
    }
}

inline unsigned blocks(long n) { return (unsigned)(n / 256 + 1 < 148L * 16 ? n / 256 + 1 : 148L * 16); }

cudaStream_t illum_stream() {
    static thread_local cudaStream_t s = nullptr;
    if (!s) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    return s;
}

template <class T>
void dropin(T *accum, T *field, size_t n) {
    if (!field || !n) return;
    cudaStream_t s = illum_stream();
    const bool fdev = device_accessible(field), adev = !accum || device_accessible(accum);
    T *df = fdev ? field : nullptr, *da = (accum && adev) ? accum : nullptr;
    bool ok = true;
    if (!fdev) ok = wfd::dMallocAsync(&df, sizeof(T) * n, s) == cudaSuccess;
    if (ok && accum && !adev) ok = wfd::dMallocAsync(&da, sizeof(T) * n, s) == cudaSuccess;
    if (!ok) {
        set_global_error(WFD_ERR_ALLOC, "illumination: device allocation failed");
    } else {
        if (!fdev) cudaMemcpyAsync(df, field, sizeof(T) * n, cudaMemcpyHostToDevice, s);
        if (accum && !adev) cudaMemcpyAsync(da, accum, sizeof(T) * n, cudaMemcpyHostToDevice, s);
        k_illum<T><<<blocks((long)n), 256, 0, s>>>(da, df, (long)n);
        if (accum && !adev) cudaMemcpyAsync(accum, da, sizeof(T) * n, cudaMemcpyDeviceToHost, s);
        if (!accum && !fdev) cudaMemcpyAsync(field, df, sizeof(T) * n, cudaMemcpyDeviceToHost, s);
    }
    if (!fdev && df) cudaFreeAsync(df, s);
    if (accum && !adev && da) cudaFreeAsync(da, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) set_global_error(WFD_ERR_CUDA, std::string("illumination: ") + cudaGetErrorString(e));
}

}  // namespace

void illum_accumulate(float *sum, const float *field, long n, cudaStream_t s) {
    if (n > 0) k_illum<float><<<blocks(n), 256, 0, s>>>(sum, const_cast<float *>(field), n);
}

}  // namespace wfd

// ---- drop-in libillumination exports (illumination.c:3-53) ------------------------------------------
extern "C" void srcillum_helper_float(float *field_ginsu, size_t n, int nthreads) {
    (void)nthreads;
    wfd::dropin<float>(nullptr, field_ginsu, n);
}
extern "C" void srcillum_helper_double(double *field_ginsu, size_t n, int nthreads) {
    (void)nthreads;
    wfd::dropin<double>(nullptr, field_ginsu, n);
}
extern "C" void illum_accumulate_float(float *field_ginsu_accum, float *field_ginsu, size_t n, int nthreads) {
    (void)nthreads;
    wfd::dropin<float>(field_ginsu_accum, field_ginsu, n);
}
extern "C" void illum_accumulate_double(double *field_ginsu_accum, double *field_ginsu, size_t n, int nthreads) {
    (void)nthreads;
    wfd::dropin<double>(field_ginsu_accum, field_ginsu, n);
}

// ---- add-on: device illumination sum for the time loop ----------------------------------------------
extern "C" int WFD_IllumAccumulate(float *accum, const float *field, long n, void *stream) {
    if (!accum || !field || n < 0) return WFD_ERR_ARG;
    if (!n) return WFD_OK;
    wfd::k_illum<float><<<wfd::blocks(n), 256, 0, (cudaStream_t)stream>>>(accum, const_cast<float *>(field), n);
    return cudaGetLastError() == cudaSuccess ? WFD_OK : WFD_ERR_CUDA;
}
