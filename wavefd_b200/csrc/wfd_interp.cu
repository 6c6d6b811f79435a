// Time interpolation between the modelling step dtmod (fine, nm samples) and the recording step
// dtrec (coarse, nd samples) with nh 8-tap filters (spacetime.cc:4-127, exported :228-330; the
// filters come from interpfilters, src/spacetime.jl:333-360), on the GPU.
//
// The reference runs, per trace, the helper calls (i, lo, hi) = (0,3,7), (1,2,7), (2,1,7),
// (3..nd-5, 0,7), (nd-4,0,6), (nd-3,0,5), (nd-2,0,4): fine sample jk = i*nh + k (if < nm) pairs
// with coarse samples i-3+l, l in [lo, hi]. Both directions are written here as gathers, one thread
// per output sample, summing its terms in the reference's loop order with separate IEEE multiply
// and add, so the results are the reference's bit for bit:
//   adjoint (coarse -> fine)  m[jk] = sum_l h[k][l] d[i-3+l]
//   forward (fine -> coarse)  d[q]  = sum over i ascending (l = q+3-i in [lo(i), hi(i)]), k ascending,
//                                     of h[k][l] m[i*nh+k]
// nd >= 7 (below that the reference reads outside its arrays).
//
// WFD_ExtractInterp streams the forward operator into receiver extraction: at fine step jk each
// receiver's sample (the grouped extraction sum, from zero) is scattered into its coarse trace at
// once. Fine samples arrive in the order the forward operator visits them (i, then k, ascending),
// so the coarse traces equal extraction into a fine buffer followed by interpforward, bit for bit,
// without the fine buffer.
#include <string.h>

#include <string>
#include <vector>

#include "wavefd_b200.h"
#include "wfd_alloc.h"
#include "wfd_points.h"
#include "wfd_prop.h"

namespace wfd {
namespace {

__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

// l range [lo, hi] of helper call i (lo > hi: no call at i); a coarse index may have two calls when
// the fixed calls overlap the loop (only for nd < 8, where nd-4 <= 3): call 0 is the fixed call
// of i in 0..2, call 1 the loop/tail call
__device__ __forceinline__ int calls_at(long i, long nd, int (&lo)[2], int (&hi)[2]) {
    int n = 0;
    if (i == 0) lo[n] = 3, hi[n++] = 7;
    else if (i == 1) lo[n] = 2, hi[n++] = 7;
    else if (i == 2) lo[n] = 1, hi[n++] = 7;
    if (i >= 3 && i < nd - 4) lo[n] = 0, hi[n++] = 7;
    if (i == nd - 4) lo[n] = 0, hi[n++] = 6;
    if (i == nd - 3) lo[n] = 0, hi[n++] = 5;
    if (i == nd - 2) lo[n] = 0, hi[n++] = 4;
    return n;
}

template <class T>
__global__ void k_interp_adjoint(const T *__restrict__ h, T *__restrict__ m, const T *__restrict__ d, long nh,
                                 long nm, long nd, long nslow) {
    const long n = nm * nslow;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const long t = e / nm, jk = e % nm;
        const long i = jk / nh, k = jk % nh;
        const T *dt = d + t * nd;
        T acc = 0;
        int lo[2], hi[2];
        const int nc = i <= nd - 2 ? calls_at(i, nd, lo, hi) : 0;
        for (int c = 0; c < nc; c++)
            for (int l = lo[c]; l <= hi[c]; l++) acc = add_rn(acc, mul_rn(h[k * 8 + l], dt[i - 3 + l]));
        m[e] = acc;
    }
}

template <class T>
__global__ void k_interp_forward(const T *__restrict__ h, T *__restrict__ d, const T *__restrict__ m, long nh,
                                 long nd, long nm, long nslow) {
    const long n = nd * nslow;
    for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const long t = e / nd, q = e % nd;
        const T *mt = m + t * nm;
        T acc = 0;
        const long i0 = q - 4 > 0 ? q - 4 : 0, i1 = q + 3 < nd - 2 ? q + 3 : nd - 2;
        for (long i = i0; i <= i1; i++) {
            const int l = (int)(q + 3 - i);
            int lo[2], hi[2];
            const int nc = calls_at(i, nd, lo, hi);
            for (int c = 0; c < nc; c++) {
                if (l < lo[c] || l > hi[c]) continue;
                for (long k = 0; k < nh; k++) {
                    const long jk = i * nh + k;
                    if (jk >= nm) break;
                    acc = add_rn(acc, mul_rn(h[k * 8 + l], mt[jk]));
                }
            }
        }
        d[e] = acc;
    }
}

// streaming extraction + forward interpolation at fine sample jk: one thread per receiver group
// (trace key), v = sum c * field[other] from zero in group order, then for the call(s) at
// i = jk / nh: coarse[key][i-3+l] += h[k][l] * v, l in [lo, hi]
__global__ void k_extract_interp(long ngroups, const long *__restrict__ key, const long *__restrict__ start,
                                 const long *__restrict__ other, const float *__restrict__ c,
                                 const float *__restrict__ field, const float *__restrict__ h, long nh, long jk,
                                 long nm, long nd, float *coarse) {
    const long gi = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gi >= ngroups || jk >= nm) return;
    const long i = jk / nh, k = jk % nh;
    if (i > nd - 2) return;
    float v = 0.0f;
    for (long j = start[gi]; j < start[gi + 1]; j++) v = add_rn(v, mul_rn(c[j], field[other[j]]));
    float *dt = coarse + key[gi] * nd;
    int lo[2], hi[2];
    const int nc = calls_at(i, nd, lo, hi);
    for (int cc = 0; cc < nc; cc++)
        for (int l = lo[cc]; l <= hi[cc]; l++) dt[i - 3 + l] = add_rn(dt[i - 3 + l], mul_rn(h[k * 8 + l], v));
}

inline unsigned blocks(long n) { return (unsigned)(n / 256 + 1 < 148L * 32 ? n / 256 + 1 : 148L * 32); }

cudaStream_t interp_stream() {
    static thread_local cudaStream_t s = nullptr;
    if (!s) cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    return s;
}

// Drop-in path: h as the reference takes it (nh host pointers to 8 values); in/out arrays host,
// device or managed. forward != 0: out = d (nd x nslow), in = m; else out = m (nm x nslow), in = d.
template <class T>
void dropin(int forward, T **h, T *out, const T *in, size_t nh, size_t nm, size_t nd, size_t nslow) {
    if (nd < 7 || nh < 1 || !h || !out || !in) {
        set_global_error(WFD_ERR_ARG, "time interpolation: needs nd >= 7, nh >= 1 and non-null arrays");
        return;
    }
    cudaStream_t s = interp_stream();
    std::vector<T> ht(nh * 8);
    for (size_t k = 0; k < nh; k++) memcpy(&ht[k * 8], h[k], 8 * sizeof(T));
    const size_t nout = (forward ? nd : nm) * nslow, nin = (forward ? nm : nd) * nslow;
    T *dh = nullptr, *dout = nullptr, *din = nullptr;
    const bool out_dev = device_accessible(out), in_dev = device_accessible(in);
    bool ok = wfd::dMallocAsync(&dh, sizeof(T) * ht.size(), s) == cudaSuccess;
    if (ok && !out_dev) ok = wfd::dMallocAsync(&dout, sizeof(T) * (nout ? nout : 1), s) == cudaSuccess;
    if (ok && !in_dev) ok = wfd::dMallocAsync(&din, sizeof(T) * (nin ? nin : 1), s) == cudaSuccess;
    if (!ok) {
        set_global_error(WFD_ERR_ALLOC, "time interpolation: device allocation failed");
    } else {
        cudaMemcpyAsync(dh, ht.data(), sizeof(T) * ht.size(), cudaMemcpyHostToDevice, s);
        if (!in_dev && nin) cudaMemcpyAsync(din, in, sizeof(T) * nin, cudaMemcpyHostToDevice, s);
        T *o = out_dev ? out : dout;
        const T *i = in_dev ? in : din;
        if (nout) {
            if (forward) k_interp_forward<T><<<blocks((long)nout), 256, 0, s>>>(dh, o, i, nh, nd, nm, nslow);
            else k_interp_adjoint<T><<<blocks((long)nout), 256, 0, s>>>(dh, o, i, nh, nm, nd, nslow);
        }
        if (!out_dev && nout) cudaMemcpyAsync(out, dout, sizeof(T) * nout, cudaMemcpyDeviceToHost, s);
    }
    cudaFreeAsync(dh, s);
    if (dout) cudaFreeAsync(dout, s);
    if (din) cudaFreeAsync(din, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) set_global_error(WFD_ERR_CUDA, std::string("time interpolation: ") + cudaGetErrorString(e));
}

}  // namespace
}  // namespace wfd

// ---- drop-in libspacetime exports (spacetime.cc:228-330) -------------------------------------------
extern "C" void interpadjoint_1d_float(float **h, float *m, float *d, size_t nh, size_t nm, size_t nd) {
    wfd::dropin<float>(0, h, m, d, nh, nm, nd, 1);
}
extern "C" void interpadjoint_1d_double(double **h, double *m, double *d, size_t nh, size_t nm, size_t nd) {
    wfd::dropin<double>(0, h, m, d, nh, nm, nd, 1);
}
extern "C" void interpforward_1d_float(float **h, float *d, float *m, size_t nh, size_t nd, size_t nm) {
    wfd::dropin<float>(1, h, d, m, nh, nm, nd, 1);
}
extern "C" void interpforward_1d_double(double **h, double *d, double *m, size_t nh, size_t nd, size_t nm) {
    wfd::dropin<double>(1, h, d, m, nh, nm, nd, 1);
}
extern "C" void interpadjoint_nd_float(float **h, float *m, float *d, size_t nh, size_t nm, size_t nd, size_t nslow,
                                       size_t nthreads) {
    (void)nthreads;
    wfd::dropin<float>(0, h, m, d, nh, nm, nd, nslow);
}
extern "C" void interpadjoint_nd_double(double **h, double *m, double *d, size_t nh, size_t nm, size_t nd,
                                        size_t nslow, size_t nthreads) {
    (void)nthreads;
    wfd::dropin<double>(0, h, m, d, nh, nm, nd, nslow);
}
extern "C" void interpforward_nd_float(float **h, float *d, float *m, size_t nh, size_t nd, size_t nm, size_t nslow,
                                       size_t nthreads) {
    (void)nthreads;
    wfd::dropin<float>(1, h, d, m, nh, nm, nd, nslow);
}
extern "C" void interpforward_nd_double(double **h, double *d, double *m, size_t nh, size_t nd, size_t nm,
                                        size_t nslow, size_t nthreads) {
    (void)nthreads;
    wfd::dropin<double>(1, h, d, m, nh, nm, nd, nslow);
}

// ---- add-ons: device-resident interpolation --------------------------------------------------------
extern "C" int WFD_Interp(int forward, const float *h, float *out, const float *in, long nh, long nm, long nd,
                          long nslow, void *stream) {
    if (nd < 7 || nh < 1 || nm < 1 || nslow < 0 || !h || !out || !in) return WFD_ERR_ARG;
    const long nout = (forward ? nd : nm) * nslow;
    if (!nout) return WFD_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (forward) wfd::k_interp_forward<float><<<wfd::blocks(nout), 256, 0, s>>>(h, out, in, nh, nd, nm, nslow);
    else wfd::k_interp_adjoint<float><<<wfd::blocks(nout), 256, 0, s>>>(h, out, in, nh, nm, nd, nslow);
    return cudaGetLastError() == cudaSuccess ? WFD_OK : WFD_ERR_CUDA;
}

namespace wfd {
void launch_extract_interp(long ngroups, const long *key, const long *start, const long *other, const float *c,
                           const float *field, const float *h, long nh, long jk, long nm, long nd, float *coarse,
                           cudaStream_t s) {
    k_extract_interp<<<(unsigned)((ngroups + 255) / 256), 256, 0, s>>>(ngroups, key, start, other, c, field, h, nh, jk,
                                                                       nm, nd, coarse);
}
}  // namespace wfd
