// An entry point that allocates no memory: the wavefield-separation imaging condition
// (the AdjointBornAccumulation_wavefieldsep family) on caller-provided device arrays.
//
// Some callers cannot call cudaMalloc at all: code running under a memory pool or allocator that
// owns all device memory of the process, callers inside a region where allocation is not allowed
// (for example while other work holds the allocator), or plug-ins whose host application forbids
// device allocations by extensions. The regular entry points allocate the Bluestein FFT tables and,
// for host arrays, staging buffers on every call. This variant keeps its scratch (the tables) in a
// fixed file-scope device array instead, builds them on the device when the FFT length differs from
// the last call's on that device, and requires every array it is given to be device or managed
// memory on the current device. The device address of the array is looked up once per device and
// kept for the life of the process, so the entry point must not be used across a cudaDeviceReset.
#include <math.h>
#include <stdlib.h>

#include <mutex>

#include "wfd_prop.h"

namespace {

constexpr long kMaxNz = 2048;               // largest nz accepted (FFT length 2nz <= 4096)
constexpr int kMaxN = 2 * (int)kMaxNz;      // 4096
constexpr int kMaxM = 8192;                 // Bluestein length for n <= 4096 (power of two >= 2n-1)
constexpr int kScratch = kMaxN + 2 * kMaxM; // float2 entries: 160 KiB

// The scratch: chirp[n], filter(+1)[m], filter(-1)[m]. Every GPU that loads the library holds it
// until the process exits. In host code this name is only a stand-in for the device symbol; the
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) float2 g_sep_scratch[kScratch];

std::mutex g_mu;
float2 *g_addr[256];  // device address of g_sep_scratch, per device ordinal
int g_tables_n[256];  // FFT length whose Bluestein tables the scratch of that device holds (0: none)

// radix-2 FFT of length m (power of two) in shared memory, double precision:
// a[k] <- sum_j a[j] e^{sign 2 pi i jk/m}
__device__ void fft_pow2_d(double2 *a, int m, int sign) {
    const int lg = 31 - __clz(m);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int j = (int)(__brev((unsigned)i) >> (32 - lg));
        if (i < j) {
            const double2 t = a[i];
            a[i] = a[j];
            a[j] = t;
        }
    }
    __syncthreads();
    for (int half = 1; half < m; half <<= 1) {
        const int len = half << 1;
        for (int t = threadIdx.x; t < m / 2; t += blockDim.x) {
            const int pos = t & (half - 1);
            const int i = (t / half) * len + pos;
            const int j = i + half;
            double s, c;
            sincospi((double)(2 * pos) / (double)len, &s, &c);
            const double wr = c, wi = sign * s;
            const double2 u = a[i], v = a[j];
            const double2 vw = make_double2(v.x * wr - v.y * wi, v.x * wi + v.y * wr);
            a[i] = make_double2(u.x + vw.x, u.y + vw.y);
            a[j] = make_double2(u.x - vw.x, u.y - vw.y);
        }
        __syncthreads();
    }
}

// Bluestein tables for FFT length n: chirp e^{+i pi j^2/n} and, for sign +1 and -1, the forward
// transform (sign -1) of the wrapped conjugate chirp filter of length m. One CTA.
__global__ void k_sep_tables(int n, int m, float2 *out) {
    extern __shared__ double2 a[];
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const long q = ((long)j * j) % (2L * n);  // phase pi*j^2/n reduced exactly
        double s, c;
        sincospi((double)q / (double)n, &s, &c);
        out[j] = make_float2((float)c, (float)s);
    }
    for (int sg = 0; sg < 2; sg++) {
        const double sign = sg == 0 ? 1.0 : -1.0;
        for (int j = threadIdx.x; j < m; j += blockDim.x) a[j] = make_double2(0.0, 0.0);
        __syncthreads();
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const long q = ((long)j * j) % (2L * n);
            double s, c;
            sincospi((double)q / (double)n, &s, &c);
            const double2 v = make_double2(c, -sign * s);  // conj of e^{sign i pi j^2/n}
            a[j] = v;
            if (j > 0) a[m - j] = v;  // m >= 2n-1: never overlaps a[0..n)
        }
        __syncthreads();
        fft_pow2_d(a, m, -1);
        for (int j = threadIdx.x; j < m; j += blockDim.x)
            out[n + sg * m + j] = make_float2((float)a[j].x, (float)a[j].y);
        __syncthreads();
    }
}

int fail(const char *msg) {
    wfd::set_global_error(WFD_ERR_ARG, msg);
    return WFD_ERR_ARG;
}

}  // namespace

extern "C" int WFD_AdjointBornAccumulation_wavefieldsep_NoAlloc(long nx, long ny, long nz, long isFWI,
                                                                 const float *v, const float *b,
                                                                 const float *wavefieldDP, const float *pOld,
                                                                 const float *wavefieldDM, const float *mOld,
                                                                 float *dVel, void *stream) {
    if (nx < 1 || ny < 1 || nz < 1) return fail("wavefieldsep_NoAlloc: grid sizes must be positive");
    if (nz > kMaxNz) return fail("wavefieldsep_NoAlloc: nz exceeds the maximum of 2048 (fixed scratch size)");
    if (!v || !b || !wavefieldDP || !pOld || !dVel) return fail("wavefieldsep_NoAlloc: null array");
    if ((wavefieldDM == nullptr) != (mOld == nullptr))
        return fail("wavefieldsep_NoAlloc: wavefieldDM and mOld must be given together");
    const void *arrays[7] = {v, b, wavefieldDP, pOld, dVel, wavefieldDM, mOld};
    for (int i = 0; i < 7; i++)
        if (arrays[i] && !wfd::device_accessible(arrays[i]))
            return fail("wavefieldsep_NoAlloc: every array must be device or managed memory");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return fail("wavefieldsep_NoAlloc: no device");
    // the arrays must live on the current device: the scratch address below is this device's
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, dVel) != cudaSuccess ||
        (attr.type == cudaMemoryTypeDevice && attr.device != dev))
        return fail("wavefieldsep_NoAlloc: the image is not on the current device");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = (int)(2 * nz);
    int m = 0;
    if (n & (n - 1)) {
        m = 1;
        while (m < 2 * n - 1) m <<= 1;
    }
    float2 *scratch = nullptr;
    {
        // set-up, once per device, with that device current: the device address of the file-scope
        // scratch array (the host name g_sep_scratch is not a device address)
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_addr[dev]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_sep_scratch);
            if (e != cudaSuccess) {
                wfd::set_global_error(WFD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
                return WFD_ERR_CUDA;
            }
            g_addr[dev] = static_cast<float2 *>(p);
            g_tables_n[dev] = 0;
        }
        scratch = g_addr[dev];
        // the Bluestein tables depend on n only: rebuilt when the last call on this device had another n
        if (m && g_tables_n[dev] != n) {
            const int smem = (int)(sizeof(double2) * (size_t)m);
            const cudaError_t e = cudaFuncSetAttribute(k_sep_tables, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (e != cudaSuccess) {
                wfd::set_global_error(WFD_ERR_CUDA, std::string("wavefieldsep_NoAlloc: shared memory for the tables: ") +
                                                        cudaGetErrorString(e));
                return WFD_ERR_CUDA;
            }
            k_sep_tables<<<1, 1024, smem, s>>>(n, m, scratch);
            g_tables_n[dev] = n;
        }
    }
    wfd::Grid g{};
    g.ndim = ny > 1 ? 3 : 2;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.sy = nz;
    g.sx = ny * nz;
    g.n = nx * ny * nz;
    wfd::Fields F{};
    F.v = const_cast<float *>(v);
    F.b = const_cast<float *>(b);
    F.pold = const_cast<float *>(pOld);
    F.mold = const_cast<float *>(mOld);
    // the bitwise-parity build when WAVEFD_B200_STRICT=1, as for new propagator objects
    const char *mode = getenv("WAVEFD_B200_STRICT");
    if (mode && mode[0] == '1')
        wfd_strict::image_wavefieldsep_tables(g, isFWI, F, wavefieldDP, wavefieldDM, dVel, scratch, m, s);
    else
        wfd_fast::image_wavefieldsep_tables(g, isFWI, F, wavefieldDP, wavefieldDM, dVel, scratch, m, s);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> lk(g_mu);
        g_tables_n[dev] = 0;  // the tables may not have been built
        wfd::set_global_error(WFD_ERR_CUDA, std::string("wavefieldsep_NoAlloc launch: ") + cudaGetErrorString(e));
        return WFD_ERR_CUDA;
    }
    return WFD_OK;
}
