// Wavefield-separation imaging condition (prop3DAcoIsoDenQ_DEO2_FDTD.h:673-765; VTI
// prop3DAcoVTIDenQ_DEO2_FDTD.h:606-725; TTI prop3DAcoTTIDenQ_DEO2_FDTD.h:609-728; 2D Iso
// prop2DAcoIsoDenQ_DEO2_FDTD.h:584-672), with a hand-written batched column FFT.
//
// Per (x,y) column and per field: zero-pad the column to nfft = 2nz, scale by 1/nfft,
// transform with sign +1 (FFTW's "forward" here is +1), zero bins [n/2+1, n) of the forward
// field and [kadj+1, kadj+n/2) of the adjoint field (kadj = 0 FWI, n/2 RTM), transform back
// with sign -1, and accumulate 2B/V^3 * Re(a*b). One CTA per column, everything in shared
// memory: radix-2 when nfft is a power of two, Bluestein's chirp-z convolution otherwise.
#include <math.h>

#include <vector>

#include "wfd_kernels.h"
#include "wfd_alloc.h"

namespace WFD_NS {
using namespace wfd;

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// in-place radix-2 FFT of length m (power of two) in shared memory: a[k] = sum_j a[j] e^{sign 2 pi i jk/m}
__device__ void fft_pow2(float2 *a, int m, int sign) {
    const int lg = 31 - __clz(m);
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        const int j = (int)(__brev((unsigned)i) >> (32 - lg));
        if (i < j) {
            const float2 t = a[i];
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
            float s, c;
            sincospif((float)(2 * pos) / (float)len, &s, &c);
            const float2 w = make_float2(c, sign * s);
            const float2 u = a[i];
            const float2 v = cmul(a[j], w);
            a[i] = make_float2(u.x + v.x, u.y + v.y);
            a[j] = make_float2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }
}

struct SepTables {
    const float2 *chirp;  // e^{+i pi j^2 / n}, j < n (Bluestein only)
    const float2 *vplus;  // FFT_M of the conjugate chirp filter for sign +1
    const float2 *vminus; // same for sign -1
    int n, m;             // transform length and Bluestein length (m = 0: radix-2)
};

// buf[0..n) <- DFT_n(buf) with the given sign; bb is an m-long scratch for Bluestein
__device__ void dft_n(float2 *buf, float2 *bb, const SepTables &T, int sign) {
    if (T.m == 0) {
        fft_pow2(buf, T.n, sign);
        return;
    }
    const int n = T.n, m = T.m;
    for (int j = threadIdx.x; j < m; j += blockDim.x) {
        if (j < n) {
            float2 c = T.chirp[j];
            if (sign < 0) c.y = -c.y;
            bb[j] = cmul(buf[j], c);
        } else {
            bb[j] = make_float2(0.0f, 0.0f);
        }
    }
    __syncthreads();
    fft_pow2(bb, m, -1);
    const float2 *V = sign > 0 ? T.vplus : T.vminus;
    for (int j = threadIdx.x; j < m; j += blockDim.x) bb[j] = cmul(bb[j], V[j]);
    __syncthreads();
    fft_pow2(bb, m, +1);
    const float inv = 1.0f / (float)m;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        float2 c = T.chirp[k];
        if (sign < 0) c.y = -c.y;
        const float2 y = make_float2(bb[k].x * inv, bb[k].y * inv);
        buf[k] = cmul(y, c);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_wavefieldsep(Grid g, long isfwi, Fields F, const float *__restrict__ dp,
                                                      const float *__restrict__ dm, float *dv, SepTables T, long col0) {
    extern __shared__ float2 sm[];
    const int n = T.n;
    const int nz = (int)g.nz;
    float2 *buf = sm;                          // n
    float2 *res = buf + n;                     // nz
    float *acc = (float *)(res + nz);          // nz
    float2 *bb = (float2 *)(acc + nz + (nz & 1));  // m (Bluestein)
    const long col = col0 + blockIdx.x;
    if (col >= g.nx * g.ny) return;
    const long base = col * g.nz;
    const float scale = 1.0f / (float)n;
    const int kadj = isfwi ? 0 : n / 2;
    for (int z = threadIdx.x; z < nz; z += blockDim.x) acc[z] = 0.0f;
    const int nfield = dm ? 2 : 1;
    for (int fld = 0; fld < nfield; fld++) {
        const float *nlf = fld == 0 ? dp : dm;
        const float *adj = fld == 0 ? F.pold : F.mold;
        for (int pass = 0; pass < 2; pass++) {
            const float *src = pass == 0 ? nlf : adj;
            for (int j = threadIdx.x; j < n; j += blockDim.x)
                buf[j] = make_float2(j < nz ? scale * src[base + j] : 0.0f, 0.0f);
            __syncthreads();
            dft_n(buf, bb, T, +1);
            const int z0 = pass == 0 ? n / 2 : kadj;  // up-going: drop positive bins; down-going: negative
            for (int k = 1 + threadIdx.x; k < n / 2; k += blockDim.x) buf[z0 + k] = make_float2(0.0f, 0.0f);
            __syncthreads();
            dft_n(buf, bb, T, -1);
            for (int z = threadIdx.x; z < nz; z += blockDim.x) {
                if (pass == 0) res[z] = buf[z];
                else acc[z] += res[z].x * buf[z].x - res[z].y * buf[z].y;
            }
            __syncthreads();
        }
    }
    for (int z = threadIdx.x; z < nz; z += blockDim.x) {
        const long k = base + z;
        const float V = F.v[k];
        const float B = F.b[k];
        const float factor = 2 * B / (V * V * V);
        dv[k] += factor * acc[z];
    }
}

// host double-precision radix-2 FFT for the Bluestein filter tables
void host_fft(std::vector<double> &re, std::vector<double> &im, int sign) {
    const size_t m = re.size();
    for (size_t i = 1, j = 0; i < m; i++) {
        size_t bit = m >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            std::swap(re[i], re[j]);
            std::swap(im[i], im[j]);
        }
    }
    for (size_t len = 2; len <= m; len <<= 1) {
        const double ang = sign * 2.0 * M_PI / (double)len;
        for (size_t i = 0; i < m; i += len)
            for (size_t k = 0; k < len / 2; k++) {
                const double c = cos(ang * k), s = sin(ang * k);
                const size_t a = i + k, b = i + k + len / 2;
                const double vr = re[b] * c - im[b] * s, vi = re[b] * s + im[b] * c;
                re[b] = re[a] - vr;
                im[b] = im[a] - vi;
                re[a] += vr;
                im[a] += vi;
            }
    }
}

}  // namespace

// Launch with Bluestein tables already on the device ({chirp[n], filter(+1)[m], filter(-1)[m]},
// m = 0 for power-of-two n); allocates nothing.
void image_wavefieldsep_tables(const Grid &g, long isfwi, const Fields &F, const float *dp, const float *dm,
                               float *dv, const float2 *tables, int m, cudaStream_t s) {
    const int n = (int)(2 * g.nz);
    SepTables T{nullptr, nullptr, nullptr, n, m};
    if (m) {
        T.chirp = tables;
        T.vplus = tables + n;
        T.vminus = tables + n + m;
    }
    const long nz = g.nz;
    const size_t smem = sizeof(float2) * (size_t)n + sizeof(float2) * (size_t)nz +
                        sizeof(float) * (size_t)(nz + (nz & 1)) + sizeof(float2) * (size_t)m;
    cudaFuncSetAttribute(k_wavefieldsep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long ncols = g.nx * g.ny;
    const long chunk = 65535;
    for (long c0 = 0; c0 < ncols; c0 += chunk) {
        const long nb = ncols - c0 < chunk ? ncols - c0 : chunk;
        k_wavefieldsep<<<(unsigned)nb, 256, smem, s>>>(g, isfwi, F, dp, dm, dv, T, c0);
    }
}

void image_wavefieldsep(const Grid &g, long isfwi, const Fields &F, const float *dp, const float *dm, float *dv,
                        float2 *work, long ncols_per_pass, cudaStream_t s) {
    (void)work;
    (void)ncols_per_pass;
    const int n = (int)(2 * g.nz);
    const bool pow2 = (n & (n - 1)) == 0;
    int m = 0;
    SepTables T{nullptr, nullptr, nullptr, n, 0};
    float2 *tables = nullptr;
    if (!pow2) {
        m = 1;
        while (m < 2 * n - 1) m <<= 1;
        T.m = m;
        std::vector<float2> h((size_t)n + 2 * (size_t)m);
        std::vector<double> cr(n), ci(n);
        for (long j = 0; j < n; j++) {
            const long q = (j * j) % (2L * n);  // exact phase pi*j^2/n reduced mod 2 pi
            cr[j] = cos(M_PI * (double)q / (double)n);
            ci[j] = sin(M_PI * (double)q / (double)n);
            h[j] = make_float2((float)cr[j], (float)ci[j]);
        }
        for (int sgn = 0; sgn < 2; sgn++) {
            const double sg = sgn == 0 ? 1.0 : -1.0;
            std::vector<double> vr(m, 0.0), vi(m, 0.0);
            for (long j = 0; j < n; j++) {
                // conj(c_s[j]) with c_s = e^{s i pi j^2/n}
                vr[j] = cr[j];
                vi[j] = -sg * ci[j];
                if (j > 0) {
                    vr[m - j] = vr[j];
                    vi[m - j] = vi[j];
                }
            }
            host_fft(vr, vi, -1);
            for (int j = 0; j < m; j++) h[(size_t)n + (size_t)sgn * m + j] = make_float2((float)vr[j], (float)vi[j]);
        }
        wfd::dMallocAsync(&tables, sizeof(float2) * h.size(), s);
        cudaMemcpyAsync(tables, h.data(), sizeof(float2) * h.size(), cudaMemcpyHostToDevice, s);
        T.chirp = tables;
        T.vplus = tables + n;
        T.vminus = tables + n + m;
    }
    const long nz = g.nz;
    size_t smem = sizeof(float2) * (size_t)n + sizeof(float2) * (size_t)nz + sizeof(float) * (size_t)(nz + (nz & 1));
    smem += sizeof(float2) * (size_t)m;
    cudaFuncSetAttribute(k_wavefieldsep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    const long ncols = g.nx * g.ny;
    const long chunk = 65535;
    for (long c0 = 0; c0 < ncols; c0 += chunk) {
        const long nb = ncols - c0 < chunk ? ncols - c0 : chunk;
        k_wavefieldsep<<<(unsigned)nb, 256, smem, s>>>(g, isfwi, F, dp, dm, dv, T, c0);
    }
    if (tables) cudaFreeAsync(tables, s);
}

}  // namespace WFD_NS
