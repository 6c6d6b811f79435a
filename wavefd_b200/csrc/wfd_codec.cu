// Learned wavefield codec: a small 3D convolutional autoencoder that compresses the saved forward
// wavefield of Born/adjoint imaging (the role CvxCompress plays for the reference: src/compressedio.jl
// :1-137 writes, and reads back, the saved p and m fields through CvxCompress). No counterpart in the
// reference's arithmetic; designed from scratch.
//
// Network (strided, non-overlapping convolutions; BF16 weights and activations, FP32 accumulation):
//   E1  conv 4^3 / stride 4,   1 -> 16 channels, leaky ReLU      (per 4^3 sub-block: 64 -> 16)
//   E2  conv 2^3 / stride 2,  16 -> 32 channels = the latent     (per 8^3 block: 8 x 16 -> 32)
//   D1  transposed conv 2^3,  32 -> 16 channels, leaky ReLU      (32 -> 8 x 16)
//   D2  transposed conv 4^3,  16 ->  1 channel                   (16 -> 64 per sub-block)
// Every 8^3 block is scaled by its max |value| (kept in FP32) before E1 and after D2. A block's
// code is 32 BF16 values + 1 FP32 scale (16x fewer values than the block). Trained on 32^3 patches
// of propagated wavefields; applied to whole grids (zero padding to multiples of 8).
// Raw fallback: the encoder also decodes each block and records its absolute error energy; the 1 %
// of blocks with the largest error (the few blocks around a source, where the field is not smooth
// on the block scale) are kept in FP32 beside the codes and written back over the decoded field.
// Code buffer per field: the raw-block selection state (16 B and an 8 KB histogram), scales, error
// energies, the raw slots' block ids, BF16 codes and raw blocks: about 97 bytes per 512 cells
// (2048 in FP32), 21x fewer bytes. Which blocks of the lowest selected error bin are kept raw
// depends on the order CTAs reach them; everything else is deterministic.
//
// Inference (encode / decode) runs the four layers as BF16 tensor-core MMAs (mma.sync m16n8k16,
// FP32 accumulate) on slabs of 32(z) x 32(y) x 8(x) cells staged in shared memory (the encoder
// double-buffers them with cp.async); at about 12 flop per byte it is bound by HBM, not by the
// tensor pipe. Training runs forward and backward on
// CUDA cores in FP32 from the same BF16 weights and BF16-rounded activations (straight-through
// gradients of the roundings), then Adam on FP32 master weights.
//
// Cell order inside a block (training blocks and the kernels agree): index = s*64 + k, sub-block
// s = (sx*2 + sy)*2 + sz, cell k = (dx*4 + dy)*4 + dz, position (4sx+dx, 4sy+dy, 4sz+dz) in (x,y,z).
// Latent of block (bx, by, bz): index (bx*nby + by)*nbz + bz, nb* = ceil(n*/8).
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "wavefd_b200.h"
#include "wfd_alloc.h"
#include "wfd_prop.h"
#include "wfd_tma.cuh"
#include "wfd_umma.cuh"

namespace wfd {
namespace codec {

typedef __nv_bfloat16 bf16;

// parameter vector (FP32 master; the BF16 copy uses the same offsets). W*t[n][k]: output n, input k.
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + 16 * 64, OFF_W2 = OFF_B1 + 16, OFF_B2 = OFF_W2 + 32 * 128,
              OFF_W3 = OFF_B2 + 32, OFF_B3 = OFF_W3 + 128 * 32, OFF_W4 = OFF_B3 + 128, OFF_B4 = OFF_W4 + 64 * 16,
              NPARAM = OFF_B4 + 64;
constexpr float LEAK = 0.5f;

__device__ __forceinline__ float act(float x) { return x >= 0.0f ? x : LEAK * x; }
__device__ __forceinline__ float dact(float x) { return x >= 0.0f ? 1.0f : LEAK; }
__device__ __forceinline__ float rbf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ uint32_t pack2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ uint32_t ld32(const bf16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

__device__ __forceinline__ void mma16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// ---- slabs ------------------------------------------------------------------------------------------
constexpr int SZ = 32, SY = 32, SX = 8, SLAB = SZ * SY * SX;  // 16 blocks of 8^3, 128 sub-blocks
constexpr int HROW = 136;                                     // bf16 row of one block's 8 x 16 (padded)
constexpr int W1P = 72, W2P = 136, W3P = 40, W4P = 24, LATP = 40;  // padded bf16 rows (bank spread)
constexpr int NTC = 128;                                      // threads of the codec kernels

struct Dims {
    int nx, ny, nz;
    int nsx, nsy, nsz;  // slabs per axis
    int nbx, nby, nbz;  // blocks per axis
};

// slab (xi, yi, zi) -> its 16 blocks: block b = by_local*4 + bz_local, x one block
__device__ __forceinline__ void slab_of(const Dims &d, long s, int &xi, int &yi, int &zi) {
    zi = (int)(s % d.nsz);
    yi = (int)((s / d.nsz) % d.nsy);
    xi = (int)(s / ((long)d.nsz * d.nsy));
}

__device__ __forceinline__ long block_id(const Dims &d, int xi, int yi, int zi, int b, bool &valid) {
    const int bx = xi, by = yi * 4 + b / 4, bz = zi * 4 + (b & 3);
    valid = bx < d.nbx && by < d.nby && bz < d.nbz;
    return ((long)bx * d.nby + by) * d.nbz + bz;
}

// Slab layout in shared memory: row (x, y) holds 32 z values, z stored at z ^ swz(x, y). The XOR
// touches bits 2-4 only (float4 groups stay whole) and spreads the rows of a fragment load over
// the banks (the sub-blocks of a fragment differ in x bit 2, y bit 2 and y bit 0).
__device__ __forceinline__ int swz(int x, int y) { return (((x >> 2) & 1) << 4) | (((y >> 2) & 1) << 3) | ((y & 1) << 2); }
__device__ __forceinline__ int soff(int x, int y, int z) { return (x * SY + y) * SZ + (z ^ swz(x, y)); }

// slab load (zero outside the grid) into sm[x][y][z]
__device__ __forceinline__ void load_slab(const Dims &d, const float *__restrict__ f, int xi, int yi, int zi,
                                          float *sm) {
    const int x0 = xi * SX, y0 = yi * SY, z0 = zi * SZ;
    const bool vec = (d.nz % 4) == 0;
    for (int q = threadIdx.x; q < SLAB / 4; q += NTC) {
        const int z = (q % (SZ / 4)) * 4, y = (q / (SZ / 4)) % SY, x = q / (SZ / 4 * SY);
        const int gx = x0 + x, gy = y0 + y, gz = z0 + z;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gx < d.nx && gy < d.ny) {
            const float *p = f + ((long)gx * d.ny + gy) * d.nz + gz;
            if (vec && gz + 3 < d.nz) {
                v = __ldg(reinterpret_cast<const float4 *>(p));
            } else {
                v.x = gz < d.nz ? p[0] : 0.f;
                v.y = gz + 1 < d.nz ? p[1] : 0.f;
                v.z = gz + 2 < d.nz ? p[2] : 0.f;
                v.w = gz + 3 < d.nz ? p[3] : 0.f;
            }
        }
        *reinterpret_cast<float4 *>(sm + soff(x, y, z)) = v;
    }
}

// the same load with cp.async (16-byte copies, zero fill outside the grid); needs nz % 4 == 0 and a
// 16-byte-aligned field. Completion: cp.async.wait_group, then a CTA barrier.
__device__ __forceinline__ void load_slab_async(const Dims &d, const float *__restrict__ f, int xi, int yi, int zi,
                                                float *sm) {
    const int x0 = xi * SX, y0 = yi * SY, z0 = zi * SZ;
    for (int q = threadIdx.x; q < SLAB / 4; q += NTC) {
        const int z = (q % (SZ / 4)) * 4, y = (q / (SZ / 4)) % SY, x = q / (SZ / 4 * SY);
        const int gx = x0 + x, gy = y0 + y, gz = z0 + z;
        const bool in = gx < d.nx && gy < d.ny && gz < d.nz;
        const float *src = in ? f + ((long)gx * d.ny + gy) * d.nz + gz : f;
        const uint32_t dst = static_cast<uint32_t>(__cvta_generic_to_shared(sm + soff(x, y, z)));
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(in ? 16 : 0)
                     : "memory");
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void store_slab(const Dims &d, float *__restrict__ f, int xi, int yi, int zi,
                                           const float *sm) {
    const int x0 = xi * SX, y0 = yi * SY, z0 = zi * SZ;
    const bool vec = (d.nz % 4) == 0;
    for (int q = threadIdx.x; q < SLAB / 4; q += NTC) {
        const int z = (q % (SZ / 4)) * 4, y = (q / (SZ / 4)) % SY, x = q / (SZ / 4 * SY);
        const int gx = x0 + x, gy = y0 + y, gz = z0 + z;
        if (gx >= d.nx || gy >= d.ny || gz >= d.nz) continue;
        const float4 v = *reinterpret_cast<const float4 *>(sm + soff(x, y, z));
        float *p = f + ((long)gx * d.ny + gy) * d.nz + gz;
        if (vec && gz + 3 < d.nz) {
            *reinterpret_cast<float4 *>(p) = v;
        } else {
            p[0] = v.x;
            if (gz + 1 < d.nz) p[1] = v.y;
            if (gz + 2 < d.nz) p[2] = v.z;
            if (gz + 3 < d.nz) p[3] = v.w;
        }
    }
}

// smem offset of cell (sub-row r = b*8+s, cell k) in the slab
__device__ __forceinline__ int cell_off(int r, int k) {
    const int b = r >> 3, s = r & 7;
    const int x = (s >> 2) * 4 + (k >> 4);
    const int y = (b >> 2) * 8 + ((s >> 1) & 1) * 4 + ((k >> 2) & 3);
    const int z = (b & 3) * 8 + (s & 1) * 4 + (k & 3);
    return soff(x, y, z);
}

// ---- encode -----------------------------------------------------------------------------------------
// Codes and scales of every block, and its error energy: the block is decoded here too (D1, D2 on
// the same tiles) and sum((decoded - field)^2) over its cells is stored in err_out.
__global__ void __launch_bounds__(NTC, 2)
    k_encode(Dims d, const float *__restrict__ f, const bf16 *__restrict__ wb, const float *__restrict__ wp,
             float *__restrict__ scale_out, float *__restrict__ err_out, bf16 *__restrict__ lat_out) {
    extern __shared__ __align__(16) float smf[];
    float *slabs = smf;                                    // 2 x SLAB floats (double buffer)
    float *bscale = slabs + 2 * SLAB;                      // 16
    float *binv = bscale + 16;                             // 16
    float *berr = binv + 16;                               // 16
    float *sb1 = berr + 16;                                // 16
    float *sb2 = sb1 + 16;                                 // 32
    float *sb3 = sb2 + 32;                                 // 128
    float *sb4 = sb3 + 128;                                // 64
    bf16 *H1 = reinterpret_cast<bf16 *>(sb4 + 64);         // 16 * HROW (reused for D1's output)
    bf16 *lat = H1 + 16 * HROW;                            // 16 * LATP
    bf16 *sW1 = lat + 16 * LATP;                           // 16 * W1P
    bf16 *sW2 = sW1 + 16 * W1P;                            // 32 * W2P
    bf16 *sW3 = sW2 + 32 * W2P;                            // 128 * W3P
    bf16 *sW4 = sW3 + 128 * W3P;                           // 64 * W4P
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, c = lane & 3;
    for (int i = tid; i < 16 * 64; i += NTC) sW1[(i / 64) * W1P + i % 64] = wb[OFF_W1 + i];
    for (int i = tid; i < 32 * 128; i += NTC) sW2[(i / 128) * W2P + i % 128] = wb[OFF_W2 + i];
    for (int i = tid; i < 128 * 32; i += NTC) sW3[(i / 32) * W3P + i % 32] = wb[OFF_W3 + i];
    for (int i = tid; i < 64 * 16; i += NTC) sW4[(i / 16) * W4P + i % 16] = wb[OFF_W4 + i];
    if (tid < 16) sb1[tid] = wp[OFF_B1 + tid];
    if (tid < 32) sb2[tid] = wp[OFF_B2 + tid];
    sb3[tid] = wp[OFF_B3 + tid];
    if (tid < 64) sb4[tid] = wp[OFF_B4 + tid];
    const long nslab = (long)d.nsx * d.nsy * d.nsz;
    const bool async = (d.nz % 4) == 0 && (reinterpret_cast<uintptr_t>(f) & 15) == 0;
    if (async && blockIdx.x < nslab) {
        int xi, yi, zi;
        slab_of(d, blockIdx.x, xi, yi, zi);
        load_slab_async(d, f, xi, yi, zi, slabs);
    }
    int buf = 0;
    for (long sl = blockIdx.x; sl < nslab; sl += gridDim.x, buf ^= 1) {
        int xi, yi, zi;
        slab_of(d, sl, xi, yi, zi);
        float *slab = slabs + buf * SLAB;
        __syncthreads();  // the other buffer's readers (the previous slab) are done
        if (async) {
            // the next slab's copies go into the other buffer while this one is processed
            if (sl + gridDim.x < nslab) {
                int xn, yn, zn;
                slab_of(d, sl + gridDim.x, xn, yn, zn);
                load_slab_async(d, f, xn, yn, zn, slabs + (buf ^ 1) * SLAB);
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            }
        } else {
            load_slab(d, f, xi, yi, zi, slab);
        }
        __syncthreads();
        {  // block max |value|: 8 threads per block, one x plane each
            const int b = tid >> 3, x = tid & 7;
            float m = 0.0f;
#pragma unroll
            for (int yy = 0; yy < 8; yy++) {
                const int y = (b >> 2) * 8 + yy, z = (b & 3) * 8;
                const float4 u = *reinterpret_cast<const float4 *>(slab + soff(x, y, z));
                const float4 v = *reinterpret_cast<const float4 *>(slab + soff(x, y, z + 4));
                m = fmaxf(m, fmaxf(fmaxf(fabsf(u.x), fabsf(u.y)), fmaxf(fabsf(u.z), fabsf(u.w))));
                m = fmaxf(m, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
            }
            m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 1));
            m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 2));
            m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 4));
            if (x == 0) {
                bscale[b] = m;
                binv[b] = m > 0.0f ? 1.0f / m : 0.0f;
            }
        }
        __syncthreads();
        // E1: rows = sub-blocks (128), K = 64, N = 16; warp w: m-tiles 2w, 2w+1
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            const int r0 = (2 * warp + mt) * 16 + g, r1 = r0 + 8;
            const float i0 = binv[r0 >> 3], i1 = binv[r1 >> 3];
            float acc[2][4] = {};
#pragma unroll
            for (int kk = 0; kk < 4; kk++) {
                const int ka = 16 * kk + 2 * c, kb = ka + 8;
                const float2 x00 = *reinterpret_cast<const float2 *>(slab + cell_off(r0, ka));
                const float2 x10 = *reinterpret_cast<const float2 *>(slab + cell_off(r1, ka));
                const float2 x01 = *reinterpret_cast<const float2 *>(slab + cell_off(r0, kb));
                const float2 x11 = *reinterpret_cast<const float2 *>(slab + cell_off(r1, kb));
                const uint32_t a0 = pack2(x00.x * i0, x00.y * i0), a1 = pack2(x10.x * i1, x10.y * i1);
                const uint32_t a2 = pack2(x01.x * i0, x01.y * i0), a3 = pack2(x11.x * i1, x11.y * i1);
#pragma unroll
                for (int nt = 0; nt < 2; nt++) {
                    const bf16 *wr = sW1 + (nt * 8 + g) * W1P + 16 * kk + 2 * c;
                    mma16816(acc[nt], a0, a1, a2, a3, ld32(wr), ld32(wr + 8));
                }
            }
#pragma unroll
            for (int nt = 0; nt < 2; nt++) {
                const int ch = nt * 8 + 2 * c;
                const float bb0 = sb1[ch], bb1 = sb1[ch + 1];
                *reinterpret_cast<uint32_t *>(H1 + (r0 >> 3) * HROW + (r0 & 7) * 16 + ch) =
                    pack2(act(acc[nt][0] + bb0), act(acc[nt][1] + bb1));
                *reinterpret_cast<uint32_t *>(H1 + (r1 >> 3) * HROW + (r1 & 7) * 16 + ch) =
                    pack2(act(acc[nt][2] + bb0), act(acc[nt][3] + bb1));
            }
        }
        __syncthreads();
        // E2: rows = blocks (16), K = 128, N = 32; warp w: n-tile w
        {
            float acc[4] = {};
#pragma unroll
            for (int kk = 0; kk < 8; kk++) {
                const bf16 *h0 = H1 + g * HROW + 16 * kk + 2 * c, *h1 = h0 + 8 * HROW;
                const bf16 *wr = sW2 + (warp * 8 + g) * W2P + 16 * kk + 2 * c;
                mma16816(acc, ld32(h0), ld32(h1), ld32(h0 + 8), ld32(h1 + 8), ld32(wr), ld32(wr + 8));
            }
            const int n = warp * 8 + 2 * c;
            const uint32_t q0 = pack2(acc[0] + sb2[n], acc[1] + sb2[n + 1]);
            const uint32_t q1 = pack2(acc[2] + sb2[n], acc[3] + sb2[n + 1]);
            *reinterpret_cast<uint32_t *>(lat + g * LATP + n) = q0;
            *reinterpret_cast<uint32_t *>(lat + (g + 8) * LATP + n) = q1;
            bool v0, v1;
            const long id0 = block_id(d, xi, yi, zi, g, v0), id1 = block_id(d, xi, yi, zi, g + 8, v1);
            if (v0) *reinterpret_cast<uint32_t *>(lat_out + id0 * 32 + n) = q0;
            if (v1) *reinterpret_cast<uint32_t *>(lat_out + id1 * 32 + n) = q1;
        }
        __syncthreads();
        // decode in place: D1 (blocks x 32 -> 128) into H1, then D2 against the slab
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int nt = 4 * warp + j;
            float acc[4] = {};
#pragma unroll
            for (int kk = 0; kk < 2; kk++) {
                const bf16 *l0 = lat + g * LATP + 16 * kk + 2 * c, *l1 = l0 + 8 * LATP;
                const bf16 *wr = sW3 + (nt * 8 + g) * W3P + 16 * kk + 2 * c;
                mma16816(acc, ld32(l0), ld32(l1), ld32(l0 + 8), ld32(l1 + 8), ld32(wr), ld32(wr + 8));
            }
            const int n = nt * 8 + 2 * c;
            *reinterpret_cast<uint32_t *>(H1 + g * HROW + n) = pack2(act(acc[0] + sb3[n]), act(acc[1] + sb3[n + 1]));
            *reinterpret_cast<uint32_t *>(H1 + (g + 8) * HROW + n) =
                pack2(act(acc[2] + sb3[n]), act(acc[3] + sb3[n + 1]));
        }
        __syncthreads();
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            const int r0 = (2 * warp + mt) * 16 + g, r1 = r0 + 8;
            const bf16 *h0 = H1 + (r0 >> 3) * HROW + (r0 & 7) * 16 + 2 * c;
            const bf16 *h1 = H1 + (r1 >> 3) * HROW + (r1 & 7) * 16 + 2 * c;
            const uint32_t a0 = ld32(h0), a1 = ld32(h1), a2 = ld32(h0 + 8), a3 = ld32(h1 + 8);
            const float s0 = bscale[r0 >> 3], s1 = bscale[r1 >> 3];
            float e0 = 0.0f, e1 = 0.0f;
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                float acc[4] = {};
                const bf16 *wr = sW4 + (nt * 8 + g) * W4P + 2 * c;
                mma16816(acc, a0, a1, a2, a3, ld32(wr), ld32(wr + 8));
                const int k = nt * 8 + 2 * c;
                const float2 x0 = *reinterpret_cast<const float2 *>(slab + cell_off(r0, k));
                const float2 x1 = *reinterpret_cast<const float2 *>(slab + cell_off(r1, k));
                const float d00 = (acc[0] + sb4[k]) * s0 - x0.x, d01 = (acc[1] + sb4[k + 1]) * s0 - x0.y;
                const float d10 = (acc[2] + sb4[k]) * s1 - x1.x, d11 = (acc[3] + sb4[k + 1]) * s1 - x1.y;
                e0 += d00 * d00 + d01 * d01;
                e1 += d10 * d10 + d11 * d11;
            }
            // rows r0 of this m-tile all belong to block r0 >> 3, rows r1 to the next block: one
            // warp owns both blocks' sums (a fixed-order reduction)
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                e0 += __shfl_xor_sync(0xffffffffu, e0, o);
                e1 += __shfl_xor_sync(0xffffffffu, e1, o);
            }
            if (lane == 0) {
                berr[r0 >> 3] = e0;
                berr[r1 >> 3] = e1;
            }
        }
        __syncthreads();
        if (tid < 16) {
            bool v;
            const long id = block_id(d, xi, yi, zi, tid, v);
            if (v) {
                scale_out[id] = bscale[tid];
                err_out[id] = berr[tid];
            }
        }
    }
}

// Raw fallback, step 1: histogram of the error energies (2048 bins of the float's top bits, i.e.
// 1/8-octave bins; energies are >= 0 so their bit patterns order like the values).
__global__ void k_err_hist(long nb, const float *__restrict__ err, unsigned *__restrict__ hist) {
    __shared__ unsigned h[2048];
    for (int i = threadIdx.x; i < 2048; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (long b = (long)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (long)gridDim.x * blockDim.x)
        atomicAdd(&h[__float_as_uint(err[b]) >> 20], 1u);
    __syncthreads();
    for (int i = threadIdx.x; i < 2048; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], h[i]);
}

// step 2 (one CTA of 1024 threads): with S(t) = the blocks in bins >= t, the threshold bin T is
// the largest t >= 1 with S(t) > cap (0 if none); every block above T is kept raw and ctl[1] =
// cap - S(T+1) slots are left for blocks in bin T. S is non-increasing, so T = #{t >= 1 : S(t) >
// cap}. Thread i holds bins 2047-2i and 2046-2i; a prefix sum over threads is a suffix sum over
// bins. Bin 0 (zero error) is never kept.
__global__ void __launch_bounds__(1024) k_err_threshold(const unsigned *__restrict__ hist, long cap,
                                                         int *__restrict__ ctl) {
    __shared__ unsigned long long wsum[32];
    __shared__ int count;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const int b0 = 2047 - 2 * t, b1 = b0 - 1;
    const unsigned long long h0 = hist[b0], h1 = hist[b1];
    unsigned long long x = h0 + h1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (t == 0) count = 0;
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        unsigned long long y = wsum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long z = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) y += z;
        }
        wsum[lane] = y;
    }
    __syncthreads();
    const unsigned long long above = (wid ? wsum[wid - 1] : 0ull) + x - (h0 + h1);  // bins > b0
    const unsigned long long s0 = above + h0, s1 = s0 + h1;                         // S(b0), S(b1)
    const unsigned long long ucap = (unsigned long long)cap;
    const int c = (b0 >= 1 && s0 > ucap ? 1 : 0) + (b1 >= 1 && s1 > ucap ? 1 : 0);
    const int wc = __reduce_add_sync(0xffffffffu, (unsigned)c);
    if (lane == 0 && wc) atomicAdd(&count, wc);
    __syncthreads();
    const int T = count;
    // S(T+1): the blocks above the threshold bin (none when T = 2047)
    unsigned long long used = 0;
    bool mine = false;
    if (T == 2047) mine = t == 0;
    else if (b0 == T + 1) mine = true, used = s0;
    else if (b1 == T + 1) mine = true, used = s1;
    if (mine) {
        ctl[0] = T;                                     // bins > T: raw
        ctl[1] = T > 0 ? (int)(cap - (long)used) : 0;  // slots for bin T
        ctl[2] = 0;                                     // slots taken (step 3)
        ctl[3] = 0;                                     // slots taken in bin T
    }
}

// step 3: assign raw slots, one block per thread with warp-aggregated counters
__global__ void k_err_pick(long nb, const float *__restrict__ err, long cap, int *__restrict__ ctl,
                           int *__restrict__ raw_id) {
    const int T = ctl[0], tslots = ctl[1];
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long base = (long)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < nb; base += stride) {
        const long b = base + lane;
        const int bin = b < nb ? (int)(__float_as_uint(err[b]) >> 20) : 0;
        const bool hi = b < nb && bin > T;
        const bool eq = b < nb && bin == T && bin > 0;
        const unsigned meq = __ballot_sync(0xffffffffu, eq);
        int ebase = 0;
        if (meq) {
            if (lane == 0) ebase = atomicAdd(&ctl[3], __popc(meq));
            ebase = __shfl_sync(0xffffffffu, ebase, 0);
        }
        const bool take = hi || (eq && ebase + __popc(meq & below) < tslots);
        const unsigned mt = __ballot_sync(0xffffffffu, take);
        if (mt) {
            int sbase = 0;
            if (lane == 0) sbase = atomicAdd(&ctl[2], __popc(mt));
            sbase = __shfl_sync(0xffffffffu, sbase, 0);
            const int sl = sbase + __popc(mt & below);
            if (take && sl < cap) raw_id[sl] = (int)b;
        }
    }
}

// step 4: copy the raw blocks' cells (x, y, z order; zero outside the grid), one CTA per block
__global__ void k_raw_gather(Dims d, const float *__restrict__ f, const int *__restrict__ ctl, long cap,
                             const int *__restrict__ raw_id, float *__restrict__ raw) {
    const int nraw = ctl[2] < cap ? ctl[2] : (int)cap;
    for (int s = blockIdx.x; s < nraw; s += gridDim.x) {
        const long b = raw_id[s];
        const int bz = (int)(b % d.nbz), by = (int)((b / d.nbz) % d.nby), bx = (int)(b / ((long)d.nbz * d.nby));
        for (int j = threadIdx.x; j < 512; j += blockDim.x) {
            const int x = bx * 8 + (j >> 6), y = by * 8 + ((j >> 3) & 7), z = bz * 8 + (j & 7);
            raw[(long)s * 512 + j] = (x < d.nx && y < d.ny && z < d.nz) ? f[((long)x * d.ny + y) * d.nz + z] : 0.0f;
        }
    }
}

// decode's last step: raw blocks written over the decoded field
__global__ void k_raw_scatter(Dims d, const int *__restrict__ ctl, long cap, const int *__restrict__ raw_id,
                              const float *__restrict__ raw, float *__restrict__ f) {
    const int nraw = ctl[2] < cap ? ctl[2] : (int)cap;
    for (int s = blockIdx.x; s < nraw; s += gridDim.x) {
        const long b = raw_id[s];
        const int bz = (int)(b % d.nbz), by = (int)((b / d.nbz) % d.nby), bx = (int)(b / ((long)d.nbz * d.nby));
        for (int j = threadIdx.x; j < 512; j += blockDim.x) {
            const int x = bx * 8 + (j >> 6), y = by * 8 + ((j >> 3) & 7), z = bz * 8 + (j & 7);
            if (x < d.nx && y < d.ny && z < d.nz) f[((long)x * d.ny + y) * d.nz + z] = raw[(long)s * 512 + j];
        }
    }
}

// ---- decode -----------------------------------------------------------------------------------------
__global__ void __launch_bounds__(NTC, 4)
    k_decode(Dims d, const float *__restrict__ scale_in, const bf16 *__restrict__ lat_in, const bf16 *__restrict__ wb,
             const float *__restrict__ wp, float *__restrict__ f) {
    extern __shared__ __align__(16) float smf[];
    float *slab = smf;               // SLAB
    float *bscale = slab + SLAB;     // 16
    float *sb3 = bscale + 16;        // 128
    float *sb4 = sb3 + 128;          // 64
    bf16 *lat = reinterpret_cast<bf16 *>(sb4 + 64);  // 16 * LATP
    bf16 *H2 = lat + 16 * LATP;                      // 16 * HROW
    bf16 *sW3 = H2 + 16 * HROW;                      // 128 * W3P
    bf16 *sW4 = sW3 + 128 * W3P;                     // 64 * W4P
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, c = lane & 3;
    for (int i = tid; i < 128 * 32; i += NTC) sW3[(i / 32) * W3P + i % 32] = wb[OFF_W3 + i];
    for (int i = tid; i < 64 * 16; i += NTC) sW4[(i / 16) * W4P + i % 16] = wb[OFF_W4 + i];
    for (int i = tid; i < 128; i += NTC) sb3[i] = wp[OFF_B3 + i];
    if (tid < 64) sb4[tid] = wp[OFF_B4 + tid];
    const long nslab = (long)d.nsx * d.nsy * d.nsz;
    for (long sl = blockIdx.x; sl < nslab; sl += gridDim.x) {
        int xi, yi, zi;
        slab_of(d, sl, xi, yi, zi);
        __syncthreads();
        {  // latents and scales of the slab's 16 blocks (zero outside the grid)
            const int b = tid >> 3, part = tid & 7;  // 8 threads x 4 values per block
            bool v;
            const long id = block_id(d, xi, yi, zi, b, v);
            uint2 q = make_uint2(0u, 0u);
            if (v) q = *reinterpret_cast<const uint2 *>(lat_in + id * 32 + 4 * part);
            *reinterpret_cast<uint2 *>(lat + b * LATP + 4 * part) = q;
            if (part == 0) bscale[b] = v ? scale_in[id] : 0.0f;
        }
        __syncthreads();
        // D1: rows = blocks (16), K = 32, N = 128; warp w: n-tiles 4w .. 4w+3
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int nt = 4 * warp + j;
            float acc[4] = {};
#pragma unroll
            for (int kk = 0; kk < 2; kk++) {
                const bf16 *l0 = lat + g * LATP + 16 * kk + 2 * c, *l1 = l0 + 8 * LATP;
                const bf16 *wr = sW3 + (nt * 8 + g) * W3P + 16 * kk + 2 * c;
                mma16816(acc, ld32(l0), ld32(l1), ld32(l0 + 8), ld32(l1 + 8), ld32(wr), ld32(wr + 8));
            }
            const int n = nt * 8 + 2 * c;
            *reinterpret_cast<uint32_t *>(H2 + g * HROW + n) = pack2(act(acc[0] + sb3[n]), act(acc[1] + sb3[n + 1]));
            *reinterpret_cast<uint32_t *>(H2 + (g + 8) * HROW + n) =
                pack2(act(acc[2] + sb3[n]), act(acc[3] + sb3[n + 1]));
        }
        __syncthreads();
        // D2: rows = sub-blocks (128), K = 16, N = 64; warp w: m-tiles 2w, 2w+1
#pragma unroll
        for (int mt = 0; mt < 2; mt++) {
            const int r0 = (2 * warp + mt) * 16 + g, r1 = r0 + 8;
            const bf16 *h0 = H2 + (r0 >> 3) * HROW + (r0 & 7) * 16 + 2 * c;
            const bf16 *h1 = H2 + (r1 >> 3) * HROW + (r1 & 7) * 16 + 2 * c;
            const uint32_t a0 = ld32(h0), a1 = ld32(h1), a2 = ld32(h0 + 8), a3 = ld32(h1 + 8);
            const float s0 = bscale[r0 >> 3], s1 = bscale[r1 >> 3];
#pragma unroll
            for (int nt = 0; nt < 8; nt++) {
                float acc[4] = {};
                const bf16 *wr = sW4 + (nt * 8 + g) * W4P + 2 * c;
                mma16816(acc, a0, a1, a2, a3, ld32(wr), ld32(wr + 8));
                const int k = nt * 8 + 2 * c;
                *reinterpret_cast<float2 *>(slab + cell_off(r0, k)) =
                    make_float2((acc[0] + sb4[k]) * s0, (acc[1] + sb4[k + 1]) * s0);
                *reinterpret_cast<float2 *>(slab + cell_off(r1, k)) =
                    make_float2((acc[2] + sb4[k]) * s1, (acc[3] + sb4[k + 1]) * s1);
            }
        }
        __syncthreads();
        store_slab(d, f, xi, yi, zi, slab);
    }
}

constexpr size_t ENC_SMEM = (size_t)(2 * SLAB + 16 * 4 + 32 + 128 + 64) * 4 +
                            (size_t)(16 * HROW + 16 * LATP + 16 * W1P + 32 * W2P + 128 * W3P + 64 * W4P) * 2;
constexpr size_t DEC_SMEM =
    (size_t)(SLAB + 16 + 128 + 64) * 4 + (size_t)(16 * LATP + 16 * HROW + 128 * W3P + 64 * W4P) * 2;

#include "wfd_codec_umma.cuh"

// ---- training blocks --------------------------------------------------------------------------------
// blocks[i] = field block at origin (ox, oy, oz)[i] in the codec's cell order, divided by its max
// |value| (zero blocks stay zero); scale[i] = that max. Cells outside the grid read as zero.
__global__ void k_gather_blocks(int nx, int ny, int nz, const float *__restrict__ f, const int *__restrict__ org,
                                long n, float *__restrict__ out, float *__restrict__ scale) {
    const long i = blockIdx.x;
    if (i >= n) return;
    const int ox = org[3 * i], oy = org[3 * i + 1], oz = org[3 * i + 2];
    __shared__ float v[512];
    __shared__ float red[32];
    float m = 0.0f;
    for (int j = threadIdx.x; j < 512; j += blockDim.x) {
        const int s = j >> 6, k = j & 63;
        const int x = ox + (s >> 2) * 4 + (k >> 4), y = oy + ((s >> 1) & 1) * 4 + ((k >> 2) & 3),
                  z = oz + (s & 1) * 4 + (k & 3);
        float a = 0.0f;
        if (x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz) a = f[((long)x * ny + y) * nz + z];
        v[j] = a;
        m = fmaxf(m, fabsf(a));
    }
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float mm = 0.0f;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) mm = fmaxf(mm, red[w]);
        red[0] = mm;
    }
    __syncthreads();
    const float mm = red[0], inv = mm > 0.0f ? 1.0f / mm : 0.0f;
    for (int j = threadIdx.x; j < 512; j += blockDim.x) out[i * 512 + j] = v[j] * inv;
    if (threadIdx.x == 0 && scale) scale[i] = mm;
}

// ---- training: forward + backward on CUDA cores -----------------------------------------------------
constexpr int NTT = 256;

struct TrainSmem {
    float W[NPARAM];    // BF16 weights widened to FP32 (biases FP32 master)
    float G[NPARAM];    // this CTA's gradient
    float X[512], Xq[512], Y[512], dY[512];
    float H1p[128], H1q[128], dH1[128];
    float Z[32], Zq[32], dZ[32];
    float H2p[128], H2q[128], dH2[128];
    float red[NTT / 32];
};

__global__ void __launch_bounds__(NTT)
    k_train(const float *__restrict__ blocks, long n, float inv_count, const bf16 *__restrict__ wb,
            const float *__restrict__ wp, float *__restrict__ grad, float *__restrict__ loss) {
    extern __shared__ __align__(16) float smraw[];
    TrainSmem &S = *reinterpret_cast<TrainSmem *>(smraw);
    const int t = threadIdx.x, lane = t & 31;
    for (int i = t; i < NPARAM; i += NTT) {
        const bool bias = (i >= OFF_B1 && i < OFF_W2) || (i >= OFF_B2 && i < OFF_W3) || (i >= OFF_B3 && i < OFF_W4) ||
                          i >= OFF_B4;
        S.W[i] = bias ? wp[i] : __bfloat162float(wb[i]);
        S.G[i] = 0.0f;
    }
    const float *W1 = S.W + OFF_W1, *B1 = S.W + OFF_B1, *W2 = S.W + OFF_W2, *B2 = S.W + OFF_B2;
    const float *W3 = S.W + OFF_W3, *B3 = S.W + OFF_B3, *W4 = S.W + OFF_W4, *B4 = S.W + OFF_B4;
    float *G1 = S.G + OFF_W1, *Gb1 = S.G + OFF_B1, *G2 = S.G + OFF_W2, *Gb2 = S.G + OFF_B2;
    float *G3 = S.G + OFF_W3, *Gb3 = S.G + OFF_B3, *G4 = S.G + OFF_W4, *Gb4 = S.G + OFF_B4;
    float lsum = 0.0f;
    __syncthreads();
    for (long bi = blockIdx.x; bi < n; bi += gridDim.x) {
        for (int j = t; j < 512; j += NTT) {
            const float x = blocks[bi * 512 + j];
            S.X[j] = x;
            S.Xq[j] = rbf(x);
        }
        __syncthreads();
        // E1: H1p[s*16+ch] = b1 + W1[ch] . Xq[s]
        if (t < 128) {
            const int s = t >> 4, ch = t & 15;
            float a = 0.0f;
            for (int k = 0; k < 64; k++) a += W1[ch * 64 + k] * S.Xq[s * 64 + k];
            a += B1[ch];
            S.H1p[t] = a;
            S.H1q[t] = rbf(act(a));
        }
        __syncthreads();
        // E2: Z[n] = b2 + W2[n] . H1q; 8 threads per output
        {
            const int nn = t >> 3, part = t & 7;
            float a = 0.0f;
            for (int k = part * 16; k < part * 16 + 16; k++) a += W2[nn * 128 + k] * S.H1q[k];
            a += __shfl_xor_sync(0xffffffffu, a, 1);
            a += __shfl_xor_sync(0xffffffffu, a, 2);
            a += __shfl_xor_sync(0xffffffffu, a, 4);
            if (part == 0) {
                a += B2[nn];
                S.Z[nn] = a;
                S.Zq[nn] = rbf(a);
            }
        }
        __syncthreads();
        // D1: H2p[n] = b3 + W3[n] . Zq
        if (t < 128) {
            float a = 0.0f;
            for (int k = 0; k < 32; k++) a += W3[t * 32 + k] * S.Zq[k];
            a += B3[t];
            S.H2p[t] = a;
            S.H2q[t] = rbf(act(a));
        }
        __syncthreads();
        // D2: Y[s*64+k] = b4 + W4[k] . H2q[s]; loss and dY
        for (int o = t; o < 512; o += NTT) {
            const int s = o >> 6, k = o & 63;
            float a = 0.0f;
            for (int j = 0; j < 16; j++) a += W4[k * 16 + j] * S.H2q[s * 16 + j];
            a += B4[k];
            S.Y[o] = a;
            const float e = a - S.X[o];
            lsum += e * e;
            S.dY[o] = 2.0f * e * inv_count;
        }
        __syncthreads();
        // dW4[k][j] += sum_s dY[s,k] H2q[s,j]; db4; dH2[s*16+j] = sum_k W4[k][j] dY[s,k]
        for (int e = t; e < 64 * 16; e += NTT) {
            const int k = e >> 4, j = e & 15;
            float a = 0.0f;
            for (int s = 0; s < 8; s++) a += S.dY[s * 64 + k] * S.H2q[s * 16 + j];
            G4[e] += a;
        }
        if (t < 64) {
            float a = 0.0f;
            for (int s = 0; s < 8; s++) a += S.dY[s * 64 + t];
            Gb4[t] += a;
        }
        if (t < 128) {
            const int s = t >> 4, j = t & 15;
            float a = 0.0f;
            for (int k = 0; k < 64; k++) a += W4[k * 16 + j] * S.dY[s * 64 + k];
            S.dH2[t] = a * dact(S.H2p[t]);
        }
        __syncthreads();
        // dW3[n][k] += dH2[n] Zq[k]; db3; dZ[k] = sum_n W3[n][k] dH2[n]
        for (int e = t; e < 128 * 32; e += NTT) G3[e] += S.dH2[e >> 5] * S.Zq[e & 31];
        if (t < 128) Gb3[t] += S.dH2[t];
        {
            const int k = t >> 3, part = t & 7;
            float a = 0.0f;
            for (int nn = part * 16; nn < part * 16 + 16; nn++) a += W3[nn * 32 + k] * S.dH2[nn];
            a += __shfl_xor_sync(0xffffffffu, a, 1);
            a += __shfl_xor_sync(0xffffffffu, a, 2);
            a += __shfl_xor_sync(0xffffffffu, a, 4);
            if (part == 0) S.dZ[k] = a;
        }
        __syncthreads();
        // dW2[n][k] += dZ[n] H1q[k]; db2; dH1[k] = sum_n W2[n][k] dZ[n]
        for (int e = t; e < 32 * 128; e += NTT) G2[e] += S.dZ[e >> 7] * S.H1q[e & 127];
        if (t < 32) Gb2[t] += S.dZ[t];
        if (t < 128) {
            float a = 0.0f;
            for (int nn = 0; nn < 32; nn++) a += W2[nn * 128 + t] * S.dZ[nn];
            S.dH1[t] = a * dact(S.H1p[t]);
        }
        __syncthreads();
        // dW1[ch][k] += sum_s dH1[s*16+ch] Xq[s*64+k]; db1
        for (int e = t; e < 16 * 64; e += NTT) {
            const int ch = e >> 6, k = e & 63;
            float a = 0.0f;
            for (int s = 0; s < 8; s++) a += S.dH1[s * 16 + ch] * S.Xq[s * 64 + k];
            G1[e] += a;
        }
        if (t < 16) {
            float a = 0.0f;
            for (int s = 0; s < 8; s++) a += S.dH1[s * 16 + t];
            Gb1[t] += a;
        }
        __syncthreads();
    }
    for (int i = t; i < NPARAM; i += NTT) atomicAdd(&grad[i], S.G[i]);
    for (int o = 16; o; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane == 0) S.red[t >> 5] = lsum;
    __syncthreads();
    if (t == 0) {
        float a = 0.0f;
        for (int w = 0; w < NTT / 32; w++) a += S.red[w];
        atomicAdd(loss, a * inv_count);
    }
}

// Adam on the FP32 master weights, then the BF16 copy; the gradient is cleared for the next step.
__global__ void k_adam(int n, float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                       float *__restrict__ grad, bf16 *__restrict__ wb, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    wb[i] = __float2bfloat16_rn(wi);
    grad[i] = 0.0f;
}

__global__ void k_to_bf16(int n, const float *__restrict__ w, bf16 *__restrict__ wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) wb[i] = __float2bfloat16_rn(w[i]);
}

// ---- host object ------------------------------------------------------------------------------------
struct Codec {
    float *w = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *loss = nullptr;
    bf16 *wb = nullptr;
    long step = 0;
    int device = 0;
    int grid_enc = 0, grid_dec = 0, grid_train = 0;
    int engine = 0;  // 0: mma.sync, 1: tcgen05 (UMMA, tensor memory), 2: encode mma.sync, decode tcgen05
    int grid_enc_u = 0, grid_dec_u = 0;
};

Dims dims(long nx, long ny, long nz) {
    Dims d;
    d.nx = (int)nx;
    d.ny = (int)ny;
    d.nz = (int)nz;
    d.nsx = (int)((nx + SX - 1) / SX);
    d.nsy = (int)((ny + SY - 1) / SY);
    d.nsz = (int)((nz + SZ - 1) / SZ);
    d.nbx = (int)((nx + 7) / 8);
    d.nby = (int)((ny + 7) / 8);
    d.nbz = (int)((nz + 7) / 8);
    return d;
}

long nblocks(long nx, long ny, long nz) { return ((nx + 7) / 8) * ((ny + 7) / 8) * ((nz + 7) / 8); }

// code buffer of one field, each part 256-byte aligned: ctl (4 ints + 2048 histogram bins),
// scales [nb] FP32, error energies [nb] FP32, raw slots' block ids [cap] int, codes [nb][32] BF16,
// raw blocks [cap][512] FP32; cap = 1 % of the blocks (at least 1)
long raw_cap(long nb) { return nb / 100 > 1 ? nb / 100 : 1; }
size_t al(size_t b) { return (b + 255) / 256 * 256; }
struct Layout {
    size_t ctl, hist, scale, err, raw_id, lat, raw, total;
};
Layout layout(long nb) {
    Layout L;
    const long cap = raw_cap(nb);
    L.ctl = 0;
    L.hist = 16;
    L.scale = al(16 + 2048 * 4);
    L.err = L.scale + al((size_t)nb * 4);
    L.raw_id = L.err + al((size_t)nb * 4);
    L.lat = L.raw_id + al((size_t)cap * 4);
    L.raw = L.lat + al((size_t)nb * 64);
    L.total = L.raw + (size_t)cap * 2048;
    return L;
}
size_t latent_bytes(long nx, long ny, long nz) { return layout(nblocks(nx, ny, nz)).total; }

void init_weights(std::vector<float> &w, unsigned seed) {
    std::mt19937 rng(seed);
    w.assign(NPARAM, 0.0f);
    auto fill = [&](int off, int nout, int nin) {
        const float a = std::sqrt(6.0f / (float)(nin + nout));
        std::uniform_real_distribution<float> u(-a, a);
        for (int i = 0; i < nout * nin; i++) w[off + i] = u(rng);
    };
    fill(OFF_W1, 16, 64);
    fill(OFF_W2, 32, 128);
    fill(OFF_W3, 128, 32);
    fill(OFF_W4, 64, 16);
}

bool valid_dims(long nx, long ny, long nz) {
    return nx > 0 && ny > 0 && nz > 0 && nx < (1L << 30) && ny < (1L << 30) && nz < (1L << 30);
}

}  // namespace codec
}  // namespace wfd

using wfd::codec::Codec;

namespace {
Codec *C(void *p) { return reinterpret_cast<Codec *>(p); }

int cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return WFD_OK;
    wfd::set_global_error(WFD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return WFD_ERR_CUDA;
}
}  // namespace

extern "C" long WFD_Codec_NumParams(void) { return wfd::codec::NPARAM; }

extern "C" long WFD_Codec_LatentBytes(long nx, long ny, long nz) {
    if (!wfd::codec::valid_dims(nx, ny, nz)) return -1;
    return (long)wfd::codec::latent_bytes(nx, ny, nz);
}

extern "C" void *WFD_Codec_Create(unsigned seed) {
    using namespace wfd::codec;
    Codec *c = new Codec();
    cudaGetDevice(&c->device);
    const size_t nb = sizeof(float) * NPARAM;
    bool ok = wfd::dMalloc(&c->w, nb) == cudaSuccess && wfd::dMalloc(&c->m, nb) == cudaSuccess &&
              wfd::dMalloc(&c->v, nb) == cudaSuccess && wfd::dMalloc(&c->grad, nb) == cudaSuccess &&
              wfd::dMalloc(&c->loss, sizeof(float)) == cudaSuccess &&
              wfd::dMalloc(&c->wb, sizeof(bf16) * NPARAM) == cudaSuccess;
    if (!ok) {
        wfd::set_global_error(WFD_ERR_ALLOC, "WFD_Codec_Create: device allocation failed");
        cudaFree(c->w), cudaFree(c->m), cudaFree(c->v), cudaFree(c->grad), cudaFree(c->loss), cudaFree(c->wb);
        delete c;
        return nullptr;
    }
    std::vector<float> w;
    init_weights(w, seed);
    cudaMemcpy(c->w, w.data(), nb, cudaMemcpyHostToDevice);
    cudaMemset(c->m, 0, nb);
    cudaMemset(c->v, 0, nb);
    cudaMemset(c->grad, 0, nb);
    k_to_bf16<<<(NPARAM + 255) / 256, 256>>>(NPARAM, c->w, c->wb);
    cudaFuncSetAttribute(k_encode, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ENC_SMEM);
    cudaFuncSetAttribute(k_decode, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DEC_SMEM);
    cudaFuncSetAttribute(k_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TrainSmem));
    int sms = 0, pe = 0, pd = 0, pt = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pe, k_encode, NTC, ENC_SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pd, k_decode, NTC, DEC_SMEM);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pt, k_train, NTT, sizeof(TrainSmem));
    c->grid_enc = sms * (pe > 0 ? pe : 1);
    c->grid_dec = sms * (pd > 0 ? pd : 1);
    c->grid_train = sms * (pt > 0 ? pt : 1);
    // tcgen05 encode/decode: each CTA holds 64 tensor-memory columns, so up to 8 CTAs per SM fit the
    // 512 columns; shared memory allows 2 encode and 4 decode CTAs
    int peu = 0, pdu = 0;
    const bool umma_ok =
        cudaFuncSetAttribute(k_encode_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, umma_layout::E_BYTES) ==
            cudaSuccess &&
        cudaFuncSetAttribute(k_decode_umma, cudaFuncAttributeMaxDynamicSharedMemorySize, umma_layout::D_BYTES) ==
            cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&peu, k_encode_umma, NTC, umma_layout::E_BYTES) == cudaSuccess &&
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pdu, k_decode_umma, NTC, umma_layout::D_BYTES) == cudaSuccess &&
        peu > 0 && pdu > 0;
    // CTAs per SM from the kernels' own resource use (shared memory, registers, and 64 of the 512
    // tensor-memory columns each), where that exceeds the occupancy query's answer (which returned 1
    // per SM for these kernels on a B200 where ncu reports 4 decode CTAs fitting); a grid larger than
    // what fits only runs in more waves, the CTAs never wait on one another
    auto fit = [&](const void *kern, int bytes) {
        cudaFuncAttributes a{};
        int smem_sm = 0, regs_sm = 0;
        if (cudaFuncGetAttributes(&a, kern) != cudaSuccess) return 1;
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->device);
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, c->device);
        const int by_smem = smem_sm / (bytes + (int)a.sharedSizeBytes + 1024);
        const int by_regs = a.numRegs > 0 ? regs_sm / (a.numRegs * NTC) : 1;
        int n = by_smem < by_regs ? by_smem : by_regs;
        n = n < 512 / umma_layout::TMEM_COLS ? n : 512 / umma_layout::TMEM_COLS;
        return n > 0 ? n : 1;
    };
    if (umma_ok) {
        const int fe = fit((const void *)k_encode_umma, umma_layout::E_BYTES);
        const int fd = fit((const void *)k_decode_umma, umma_layout::D_BYTES);
        peu = peu > fe ? peu : fe;
        pdu = pdu > fd ? pdu : fd;
    }
    c->grid_enc_u = umma_ok ? sms * (peu < 8 ? peu : 8) : 0;
    c->grid_dec_u = umma_ok ? sms * (pdu < 8 ? pdu : 8) : 0;
    // default: encode on mma.sync, decode on tcgen05, the faster kernel of each direction as measured
    // at 512x512x400 (encode 0.28 against 0.34 ms: four dependent UMMA rounds per slab wait on their
    // completion, where the mma.sync kernel keeps each layer's operands in registers; decode 0.153
    // against 0.160 ms). WAVEFD_B200_CODEC=mma or =tcgen05 puts both directions on one engine.
    const char *eng = getenv("WAVEFD_B200_CODEC");
    c->engine = !umma_ok || (eng && strcmp(eng, "mma") == 0) ? 0 : (eng && strcmp(eng, "tcgen05") == 0 ? 1 : 2);
    if (cuda_status(cudaDeviceSynchronize(), "WFD_Codec_Create")) {
        WFD_Codec_Free(c);
        return nullptr;
    }
    return c;
}

extern "C" void WFD_Codec_Free(void *codec) {
    Codec *c = C(codec);
    if (!c) return;
    cudaDeviceSynchronize();
    cudaFree(c->w), cudaFree(c->m), cudaFree(c->v), cudaFree(c->grad), cudaFree(c->loss), cudaFree(c->wb);
    delete c;
}

extern "C" int WFD_Codec_SetWeights(void *codec, const float *w, long n) {
    using namespace wfd::codec;
    Codec *c = C(codec);
    if (!c || !w || n != NPARAM) return WFD_ERR_ARG;
    cudaMemcpy(c->w, w, sizeof(float) * NPARAM, cudaMemcpyHostToDevice);
    cudaMemset(c->m, 0, sizeof(float) * NPARAM);
    cudaMemset(c->v, 0, sizeof(float) * NPARAM);
    c->step = 0;
    k_to_bf16<<<(NPARAM + 255) / 256, 256>>>(NPARAM, c->w, c->wb);
    return cuda_status(cudaDeviceSynchronize(), "WFD_Codec_SetWeights");
}

extern "C" int WFD_Codec_GetWeights(void *codec, float *w, long n) {
    using namespace wfd::codec;
    Codec *c = C(codec);
    if (!c || !w || n != NPARAM) return WFD_ERR_ARG;
    return cuda_status(cudaMemcpy(w, c->w, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost), "WFD_Codec_GetWeights");
}

extern "C" int WFD_Codec_Encode(void *codec, const float *field, long nx, long ny, long nz, void *latent,
                                void *stream) {
    using namespace wfd::codec;
    Codec *c = C(codec);
    if (!c || !field || !latent || !valid_dims(nx, ny, nz)) return WFD_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Dims d = dims(nx, ny, nz);
    const long nb = nblocks(nx, ny, nz), cap = raw_cap(nb);
    const Layout L = layout(nb);
    char *base = reinterpret_cast<char *>(latent);
    int *ctl = reinterpret_cast<int *>(base + L.ctl);
    unsigned *hist = reinterpret_cast<unsigned *>(base + L.hist);
    float *scale = reinterpret_cast<float *>(base + L.scale), *err = reinterpret_cast<float *>(base + L.err);
    int *raw_id = reinterpret_cast<int *>(base + L.raw_id);
    bf16 *lat = reinterpret_cast<bf16 *>(base + L.lat);
    float *raw = reinterpret_cast<float *>(base + L.raw);
    const long nslab = (long)d.nsx * d.nsy * d.nsz;
    const int grid = (int)(nslab < c->grid_enc ? nslab : c->grid_enc);
    cudaMemsetAsync(base, 0, L.scale, st);  // ctl and histogram
    if (c->engine == 1)
        k_encode_umma<<<(int)(nslab < c->grid_enc_u ? nslab : c->grid_enc_u), NTC, umma_layout::E_BYTES, st>>>(
            d, field, c->wb, c->w, scale, err, lat);
    else
        k_encode<<<grid, NTC, ENC_SMEM, st>>>(d, field, c->wb, c->w, scale, err, lat);
    const int gb = (int)((nb + 255) / 256 < 1184 ? (nb + 255) / 256 : 1184);
    k_err_hist<<<gb, 256, 0, st>>>(nb, err, hist);
    k_err_threshold<<<1, 1024, 0, st>>>(hist, cap, ctl);
    k_err_pick<<<gb, 256, 0, st>>>(nb, err, cap, ctl, raw_id);
    k_raw_gather<<<(unsigned)(cap < 1184 ? cap : 1184), 128, 0, st>>>(d, field, ctl, cap, raw_id, raw);
    return cuda_status(cudaGetLastError(), "WFD_Codec_Encode");
}

extern "C" int WFD_Codec_Decode(void *codec, const void *latent, long nx, long ny, long nz, float *field,
                                void *stream) {
    using namespace wfd::codec;
    Codec *c = C(codec);
    if (!c || !field || !latent || !valid_dims(nx, ny, nz)) return WFD_ERR_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    const Dims d = dims(nx, ny, nz);
    const long nb = nblocks(nx, ny, nz), cap = raw_cap(nb);
    const Layout L = layout(nb);
    const char *base = reinterpret_cast<const char *>(latent);
    const int *ctl = reinterpret_cast<const int *>(base + L.ctl);
    const float *scale = reinterpret_cast<const float *>(base + L.scale);
    const int *raw_id = reinterpret_cast<const int *>(base + L.raw_id);
    const bf16 *lat = reinterpret_cast<const bf16 *>(base + L.lat);
    const float *raw = reinterpret_cast<const float *>(base + L.raw);
    const long nslab = (long)d.nsx * d.nsy * d.nsz;
    const int grid = (int)(nslab < c->grid_dec ? nslab : c->grid_dec);
    if (c->engine >= 1)
        k_decode_umma<<<(int)(nslab < c->grid_dec_u ? nslab : c->grid_dec_u), NTC, umma_layout::D_BYTES, st>>>(
            d, scale, lat, c->wb, c->w, field);
    else
        k_decode<<<grid, NTC, DEC_SMEM, st>>>(d, scale, lat, c->wb, c->w, field);
    k_raw_scatter<<<(unsigned)(cap < 1184 ? cap : 1184), 128, 0, st>>>(d, ctl, cap, raw_id, raw, field);
    return cuda_status(cudaGetLastError(), "WFD_Codec_Decode");
}

extern "C" int WFD_Codec_SetEngine(void *codec, int engine) {
    wfd::codec::Codec *c = C(codec);
    if (!c || engine < 0 || engine > 2) return WFD_ERR_ARG;
    if (engine >= 1 && (c->grid_enc_u == 0 || c->grid_dec_u == 0)) return WFD_ERR_UNSUPPORTED;
    c->engine = engine;
    return WFD_OK;
}

extern "C" int WFD_Codec_Engine(void *codec) { return codec ? C(codec)->engine : -1; }

extern "C" int WFD_Codec_Grid(void *codec, int kernel) {
    if (!codec) return -1;
    const wfd::codec::Codec *c = C(codec);
    switch (kernel) {
        case 0: return c->grid_enc;
        case 1: return c->grid_dec;
        case 2: return c->grid_enc_u;
        case 3: return c->grid_dec_u;
        default: return -1;
    }
}

extern "C" int WFD_Codec_Status(void *codec) {
    if (!codec) return WFD_ERR_ARG;
    if (cudaDeviceSynchronize() != cudaSuccess) return cuda_status(cudaGetLastError(), "WFD_Codec_Status");
    unsigned v = 0, z = 0;
    cudaMemcpyFromSymbol(&v, wfd::codec::d_codec_status, sizeof(v));
    if (v) {
        cudaMemcpyToSymbol(wfd::codec::d_codec_status, &z, sizeof(z));
        wfd::set_global_error(WFD_ERR_TIMEOUT, "codec: a tensor-core completion wait ran out");
        return WFD_ERR_TIMEOUT;
    }
    return WFD_OK;
}

extern "C" long WFD_Codec_RawBlocks(const void *latent, long nx, long ny, long nz) {
    using namespace wfd::codec;
    if (!latent || !valid_dims(nx, ny, nz)) return -1;
    int ctl[4] = {0, 0, 0, 0};
    if (cudaMemcpy(ctl, latent, sizeof(ctl), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    const long cap = raw_cap(nblocks(nx, ny, nz));
    return ctl[2] < cap ? ctl[2] : cap;
}

extern "C" int WFD_Codec_GatherBlocks(const float *field, long nx, long ny, long nz, const int *origins, long n,
                                      float *blocks, float *scales, void *stream) {
    if (!field || !origins || !blocks || n < 0 || !wfd::codec::valid_dims(nx, ny, nz)) return WFD_ERR_ARG;
    if (n == 0) return WFD_OK;
    wfd::codec::k_gather_blocks<<<(unsigned)n, 128, 0, (cudaStream_t)stream>>>((int)nx, (int)ny, (int)nz, field,
                                                                               origins, n, blocks, scales);
    return cuda_status(cudaGetLastError(), "WFD_Codec_GatherBlocks");
}

extern "C" int WFD_Codec_Gradient(void *codec, const float *blocks, long n, float *grad, float *loss) {
    using namespace wfd::codec;
    Codec *c = C(codec);
    if (!c || !blocks || n < 1 || !grad || !loss) return WFD_ERR_ARG;
    cudaMemset(c->grad, 0, sizeof(float) * NPARAM);
    cudaMemset(c->loss, 0, sizeof(float));
    const int grid = (int)(n < c->grid_train ? n : c->grid_train);
    k_train<<<grid, NTT, sizeof(TrainSmem)>>>(blocks, n, 1.0f / (float)(n * 512), c->wb, c->w, c->grad, c->loss);
    if (int rc = cuda_status(cudaDeviceSynchronize(), "WFD_Codec_Gradient")) return rc;
    cudaMemcpy(grad, c->grad, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost);
    cudaMemcpy(loss, c->loss, sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemset(c->grad, 0, sizeof(float) * NPARAM);
    return cuda_status(cudaGetLastError(), "WFD_Codec_Gradient");
}

extern "C" int WFD_Codec_TrainStep(void *codec, const float *blocks, long n, float lr, float *loss, void *stream) {
    using namespace wfd::codec;
    Codec *c = C(codec);
    if (!c || !blocks || n < 1 || lr <= 0.0f) return WFD_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    cudaMemsetAsync(c->loss, 0, sizeof(float), s);
    const int grid = (int)(n < c->grid_train ? n : c->grid_train);
    k_train<<<grid, NTT, sizeof(TrainSmem), s>>>(blocks, n, 1.0f / (float)(n * 512), c->wb, c->w, c->grad, c->loss);
    c->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)c->step), c2 = 1.0f - std::pow(b2, (float)c->step);
    k_adam<<<(NPARAM + 255) / 256, 256, 0, s>>>(NPARAM, c->w, c->m, c->v, c->grad, c->wb, lr, b1, b2, 1e-8f, c1, c2);
    if (loss) cudaMemcpyAsync(loss, c->loss, sizeof(float), cudaMemcpyDeviceToHost, s);
    return cuda_status(cudaGetLastError(), "WFD_Codec_TrainStep");
}
