// The codec's encode and decode on the tcgen05 tensor cores (included by wfd_codec.cu inside
// namespace wfd::codec, after the slab helpers). Same network, same slabs (32 x 32 x 8 cells = 16
// blocks of 8^3 = 128 sub-blocks of 4^3), same BF16 roundings as the mma.sync kernels; the four
// layers become four single-CTA UMMA rounds with M = 128 and the accumulators in tensor memory:
//   E1  D[sub-block r][channel]     = A1[r][cell] . W1[channel][cell]          M 128, N 16, K 64
//   E2  D[block b][latent]          = A2[b][s*16+ch] . W2[latent][s*16+ch]     M 128 (16 rows used), N 32, K 128
//   D1  D[s*16+ch][block b]         = W3[s*16+ch][latent] . L[b][latent]       M 128, N 16, K 32
//   D2  D[sub-block r][cell]        = A4[r][channel] . W4[cell][channel]       M 128, N 64, K 16
// (D1 is computed transposed so that its M is the 128 outputs rather than the 16 blocks.) E2 has
// only 16 rows: the descriptor's row-group stride (SBO) is smaller than its K stride (LBO), so the
// 112 unused rows read bytes of the same 6 KB buffer and their outputs are never loaded.
// Operands are written by the threads in the no-swizzle K-major core-matrix layout (wfd_umma.cuh);
// one thread (thread 0) issues the MMAs and commits them to an mbarrier, every thread waits for it
// (bounded) and reads its accumulator lane back with tcgen05.ld. Each CTA holds 64 tensor-memory
// columns (the four rounds reuse them).

__device__ unsigned d_codec_status;

namespace umma_layout {
// byte offsets in dynamic shared memory (every buffer 128-byte aligned)
constexpr int E_SLABS = 0;                      // 2 x SLAB floats
constexpr int E_A1 = E_SLABS + 2 * SLAB * 4;    // [128 rows][64] bf16: LBO 128, SBO 1024
constexpr int E_A2 = E_A1 + 16384;              // [16 rows][128] bf16: LBO 256, SBO 128 (+2 KB read by unused rows)
constexpr int E_LAT = E_A2 + 6144;              // B of D1: [16 blocks][32] bf16: LBO 128, SBO 512
constexpr int E_A4 = E_LAT + 1024;              // [128 rows][16] bf16: LBO 128, SBO 256
constexpr int E_W1 = E_A4 + 4096;               // B of E1: [16][64]: LBO 128, SBO 1024
constexpr int E_W2 = E_W1 + 2048;               // B of E2: [32][128]: LBO 128, SBO 2048
constexpr int E_W3 = E_W2 + 8192;               // A of D1: [128][32]: LBO 128, SBO 512
constexpr int E_W4 = E_W3 + 8192;               // B of D2: [64][16]: LBO 128, SBO 256
constexpr int E_F = E_W4 + 2048;                // floats: scale 16, inv 16, err 16, b1 16, b2 32, b3 128, b4 64
constexpr int E_BAR = E_F + 288 * 4;            // mbarrier (8 B) + tensor-memory address (4 B)
constexpr int E_BYTES = E_BAR + 16;

constexpr int D_SLAB = 0;                       // SLAB floats
constexpr int D_LAT = D_SLAB + SLAB * 4;
constexpr int D_A4 = D_LAT + 1024;
constexpr int D_W3 = D_A4 + 4096;
constexpr int D_W4 = D_W3 + 8192;
constexpr int D_F = D_W4 + 2048;                // floats: scale 16, b3 128, b4 64
constexpr int D_BAR = D_F + 208 * 4;
constexpr int D_BYTES = D_BAR + 16;

static_assert(E_A1 % 128 == 0 && E_A2 % 128 == 0 && E_LAT % 128 == 0 && E_A4 % 128 == 0 && E_W1 % 128 == 0 &&
                  E_W2 % 128 == 0 && E_W3 % 128 == 0 && E_W4 % 128 == 0 && E_F % 128 == 0 && E_BAR % 8 == 0,
              "operand alignment");
static_assert(D_LAT % 128 == 0 && D_A4 % 128 == 0 && D_W3 % 128 == 0 && D_W4 % 128 == 0 && D_BAR % 8 == 0,
              "operand alignment");
static_assert(E_BYTES <= 114 * 1024, "two encode CTAs per SM");
static_assert(D_BYTES <= 56 * 1024, "four decode CTAs per SM");

// byte offset of element (row, k) in a K-major no-swizzle operand
__host__ __device__ constexpr int kmaj(int row, int k, int lbo, int sbo) {
    return (row >> 3) * sbo + (k >> 3) * lbo + (row & 7) * 16 + (k & 7) * 2;
}
constexpr int TMEM_COLS = 64;

// Last byte an MMA's operand descriptor reads (rows / 8 row groups, two core matrices along K):
// every MMA below stays inside its buffer.
constexpr int desc_end(int start, int rows, int lbo, int sbo) { return start + (rows / 8 - 1) * sbo + lbo + 127; }
static_assert(desc_end(E_A1 + 3 * 256, 128, 128, 1024) < E_A1 + 16384, "E1 A");
static_assert(desc_end(E_W1 + 3 * 256, 16, 128, 1024) < E_W1 + 2048, "E1 B");
static_assert(desc_end(E_A2 + 7 * 512, 128, 256, 128) < E_A2 + 6144, "E2 A (128 rows read, 16 used)");
static_assert(desc_end(E_W2 + 7 * 256, 32, 128, 2048) < E_W2 + 8192, "E2 B");
static_assert(desc_end(E_W3 + 256, 128, 128, 512) < E_W3 + 8192, "D1 A");
static_assert(desc_end(E_LAT + 256, 16, 128, 512) < E_LAT + 1024, "D1 B");
static_assert(desc_end(E_A4, 128, 128, 256) < E_A4 + 4096, "D2 A");
static_assert(desc_end(E_W4, 64, 128, 256) < E_W4 + 2048, "D2 B");
static_assert(desc_end(D_W3 + 256, 128, 128, 512) < D_W3 + 8192, "D1 A");
static_assert(desc_end(D_LAT + 256, 16, 128, 512) < D_LAT + 1024, "D1 B");
static_assert(desc_end(D_A4, 128, 128, 256) < D_A4 + 4096, "D2 A");
static_assert(desc_end(D_W4, 64, 128, 256) < D_W4 + 2048, "D2 B");
// and the threads' writes: the last element of each operand
static_assert(kmaj(127, 63, 128, 1024) + 2 <= 16384 && kmaj(15, 127, 256, 128) + 2 <= 4096 &&
                  kmaj(15, 31, 128, 512) + 2 <= 1024 && kmaj(127, 15, 128, 256) + 2 <= 4096 &&
                  kmaj(15, 63, 128, 1024) + 2 <= 2048 && kmaj(31, 127, 128, 2048) + 2 <= 8192 &&
                  kmaj(127, 31, 128, 512) + 2 <= 8192 && kmaj(63, 15, 128, 256) + 2 <= 2048,
              "operand writes");
}  // namespace umma_layout

// weights into their operand layouts (bf16), biases into shared memory
__device__ __forceinline__ void umma_load_weights(char *sm, const bf16 *__restrict__ wb, const float *__restrict__ wp,
                                                  bool encoder, int w1, int w2, int w3, int w4, float *b1, float *b2,
                                                  float *b3, float *b4) {
    using namespace umma_layout;
    const int tid = threadIdx.x;
    if (encoder) {
        for (int i = tid; i < 16 * 64; i += NTC)
            *reinterpret_cast<bf16 *>(sm + w1 + kmaj(i / 64, i % 64, 128, 1024)) = wb[OFF_W1 + i];
        for (int i = tid; i < 32 * 128; i += NTC)
            *reinterpret_cast<bf16 *>(sm + w2 + kmaj(i / 128, i % 128, 128, 2048)) = wb[OFF_W2 + i];
        if (tid < 16) b1[tid] = wp[OFF_B1 + tid];
        if (tid < 32) b2[tid] = wp[OFF_B2 + tid];
    }
    for (int i = tid; i < 128 * 32; i += NTC)
        *reinterpret_cast<bf16 *>(sm + w3 + kmaj(i / 32, i % 32, 128, 512)) = wb[OFF_W3 + i];
    for (int i = tid; i < 64 * 16; i += NTC)
        *reinterpret_cast<bf16 *>(sm + w4 + kmaj(i / 16, i % 16, 128, 256)) = wb[OFF_W4 + i];
    for (int i = tid; i < 128; i += NTC) b3[i] = wp[OFF_B3 + i];
    if (tid < 64) b4[tid] = wp[OFF_B4 + tid];
}

// One UMMA round: operands written by the threads are fenced to the async proxy, thread 0 issues
// `issue()` and commits, every thread waits (bounded) for the commit's phase. Returns false, for
// every thread alike, when some thread's wait ran out (the status word then says so).
template <class F>
__device__ __forceinline__ bool umma_round(uint64_t *bar, unsigned &phase, F issue) {
    wfd_umma::fence_async_smem();
    wfd_umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
        wfd_umma::fence_after_sync();
        issue();
        wfd_umma::mma_commit(bar);
    }
    const bool ok = wfd_dev::mbar_wait(bar, phase);
    phase ^= 1u;
    const bool bad = __syncthreads_or(!ok) != 0;
    wfd_umma::fence_after_sync();
    if (bad && threadIdx.x == 0) atomicOr(&d_codec_status, 1u);
    return !bad;
}

// D1 (transposed) then D2 for the slab's 16 blocks whose BF16 latents sit in `lat` (B layout) and
// whose scales sit in `bscale`: thread r then hands the decoded cells of sub-block r (scaled back)
// to consume(q, v), 16 at a time (cells 16q .. 16q+15). Returns false when a wait ran out.
template <class Consume>
__device__ __forceinline__ bool umma_decode_slab(char *sm, int lat_off, int a4_off, int w3_off, int w4_off,
                                                 const float *b3, const float *b4, const float *bscale,
                                                 uint32_t tm, uint64_t *bar, unsigned &phase, Consume consume) {
    using namespace umma_layout;
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t sbase = wfd_umma::smem_addr(sm);
    const uint32_t tl = tm + ((uint32_t)(32 * warp) << 16);  // this warp's lane quarter
    // D1^T: lanes = outputs s*16+ch (128), columns = blocks (16), K = 32 latents
    if (!umma_round(bar, phase, [&] {
            for (int kk = 0; kk < 2; kk++)
                wfd_umma::mma_bf16(tm, wfd_umma::smem_desc(sbase + w3_off + kk * 256, 128, 512),
                                   wfd_umma::smem_desc(sbase + lat_off + kk * 256, 128, 512),
                                   wfd_umma::idesc_bf16(128, 16), kk > 0);
        }))
        return false;
    {
        float v[16];
        wfd_umma::tmem_ld16(tl, v);
        const int L = tid, s = L >> 4, ch = L & 15;
        const float bias = b3[L];
#pragma unroll
        for (int b = 0; b < 16; b++) {
            // sub-block row b*8+s, channel ch; even channels store the pair with their odd neighbour
            const float h = act(v[b] + bias);
            const float hn = __shfl_down_sync(0xffffffffu, h, 1);
            if ((ch & 1) == 0)
                *reinterpret_cast<uint32_t *>(sm + a4_off + kmaj(b * 8 + s, ch, 128, 256)) = pack2(h, hn);
        }
    }
    // D2: lanes = sub-blocks (128), columns = cells (64), K = 16 channels
    if (!umma_round(bar, phase, [&] {
            wfd_umma::mma_bf16(tm, wfd_umma::smem_desc(sbase + a4_off, 128, 256),
                               wfd_umma::smem_desc(sbase + w4_off, 128, 256), wfd_umma::idesc_bf16(128, 64), false);
        }))
        return false;
    const float sc = bscale[tid >> 3];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        float v[16];
        wfd_umma::tmem_ld16(tl + 16 * q, v);
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = (v[i] + b4[16 * q + i]) * sc;
        consume(q, v);
    }
    return true;
}

// ---- encode (tcgen05) -------------------------------------------------------------------------------
__global__ void __launch_bounds__(NTC, 2)
    k_encode_umma(Dims d, const float *__restrict__ f, const bf16 *__restrict__ wb, const float *__restrict__ wp,
                  float *__restrict__ scale_out, float *__restrict__ err_out, bf16 *__restrict__ lat_out) {
    using namespace umma_layout;
    extern __shared__ __align__(1024) char sm[];
    float *slabs = reinterpret_cast<float *>(sm + E_SLABS);
    float *fl = reinterpret_cast<float *>(sm + E_F);
    float *bscale = fl, *binv = fl + 16, *berr = fl + 32, *b1 = fl + 48, *b2 = fl + 64, *b3 = fl + 96,
          *b4 = fl + 224;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + E_BAR);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + E_BAR + 8);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t sbase = wfd_umma::smem_addr(sm);

    umma_load_weights(sm, wb, wp, true, E_W1, E_W2, E_W3, E_W4, b1, b2, b3, b4);
    for (int i = tid; i < 6144 / 16; i += NTC) reinterpret_cast<uint4 *>(sm + E_A2)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        wfd_dev::mbar_init(bar, 1);
        wfd_dev::fence_mbar_init();
    }
    if (warp == 0) wfd_umma::tmem_alloc(tslot, TMEM_COLS);
    wfd_umma::fence_before_sync();
    __syncthreads();
    wfd_umma::fence_after_sync();
    const uint32_t tm = *tslot;
    const uint32_t tl = tm + ((uint32_t)(32 * warp) << 16);
    unsigned phase = 0;

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
        {  // A1: sub-block r = tid, its 64 cells scaled by the block's 1/max, in chunks of 8 cells
            const int r = tid;
            const float inv = binv[r >> 3];
#pragma unroll
            for (int c = 0; c < 8; c++) {
                const float4 u = *reinterpret_cast<const float4 *>(slab + cell_off(r, 8 * c));
                const float4 v = *reinterpret_cast<const float4 *>(slab + cell_off(r, 8 * c + 4));
                uint4 q;
                q.x = pack2(u.x * inv, u.y * inv);
                q.y = pack2(u.z * inv, u.w * inv);
                q.z = pack2(v.x * inv, v.y * inv);
                q.w = pack2(v.z * inv, v.w * inv);
                *reinterpret_cast<uint4 *>(sm + E_A1 + kmaj(r, 8 * c, 128, 1024)) = q;
            }
        }
        // E1
        if (!umma_round(bar, phase, [&] {
                for (int kk = 0; kk < 4; kk++)
                    wfd_umma::mma_bf16(tm, wfd_umma::smem_desc(sbase + E_A1 + kk * 256, 128, 1024),
                                       wfd_umma::smem_desc(sbase + E_W1 + kk * 256, 128, 1024),
                                       wfd_umma::idesc_bf16(128, 16), kk > 0);
            }))
            break;
        {  // E1 epilogue: bias, leaky ReLU, BF16 into A2 row b = r/8, columns s*16 .. s*16+15
            float v[16];
            wfd_umma::tmem_ld16(tl, v);
            const int r = tid, b = r >> 3, s = r & 7;
            uint4 q0, q1;
            q0.x = pack2(act(v[0] + b1[0]), act(v[1] + b1[1]));
            q0.y = pack2(act(v[2] + b1[2]), act(v[3] + b1[3]));
            q0.z = pack2(act(v[4] + b1[4]), act(v[5] + b1[5]));
            q0.w = pack2(act(v[6] + b1[6]), act(v[7] + b1[7]));
            q1.x = pack2(act(v[8] + b1[8]), act(v[9] + b1[9]));
            q1.y = pack2(act(v[10] + b1[10]), act(v[11] + b1[11]));
            q1.z = pack2(act(v[12] + b1[12]), act(v[13] + b1[13]));
            q1.w = pack2(act(v[14] + b1[14]), act(v[15] + b1[15]));
            *reinterpret_cast<uint4 *>(sm + E_A2 + kmaj(b, 16 * s, 256, 128)) = q0;
            *reinterpret_cast<uint4 *>(sm + E_A2 + kmaj(b, 16 * s + 8, 256, 128)) = q1;
        }
        // E2 (rows 16..127 of the MMA are unused)
        if (!umma_round(bar, phase, [&] {
                for (int kk = 0; kk < 8; kk++)
                    wfd_umma::mma_bf16(tm, wfd_umma::smem_desc(sbase + E_A2 + kk * 512, 256, 128),
                                       wfd_umma::smem_desc(sbase + E_W2 + kk * 256, 128, 2048),
                                       wfd_umma::idesc_bf16(128, 32), kk > 0);
            }))
            break;
        if (warp == 0) {  // E2 epilogue: block b = lane (< 16): latent codes, to global memory and to D1's B
            float v0[16], v1[16];
            wfd_umma::tmem_ld16(tl, v0);
            wfd_umma::tmem_ld16(tl + 16, v1);
            if (lane < 16) {
                const int b = lane;
                uint32_t q[16];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    q[i] = pack2(v0[2 * i] + b2[2 * i], v0[2 * i + 1] + b2[2 * i + 1]);
                    q[8 + i] = pack2(v1[2 * i] + b2[16 + 2 * i], v1[2 * i + 1] + b2[16 + 2 * i + 1]);
                }
#pragma unroll
                for (int c = 0; c < 4; c++)
                    *reinterpret_cast<uint4 *>(sm + E_LAT + kmaj(b, 8 * c, 128, 512)) =
                        make_uint4(q[4 * c], q[4 * c + 1], q[4 * c + 2], q[4 * c + 3]);
                bool valid;
                const long id = block_id(d, xi, yi, zi, b, valid);
                if (valid) {
                    uint4 *dst = reinterpret_cast<uint4 *>(lat_out + id * 32);
#pragma unroll
                    for (int c = 0; c < 4; c++) dst[c] = make_uint4(q[4 * c], q[4 * c + 1], q[4 * c + 2], q[4 * c + 3]);
                }
            }
        }
        // decode in place and the error energy of every block (the slab is still in shared memory)
        float e = 0.0f;
        const bool ok = umma_decode_slab(sm, E_LAT, E_A4, E_W3, E_W4, b3, b4, bscale, tm, bar, phase,
                                         [&](int q, const float (&v)[16]) {
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const float4 x = *reinterpret_cast<const float4 *>(slab + cell_off(tid, 16 * q + 4 * c));
                const float d0 = v[4 * c] - x.x, d1 = v[4 * c + 1] - x.y, d2 = v[4 * c + 2] - x.z,
                            d3 = v[4 * c + 3] - x.w;
                e += d0 * d0 + d1 * d1 + d2 * d2 + d3 * d3;
            }
        });
        if (!ok) break;
        // the 8 sub-blocks of a block are 8 consecutive lanes (fixed-order reduction)
        e += __shfl_xor_sync(0xffffffffu, e, 1);
        e += __shfl_xor_sync(0xffffffffu, e, 2);
        e += __shfl_xor_sync(0xffffffffu, e, 4);
        if ((tid & 7) == 0) berr[tid >> 3] = e;
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
    // copies still in flight (a loop left early) land before the CTA ends
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    wfd_umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        wfd_umma::fence_after_sync();
        wfd_umma::tmem_dealloc(tm, TMEM_COLS);
    }
}

// ---- decode (tcgen05) -------------------------------------------------------------------------------
__global__ void __launch_bounds__(NTC, 4)
    k_decode_umma(Dims d, const float *__restrict__ scale_in, const bf16 *__restrict__ lat_in,
                  const bf16 *__restrict__ wb, const float *__restrict__ wp, float *__restrict__ f) {
    using namespace umma_layout;
    extern __shared__ __align__(1024) char sm[];
    float *slab = reinterpret_cast<float *>(sm + D_SLAB);
    float *fl = reinterpret_cast<float *>(sm + D_F);
    float *bscale = fl, *b3 = fl + 16, *b4 = fl + 144;
    uint64_t *bar = reinterpret_cast<uint64_t *>(sm + D_BAR);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + D_BAR + 8);
    const int tid = threadIdx.x, warp = tid >> 5;

    umma_load_weights(sm, wb, wp, false, 0, 0, D_W3, D_W4, nullptr, nullptr, b3, b4);
    if (tid == 0) {
        wfd_dev::mbar_init(bar, 1);
        wfd_dev::fence_mbar_init();
    }
    if (warp == 0) wfd_umma::tmem_alloc(tslot, TMEM_COLS);
    wfd_umma::fence_before_sync();
    __syncthreads();
    wfd_umma::fence_after_sync();
    const uint32_t tm = *tslot;
    unsigned phase = 0;

    const long nslab = (long)d.nsx * d.nsy * d.nsz;
    for (long sl = blockIdx.x; sl < nslab; sl += gridDim.x) {
        int xi, yi, zi;
        slab_of(d, sl, xi, yi, zi);
        __syncthreads();  // the previous slab's store has read the staging slab
        {  // latents (D1's B operand) and scales of the slab's 16 blocks, zero outside the grid
            const int b = tid >> 3, part = tid & 7;  // 8 threads x 4 latents per block
            bool v;
            const long id = block_id(d, xi, yi, zi, b, v);
            uint2 q = make_uint2(0u, 0u);
            if (v) q = *reinterpret_cast<const uint2 *>(lat_in + id * 32 + 4 * part);
            *reinterpret_cast<uint2 *>(sm + D_LAT + kmaj(b, 4 * part, 128, 512)) = q;
            if (part == 0) bscale[b] = v ? scale_in[id] : 0.0f;
        }
        const bool ok = umma_decode_slab(sm, D_LAT, D_A4, D_W3, D_W4, b3, b4, bscale, tm, bar, phase,
                                         [&](int q, const float (&v)[16]) {
#pragma unroll
                                             for (int c = 0; c < 4; c++)
                                                 *reinterpret_cast<float4 *>(slab + cell_off(tid, 16 * q + 4 * c)) =
                                                     make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
                                         });
        if (!ok) break;
        __syncthreads();
        store_slab(d, f, xi, yi, zi, slab);
    }
    wfd_umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        wfd_umma::fence_after_sync();
        wfd_umma::tmem_dealloc(tm, TMEM_COLS);
    }
}
