// Fused single-sweep 3D Iso step with TMA-staged tiles (prop3DAcoIsoDenQ_DEO2_FDTD.h:247-261 in one
// kernel; 28 B/cell of HBM traffic: read pCur, pOld, V, B, Q; write pOld, pSpace).
//
// A CTA (128 threads) owns a (z,y) tile of 32 x 16 columns and sweeps a chunk of x planes. For each
// plane j one thread issues, D planes ahead, a group of TMA tile loads completed on one mbarrier:
//   pCur(j) with its halo (48 x 30 at z0-8, y0-7), pCur(j+7) (32 x 16),
//   B(j) with its halo (40 x 24 at z0-4, y0-4), B(j+3) (32 x 16), pOld(j), V(j), Q(j) (32 x 16).
// pCur and B are read twice (the second time from L2), which keeps the stage small enough for
// three CTAs per SM. A thread owns 4 consecutive z cells of one row (float4 shared-memory
// accesses) and keeps along x register queues of pCur and of the pass-1 x output, 8 planes each.
// At plane j, warps 0-1 form the pass-1 y output on the 24 halo-extended rows (3 rows per thread,
// sliding along y) and warps 2-3 the pass-1 z output on the 40 halo-extended columns; then every
// thread applies D- and the time update to its 4 cells and stores pOld and pSpace as float4.
// Tiles whose halo lies wholly inside the interior take a branch-free path.
// Persistent CTAs loop over (tile, x-chunk) items; a chunk starts with 14 warm-up planes that only
// fill the queues. Waits are bounded; on timeout the kernel records an error in a device status
// word and leaves. Requires nz % 4 == 0 (TMA row pitch); the caller falls back otherwise.
#include "wfd_kernels.h"
#include "wfd_tma.cuh"

namespace WFD_NS {
using namespace wfd;
using namespace wfd_dev;

namespace {

constexpr int TZ = 32;
constexpr int TY = 16;
constexpr int NT = 128;
constexpr int D = 2;       // prefetch distance in planes
constexpr int NS = D + 1;  // stages (and mbarriers)
constexpr int PZW = TZ + 16, PYH = TY + 14;
constexpr int BZW = TZ + 8, BYH = TY + 8;
constexpr int PH_ = PYH * PZW, BH_ = BYH * BZW, OS = TY * TZ;
constexpr int TYR = TY + 8;  // pass-1 y output rows y0-4 .. y0+19 (23 used)
constexpr int TZW = TZ + 8;  // pass-1 z output columns z0-4 .. z0+35 (39 used)
// stage layout (floats): P halo, B halo, P own (j+7), B own (j+3), pOld, V, Q
constexpr int S_PH = 0, S_BH = S_PH + PH_, S_PN = S_BH + BH_, S_BN = S_PN + OS, S_PO = S_BN + OS, S_V = S_PO + OS,
              S_Q = S_V + OS, STAGE = S_Q + OS;
constexpr unsigned GROUP_BYTES = 4u * STAGE;
constexpr int WARMUP = 14;
constexpr int OFF_TY = NS * STAGE;
constexpr int OFF_TZ = OFF_TY + TYR * TZ;
constexpr int OFF_BAR = OFF_TZ + TY * TZW;
constexpr size_t SMEM_BYTES = (size_t)OFF_BAR * 4 + NS * 8 + 16;
static_assert(OFF_BAR % 2 == 0, "mbarrier alignment");
static_assert((STAGE * 4) % 128 == 0 && (S_BH * 4) % 128 == 0 && (S_PN * 4) % 128 == 0, "TMA destination alignment");

__device__ unsigned int d_status;

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float at(const float4 &v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// D+ at the centre of an 8-sample window w[0..7] = f(k-3..k+4); D- with w[0..7] = f(k-4..k+3)
__device__ __forceinline__ float st8(const Grid &g, float w0, float w1, float w2, float w3, float w4, float w5,
                                     float w6, float w7) {
    return g.c1 * (-w3 + w4) + g.c2 * (-w2 + w5) + g.c3 * (-w1 + w6) + g.c4 * (-w0 + w7);
}

// pass-1 y/z outputs of the centre plane j into TYs/TZs
template <bool INTERIOR>
__device__ __forceinline__ void ext_stage(const Grid &g, const long j, const int z0, const int y0, const float *st,
                                          float *TYs, float *TZs) {
    const int tid = threadIdx.x;
    const float *Pc = st + S_PH;
    const float *Bc = st + S_BH;
    const bool xin = INTERIOR || (j >= 4 && j < g.nx - 4);
    if (tid < 64) {
        const int zq = tid & 7;
        const int r0 = (tid >> 3) * 3;  // rows r0..r0+2 of the 24 extended rows
        const int zz0 = z0 + 4 * zq;
        float4 w[10];
#pragma unroll
        for (int i = 0; i < 10; i++)  // row 30 would only feed the unused padding row 23
            w[i] = r0 + i < PYH ? ld4(Pc + (r0 + i) * PZW + 8 + 4 * zq) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int rr = 0; rr < 3; rr++) {
            const int r = r0 + rr;
            const int y = y0 - 4 + r;
            const bool ok = INTERIOR || (xin && y >= 4 && y < g.ny - 4);
            const float4 b = ld4(Bc + r * BZW + 4 + 4 * zq);
            float out[4];
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const int zz = zz0 + m;
                float t = 0.0f;
                // region 1, or free-surface rows 1..3 (row 0 holds B*0 = 0)
                if (INTERIOR || (ok && zz < g.nz - 4 && (zz >= 4 || (g.fs && zz > 0)))) {
                    const float s = st8(g, at(w[rr], m), at(w[rr + 1], m), at(w[rr + 2], m), at(w[rr + 3], m),
                                        at(w[rr + 4], m), at(w[rr + 5], m), at(w[rr + 6], m), at(w[rr + 7], m));
                    t = at(b, m) * (g.idy * s);
                }
                out[m] = t;
            }
            st4(TYs + r * TZ + 4 * zq, make_float4(out[0], out[1], out[2], out[3]));
        }
    } else {
        // 16 rows x 10 quads = 160 items over 64 threads
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int item = tid - 64 + 64 * k;
            if (item >= TY * (TZW / 4)) break;
            const int r = item / (TZW / 4);
            const int qi = item - r * (TZW / 4);
            const int y = y0 + r;
            const int zb = z0 - 4 + 4 * qi;  // first z of this quad
            const bool ok = INTERIOR || (xin && y >= 4 && y < g.ny - 4);
            const float *rowp = Pc + (r + 7) * PZW;
            const float4 a0 = ld4(rowp + 4 * qi), a1 = ld4(rowp + 4 * qi + 4), a2 = ld4(rowp + 4 * qi + 8);
            const float v[12] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w, a2.x, a2.y, a2.z, a2.w};
            const float4 b = ld4(Bc + (r + 4) * BZW + 4 * qi);
            float out[4];
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const int zz = zb + m;
                float t = 0.0f;
                if (INTERIOR || (ok && zz >= 0 && zz < g.nz - 4 && (zz >= 4 || g.fs))) {
                    float s;
                    if (INTERIOR || zz >= 3) {
                        s = st8(g, v[m + 1], v[m + 2], v[m + 3], v[m + 4], v[m + 5], v[m + 6], v[m + 7], v[m + 8]);
                    } else {
                        // antisymmetric image above the free surface, p[-j] = -p[j] (z0 == 0 here)
                        auto pm = [&](int jz) { return jz >= 0 ? rowp[jz + 8] : -rowp[-jz + 8]; };
                        s = st8(g, pm(zz - 3), pm(zz - 2), pm(zz - 1), pm(zz), pm(zz + 1), pm(zz + 2), pm(zz + 3),
                                pm(zz + 4));
                    }
                    t = at(b, m) * (g.idz * s);
                }
                out[m] = t;
            }
            st4(TZs + r * TZW + 4 * qi, make_float4(out[0], out[1], out[2], out[3]));
        }
    }
}

// D- in y and z, the time update and the stores of this thread's 4 cells
template <bool INTERIOR>
__device__ __forceinline__ void fin_stage(const Grid &g, const long j, const int z, const int y, const int zq,
                                          const int row, const float *sx, const float *pc, const float *st,
                                          const float *TYs, const float *TZs, float *po, float *ps) {
    const bool xin = INTERIOR || (j >= 4 && j < g.nx - 4);
    const bool yin = INTERIOR || (y >= 4 && y < g.ny - 4);
    const int o = row * TZ + 4 * zq;
    const float4 pold4 = ld4(st + S_PO + o), v4 = ld4(st + S_V + o), q4 = ld4(st + S_Q + o);
    const float4 b4 = ld4(st + S_BH + (4 + row) * BZW + 4 + 4 * zq);
    float4 ty[8];
#pragma unroll
    for (int i = 0; i < 8; i++) ty[i] = ld4(TYs + (row + i) * TZ + 4 * zq);
    const float *tzr = TZs + row * TZW;
    const float4 t0 = ld4(tzr + 4 * zq), t1 = ld4(tzr + 4 * zq + 4), t2 = ld4(tzr + 4 * zq + 8);
    const float w[12] = {t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w, t2.x, t2.y, t2.z, t2.w};
    float npo[4], nps[4];
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const int zz = z + m;
        const float pcv = pc[m];
        const float pov = at(pold4, m);
        const bool r1 = INTERIOR || (xin && yin && zz >= 4 && zz < g.nz - 4);
        const bool r2 = !INTERIOR && xin && yin && g.fs && zz < 4 && zz < g.nz - 4;
        if (!r1 && !r2) {
            npo[m] = pov;  // not updated
            nps[m] = 0.0f;
            continue;
        }
        float L;
        if (!INTERIOR && r2 && zz == 0) {
            L = 0.0f + 0.0f + 0.0f;
        } else {
            const float sy = st8(g, at(ty[0], m), at(ty[1], m), at(ty[2], m), at(ty[3], m), at(ty[4], m),
                                 at(ty[5], m), at(ty[6], m), at(ty[7], m));
            float sz;
            if (INTERIOR || zz >= 4) {
                sz = st8(g, w[m], w[m + 1], w[m + 2], w[m + 3], w[m + 4], w[m + 5], w[m + 6], w[m + 7]);
            } else {
                // symmetric image above the free surface, t[-j] = t[j-1] (z0 == 0: column of z is z+4)
                auto tm = [&](int jz) { return tzr[(jz >= 0 ? jz : -jz - 1) + 4]; };
                sz = st8(g, tm(zz - 4), tm(zz - 3), tm(zz - 2), tm(zz - 1), tm(zz), tm(zz + 1), tm(zz + 2),
                         tm(zz + 3));
            }
            const float dx = g.idx * sx[m];
            const float dy = g.idy * sy;
            const float dz = g.idz * sz;
            L = dx + dy + dz;
        }
        const float V = at(v4, m);
        const float dt2V2_B = g.dt2 * V * V / at(b4, m);
        npo[m] = dt2V2_B * L - at(q4, m) * (pcv - pov) - pov + 2 * pcv;
        nps[m] = L;
    }
    const long k = j * g.sx + (long)y * g.nz + z;
    st4(po + k, make_float4(npo[0], npo[1], npo[2], npo[3]));
    st4(ps + k, make_float4(nps[0], nps[1], nps[2], nps[3]));
}

__global__ void __launch_bounds__(NT, 3)
    k_iso3d_tma(Grid g, Fields F, const __grid_constant__ CUtensorMap mPH, const __grid_constant__ CUtensorMap mPN,
                const __grid_constant__ CUtensorMap mBH, const __grid_constant__ CUtensorMap mBN,
                const __grid_constant__ CUtensorMap mPO, const __grid_constant__ CUtensorMap mV,
                const __grid_constant__ CUtensorMap mQ, int ntz, int nty, int nch, int xchunk) {
    extern __shared__ __align__(1024) float sm[];
    float *TYs = sm + OFF_TY;
    float *TZs = sm + OFF_TZ;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + OFF_BAR);
    int *abort_flag = reinterpret_cast<int *>(bars + NS);

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    if (tid == 0) {
        for (int s = 0; s < NS; s++) mbar_init(&bars[s], 1);
        fence_mbar_init();
        prefetch_tensor_map(&mPH);
        prefetch_tensor_map(&mPN);
        prefetch_tensor_map(&mBH);
        prefetch_tensor_map(&mBN);
        prefetch_tensor_map(&mPO);
        prefetch_tensor_map(&mV);
        prefetch_tensor_map(&mQ);
        *abort_flag = 0;
    }
    __syncthreads();

    const long total = (long)ntz * nty * nch;
    unsigned gseq = 0;                  // groups consumed so far by this CTA
    unsigned out_from = 0, out_to = 0;  // groups issued but not yet consumed (thread 0)
    const int zq = lane & 7;
    const int row = 4 * warp + (lane >> 3);

    for (long w = blockIdx.x; w < total; w += gridDim.x) {
        const int tzi = (int)(w % ntz);
        const int tyi = (int)((w / ntz) % nty);
        const int chi = (int)(w / ((long)ntz * nty));
        const int z0 = tzi * TZ;
        const int y0 = tyi * TY;
        const int z = z0 + 4 * zq;
        const int y = y0 + row;
        const bool own = z < g.nz && y < g.ny;
        const bool yin = y >= 4 && y < g.ny - 4;
        const long xbeg = (long)chi * xchunk;
        const long xend = xbeg + xchunk < g.nx ? xbeg + xchunk : g.nx;
        const long jstart = xbeg - WARMUP;
        const int ngroups = (int)(xend - jstart);
        // the tile and its halo of extended rows/columns lie inside [4, n-4) in y and z
        const bool tile_inner = z0 - 4 >= 4 && z0 + TZ + 4 <= g.nz - 4 && y0 - 4 >= 4 && y0 + TY + 4 <= g.ny - 4;

        auto issue = [&](long jj, unsigned gs) {
            uint64_t *bar = &bars[gs % NS];
            float *s = sm + (gs % NS) * STAGE;
            mbar_expect_tx(bar, GROUP_BYTES);
            tma_load_3d(s + S_PH, &mPH, bar, z0 - 8, y0 - 7, (int)jj);
            tma_load_3d(s + S_BH, &mBH, bar, z0 - 4, y0 - 4, (int)jj);
            tma_load_3d(s + S_PN, &mPN, bar, z0, y0, (int)(jj + 7));
            tma_load_3d(s + S_BN, &mBN, bar, z0, y0, (int)(jj + 3));
            tma_load_3d(s + S_PO, &mPO, bar, z0, y0, (int)jj);
            tma_load_3d(s + S_V, &mV, bar, z0, y0, (int)jj);
            tma_load_3d(s + S_Q, &mQ, bar, z0, y0, (int)jj);
        };
        if (tid == 0) {
            for (int q = 0; q < D && q < ngroups; q++) issue(jstart + q, gseq + q);
            out_from = gseq;
            out_to = gseq + (D < ngroups ? D : ngroups);
        }
        // queues: qp[i] = pCur(j+i), qt[i] = pass-1 x output at plane j-4+i
        float qp[8][4], qt[8][4];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int m = 0; m < 4; m++) {
                qp[i][m] = 0.0f;
                qt[i][m] = 0.0f;
            }

        bool stop = false;
        for (int q = 0; q < ngroups; q++) {
            const long j = jstart + q;
            const unsigned gs = gseq + q;
            if (tid == 0 && q + D < ngroups) {
                issue(j + D, gs + D);
                out_to = gs + D + 1;
            }
            if (!mbar_wait(&bars[gs % NS], (gs / NS) & 1u)) {
                atomicExch(abort_flag, 1);
                atomicOr(&d_status, 1u);
            }
            if (tid == 0) out_from = gs + 1;
            const float *st = sm + (gs % NS) * STAGE;
            // ---- queues: newest pCur plane j+7, pass-1 x output at plane j+3 -----------------------
            {
                const int o = row * TZ + 4 * zq;
                const float4 pn = ld4(st + S_PN + o);
                const float4 bn = ld4(st + S_BN + o);
#pragma unroll
                for (int i = 0; i < 7; i++)
#pragma unroll
                    for (int m = 0; m < 4; m++) qp[i][m] = qp[i + 1][m];
                qp[7][0] = pn.x;
                qp[7][1] = pn.y;
                qp[7][2] = pn.z;
                qp[7][3] = pn.w;
                const long xa = j + 3;
                const bool xin = xa >= 4 && xa < g.nx - 4;
#pragma unroll
                for (int i = 0; i < 7; i++)
#pragma unroll
                    for (int m = 0; m < 4; m++) qt[i][m] = qt[i + 1][m];
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    const int zz = z + m;
                    float t = 0.0f;
                    if (xin && yin && zz < g.nz - 4 && (zz >= 4 || (g.fs && zz > 0))) {
                        const float s = st8(g, qp[0][m], qp[1][m], qp[2][m], qp[3][m], qp[4][m], qp[5][m], qp[6][m],
                                            qp[7][m]);
                        t = at(bn, m) * (g.idx * s);
                    }
                    qt[7][m] = t;
                }
            }
            if (j >= xbeg) {
                const bool inner = tile_inner && j >= 4 && j < g.nx - 4;
                if (inner) ext_stage<true>(g, j, z0, y0, st, TYs, TZs);
                else ext_stage<false>(g, j, z0, y0, st, TYs, TZs);
                __syncthreads();
                if (own) {
                    float sx[4], pc[4];
#pragma unroll
                    for (int m = 0; m < 4; m++) {
                        sx[m] = st8(g, qt[0][m], qt[1][m], qt[2][m], qt[3][m], qt[4][m], qt[5][m], qt[6][m], qt[7][m]);
                        pc[m] = qp[0][m];
                    }
                    if (inner) fin_stage<true>(g, j, z, y, zq, row, sx, pc, st, TYs, TZs, F.pold, F.pspace);
                    else fin_stage<false>(g, j, z, y, zq, row, sx, pc, st, TYs, TZs, F.pold, F.pspace);
                }
            }
            __syncthreads();
            if (*abort_flag) {
                stop = true;
                break;
            }
        }
        gseq += ngroups;
        if (stop) break;
    }
    if (*abort_flag && tid == 0) {
        // let copies still in flight land before the CTA leaves (bounded)
        for (unsigned gs = out_from; gs < out_to; gs++) mbar_wait(&bars[gs % NS], (gs / NS) & 1u, 100000000ull);
    }
}

}  // namespace

bool fused_iso3d_tma(const Grid &g, const Fields &F, cudaStream_t s) {
    if (g.nz % 4 != 0) return false;
    CUtensorMap mPH, mPN, mBH, mBN, mPO, mV, mQ;
    if (!make_tensor_map_3d(&mPH, F.pcur, g.nx, g.ny, g.nz, PZW, PYH, 1)) return false;
    if (!make_tensor_map_3d(&mPN, F.pcur, g.nx, g.ny, g.nz, TZ, TY, 1)) return false;
    if (!make_tensor_map_3d(&mBH, F.b, g.nx, g.ny, g.nz, BZW, BYH, 1)) return false;
    if (!make_tensor_map_3d(&mBN, F.b, g.nx, g.ny, g.nz, TZ, TY, 1)) return false;
    if (!make_tensor_map_3d(&mPO, F.pold, g.nx, g.ny, g.nz, TZ, TY, 1)) return false;
    if (!make_tensor_map_3d(&mV, F.v, g.nx, g.ny, g.nz, TZ, TY, 1)) return false;
    if (!make_tensor_map_3d(&mQ, F.q, g.nx, g.ny, g.nz, TZ, TY, 1)) return false;
    static int grid_cap = 0;
    if (!grid_cap) {
        cudaFuncSetAttribute(k_iso3d_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_iso3d_tma, NT, SMEM_BYTES);
        grid_cap = sms * (per > 0 ? per : 1);
    }
    const int ntz = (int)((g.nz + TZ - 1) / TZ);
    const int nty = (int)((g.ny + TY - 1) / TY);
    // x-chunking: balance the last wave of persistent CTAs against the warm-up planes per chunk
    const long tiles = (long)ntz * nty;
    int best_nch = 1;
    double best_cost = 1e30;
    for (int nch = 1; nch <= 64 && nch <= g.nx / 16 + 1; nch++) {
        const long chunk = (g.nx + nch - 1) / nch;
        const long items = tiles * nch;
        const double waves = (double)((items + grid_cap - 1) / grid_cap);
        const double cost = waves * (double)(chunk + WARMUP * 0.35);
        if (cost < best_cost) {
            best_cost = cost;
            best_nch = nch;
        }
    }
    const int xchunk = (int)((g.nx + best_nch - 1) / best_nch);
    const int nch = (int)((g.nx + xchunk - 1) / xchunk);
    const long work = tiles * nch;
    const int grid = (int)(work < grid_cap ? work : grid_cap);
    k_iso3d_tma<<<grid, NT, SMEM_BYTES, s>>>(g, F, mPH, mPN, mBH, mBN, mPO, mV, mQ, ntz, nty, nch, xchunk);
    return true;
}

unsigned fused_status_and_clear() {
    unsigned v = 0, z = 0;
    cudaMemcpyFromSymbol(&v, d_status, sizeof(v));
    if (v) cudaMemcpyToSymbol(d_status, &z, sizeof(z));
    return v;
}

}  // namespace WFD_NS
