// Fused 2D VTI and TTI steps: both reference passes of prop2DAcoVTIDenQ_DEO2_FDTD (pass 1 D+ and the
// sandwich :771-779, pass 2 D- and the update with Q :992-1247, linear :1252-1480) and of
// prop2DAcoTTIDenQ_DEO2_FDTD (pass 1 with the rotation :672-760, pass 2 with the back-rotation inside
// the D- stencils :997-1135) in one launch. A 2D grid is small and L2-resident, so a step is bound
// by latency, not bandwidth: one kernel instead of two, and no scratch arrays in global memory.
//
// A CTA of 512 threads owns a tile of 16 (x) x 64 (z) cells. It loads pCur and mCur with 7 cells of
// halo on every side (the antisymmetric image above kz = 0) and the materials with 4, evaluates
// pass 1 on the tile extended by 4 cells before and 3 after on both axes (the TTI rotation needs
// both derivatives at every output, so the halo cells of both directions are evaluated; for VTI the
// same rectangle keeps one code path), then D- and the update on its cells. The D- z stencils read
// the symmetric image above the free surface by reflecting the column index (t[-j] = t[j-1], the
// weights of the TTI back-rotation with it). Cell arithmetic is the expression trees of the
// two-pass kernels (wfd_generic.cu), so the strict build gives their bits.
#include "wfd_gridbar.cuh"
#include "wfd_kernels.h"

namespace WFD_NS {
using namespace wfd;

namespace {

constexpr int TX = 16, TZ = 64, NT = 512;
constexpr int PXH = TX + 14, PZW = TZ + 14;  // pCur/mCur boxes: rows x0-7 .., columns z0-7 ..
constexpr int MXH = TX + 8, MZW = TZ + 8;    // material boxes: rows x0-4 .., columns z0-4 ..
constexpr int OXH = TX + 7, OZW = TZ + 7;    // pass-1 outputs: rows x0-4 .. x0+TX+2, columns z0-4 .. z0+TZ+2
constexpr int WZ = 32, WX = NT / WZ;
enum { MT2_B = 0, MT2_E, MT2_A, MT2_F, MT2_ST, MT2_CT };
constexpr int NMAT_MAX = 6;
// shared memory (floats): P, M boxes; materials; pass-1 outputs t0, t2 (P), t3, t5 (M)
constexpr int O_PM = 0;
constexpr int O_MAT = O_PM + 2 * PXH * PZW;
constexpr int O_OUT = O_MAT + NMAT_MAX * MXH * MZW;
constexpr int SMEM_FLOATS = O_OUT + 4 * OXH * OZW;
constexpr size_t SMEM_BYTES = (size_t)SMEM_FLOATS * 4;

__device__ __forceinline__ int region2(const Grid &g, long x, long z) {
    if (x < 4 || x >= g.nx - 4 || z >= g.nz - 4) return 0;
    if (z >= 4) return 1;
    return g.fs ? 2 : 0;
}

template <class W>
__device__ __forceinline__ float stp(const Grid &g, const W &w) {
    return g.c1 * (-w(0) + w(1)) + g.c2 * (-w(-1) + w(2)) + g.c3 * (-w(-2) + w(3)) + g.c4 * (-w(-3) + w(4));
}
template <class W>
__device__ __forceinline__ float stm(const Grid &g, const W &w) {
    return g.c1 * (-w(-1) + w(0)) + g.c2 * (-w(-2) + w(1)) + g.c3 * (-w(-3) + w(2)) + g.c4 * (-w(-4) + w(3));
}

// loads of the fields a step writes: past L1 in the whole-loop launch (other CTAs rewrite them
// between steps)
template <bool RUN>
__device__ __forceinline__ float ldf(const float *p) {
    return RUN ? __ldcg(p) : *p;
}

// One step of the tile at (x0, z0) (shared memory sm of SMEM_BYTES); in the whole-loop launch
// (RUN) also the step's source injection at time index it into the tile's cells of the new pCur,
// each group's contributions in order, separate IEEE multiply and add, as the injection kernel does.
// load_mat false: the material boxes are those of this tile from the step before.
template <int PHYS, bool LINEAR, bool RUN>
__device__ __forceinline__ void aniso_tile_step(const Grid &g, const Fields &F, const long x0, const long z0,
                                                float *sm, const long it, const bool load_mat = true) {
    float(*P)[PZW] = reinterpret_cast<float(*)[PZW]>(sm + O_PM);
    float(*Mf)[PZW] = reinterpret_cast<float(*)[PZW]>(sm + O_PM + PXH * PZW);
    auto mat = [&](int m) { return reinterpret_cast<float(*)[MZW]>(sm + O_MAT + m * MXH * MZW); };
    auto out = [&](int o) { return reinterpret_cast<float(*)[OZW]>(sm + O_OUT + o * OXH * OZW); };
    const int tz = threadIdx.x % WZ, tx = threadIdx.x / WZ;
    const long nx = g.nx, nz = g.nz;
    constexpr int nmat = PHYS == TTI ? 6 : 4;

    // pCur, mCur with the antisymmetric image above kz = 0 (zero outside the grid elsewhere)
    for (int r = tx; r < PXH; r += WX) {
        const long x = x0 - 7 + r;
        const bool xin = x >= 0 && x < nx;
        for (int c = tz; c < PZW; c += WZ) {
            const long z = z0 - 7 + c;
            float vp = 0.0f, vm = 0.0f;
            if (xin) {
                if (z >= 0 && z < nz) {
                    vp = ldf<RUN>(F.pcur + x * nz + z);
                    vm = ldf<RUN>(F.mcur + x * nz + z);
                } else if (z < 0 && -z < nz) {
                    vp = -ldf<RUN>(F.pcur + x * nz - z);
                    vm = -ldf<RUN>(F.mcur + x * nz - z);
                }
            }
            P[r][c] = vp;
            Mf[r][c] = vm;
        }
    }
    const float *msrc[NMAT_MAX] = {F.b, F.eps, F.eta, F.f, F.st, F.ct};
    for (int m = 0; m < nmat && load_mat; m++) {  // (already in shared memory when the tile stays)
        float(*Ms)[MZW] = mat(m);
        for (int r = tx; r < MXH; r += WX) {
            const long x = x0 - 4 + r;
            for (int c = tz; c < MZW; c += WZ) {
                const long z = z0 - 4 + c;
                Ms[r][c] = (x >= 0 && x < nx && z >= 0 && z < nz) ? msrc[m][x * nz + z] : 0.0f;
            }
        }
    }
    __syncthreads();

    // pass 1 on rows x0-4 .. x0+TX+2, columns z0-4 .. z0+TZ+2 (cells above kz = 0 are left zero:
    // the D- z stencils read their images)
    {
        float(*B_)[MZW] = mat(MT2_B);
        float(*E_)[MZW] = mat(MT2_E);
        float(*A_)[MZW] = mat(MT2_A);
        float(*F_)[MZW] = mat(MT2_F);
        float(*T0)[OZW] = out(0);
        float(*T2)[OZW] = out(1);
        float(*T3)[OZW] = out(2);
        float(*T5)[OZW] = out(3);
        for (int r = tx; r < OXH; r += WX) {
            const long x = x0 - 4 + r;
            for (int c = tz; c < OZW; c += WZ) {
                const long z = z0 - 4 + c;
                float o0 = 0.0f, o2 = 0.0f, o3 = 0.0f, o5 = 0.0f;
                const int reg = z >= 0 ? region2(g, x, z) : 0;
                if (reg) {
                    const int pr = r + 3, pc = c + 3;  // P/M box row and column of (x, z)
                    float dPx, dMx;
                    if (reg == 2 && z == 0) {
                        dPx = 0.0f;
                        dMx = 0.0f;
                    } else {
                        dPx = g.idx * stp(g, [&](int j) { return P[pr + j][pc]; });
                        dMx = g.idx * stp(g, [&](int j) { return Mf[pr + j][pc]; });
                    }
                    const float dPz = g.idz * stp(g, [&](int j) { return P[pr][pc + j]; });
                    const float dMz = g.idz * stp(g, [&](int j) { return Mf[pr][pc + j]; });
                    const int mr = r, mc = c;  // material box row and column of (x, z)
                    const float E = 1 + 2 * E_[mr][mc];
                    const float A = A_[mr][mc];
                    const float Fv = F_[mr][mc];
                    const float B = B_[mr][mc];
                    if (PHYS == VTI) {
                        // prop2DAcoVTIDenQ_DEO2_FDTD.h:771-779
                        o0 = B * E * dPx;
                        o2 = B * (1 - Fv * A * A) * dPz + B * Fv * A * sqrtf(1 - A * A) * dMz;
                        o3 = B * (1 - Fv) * dMx;
                        o5 = B * Fv * A * sqrtf(1 - A * A) * dPz + B * (1 - Fv + Fv * A * A) * dMz;
                    } else {
                        // prop2DAcoTTIDenQ_DEO2_FDTD.h:672-760
                        const float cosT = mat(MT2_CT)[mr][mc], sinT = mat(MT2_ST)[mr][mc];
                        const float dPG1 = cosT * dPx - sinT * dPz;
                        const float dPG3 = sinT * dPx + cosT * dPz;
                        const float dMG1 = cosT * dMx - sinT * dMz;
                        const float dMG3 = sinT * dMx + cosT * dMz;
                        o0 = B * E * dPG1;
                        o2 = B * (1 - Fv * A * A) * dPG3 + B * Fv * A * sqrtf(1 - A * A) * dMG3;
                        o3 = B * (1 - Fv) * dMG1;
                        o5 = B * Fv * A * sqrtf(1 - A * A) * dPG3 + B * (1 - Fv + Fv * A * A) * dMG3;
                    }
                }
                T0[r][c] = o0;
                T2[r][c] = o2;
                T3[r][c] = o3;
                T5[r][c] = o5;
            }
        }
    }
    __syncthreads();

    // pass 2: D-, the update with Q, pSpace/mSpace
    const bool top = z0 == 0 && g.fs;
    float(*T0)[OZW] = out(0);
    float(*T2)[OZW] = out(1);
    float(*T3)[OZW] = out(2);
    float(*T5)[OZW] = out(3);
    float(*ST)[MZW] = mat(MT2_ST);
    float(*CT)[MZW] = mat(MT2_CT);
    for (int r = tx; r < TX; r += WX) {
        for (int c = tz; c < TZ; c += WZ) {
            const long x = x0 + r, z = z0 + c;
            if (x >= nx || z >= nz) continue;
            const long k = x * nz + z;
            const int reg = region2(g, x, z);
            if (!reg) {
                if (!LINEAR) {
                    F.pspace[k] = 0.0f;
                    F.mspace[k] = 0.0f;
                }
                continue;
            }
            const int orow = r + 4, ocol = c + 4;  // output row and column of (x, z)
            // column of tap z+j in the output arrays: above the free surface the image t[-j] = t[j-1]
            auto zc = [&](int j) {
                const long zz = z + j;
                return (top && zz < 0) ? (int)(-zz - 1) + 4 : ocol + j;
            };
            float LP = 0.0f, LM = 0.0f;
            if (PHYS == VTI) {
                float dPx = 0.0f, dPz = 0.0f, dMx = 0.0f, dMz = 0.0f;
                if (!(reg == 2 && z == 0)) {
                    dPx = g.idx * stm(g, [&](int j) { return T0[orow + j][ocol]; });
                    dPz = g.idz * stm(g, [&](int j) { return T2[orow][zc(j)]; });
                    dMx = g.idx * stm(g, [&](int j) { return T3[orow + j][ocol]; });
                    dMz = g.idz * stm(g, [&](int j) { return T5[orow][zc(j)]; });
                }
                LP = dPx + dPz;
                LM = dMx + dMz;
            } else {
                float dPG1 = 0.0f, dPG3 = 0.0f, dMG1 = 0.0f, dMG3 = 0.0f;
                if (!(reg == 2 && z == 0)) {
                    // weights at the tap's own cell (mirrored with it above the free surface)
                    dPG1 = g.idx * stm(g, [&](int j) { return CT[orow + j][ocol] * T0[orow + j][ocol]; }) -
                           g.idz * stm(g, [&](int j) { return ST[orow][zc(j)] * T0[orow][zc(j)]; });
                    dPG3 = g.idx * stm(g, [&](int j) { return ST[orow + j][ocol] * T2[orow + j][ocol]; }) +
                           g.idz * stm(g, [&](int j) { return CT[orow][zc(j)] * T2[orow][zc(j)]; });
                    dMG1 = g.idx * stm(g, [&](int j) { return CT[orow + j][ocol] * T3[orow + j][ocol]; }) -
                           g.idz * stm(g, [&](int j) { return ST[orow][zc(j)] * T3[orow][zc(j)]; });
                    dMG3 = g.idx * stm(g, [&](int j) { return ST[orow + j][ocol] * T5[orow + j][ocol]; }) +
                           g.idz * stm(g, [&](int j) { return CT[orow][zc(j)] * T5[orow][zc(j)]; });
                }
                LP = dPG1 + dPG3;
                LM = dMG1 + dMG3;
            }
            if (!LINEAR) {
                F.pspace[k] = LP;
                F.mspace[k] = LM;
            }
            const float V = F.v[k];
            const float dt2V2_B = g.dt2 * V * V / F.b[k];
            const float Q = F.q[k];
            const float pc = ldf<RUN>(F.pcur + k), po = ldf<RUN>(F.pold + k);
            const float mc = ldf<RUN>(F.mcur + k), mo = ldf<RUN>(F.mold + k);
            F.pold[k] = dt2V2_B * LP - Q * (pc - po) - po + 2 * pc;
            F.mold[k] = dt2V2_B * LM - Q * (mc - mo) - mo + 2 * mc;
        }
    }
    if (RUN && F.inj.ngroups && it >= 1 && it <= F.inj.nt) {
        __syncthreads();
        for (long gi = threadIdx.x; gi < F.inj.ngroups; gi += NT) {
            const long key = F.inj.key[gi];
            const long x = key / nz, z = key - x * nz;
            if (x < x0 || x >= x0 + TX || z < z0 || z >= z0 + TZ) continue;
            float acc = __ldcg(F.pold + key);
            for (long j = F.inj.start[gi]; j < F.inj.start[gi + 1]; j++)
                acc = __fadd_rn(acc, __fmul_rn(F.inj.c[j], F.inj.wav[F.inj.other[j] * F.inj.nt + (it - 1)]));
            F.pold[key] = acc;
        }
    }
}

template <int PHYS, bool LINEAR>
__global__ void __launch_bounds__(NT) k_aniso2d_fused(Grid g, Fields F) {
    extern __shared__ __align__(16) float sm[];
    aniso_tile_step<PHYS, LINEAR, false>(g, F, (long)blockIdx.y * TX, (long)blockIdx.x * TZ, sm, 0);
}

// A whole 2D VTI or TTI time loop in one cooperative launch, as k_iso2d_run for 2D Iso: per step
// every tile's step with its source injection (CTAs take turns over the tiles; with as many CTAs as
// tiles each keeps its tile and its material boxes), a grid-wide barrier, then the receiver
// extraction from the new pCur; the pointer swaps of every step are the alternation of the two
// arrays of each field.
template <int PHYS>
__global__ void __launch_bounds__(NT) k_aniso2d_run(Grid g, Fields F, long nsteps, long it0, RunExtract ex,
                                                    unsigned *sync_words) {
    extern __shared__ __align__(16) float sm[];
    __shared__ int ok_flag;
    const long ntz = (g.nz + TZ - 1) / TZ, ntx = (g.nx + TX - 1) / TX, ntiles = ntz * ntx;
    unsigned gen = 0;
    for (long st = 0; st < nsteps; st++) {
        Fields Fs = F;
        Fs.pcur = (st & 1) ? F.pold : F.pcur;
        Fs.pold = (st & 1) ? F.pcur : F.pold;
        Fs.mcur = (st & 1) ? F.mold : F.mcur;
        Fs.mold = (st & 1) ? F.mcur : F.mold;
        const long it = it0 + st;
        for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
            // a CTA with one tile for the whole loop keeps the tile's material boxes
            aniso_tile_step<PHYS, false, true>(g, Fs, (t / ntz) * TX, (t % ntz) * TZ, sm, it,
                                               st == 0 || gridDim.x != ntiles);
            __syncthreads();  // the tile's shared memory is reused by the next tile
        }
        if (!grid_barrier(sync_words, gen, &ok_flag)) return;
        if (ex.ngroups && it >= 1 && it <= ex.nt) {
            // data[key*nt + it-1] += sum c * new pCur[other], each group in order, IEEE multiply and add
            for (long gi = (long)blockIdx.x * NT + threadIdx.x; gi < ex.ngroups; gi += (long)gridDim.x * NT) {
                float *dst = ex.data + ex.key[gi] * ex.nt + (it - 1);
                float acc = *dst;
                for (long j = ex.start[gi]; j < ex.start[gi + 1]; j++)
                    acc = __fadd_rn(acc, __fmul_rn(ex.c[j], __ldcg(Fs.pold + ex.other[j])));
                *dst = acc;
            }
        }
    }
}

template <int PHYS, bool LINEAR>
bool launch2(const Grid &g, const Fields &F, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(k_aniso2d_fused<PHYS, LINEAR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)SMEM_BYTES) != cudaSuccess)
            return false;
        attr = true;
    }
    const dim3 grid((unsigned)((g.nz + TZ - 1) / TZ), (unsigned)((g.nx + TX - 1) / TX));
    if (grid.y > 65535) return false;
    k_aniso2d_fused<PHYS, LINEAR><<<grid, NT, SMEM_BYTES, s>>>(g, F);
    return true;
}

}  // namespace

int aniso2d_run(const Grid &g, int phys, const Fields &F, long nsteps, long it0, const RunExtract &ex,
                unsigned *sync_words, cudaStream_t s) {
    if (g.ndim != 2 || (phys != VTI && phys != TTI)) return -1;
    // co-resident CTAs (0: no cooperative launch, or the shared memory cannot be granted)
    static int cap[2] = {-1, -1};
    const int which = phys == TTI ? 1 : 0;
    const void *fn = which ? (const void *)k_aniso2d_run<TTI> : (const void *)k_aniso2d_run<VTI>;
    if (cap[which] < 0) {
        int dev = 0, sms = 0, per = 0, coop = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES) == cudaSuccess)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, NT, SMEM_BYTES);
        cudaGetLastError();
        cap[which] = coop ? sms * per : 0;
    }
    if (cap[which] <= 0) return -1;
    const long ntiles = ((g.nz + TZ - 1) / TZ) * ((g.nx + TX - 1) / TX);
    const int grid = (int)(ntiles < cap[which] ? ntiles : cap[which]);
    Grid gg = g;
    Fields FF = F;
    long ns = nsteps, i0 = it0;
    RunExtract ee = ex;
    unsigned *sw = sync_words;
    void *args[] = {&gg, &FF, &ns, &i0, &ee, &sw};
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(NT), args, SMEM_BYTES, s) == cudaSuccess ? 0 : 1;
}

bool fused_aniso2d(const Grid &g, int phys, int linear, const Fields &F, cudaStream_t s) {
    if (g.ndim != 2) return false;
    if (phys == VTI) return linear ? launch2<VTI, true>(g, F, s) : launch2<VTI, false>(g, F, s);
    if (phys == TTI && !linear) return launch2<TTI, false>(g, F, s);
    return false;
}

}  // namespace WFD_NS
