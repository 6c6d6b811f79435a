// Fused 2D Iso step: both reference passes of prop2DAcoIsoDenQ_DEO2_FDTD (pass 1 D+ and the
// buoyancy sandwich, pass 2 D- and the time update with Q, .h:943) in one launch. A 2D grid is
// small (a 501 x 501 field is 1 MB and stays in L2), so a step is bound by launch latency, not by
// bandwidth: one kernel instead of two (and no scratch arrays in global memory).
//
// A CTA of 512 threads owns a tile of 16 x 64 cells (x rows, z contiguous; the fastest of the shapes
// timed on a 501 x 501 grid: 8x32, 16x32, 32x32 and 16x64 cells, 256 or 512 threads). It loads pCur
// on the tile plus 7 cells each side and B plus 4 each side into shared memory, forms the pass-1 x output
// on rows x0-4 .. x0+TX+2 of the tile's columns and the z output on columns z0-4 .. z0+TZ+2 of its
// rows (the halo is recomputed by each CTA, as neighbouring CTAs' pass-1 cells), then applies D- and
// the update to its cells. Free surface: pCur above kz = 0 is its antisymmetric image (D+ input),
// the z output above kz = 0 its symmetric image (D- input), as in propagatorStaticFunctions.h.
// Cell arithmetic is the expression trees of the two-pass kernels (wfd_generic.cu), so the strict
// build gives their bits. In a graph-replayed time loop the kernel also applies the step's source
// injection to the cells of its tile (F.inj), which saves the injection launch.
#include "wfd_gridbar.cuh"
#include "wfd_kernels.h"

namespace WFD_NS {
using namespace wfd;

namespace {

constexpr int TX = 16, TZ = 64, NT = 512;
constexpr int PXH = TX + 14, PZW = TZ + 14;  // pCur box: rows x0-7 .., columns z0-7 ..
constexpr int BXH = TX + 8, BZW = TZ + 8;    // B box: rows x0-4 .., columns z0-4 ..
constexpr int T0H = TX + 7;                  // pass-1 x output: rows x0-4 .. x0+TX+2, columns z0 ..
constexpr int T2W = TZ + 7;                  // pass-1 z output: rows x0 .., columns z0-4 .. z0+TZ+2

// region of a cell (0 outside, 1 interior, 2 free-surface row kz 0..3), as wfd::region in 2D
__device__ __forceinline__ int region2(const Grid &g, long x, long z) {
    if (x < 4 || x >= g.nx - 4 || z >= g.nz - 4) return 0;
    if (z >= 4) return 1;
    return g.fs ? 2 : 0;
}

// D+ reading w(-3..4) and D- reading w(-4..3) around the centre, the reference's term order
template <class W>
__device__ __forceinline__ float stp(const Grid &g, const W &w) {
    return g.c1 * (-w(0) + w(1)) + g.c2 * (-w(-1) + w(2)) + g.c3 * (-w(-2) + w(3)) + g.c4 * (-w(-3) + w(4));
}
template <class W>
__device__ __forceinline__ float stm(const Grid &g, const W &w) {
    return g.c1 * (-w(-1) + w(0)) + g.c2 * (-w(-2) + w(1)) + g.c3 * (-w(-3) + w(2)) + g.c4 * (-w(-4) + w(3));
}

// threads as 32 (z, fastest) x NT/32 (x); every shared-memory box is swept with compile-time trip counts
constexpr int WZ = 32, WX = NT / WZ;
static_assert(NT % WZ == 0 && TZ % WZ == 0, "thread layout");

struct Tile {
    float P[PXH][PZW];
    float Bs[BXH][BZW];
    float T0[T0H][TZ];
    float T2[TX][T2W];
};

// Pass 1 of the tile at (x0, z0) from the pCur and B boxes in shared memory (complete and visible to
// the CTA): the x output into T0, the z output into T2 with its symmetric image above the free
// surface; ends with both visible to the CTA.
__device__ __forceinline__ void pass1_tile(const Grid &g, const long x0, const long z0, Tile &sm) {
    auto &P = sm.P;
    auto &Bs = sm.Bs;
    auto &T0 = sm.T0;
    auto &T2 = sm.T2;
    const int tz = threadIdx.x % WZ, tx = threadIdx.x / WZ;
    // pass 1, x output (B * idx * D+x pCur) on rows x0-4 .. x0+TX+2
#pragma unroll
    for (int r = tx; r < T0H; r += WX) {
#pragma unroll
        for (int c = tz; c < TZ; c += WZ) {
            const long x = x0 - 4 + r, z = z0 + c;
            const int reg = region2(g, x, z);
            float t = 0.0f;
            if (reg) {
                const int pr = r + 3, pc = c + 7;  // P row/column of (x, z)
                const float dx = (reg == 2 && z == 0) ? 0.0f : g.idx * stp(g, [&](int j) { return P[pr + j][pc]; });
                t = Bs[r][c + 4] * dx;
            }
            T0[r][c] = t;
        }
    }
    // pass 1, z output (B * idz * D+z pCur, the image supplying kz < 0) on columns z0-4 .. z0+TZ+2
#pragma unroll
    for (int r = tx; r < TX; r += WX) {
        const long x = x0 + r;
#pragma unroll
        for (int c = tz; c < T2W; c += WZ) {
            const long z = z0 - 4 + c;
            float t = 0.0f;
            if (z >= 0) {
                const int reg = region2(g, x, z);
                if (reg) {
                    const int pr = r + 7, pc = c + 3;
                    const float dz = g.idz * stp(g, [&](int j) { return P[pr][pc + j]; });
                    t = Bs[r + 4][c] * dz;
                }
            }
            T2[r][c] = t;
        }
    }
    __syncthreads();
    if (z0 == 0) {
        // symmetric image of the z output above the free surface: t[-j] = t[j-1] (column of kz is kz+4)
        if (tz < 4) {
#pragma unroll
            for (int r = tx; r < TX; r += WX) T2[r][3 - tz] = T2[r][4 + tz];
        }
        __syncthreads();
    }
}

// One step of the tile at (x0, z0): F.pcur -> F.pold, F.pspace; then the source injection F.inj at
// time index it into the tile's cells of the new field (nothing when it is outside 1..nt). Ends with
// the tile's writes done by every thread of the CTA only if injecting (callers reusing the shared
// memory synchronise first).
__device__ __forceinline__ void tile_step(const Grid &g, const Fields &F, const long x0, const long z0, const long it,
                                          Tile &sm) {
    auto &P = sm.P;
    auto &Bs = sm.Bs;
    auto &T0 = sm.T0;
    auto &T2 = sm.T2;
    const int tz = threadIdx.x % WZ, tx = threadIdx.x / WZ;
    const long nx = g.nx, nz = g.nz;
    static_assert(WX == TX && TZ == 2 * WZ, "pass 2: one row and two columns per thread");

    // pass 2's per-cell inputs of this thread's two cells (row tx, columns tz and tz + 32), loaded
    // first so that their latency overlaps the tile loads and pass 1 (pCur and B come from the tile)
    float in_v[2] = {0.0f, 0.0f}, in_q[2] = {0.0f, 0.0f}, in_po[2] = {0.0f, 0.0f};
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const long x = x0 + tx, z = z0 + tz + WZ * i;
        if (x < nx && z < nz) {
            const long k = x * nz + z;
            in_v[i] = __ldg(F.v + k);
            in_q[i] = __ldg(F.q + k);
            in_po[i] = __ldcg(F.pold + k);
        }
    }

    // pCur with its antisymmetric image above kz = 0 (zero outside the grid elsewhere); read past L1
    // (in the whole-loop launch other CTAs rewrite it between steps)
#pragma unroll
    for (int r = tx; r < PXH; r += WX) {
        const long x = x0 - 7 + r;
        const bool xin = x >= 0 && x < nx;
#pragma unroll
        for (int c = tz; c < PZW; c += WZ) {
            const long z = z0 - 7 + c;
            float v = 0.0f;
            if (xin) {
                if (z >= 0 && z < nz) v = __ldcg(F.pcur + x * nz + z);
                else if (z < 0 && -z < nz) v = -__ldcg(F.pcur + x * nz - z);
            }
            P[r][c] = v;
        }
    }
#pragma unroll
    for (int r = tx; r < BXH; r += WX) {
        const long x = x0 - 4 + r;
#pragma unroll
        for (int c = tz; c < BZW; c += WZ) {
            const long z = z0 - 4 + c;
            Bs[r][c] = (x >= 0 && x < nx && z >= 0 && z < nz) ? F.b[x * nz + z] : 0.0f;
        }
    }
    __syncthreads();

    pass1_tile(g, x0, z0, sm);

    // pass 2: D-, the time update with Q, pSpace (.h:943)
#pragma unroll
    for (int r = tx; r < TX; r += WX) {
#pragma unroll
        for (int c = tz; c < TZ; c += WZ) {
            const long x = x0 + r, z = z0 + c;
            if (x >= nx || z >= nz) continue;
            const long k = x * nz + z;
            const int reg = region2(g, x, z);
            if (!reg) {
                F.pspace[k] = 0.0f;
                continue;
            }
            float dx = 0.0f, dz = 0.0f;
            if (!(reg == 2 && z == 0)) {
                dx = g.idx * stm(g, [&](int j) { return T0[r + 4 + j][c]; });
                dz = g.idz * stm(g, [&](int j) { return T2[r][c + 4 + j]; });
            }
            const float L = dx + dz;
            const int i = c / WZ;
            const float V = in_v[i];
            const float dt2V2_B = g.dt2 * V * V / Bs[r + 4][c + 4];
            const float pc = P[r + 7][c + 7], po = in_po[i];
            F.pold[k] = dt2V2_B * L - in_q[i] * (pc - po) - po + 2 * pc;
            F.pspace[k] = L;
        }
    }

    // source injection into the new field (graph-replayed loops): the groups whose cell lies in this
    // tile, after the tile's cells are written (visible to the CTA after the barrier); each group's
    // contributions in order, separate IEEE multiply and add, as the injection kernel does
    if (F.inj.ngroups) {
        if (it >= 1 && it <= F.inj.nt) {
            __syncthreads();
            for (long gi = threadIdx.x; gi < F.inj.ngroups; gi += NT) {
                const long key = F.inj.key[gi];
                const long x = key / nz, z = key - x * nz;
                if (x < x0 || x >= x0 + TX || z < z0 || z >= z0 + TZ) continue;
                float acc = F.pold[key];
                for (long j = F.inj.start[gi]; j < F.inj.start[gi + 1]; j++)
                    acc = __fadd_rn(acc, __fmul_rn(F.inj.c[j], F.inj.wav[F.inj.other[j] * F.inj.nt + (it - 1)]));
                F.pold[key] = acc;
            }
        }
    }
}


__global__ void __launch_bounds__(NT) k_iso2d_fused(Grid g, Fields F) {
    __shared__ Tile sm;
    const long it = F.inj.ngroups ? *F.inj.d_it : 0;
    tile_step(g, F, (long)blockIdx.y * TX, (long)blockIdx.x * TZ, it, sm);
}

// A whole time loop in one launch: nsteps steps, each followed by its source injection (in the step,
// per tile) and, after a grid-wide barrier, its receiver extraction from the new field, at time
// indices it0, it0+1, ...; the pointer swap of every step is the alternation of F.pcur and F.pold.
// Between two steps one barrier suffices: step s+1 writes only the array step s read (every read of
// it is done before the barrier), and the extraction of step s reads the array step s+1 only reads.
__global__ void __launch_bounds__(NT) k_iso2d_run(Grid g, Fields F, long nsteps, long it0, RunExtract ex,
                                                  unsigned *sync_words) {
    __shared__ Tile sm;
    __shared__ int ok_flag;
    const long ntz = (g.nz + TZ - 1) / TZ, ntx = (g.nx + TX - 1) / TX, ntiles = ntz * ntx;
    float *A = F.pcur, *B = F.pold;
    unsigned gen = 0;
    for (long st = 0; st < nsteps; st++) {
        Fields Fs = F;
        Fs.pcur = (st & 1) ? B : A;
        Fs.pold = (st & 1) ? A : B;
        const long it = it0 + st;
        for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
            tile_step(g, Fs, (t / ntz) * TX, (t % ntz) * TZ, it, sm);
            __syncthreads();  // the tile's shared memory is reused by the next tile
        }
        if (!grid_barrier(sync_words, gen, &ok_flag)) return;
        if (ex.ngroups && it >= 1 && it <= ex.nt) {
            // data[key*nt + it-1] += sum c * new field[other], each group in order, IEEE multiply and add
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
// The whole time loop with every tile resident in one CTA (as many CTAs as tiles, all co-resident).
// B stays in shared memory and V, Q and the tile's pOld in registers; the pCur box keeps the tile's
// own cells from the step before (its new field), so that a step reloads only the box's ring (the
// neighbours' cells and the free-surface image) from L2. pOld of a step is the pCur of the step
// before, and a cell outside the interior keeps its array value (the reference does not write it),
// so the registers and the box hold exactly what the two arrays hold. The source injection is
// applied to the box's cells, in each group's order, before the new field is stored; the new field
// is stored every step (the neighbours' rings and the receivers read it), pSpace only at the last
// step, the only one whose pSpace outlives the loop. The receivers of a step read its new field after
// the barrier, with the next step's ring loads (the last step's after the loop); barrier as
// k_iso2d_run.
constexpr int MAX_INJ = 1024;
struct InjRef {
    int group, cell;  // group index, cell offset in the pCur box
};

__global__ void __launch_bounds__(NT, 2) k_iso2d_run_res(Grid g, Fields F, long nsteps, long it0, RunExtract ex,
                                                         unsigned *sync_words) {
    __shared__ Tile sm;
    __shared__ int ok_flag, n_inj;
    __shared__ InjRef inj[MAX_INJ];
    __shared__ float Qs[TX][TZ], Ds[TX][TZ];
    auto &P = sm.P;
    auto &Bs = sm.Bs;
    auto &T0 = sm.T0;
    auto &T2 = sm.T2;
    const int tz = threadIdx.x % WZ, tx = threadIdx.x / WZ;
    const long nx = g.nx, nz = g.nz, ntz = (nz + TZ - 1) / TZ;
    const long x0 = (long)(blockIdx.x / ntz) * TX, z0 = (long)(blockIdx.x % ntz) * TZ;

    // B over the box; the thread's two cells (row tx, columns tz and tz + 32): pOld in registers,
    // Q and dt^2 V^2 / B (the same operations, in the same order, as every step would repeat) in
    // shared memory
#pragma unroll
    for (int r = tx; r < BXH; r += WX) {
        const long x = x0 - 4 + r;
#pragma unroll
        for (int c = tz; c < BZW; c += WZ) {
            const long z = z0 - 4 + c;
            Bs[r][c] = (x >= 0 && x < nx && z >= 0 && z < nz) ? F.b[x * nz + z] : 0.0f;
        }
    }
    float po[2] = {0.0f, 0.0f};
    bool mine[2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const long x = x0 + tx, z = z0 + tz + WZ * i;
        mine[i] = x < nx && z < nz;
        if (mine[i]) {
            const long k = x * nz + z;
            const float V = __ldg(F.v + k);
            Qs[tx][tz + WZ * i] = __ldg(F.q + k);
            Ds[tx][tz + WZ * i] = g.dt2 * V * V / F.b[k];
            po[i] = __ldcg(F.pold + k);
        }
    }
    // the source groups whose cell lies in this tile (tables of up to MAX_INJ groups; each group is
    // one cell, so their order does not matter)
    if (threadIdx.x == 0) n_inj = 0;
    __syncthreads();
    for (long gi = threadIdx.x; gi < F.inj.ngroups && gi < MAX_INJ; gi += NT) {
        const long key = F.inj.key[gi];
        const long x = key / nz, z = key - x * nz;
        if (x >= x0 && x < x0 + TX && z >= z0 && z < z0 + TZ)
            inj[atomicAdd(&n_inj, 1)] = InjRef{(int)gi, (int)((x - x0 + 7) * PZW + (z - z0 + 7))};
    }

    // the receiver groups of this thread (group blockIdx.x + threadIdx.x * CTAs, and every CTAs x NT
    // after it), the first one's description in registers: a group of one point, the common case,
    // has its two loads issued with the step's ring loads
    const long G = gridDim.x, egi = blockIdx.x + (long)threadIdx.x * G;
    const bool emine = egi < ex.ngroups;
    float *edst = nullptr;  // the group's trace, at time index 1
    long eoth = -1;         // the single point's cell, -1 for a group of several points
    float ec = 0.0f;
    if (emine) {
        edst = ex.data + ex.key[egi] * ex.nt;
        const long j0 = ex.start[egi];
        if (ex.start[egi + 1] - j0 == 1) {
            eoth = ex.other[j0];
            ec = ex.c[j0];
        }
    }

    float *A = F.pcur, *B = F.pold;
    unsigned gen = 0;
    for (long st = 0;; st++) {
        // pCur of step st is the new field of step st - 1, which the receivers read
        const float *pcur = (st & 1) ? B : A;
        float *pnew = (st & 1) ? A : B;
        const long it = it0 + st, ite = it - 1;
        const bool exs = st > 0 && ex.ngroups && ite >= 1 && ite <= ex.nt;
        float ed = 0.0f, ef = 0.0f;
        if (exs && emine) {
            ed = edst[ite - 1];
            if (eoth >= 0) ef = __ldcg(pcur + eoth);
        }
        // the pCur box with its antisymmetric image above kz = 0, into registers: the whole box at the
        // first step, afterwards the ring around the tile's own cells; the corners (outside the
        // tile's rows and its columns) are never read
        float rv[2][3];
        const bool ring = st < nsteps;
#pragma unroll
        for (int ri = 0; ri < 2; ri++) {
            const int r = tx + WX * ri;
            const long x = x0 - 7 + r;
            const bool xin = x >= 0 && x < nx, own_row = r >= 7 && r < 7 + TX;
#pragma unroll
            for (int ci = 0; ci < 3; ci++) {
                const int c = tz + WZ * ci;
                const bool own_col = c >= 7 && c < 7 + TZ;
                const long z = z0 - 7 + c;
                float val = 0.0f;
                if (ring && r < PXH && c < PZW && (own_row != own_col || (st == 0 && own_row)) && xin) {
                    if (z >= 0 && z < nz) val = __ldcg(pcur + x * nz + z);
                    else if (z < 0 && -z < nz) val = -__ldcg(pcur + x * nz - z);
                }
                rv[ri][ci] = val;
            }
        }
        // the extraction of step st - 1: data[key*nt + it-1] += sum c * field[other], each group in
        // order, IEEE multiply and add
        if (exs) {
            if (emine) {
                float acc = ed;
                if (eoth >= 0)
                    acc = __fadd_rn(acc, __fmul_rn(ec, ef));
                else
                    for (long j = ex.start[egi]; j < ex.start[egi + 1]; j++)
                        acc = __fadd_rn(acc, __fmul_rn(ex.c[j], __ldcg(pcur + ex.other[j])));
                edst[ite - 1] = acc;
            }
            for (long gi = egi + G * NT; gi < ex.ngroups; gi += G * NT) {
                float *dst = ex.data + ex.key[gi] * ex.nt + (ite - 1);
                float acc = *dst;
                for (long j = ex.start[gi]; j < ex.start[gi + 1]; j++)
                    acc = __fadd_rn(acc, __fmul_rn(ex.c[j], __ldcg(pcur + ex.other[j])));
                *dst = acc;
            }
        }
        if (!ring) break;
#pragma unroll
        for (int ri = 0; ri < 2; ri++) {
            const int r = tx + WX * ri;
            const bool own_row = r >= 7 && r < 7 + TX;
#pragma unroll
            for (int ci = 0; ci < 3; ci++) {
                const int c = tz + WZ * ci;
                const bool own_col = c >= 7 && c < 7 + TZ;
                if (r < PXH && c < PZW && (own_row != own_col || (st == 0 && own_row))) P[r][c] = rv[ri][ci];
            }
        }
        __syncthreads();

        pass1_tile(g, x0, z0, sm);

        // pass 2: D-, the time update with Q (.h:943); the new field into the box's own cells
        const bool last = st == nsteps - 1;
        float nv[2] = {0.0f, 0.0f};
#pragma unroll
        for (int i = 0; i < 2; i++) {
            if (!mine[i]) continue;
            const int r = tx, c = tz + WZ * i;
            const long x = x0 + r, z = z0 + c;
            const int reg = region2(g, x, z);
            const float pc = P[r + 7][c + 7];
            float n = po[i], L = 0.0f;
            if (reg) {
                float dx = 0.0f, dz = 0.0f;
                if (!(reg == 2 && z == 0)) {
                    dx = g.idx * stm(g, [&](int j) { return T0[r + 4 + j][c]; });
                    dz = g.idz * stm(g, [&](int j) { return T2[r][c + 4 + j]; });
                }
                L = dx + dz;
                n = Ds[r][c] * L - Qs[r][c] * (pc - po[i]) - po[i] + 2 * pc;
            }
            if (last) F.pspace[x * nz + z] = L;
            po[i] = pc;
            P[r + 7][c + 7] = n;
            nv[i] = n;
        }
        // the step's source injection into the new field, each group's contributions in order,
        // separate IEEE multiply and add
        if (n_inj && it >= 1 && it <= F.inj.nt) {
            __syncthreads();
            for (int li = threadIdx.x; li < n_inj; li += NT) {
                const InjRef ref = inj[li];
                float *cell = &P[0][0] + ref.cell;
                float acc = *cell;
                for (long j = F.inj.start[ref.group]; j < F.inj.start[ref.group + 1]; j++)
                    acc = __fadd_rn(acc, __fmul_rn(F.inj.c[j], F.inj.wav[F.inj.other[j] * F.inj.nt + (it - 1)]));
                *cell = acc;
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 2; i++) nv[i] = P[tx + 7][tz + WZ * i + 7];
        }
#pragma unroll
        for (int i = 0; i < 2; i++)
            if (mine[i]) pnew[(x0 + tx) * nz + z0 + tz + WZ * i] = nv[i];

        if (!grid_barrier(sync_words, gen, &ok_flag)) return;
    }
}
}  // namespace

int iso2d_run(const Grid &g, const Fields &F, long nsteps, long it0, const RunExtract &ex, unsigned *sync_words,
              cudaStream_t s) {
    if (g.ndim != 2) return -1;
    // co-resident CTAs of the two forms (0: the device has no cooperative launch)
    static int cap = -1, cap_res = 0;
    if (cap < 0) {
        int dev = 0, sms = 0, per = 0, per_res = 0, coop = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_iso2d_run, NT, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_res, k_iso2d_run_res, NT, 0);
        cap = coop ? sms * per : 0;
        cap_res = coop ? sms * per_res : 0;
    }
    const long ntiles = ((g.nz + TZ - 1) / TZ) * ((g.nx + TX - 1) / TX);
    const bool resident = ntiles <= cap_res && F.inj.ngroups <= MAX_INJ;
    if (!resident && cap <= 0) return -1;
    const int grid = (int)(resident ? ntiles : (ntiles < cap ? ntiles : cap));
    Grid gg = g;
    Fields FF = F;
    long ns = nsteps, i0 = it0;
    RunExtract ee = ex;
    unsigned *sw = sync_words;
    void *args[] = {&gg, &FF, &ns, &i0, &ee, &sw};
    const void *fn = resident ? (const void *)k_iso2d_run_res : (const void *)k_iso2d_run;
    return cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(NT), args, 0, s) == cudaSuccess ? 0 : 1;
}

bool fused_iso2d(const Grid &g, const Fields &F, cudaStream_t s) {
    if (g.ndim != 2) return false;
    const dim3 grid((unsigned)((g.nz + TZ - 1) / TZ), (unsigned)((g.nx + TX - 1) / TX));
    if (grid.y > 65535) return false;
    k_iso2d_fused<<<grid, NT, 0, s>>>(g, F);
    return true;
}

}  // namespace WFD_NS
