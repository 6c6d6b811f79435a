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

__global__ void __launch_bounds__(NT) k_iso2d_fused(Grid g, Fields F) {
    __shared__ float P[PXH][PZW];
    __shared__ float Bs[BXH][BZW];
    __shared__ float T0[T0H][TZ];
    __shared__ float T2[TX][T2W];
    const int tz = threadIdx.x % WZ, tx = threadIdx.x / WZ;
    const long z0 = (long)blockIdx.x * TZ, x0 = (long)blockIdx.y * TX;
    const long nx = g.nx, nz = g.nz;

    // pCur with its antisymmetric image above kz = 0 (zero outside the grid elsewhere)
#pragma unroll
    for (int r = tx; r < PXH; r += WX) {
        const long x = x0 - 7 + r;
        const bool xin = x >= 0 && x < nx;
#pragma unroll
        for (int c = tz; c < PZW; c += WZ) {
            const long z = z0 - 7 + c;
            float v = 0.0f;
            if (xin) {
                if (z >= 0 && z < nz) v = F.pcur[x * nz + z];
                else if (z < 0 && -z < nz) v = -F.pcur[x * nz - z];
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
            const float V = F.v[k];
            const float dt2V2_B = g.dt2 * V * V / F.b[k];
            const float pc = F.pcur[k], po = F.pold[k];
            F.pold[k] = dt2V2_B * L - F.q[k] * (pc - po) - po + 2 * pc;
            F.pspace[k] = L;
        }
    }

    // source injection into the new field (graph-replayed loops): the groups whose cell lies in this
    // tile, after the tile's cells are written (visible to the CTA after the barrier); each group's
    // contributions in order, separate IEEE multiply and add, as the injection kernel does
    if (F.inj.ngroups) {
        const long it = *F.inj.d_it;
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

}  // namespace

bool fused_iso2d(const Grid &g, const Fields &F, cudaStream_t s) {
    if (g.ndim != 2) return false;
    const dim3 grid((unsigned)((g.nz + TZ - 1) / TZ), (unsigned)((g.nx + TX - 1) / TX));
    if (grid.y > 65535) return false;
    k_iso2d_fused<<<grid, NT, 0, s>>>(g, F);
    return true;
}

}  // namespace WFD_NS
