// Fused single-sweep 3D Iso step: pass 1 (D+ and buoyancy) and pass 2 (D-, time update with the
// Q term, pSpace) of prop3DAcoIsoDenQ_DEO2_FDTD.h:247-261 in one kernel, so that each field
// crosses HBM once per step (28 B/cell: read pCur, pOld, V, B, Q; write pOld, pSpace).
//
// Tiling: a CTA owns a (z,y) tile of TZ x TY output columns and sweeps a chunk of x planes
// (x is the slowest axis). Along x, each thread keeps register queues of pCur (8 planes) and of
// the pass-1 x-output (8 planes): the x-derivatives never touch shared memory. At each output
// plane the CTA stages pCur and B with their (y,z) halos in shared memory, forms the pass-1 y and
// z outputs on the halo-extended rows/columns, and applies D- to them. The halo plane of pCur is
// re-read from L2 (it entered the chip as the newest queue plane 7 iterations earlier).
// Persistent CTAs loop over (tile, x-chunk) work items; chunks overlap by 7 warm-up planes.
#include "wfd_kernels.h"

namespace WFD_NS {
using namespace wfd;

namespace {

constexpr int TZ = 32;
constexpr int TY = 16;
constexpr int NT = 256;  // 8 warps; warp w owns rows w and w + 8
constexpr int PZW = TZ + 16;  // pCur halo tile: z0-8 .. z0+TZ+8
constexpr int PYH = TY + 14;  // rows y0-7 .. y0+TY+6
constexpr int BZW = TZ + 8;   // B halo tile: z0-4 .. z0+TZ+4
constexpr int BYH = TY + 8;   // rows y0-4 .. y0+TY+3
constexpr int XCHUNK = 128;

struct Smem {
    float P[PYH][PZW];
    float B[BYH][BZW];
    float TYs[TY + 7][TZ];      // pass-1 y output on rows y0-4 .. y0+TY+2
    float TZs[TY][TZ + 8];      // pass-1 z output on columns z0-4 .. z0+TZ+3
};

__device__ __forceinline__ float ldg(const float *p) { return __ldg(p); }

__global__ void __launch_bounds__(NT, 2) k_iso3d_fused(Grid g, Fields F, int ntz, int nty, int nch) {
    __shared__ Smem s;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const long total = (long)ntz * nty * nch;
    const float *__restrict__ pc = F.pcur;
    const float *__restrict__ vv = F.v;
    const float *__restrict__ bb = F.b;
    const float *__restrict__ qq = F.q;
    float *po = F.pold;
    float *ps = F.pspace;

    for (long w = blockIdx.x; w < total; w += gridDim.x) {
        const int tzi = (int)(w % ntz);
        const int tyi = (int)((w / ntz) % nty);
        const int chi = (int)(w / ((long)ntz * nty));
        const long z0 = (long)tzi * TZ;
        const long y0 = (long)tyi * TY;
        const long xbeg = (long)chi * XCHUNK;
        const long xend = xbeg + XCHUNK < g.nx ? xbeg + XCHUNK : g.nx;

        // this thread's two columns
        const long z = z0 + lane;
        long yy[2] = {y0 + warp, y0 + warp + 8};
        bool in[2];
        long kcol[2];  // index of (x=0, y, z)
        for (int c = 0; c < 2; c++) {
            in[c] = z < g.nz && yy[c] < g.ny;
            kcol[c] = in[c] ? yy[c] * g.nz + z : 0;
        }
        float qp[2][8];  // pCur at planes xo .. xo+7
        float qt[2][8];  // pass-1 x output at planes xo-4 .. xo+3
        const long xs = xbeg - 7;
#pragma unroll
        for (int c = 0; c < 2; c++) {
#pragma unroll
            for (int i = 0; i < 8; i++) {
                qt[c][i] = 0.0f;
                qp[c][i] = 0.0f;
            }
#pragma unroll
            for (int i = 0; i < 7; i++) {
                const long xp = xs + i;
                qp[c][i + 1] = (in[c] && xp >= 0 && xp < g.nx) ? ldg(pc + xp * g.sx + kcol[c]) : 0.0f;
            }
        }

        for (long xo = xs; xo < xend; xo++) {
            const long xa = xo + 3;  // plane of the new pass-1 x output
            const long xn = xo + 7;  // newest pCur plane
            float bxa[2], pold_[2], vo[2], qo[2];
#pragma unroll
            for (int c = 0; c < 2; c++) {
#pragma unroll
                for (int i = 0; i < 7; i++) qp[c][i] = qp[c][i + 1];
                qp[c][7] = (in[c] && xn < g.nx) ? ldg(pc + xn * g.sx + kcol[c]) : 0.0f;
                bxa[c] = (in[c] && xa >= 0 && xa < g.nx) ? ldg(bb + xa * g.sx + kcol[c]) : 0.0f;
            }
            const bool out = xo >= xbeg;
            if (out) {
#pragma unroll
                for (int c = 0; c < 2; c++) {
                    const long k = xo * g.sx + kcol[c];
                    pold_[c] = in[c] ? po[k] : 0.0f;
                    vo[c] = in[c] ? ldg(vv + k) : 0.0f;
                    qo[c] = in[c] ? ldg(qq + k) : 0.0f;
                }
                // stage pCur(xo) and B(xo) with halos
                const long xoff = xo * g.sx;
                for (int i = threadIdx.x; i < PYH * PZW; i += NT) {
                    const int r = i / PZW, cz = i % PZW;
                    const long y = y0 - 7 + r, zz = z0 - 8 + cz;
                    s.P[r][cz] = (y >= 0 && y < g.ny && zz >= 0 && zz < g.nz) ? ldg(pc + xoff + y * g.nz + zz) : 0.0f;
                }
                for (int i = threadIdx.x; i < BYH * BZW; i += NT) {
                    const int r = i / BZW, cz = i % BZW;
                    const long y = y0 - 4 + r, zz = z0 - 4 + cz;
                    s.B[r][cz] = (y >= 0 && y < g.ny && zz >= 0 && zz < g.nz) ? ldg(bb + xoff + y * g.nz + zz) : 0.0f;
                }
            }
            // pass-1 x output at plane xa for both columns (register queue)
#pragma unroll
            for (int c = 0; c < 2; c++) {
                float t = 0.0f;
                const int r = in[c] ? region(g, xa, yy[c], z) : 0;
                if (r == 1 || (r == 2 && z != 0)) {
                    const float *q = qp[c];
                    const float st = g.c1 * (-q[3] + q[4]) + g.c2 * (-q[2] + q[5]) + g.c3 * (-q[1] + q[6]) +
                                     g.c4 * (-q[0] + q[7]);
                    t = bxa[c] * (g.idx * st);
                } else if (r == 2) {
                    t = bxa[c] * 0.0f;
                }
#pragma unroll
                for (int i = 0; i < 7; i++) qt[c][i] = qt[c][i + 1];
                qt[c][7] = t;
            }
            if (!out) continue;
            __syncthreads();
            // pass-1 y output on the extended rows, pass-1 z output on the extended columns
            for (int i = threadIdx.x; i < (TY + 7) * TZ; i += NT) {
                const int r = i / TZ, cz = i % TZ;
                const long y = y0 - 4 + r, zz = z0 + cz;
                float t = 0.0f;
                const int rg = (y >= 0 && y < g.ny && zz < g.nz) ? region(g, xo, y, zz) : 0;
                if (rg == 1 || (rg == 2 && zz != 0)) {
                    const float *col = &s.P[r][cz + 8];  // P row of y is r + 3
                    const float st = g.c1 * (-col[3 * PZW] + col[4 * PZW]) + g.c2 * (-col[2 * PZW] + col[5 * PZW]) +
                                     g.c3 * (-col[1 * PZW] + col[6 * PZW]) + g.c4 * (-col[0] + col[7 * PZW]);
                    t = s.B[r][cz + 4] * (g.idy * st);
                } else if (rg == 2) {
                    t = s.B[r][cz + 4] * 0.0f;
                }
                s.TYs[r][cz] = t;
            }
            for (int i = threadIdx.x; i < TY * (TZ + 7); i += NT) {
                const int r = i / (TZ + 7), cz = i % (TZ + 7);
                const long y = y0 + r, zz = z0 - 4 + cz;
                float t = 0.0f;
                const int rg = (y < g.ny && zz >= 0 && zz < g.nz) ? region(g, xo, y, zz) : 0;
                if (rg) {
                    const float *row = &s.P[r + 7][0];
                    const int c0 = (int)(zz - (z0 - 8));  // column of zz
                    float st;
                    if (zz >= 3) {
                        st = g.c1 * (-row[c0] + row[c0 + 1]) + g.c2 * (-row[c0 - 1] + row[c0 + 2]) +
                             g.c3 * (-row[c0 - 2] + row[c0 + 3]) + g.c4 * (-row[c0 - 3] + row[c0 + 4]);
                    } else {
                        // antisymmetric image above the free surface: p[-j] = -p[j]
                        auto pm = [&](long j) { return j >= 0 ? row[j + 8] : -row[-j + 8]; };
                        st = g.c1 * (-pm(zz) + pm(zz + 1)) + g.c2 * (-pm(zz - 1) + pm(zz + 2)) +
                             g.c3 * (-pm(zz - 2) + pm(zz + 3)) + g.c4 * (-pm(zz - 3) + pm(zz + 4));
                    }
                    t = s.B[r + 4][cz] * (g.idz * st);
                }
                s.TZs[r][cz] = t;
            }
            __syncthreads();
            // D- and the time update for this thread's two cells
#pragma unroll
            for (int c = 0; c < 2; c++) {
                if (!in[c]) continue;
                const long y = yy[c];
                const long k = xo * g.sx + kcol[c];
                const int rg = region(g, xo, y, z);
                if (!rg) {
                    ps[k] = 0.0f;
                    continue;
                }
                const float pcv = qp[c][0];
                float L;
                if (rg == 2 && z == 0) {
                    L = 0.0f + 0.0f + 0.0f;
                } else {
                    const float *q = qt[c];
                    const float sx = g.c1 * (-q[3] + q[4]) + g.c2 * (-q[2] + q[5]) + g.c3 * (-q[1] + q[6]) +
                                     g.c4 * (-q[0] + q[7]);
                    const int ry = warp + (c ? 8 : 0);  // TYs row of y is ry + 4
                    const float *cy = &s.TYs[ry][lane];
                    const float sy = g.c1 * (-cy[3 * TZ] + cy[4 * TZ]) + g.c2 * (-cy[2 * TZ] + cy[5 * TZ]) +
                                     g.c3 * (-cy[1 * TZ] + cy[6 * TZ]) + g.c4 * (-cy[0] + cy[7 * TZ]);
                    const float *rz = &s.TZs[ry][0];
                    float sz;
                    if (z >= 4) {
                        const int c0 = lane + 4;
                        sz = g.c1 * (-rz[c0 - 1] + rz[c0]) + g.c2 * (-rz[c0 - 2] + rz[c0 + 1]) +
                             g.c3 * (-rz[c0 - 3] + rz[c0 + 2]) + g.c4 * (-rz[c0 - 4] + rz[c0 + 3]);
                    } else {
                        // symmetric image above the free surface: t[-j] = t[j-1] (z0 == 0 here)
                        auto tm = [&](long j) { return rz[(j >= 0 ? j : -j - 1) + 4]; };
                        sz = g.c1 * (-tm(z - 1) + tm(z)) + g.c2 * (-tm(z - 2) + tm(z + 1)) +
                             g.c3 * (-tm(z - 3) + tm(z + 2)) + g.c4 * (-tm(z - 4) + tm(z + 3));
                    }
                    const float dx = g.idx * sx;
                    const float dy = g.idy * sy;
                    const float dz = g.idz * sz;
                    L = dx + dy + dz;
                }
                const float V = vo[c];
                const float dt2V2_B = g.dt2 * V * V / s.B[(warp + (c ? 8 : 0)) + 4][lane + 4];
                const float pov = pold_[c];
                po[k] = dt2V2_B * L - qo[c] * (pcv - pov) - pov + 2 * pcv;
                ps[k] = L;
            }
            __syncthreads();
        }
    }
}

}  // namespace

bool fused_iso3d(const Grid &g, const Fields &F, cudaStream_t s) {
    const int ntz = (int)((g.nz + TZ - 1) / TZ);
    const int nty = (int)((g.ny + TY - 1) / TY);
    const int nch = (int)((g.nx + XCHUNK - 1) / XCHUNK);
    static int grid_cap = 0;
    if (!grid_cap) {
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_iso3d_fused, NT, 0);
        grid_cap = sms * (per > 0 ? per : 1);
    }
    const long work = (long)ntz * nty * nch;
    const int grid = (int)(work < grid_cap ? work : grid_cap);
    k_iso3d_fused<<<grid, NT, 0, s>>>(g, F, ntz, nty, nch);
    return true;
}

}  // namespace WFD_NS
