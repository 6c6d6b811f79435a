// Fused single-sweep 3D Iso step with TMA-staged tiles (prop3DAcoIsoDenQ_DEO2_FDTD.h:247-261 in one
// kernel; 28 B/cell of HBM traffic: read pCur, pOld, V, B, Q; write pOld, pSpace).
//
// A CTA (128 threads) owns a (z,y) tile of 32 x 16 columns and sweeps a chunk of x planes. For each
// plane j one thread issues, D planes ahead, a group of TMA tile loads completed on one mbarrier:
//   pCur(j) with its halo (48 x 30 at z0-8, y0-7), pCur(j+7) (32 x 16),
//   B(j) with its halo (40 x 24 at z0-4, y0-4), B(j+3) (32 x 16), pOld(j), V(j), Q(j) (32 x 16).
// pCur and B are read twice (the second time from L2), which keeps the stage small enough for
// three CTAs per SM. A thread owns 4 consecutive z cells of one row (float4 shared-memory
// accesses) and keeps along x register queues of pCur and of the pass-1 x output, 8 planes each;
// the queue slot of plane j+i is (q+i)&7, so the queues never move (one small case per phase).
// At plane j, warps 0-1 form the pass-1 y output on the 24 halo-extended rows (3 rows per thread,
// sliding along y) and warps 2-3 the pass-1 z output on the 40 halo-extended columns (a run of
// 2-3 quads per thread, sliding along z); then every thread applies D- and the time update to its
// 4 cells and stores pOld and pSpace as float4.
// The reference's region rules (interior [4,n-4), free-surface rows, untouched annulus) are
// applied as selects on values computed everywhere; three code variants: interior tiles (no
// selects), edge tiles (selects), and the top tile with a free surface (selects plus the image
// stencils above kz = 0, which only the first z quad needs).
// Persistent CTAs loop over (tile, x-chunk) items; a chunk starts with 14 warm-up planes that only
// fill the queues. With an illumination sum attached (single objects), each cell's pCur^2 is added
// to it as the cell is updated. Waits are bounded; on timeout the kernel records an error in a device status
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

enum Mode { INNER = 0, EDGE = 1, TOP = 2 };

__device__ unsigned int d_status;

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float at(const float4 &v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}
// cells 0-1 (h = 0) or 2-3 (h = 1) of a quad
__device__ __forceinline__ float2 half2(const float4 &v, int h) {
    return h == 0 ? make_float2(v.x, v.y) : make_float2(v.z, v.w);
}
#if WFD_STRICT
// strict build: one rounded scalar operation per lane, never contracted (the reference has no FMA)
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return add2(mul2(a, b), c); }
// a - b written as the reference's -b + a
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return add2(make_float2(-b.x, -b.y), a); }
#else
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// b * -1 + a: one packed instruction, rounded once like -b + a
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
#endif
__device__ __forceinline__ float2 div2(float2 a, float2 b) { return make_float2(a.x / b.x, a.y / b.y); }
// lane-wise keep-or-replace by two bits of a cell mask
__device__ __forceinline__ float2 keep2(unsigned mask, int bit, float2 v, float2 other) {
    return make_float2((mask >> bit) & 1u ? v.x : other.x, (mask >> bit + 1) & 1u ? v.y : other.y);
}

// D+ at the centre of an 8-sample window w[0..7] = f(k-3..k+4); D- with w[0..7] = f(k-4..k+3)
// (prop3DAcoIsoDenQ_DEO2_FDTD.h:846-864, :1113-1131), summed left to right
__device__ __forceinline__ float st8(const Grid &g, float w0, float w1, float w2, float w3, float w4, float w5,
                                     float w6, float w7) {
    return g.c1 * (-w3 + w4) + g.c2 * (-w2 + w5) + g.c3 * (-w1 + w6) + g.c4 * (-w0 + w7);
}
// the same stencil on a pair of cells whose windows sit in the same lanes (x and y directions)
__device__ __forceinline__ float2 st8p(const Grid &g, float2 w0, float2 w1, float2 w2, float2 w3, float2 w4,
                                       float2 w5, float2 w6, float2 w7) {
    float2 s = mul2(bc2(g.c1), sub2(w4, w3));
    s = fma2(bc2(g.c2), sub2(w5, w2), s);
    s = fma2(bc2(g.c3), sub2(w6, w1), s);
    return fma2(bc2(g.c4), sub2(w7, w0), s);
}

// cells of the pass-1 outputs that the reference computes: interior, or free-surface rows 1..3
// (row 0 holds B*0 = 0 for the x/y outputs)
__device__ __forceinline__ bool xy_out_z(const Grid &g, int zz) {
    return zz < g.nz - 4 && (zz >= 4 || (g.fs && zz > 0));
}
// cells of the pass-1 z output and of the update: interior, or free-surface rows 0..3
__device__ __forceinline__ bool z_out_z(const Grid &g, int zz) { return zz >= 0 && zz < g.nz - 4 && (zz >= 4 || g.fs); }
__device__ __forceinline__ bool y_in(const Grid &g, int y) { return y >= 4 && y < g.ny - 4; }

// Thread tasks of the halo stage: threads 0-63 form the y outputs of 3 extended rows x 4 cells
// (rows r0..r0+2, r0 = 3 (tid >> 3), columns 4 (tid & 7)..+3); threads 64-127 the z outputs of
// 2-3 quads of one tile row (row (tid-64) >> 2, quads {0,1,2} {3,4,5} {6,7} {8,9} of the 10
// extended-column quads at z0-4).
__device__ __forceinline__ void ext_z_task(int tid, int &r, int &qa, int &nq) {
    const int tt = tid - 64;
    const int g4 = tt & 3;
    r = tt >> 2;
    qa = g4 == 0 ? 0 : (g4 == 1 ? 3 : (g4 == 2 ? 6 : 8));
    nq = g4 < 2 ? 3 : 2;
}
// which of those cells the reference computes (given x): bit 4 rr + m (y task, row r0+rr, cell m)
// or 4 k + m (z task, quad qa+k, cell m); fixed for an item
__device__ __forceinline__ unsigned ext_mask(const Grid &g, int tid, int z0, int y0) {
    unsigned mask = 0;
    if (tid < 64) {
        const int r0 = (tid >> 3) * 3, zz0 = z0 + 4 * (tid & 7);
#pragma unroll
        for (int rr = 0; rr < 3; rr++)
#pragma unroll
            for (int m = 0; m < 4; m++)
                if (y_in(g, y0 - 4 + r0 + rr) && xy_out_z(g, zz0 + m)) mask |= 1u << (4 * rr + m);
    } else {
        int r, qa, nq;
        ext_z_task(tid, r, qa, nq);
#pragma unroll
        for (int k = 0; k < 3; k++)
#pragma unroll
            for (int m = 0; m < 4; m++)
                if (k < nq && y_in(g, y0 + r) && z_out_z(g, z0 - 4 + 4 * (qa + k) + m)) mask |= 1u << (4 * k + m);
    }
    return mask;
}

// pass-1 y/z outputs of the centre plane j into TYs/TZs (emask: ext_mask of this thread)
template <int MODE>
__device__ __forceinline__ void ext_stage(const Grid &g, const bool xin, const bool top, const int z0,
                                          const unsigned emask, const float *st, float *TYs, float *TZs) {
    const int tid = threadIdx.x;
    const float *Pc = st + S_PH;
    const float *Bc = st + S_BH;
    const unsigned em = xin ? emask : 0u;
    const float2 zero = bc2(0.0f);
    if (tid < 64) {
        const int zq = tid & 7;
        const int r0 = (tid >> 3) * 3;  // rows r0..r0+2 of the 24 extended rows
        float4 w[10];
#pragma unroll
        for (int i = 0; i < 10; i++)  // row 30 would only feed the unused padding row 23
            w[i] = r0 + i < PYH ? ld4(Pc + (r0 + i) * PZW + 8 + 4 * zq) : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int rr = 0; rr < 3; rr++) {
            const int r = r0 + rr;
            const float4 b = ld4(Bc + r * BZW + 4 + 4 * zq);
            float2 out[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const float2 s = st8p(g, half2(w[rr], h), half2(w[rr + 1], h), half2(w[rr + 2], h),
                                      half2(w[rr + 3], h), half2(w[rr + 4], h), half2(w[rr + 5], h),
                                      half2(w[rr + 6], h), half2(w[rr + 7], h));
                float2 t = mul2(half2(b, h), mul2(bc2(g.idy), s));
                if (MODE != INNER) t = keep2(em, 4 * rr + 2 * h, t, zero);
                out[h] = t;
            }
            st4(TYs + r * TZ + 4 * zq, make_float4(out[0].x, out[0].y, out[1].x, out[1].y));
        }
    } else {
        // each thread slides along z over its contiguous quads (scalar stencils: a pair of
        // neighbouring z cells has its windows one lane apart)
        int r, qa, nq;
        ext_z_task(tid, r, qa, nq);
        const float *rowp = Pc + (r + 7) * PZW;
        float v[20];
#pragma unroll
        for (int i = 0; i < 5; i++) {
            const float4 a = (i < nq + 2) ? ld4(rowp + 4 * (qa + i)) : make_float4(0.f, 0.f, 0.f, 0.f);
            v[4 * i] = a.x;
            v[4 * i + 1] = a.y;
            v[4 * i + 2] = a.z;
            v[4 * i + 3] = a.w;
        }
#pragma unroll
        for (int k = 0; k < 3; k++) {
            if (k >= nq) break;
            const int qi = qa + k;
            const int zb = z0 - 4 + 4 * qi;  // first z of this quad
            const float4 b = ld4(Bc + (r + 4) * BZW + 4 * qi);
            float out[4];
#pragma unroll
            for (int m = 0; m < 4; m++) {
                const int o = 4 * k + m;
                float s = st8(g, v[o + 1], v[o + 2], v[o + 3], v[o + 4], v[o + 5], v[o + 6], v[o + 7], v[o + 8]);
                if (top && zb == 0 && m < 3) {
                    // antisymmetric image above the free surface, p[-j] = -p[j]; column of z is z+8
                    auto pm = [&](int jz) { return jz >= 0 ? rowp[jz + 8] : -rowp[-jz + 8]; };
                    s = st8(g, pm(m - 3), pm(m - 2), pm(m - 1), pm(m), pm(m + 1), pm(m + 2), pm(m + 3), pm(m + 4));
                }
                float t = at(b, m) * (g.idz * s);
                if (MODE != INNER) t = ((em >> (4 * k + m)) & 1u) ? t : 0.0f;
                out[m] = t;
            }
            st4(TZs + r * TZW + 4 * qi, make_float4(out[0], out[1], out[2], out[3]));
        }
    }
}

// D- in y and z, the time update and the stores of this thread's 4 cells (fmask bit m: the
// reference updates cell m, given x)
template <int MODE, bool EPI>
__device__ __forceinline__ void fin_stage(const Grid &g, const long j, const bool xin, const bool top, const int z,
                                          const int y, const unsigned fmask, const int zq, const int row,
                                          const float2 *sx, const float2 *pc, const float *st, const float *TYs,
                                          const float *TZs, float *po, float *ps, float *illum,
                                          const StepEpilogue *epi, const float4 ea, const float4 eb) {
    const int o = row * TZ + 4 * zq;
    const float4 pold4 = ld4(st + S_PO + o), v4 = ld4(st + S_V + o), q4 = ld4(st + S_Q + o);
    const float4 b4 = ld4(st + S_BH + (4 + row) * BZW + 4 + 4 * zq);
    float4 ty[8];
#pragma unroll
    for (int i = 0; i < 8; i++) ty[i] = ld4(TYs + (row + i) * TZ + 4 * zq);
    const float *tzr = TZs + row * TZW;
    const float4 t0 = ld4(tzr + 4 * zq), t1 = ld4(tzr + 4 * zq + 4), t2 = ld4(tzr + 4 * zq + 8);
    const float w[12] = {t0.x, t0.y, t0.z, t0.w, t1.x, t1.y, t1.z, t1.w, t2.x, t2.y, t2.z, t2.w};
    const unsigned fm = xin ? fmask : 0u;
    float2 npo[2], nps[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int m0 = 2 * h;
        const float2 sy = st8p(g, half2(ty[0], h), half2(ty[1], h), half2(ty[2], h), half2(ty[3], h),
                               half2(ty[4], h), half2(ty[5], h), half2(ty[6], h), half2(ty[7], h));
        const float2 sz = make_float2(
            st8(g, w[m0], w[m0 + 1], w[m0 + 2], w[m0 + 3], w[m0 + 4], w[m0 + 5], w[m0 + 6], w[m0 + 7]),
            st8(g, w[m0 + 1], w[m0 + 2], w[m0 + 3], w[m0 + 4], w[m0 + 5], w[m0 + 6], w[m0 + 7], w[m0 + 8]));
#if WFD_STRICT
        float2 L = add2(add2(mul2(bc2(g.idx), sx[h]), mul2(bc2(g.idy), sy)), mul2(bc2(g.idz), sz));
#else
        float2 L = fma2(bc2(g.idx), sx[h], fma2(bc2(g.idy), sy, mul2(bc2(g.idz), sz)));
#endif
        if (top && z == 0) {
            // the free surface row (cell 0): all derivatives are zero; cells 1-3: symmetric image
            // above the free surface, t[-j] = t[j-1] (column of z is z+4)
            float Ll[2] = {L.x, L.y};
            const float sxl[2] = {sx[h].x, sx[h].y}, syl[2] = {sy.x, sy.y};
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int m = m0 + e;
                if (m == 0) {
                    Ll[e] = 0.0f + 0.0f + 0.0f;
                } else {
                    auto tm = [&](int jz) { return tzr[(jz >= 0 ? jz : -jz - 1) + 4]; };
                    const float szi =
                        st8(g, tm(m - 4), tm(m - 3), tm(m - 2), tm(m - 1), tm(m), tm(m + 1), tm(m + 2), tm(m + 3));
                    const float dx = g.idx * sxl[e];
                    const float dy = g.idy * syl[e];
                    const float dz = g.idz * szi;
                    Ll[e] = dx + dy + dz;
                }
            }
            L = make_float2(Ll[0], Ll[1]);
        }
        const float2 V = half2(v4, h), pcv = pc[h], pov = half2(pold4, h);
        // dt^2 V^2 / B L - Q (pCur - pOld) - pOld + 2 pCur, left to right (:247-261)
        const float2 k2 = div2(mul2(mul2(bc2(g.dt2), V), V), half2(b4, h));
        const float2 t = sub2(sub2(mul2(k2, L), mul2(half2(q4, h), sub2(pcv, pov))), pov);
        float2 np = add2(t, mul2(bc2(2.0f), pcv));
        float2 nl = L;
        if (MODE != INNER) {
            np = keep2(fm, m0, np, pov);  // cells the reference leaves alone
            nl = keep2(fm, m0, nl, bc2(0.0f));
        }
        if (EPI && epi->scale_space)  // ScaleSpatialDerivatives fused (.h:269-291): pSpace *= V^2/B
            nl = mul2(nl, div2(mul2(V, V), half2(b4, h)));
        if (EPI && epi->born_dv) {
            // Born-V injection fused after the step (prop3DAcoIsoDenQ_DEO2_FDTD.h:305-334), every cell:
            // new += dt^2 V^2/B * DP * (2 B dV / V^3); ea = dV, eb = DP (loaded early)
            const float2 B = half2(b4, h);
            const float2 fv = div2(mul2(mul2(bc2(2.0f), B), half2(ea, h)), mul2(mul2(V, V), V));
            np = add2(np, mul2(mul2(k2, half2(eb, h)), fv));
        }
        if (EPI && epi->img) {
            // imaging condition fused after the step (.h:518-546): img += 2B/V^3 DP pOld, pOld being
            // this step's input pCur; ea = the image, eb = DP (loaded early)
            const long kc = j * g.sx + (long)y * g.nz + z + m0;
            const float2 fv = div2(mul2(bc2(2.0f), half2(b4, h)), mul2(mul2(V, V), V));
            st2(epi->img + kc, add2(half2(ea, h), mul2(mul2(fv, half2(eb, h)), pcv)));
        }
        npo[h] = np;
        nps[h] = nl;
    }
    const long k = j * g.sx + (long)y * g.nz + z;
    st4(po + k, make_float4(npo[0].x, npo[0].y, npo[1].x, npo[1].y));
    st4(ps + k, make_float4(nps[0].x, nps[0].y, nps[1].x, nps[1].y));
    if (illum) {
        // source illumination, every cell: sum += pCur^2 (separate IEEE multiply and add, as
        // illumination.c:31-53 does)
        float4 a = ld4(illum + k);
        a.x = __fadd_rn(a.x, __fmul_rn(pc[0].x, pc[0].x));
        a.y = __fadd_rn(a.y, __fmul_rn(pc[0].y, pc[0].y));
        a.z = __fadd_rn(a.z, __fmul_rn(pc[1].x, pc[1].x));
        a.w = __fadd_rn(a.w, __fmul_rn(pc[1].y, pc[1].y));
        st4(illum + k, a);
    }
}

// Queue update of phase PH = q & 7: pCur(j+7) enters slot (PH+7)&7, the pass-1 x output at plane
// j+3 enters qt slot (PH+7)&7; returns the D- x stencil at plane j and pCur(j). Queues hold the
// quad as two cell pairs.
template <int PH>
__device__ __forceinline__ void queue_phase(float2 (&qp)[8][2], float2 (&qt)[8][2], const Grid &g, const bool xin_a,
                                            const unsigned txmask, const float4 pn, const float4 bn, float2 *sx,
                                            float2 *pc) {
    constexpr int N = (PH + 7) & 7;
    qp[N][0] = half2(pn, 0);
    qp[N][1] = half2(pn, 1);
    const unsigned tm = xin_a ? txmask : 0u;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const float2 s = st8p(g, qp[(PH + 0) & 7][h], qp[(PH + 1) & 7][h], qp[(PH + 2) & 7][h], qp[(PH + 3) & 7][h],
                              qp[(PH + 4) & 7][h], qp[(PH + 5) & 7][h], qp[(PH + 6) & 7][h], qp[N][h]);
        const float2 t = mul2(half2(bn, h), mul2(bc2(g.idx), s));
        qt[N][h] = keep2(tm, 2 * h, t, bc2(0.0f));
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        sx[h] = st8p(g, qt[(PH + 0) & 7][h], qt[(PH + 1) & 7][h], qt[(PH + 2) & 7][h], qt[(PH + 3) & 7][h],
                     qt[(PH + 4) & 7][h], qt[(PH + 5) & 7][h], qt[(PH + 6) & 7][h], qt[N][h]);
        pc[h] = qp[PH][h];
    }
}

// BATCH = false: one propagator object, its tensor maps in the kernel parameters, items w =
// blockIdx.x, blockIdx.x + gridDim.x, ... of its (tile, x-chunk) list.
// BATCH = true: many objects (shots) of different sizes; every item names its shot, whose sizes,
// output pointers and tensor maps sit in a descriptor in global memory; CTAs take items from a
// shared counter (dynamic scheduling over shots of uneven size, in the order the caller packed).
template <bool BATCH, bool EPI = false>
__global__ void __launch_bounds__(NT, 3)
    k_iso3d_tma(Grid g0, Fields F, const __grid_constant__ IsoMaps M, int ntz0, int nty0, int nch0, int xchunk0,
                const IsoShotDesc *__restrict__ shots, const int *__restrict__ sel, const int2 *__restrict__ items,
                int nitems, int *counter) {
    extern __shared__ __align__(1024) float sm[];
    float *TYs = sm + OFF_TY;
    float *TZs = sm + OFF_TZ;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + OFF_BAR);
    int *abort_flag = reinterpret_cast<int *>(bars + NS);
    int *item_slot = abort_flag + 1;

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    if (tid == 0) {
        for (int s = 0; s < NS; s++) mbar_init(&bars[s], 1);
        fence_mbar_init();
        if (!BATCH)
            for (int i = 0; i < 7; i++) prefetch_tensor_map(&M.m[i]);
        *abort_flag = 0;
    }
    __syncthreads();

    const long total = (long)ntz0 * nty0 * nch0;
    unsigned gseq = 0;                  // groups consumed so far by this CTA
    unsigned out_from = 0, out_to = 0;  // groups issued but not yet consumed (thread 0)
    const int zq = lane & 7;
    const int row = 4 * warp + (lane >> 3);

    for (long wstat = blockIdx.x;; wstat += gridDim.x) {
        Grid g = g0;
        const CUtensorMap *maps = M.m;
        float *out_pold = F.pold, *out_pspace = F.pspace;
        int ntz = ntz0, nty = nty0, xchunk = xchunk0;
        long w = wstat;
        if (BATCH) {
            if (tid == 0) *item_slot = atomicAdd(counter, 1);
            __syncthreads();
            const int wi = *item_slot;
            __syncthreads();
            if (wi >= nitems) break;
            const int2 it = items[wi];
            const IsoShotDesc *d = shots + sel[it.x];
            g.nx = d->nx;
            g.ny = d->ny;
            g.nz = d->nz;
            g.sy = d->nz;
            g.sx = (long)d->ny * d->nz;
            g.n = g.nx * g.sx;
            maps = d->m;
            out_pold = d->pold;
            out_pspace = d->pspace;
            ntz = d->ntz;
            nty = d->nty;
            xchunk = d->xchunk;
            w = it.y;
        } else if (wstat >= total) {
            break;
        }
        const CUtensorMap *mPH = maps + 0, *mPN = maps + 1, *mBH = maps + 2, *mBN = maps + 3, *mPO = maps + 4,
                          *mV = maps + 5, *mQ = maps + 6;
        const int tzi = (int)(w % ntz);
        const int tyi = (int)((w / ntz) % nty);
        const int chi = (int)(w / ((long)ntz * nty));
        const int z0 = tzi * TZ;
        const int y0 = tyi * TY;
        const int z = z0 + 4 * zq;
        const int y = y0 + row;
        const bool own = z < g.nz && y < g.ny;
        const long xbeg = (long)chi * xchunk;
        const long xend = xbeg + xchunk < g.nx ? xbeg + xchunk : g.nx;
        const long jstart = xbeg - WARMUP;
        const int ngroups = (int)(xend - jstart);
        const bool tile_top = z0 == 0 && g.fs;
        unsigned txmask = 0;  // cells of this thread whose pass-1 x output is computed (given x)
        unsigned fmask = 0;   // cells of this thread that are updated (given x)
#pragma unroll
        for (int m = 0; m < 4; m++) {
            if (y_in(g, y) && xy_out_z(g, z + m)) txmask |= 1u << m;
            if (y_in(g, y) && z_out_z(g, z + m)) fmask |= 1u << m;
        }
        const unsigned emask = ext_mask(g, tid, z0, y0);

        auto issue = [&](long jj, unsigned gs) {
            uint64_t *bar = &bars[gs % NS];
            float *s = sm + (gs % NS) * STAGE;
            mbar_expect_tx(bar, GROUP_BYTES);
            tma_load_3d(s + S_PH, mPH, bar, z0 - 8, y0 - 7, (int)jj);
            tma_load_3d(s + S_BH, mBH, bar, z0 - 4, y0 - 4, (int)jj);
            tma_load_3d(s + S_PN, mPN, bar, z0, y0, (int)(jj + 7));
            tma_load_3d(s + S_BN, mBN, bar, z0, y0, (int)(jj + 3));
            tma_load_3d(s + S_PO, mPO, bar, z0, y0, (int)jj);
            tma_load_3d(s + S_V, mV, bar, z0, y0, (int)jj);
            tma_load_3d(s + S_Q, mQ, bar, z0, y0, (int)jj);
        };
        if (tid == 0) {
            for (int q = 0; q < D && q < ngroups; q++) issue(jstart + q, gseq + q);
            out_from = gseq;
            out_to = gseq + (D < ngroups ? D : ngroups);
        }
        // queues: qp[(q+i)&7] = pCur(j+i), qt[(q+i)&7] = pass-1 x output at plane j-4+i
        float2 qp[8][2], qt[8][2];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                qp[i][h] = bc2(0.0f);
                qt[i][h] = bc2(0.0f);
            }
        unsigned slot = gseq % NS, par = (gseq / NS) & 1u;  // stage and phase of group gseq + q

        bool stop = false;
        for (int q = 0; q < ngroups; q++) {
            const long j = jstart + q;
            const unsigned gs = gseq + q;
            if (tid == 0 && q + D < ngroups) {
                issue(j + D, gs + D);
                out_to = gs + D + 1;
            }
            // the epilogue's inputs of plane j, loaded now so that their latency hides behind the wait
            // and the queue work (born: dV, DP; imaging: the image, DP)
            float4 ea = make_float4(0.0f, 0.0f, 0.0f, 0.0f), eb = ea;
            if (EPI && own && j >= xbeg) {
                const long k = j * g.sx + (long)y * g.nz + z;
                if (F.epi.born_dv) {
                    ea = __ldg(reinterpret_cast<const float4 *>(F.epi.born_dv + k));
                    eb = __ldg(reinterpret_cast<const float4 *>(F.epi.born_dp + k));
                } else if (F.epi.img) {
                    ea = ld4(F.epi.img + k);
                    eb = __ldg(reinterpret_cast<const float4 *>(F.epi.img_dp + k));
                }
            }
            const bool landed = mbar_wait(&bars[slot], par);
            if (!landed) {
                atomicExch(abort_flag, 1);
                atomicOr(&d_status, 1u);
            }
            // a group whose wait ran out may still be in flight: the drain below waits for it
            if (tid == 0 && landed) out_from = gs + 1;
            const float *st = sm + slot * STAGE;
            slot = slot + 1 == NS ? 0u : slot + 1;
            par ^= slot == 0 ? 1u : 0u;
            float2 sx[2], pc[2];
            {
                const int o = row * TZ + 4 * zq;
                const float4 pn = ld4(st + S_PN + o);
                const float4 bn = ld4(st + S_BN + o);
                const bool xin_a = j + 3 >= 4 && j + 3 < g.nx - 4;
                switch (q & 7) {
                    case 0: queue_phase<0>(qp, qt, g, xin_a, txmask, pn, bn, sx, pc); break;
                    case 1: queue_phase<1>(qp, qt, g, xin_a, txmask, pn, bn, sx, pc); break;
                    case 2: queue_phase<2>(qp, qt, g, xin_a, txmask, pn, bn, sx, pc); break;
                    case 3: queue_phase<3>(qp, qt, g, xin_a, txmask, pn, bn, sx, pc); break;
                    case 4: queue_phase<4>(qp, qt, g, xin_a, txmask, pn, bn, sx, pc); break;
                    case 5: queue_phase<5>(qp, qt, g, xin_a, txmask, pn, bn, sx, pc); break;
                    case 6: queue_phase<6>(qp, qt, g, xin_a, txmask, pn, bn, sx, pc); break;
                    default: queue_phase<7>(qp, qt, g, xin_a, txmask, pn, bn, sx, pc); break;
                }
            }
            if (j >= xbeg) {
                const bool xin = j >= 4 && j < g.nx - 4;
                // one code path for every tile (the selects are cheap, code size is not)
                ext_stage<EDGE>(g, xin, tile_top, z0, emask, st, TYs, TZs);
                __syncthreads();
                if (own) fin_stage<EDGE, EPI>(g, j, xin, tile_top, z, y, fmask, zq, row, sx, pc, st, TYs, TZs, out_pold,
                                               out_pspace, BATCH ? nullptr : F.illum, EPI ? &F.epi : nullptr, ea, eb);
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

namespace {

int iso_grid_cap() {
    static int cap = 0;
    if (!cap) {
        int dev = 0, sms = 0, per = 0;
        for (auto kern : {k_iso3d_tma<false>, k_iso3d_tma<true>, k_iso3d_tma<false, true>})
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_iso3d_tma<false>, NT, SMEM_BYTES);
        cap = sms * (per > 0 ? per : 1);
    }
    return cap;
}

bool iso_maps(const Grid &g, const Fields &F, CUtensorMap *m) {
    return make_tensor_map_3d(&m[0], F.pcur, g.nx, g.ny, g.nz, PZW, PYH, 1) &&
           make_tensor_map_3d(&m[1], F.pcur, g.nx, g.ny, g.nz, TZ, TY, 1) &&
           make_tensor_map_3d(&m[2], F.b, g.nx, g.ny, g.nz, BZW, BYH, 1) &&
           make_tensor_map_3d(&m[3], F.b, g.nx, g.ny, g.nz, TZ, TY, 1) &&
           make_tensor_map_3d(&m[4], F.pold, g.nx, g.ny, g.nz, TZ, TY, 1) &&
           make_tensor_map_3d(&m[5], F.v, g.nx, g.ny, g.nz, TZ, TY, 1) &&
           make_tensor_map_3d(&m[6], F.q, g.nx, g.ny, g.nz, TZ, TY, 1);
}

}  // namespace

bool fused_iso3d_tma(const Grid &g, const Fields &F, cudaStream_t s) {
    if (g.nz % 4 != 0) return false;
    IsoMaps M;
    if (!iso_maps(g, F, M.m)) return false;
    const int grid_cap = iso_grid_cap();
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
if (F.epi.born_dv || F.epi.img || F.epi.scale_space)
            k_iso3d_tma<false, true><<<grid, NT, SMEM_BYTES, s>>>(g, F, M, ntz, nty, nch, xchunk, nullptr, nullptr, nullptr, 0,
                                                    nullptr);
    else
            k_iso3d_tma<false><<<grid, NT, SMEM_BYTES, s>>>(g, F, M, ntz, nty, nch, xchunk, nullptr, nullptr, nullptr, 0,
                                                    nullptr);
    return true;
}

bool iso3d_tma_describe(const Grid &g, const Fields &F, int xchunk, IsoShotDesc *d, TileInfo *t) {
    if (g.ndim != 3 || g.nz % 4 != 0 || xchunk < 1) return false;
    if (d) {
        if (!iso_maps(g, F, d->m)) return false;
        d->pold = F.pold;
        d->pspace = F.pspace;
        d->nx = (int)g.nx;
        d->ny = (int)g.ny;
        d->nz = (int)g.nz;
        d->ntz = (int)((g.nz + TZ - 1) / TZ);
        d->nty = (int)((g.ny + TY - 1) / TY);
        d->xchunk = xchunk;
    }
    if (t) {
        t->tz = TZ;
        t->ty = TY;
        t->warmup = WARMUP;
        t->grid_cap = iso_grid_cap();
    }
    return true;
}

void iso3d_tma_batch(const Grid &gc, const IsoShotDesc *shots, const int *sel, const int2 *items, int nitems,
                     int *counter, int grid, cudaStream_t s) {
    k_iso3d_tma<true><<<grid, NT, SMEM_BYTES, s>>>(gc, Fields{}, IsoMaps{}, 0, 0, 0, 1, shots, sel, items, nitems,
                                                   counter);
}

void iso3d_set_pipeline_wait(unsigned long long ns) {
    const uint64_t v = ns;
    cudaMemcpyToSymbol(wfd_dev::d_pipeline_wait_ns, &v, sizeof(v));
}

unsigned iso3d_status_and_clear() {
    unsigned v = 0, z = 0;
    cudaMemcpyFromSymbol(&v, d_status, sizeof(v));
    if (v) cudaMemcpyToSymbol(d_status, &z, sizeof(z));
    return v;
}

}  // namespace WFD_NS
