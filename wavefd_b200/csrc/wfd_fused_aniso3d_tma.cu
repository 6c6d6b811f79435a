// Fused single-sweep 3D VTI and TTI steps with TMA-staged tiles: both reference passes in one
// kernel (TTI: prop3DAcoTTIDenQ_DEO2_FDTD.h:359-385, pass 1 :885-976, pass 2 update :1420-1421;
// VTI: prop3DAcoVTIDenQ_DEO2_FDTD.h:326-376, pass 1 :945-957, update :1372-1378, linear :1697-1698).
// HBM traffic per cell: TTI reads pCur, mCur, pOld, mOld, V, B, eps, eta, f, Q, sin/cos theta,
// sin/cos phi and writes pOld, mOld, pSpace, mSpace (72 B); VTI drops the four angle arrays (56 B,
// 48 B for the linear step, which writes no pSpace/mSpace).
//
// A CTA of 256 threads owns a (z,y) tile of 32 x 16 columns and sweeps a chunk of x planes; one
// CTA per SM. In TTI the pass-1 outputs at a halo point need all three derivatives there (the
// rotation mixes them), so the x derivative is needed on the halo too; it comes from a ring of
// pCur/mCur planes in shared memory (10 slots of 48 x 30 at z0-8, y0-7, filled by TMA two planes
// ahead). Iteration j applies pass 1 at the lead plane P = j+3 on the tile (all six outputs) and on
// its halo (7 extended rows for the y outputs, 2 x 4 extended columns for the z outputs), then
// pass 2 at plane j: the x outputs of planes j-4..j+3 sit in an 8-deep register queue per thread,
// the y/z outputs of plane j (computed three iterations earlier and held in 4-deep register
// queues) are written to shared memory for the y and z D- stencils. Materials of plane P
// (40 x 24 boxes) and the update fields of plane j (32 x 16 boxes) come one plane ahead.
// A thread owns a pair of consecutive z cells of one row; arithmetic is on float2 pairs with the
// packed FP32 instructions (FFMA2/FADD2/FMUL2). The strict build uses the packed multiply and add
// (no contraction) in the reference's order of operations, which reproduces the reference's FP32
// results bit for bit.
// Region rules (interior [4,n-4), free-surface rows, untouched annulus) are selects. The free
// surface images are written into shared memory: the antisymmetric image of pCur/mCur above
// kz = 0 into each ring plane of the top tile, the symmetric image of the z outputs into the halo
// columns of the top tile. With an illumination sum attached (single objects), each cell's pCur^2
// is added to it as the cell is updated. Waits are bounded; on timeout the kernel records an error
// in a device status word and leaves. Requires nz % 4 == 0 (TMA row pitch).
#include "wfd_kernels.h"
#include "wfd_tma.cuh"

namespace WFD_NS {
using namespace wfd;
using namespace wfd_dev;

namespace {

constexpr int TZ = 32, TY = 16, NT = 256;
constexpr int DR = 2;       // ring prefetch distance (planes)
constexpr int NR = 8 + DR;  // ring slots
constexpr int DM = 1;       // prefetch distance of materials and update fields
constexpr int NM = 1 + DM;  // their stages
constexpr int RZW = TZ + 16, RYH = TY + 14, RBOX = RZW * RYH;  // ring box 48 x 30 at (z0-8, y0-7)
constexpr int MZW = TZ + 8, MYH = TY + 8, MBOX = MZW * MYH;    // material box 40 x 24 at (z0-4, y0-4)
constexpr int CBOX = TZ * TY;                                   // update-field box 32 x 16 at (z0, y0)
constexpr int NMAT = 8;                                         // b, eps, eta, f, st, ct, sp, cp
constexpr int NCORE = 5;                                        // pOld, mOld, V, Q, b
enum { MT_B = 0, MT_E, MT_A, MT_F, MT_ST, MT_CT, MT_SP, MT_CP };
enum { C_PO = 0, C_MO, C_V, C_Q, C_B };
constexpr int TYR = TY + 8, TZW = TZ + 8;  // y outputs: rows y0-4..y0+19; z outputs: columns z0-4..z0+35
constexpr int R_SLOT = 2 * RBOX;
constexpr int M_STAGE = NMAT * MBOX + NCORE * CBOX;
constexpr int OFF_RING = 0;
constexpr int OFF_MAT = OFF_RING + NR * R_SLOT;
constexpr int OFF_TY = OFF_MAT + NM * M_STAGE;
constexpr int OFF_TZ = OFF_TY + 2 * TYR * TZ;
constexpr int OFF_BAR = OFF_TZ + 2 * TY * TZW;
constexpr size_t SMEM_BYTES = (size_t)OFF_BAR * 4 + (NR + NM) * 8 + 16;
constexpr int WARMUP = 7;  // pass-1-only iterations before the first plane of a chunk
// The thread that issues the TMA copies: lane 0 of warp 6, a warp without halo work (warps 0-3 do
// the y-halo pairs, 4-5 the z-halo pairs), so that the issue does not lengthen the busiest warps'
// planes.
constexpr int ISSUER = 192;
static_assert((RBOX * 4) % 128 == 0 && (MBOX * 4) % 128 == 0 && (CBOX * 4) % 128 == 0, "TMA alignment");
static_assert((OFF_MAT * 4) % 128 == 0 && (M_STAGE * 4) % 128 == 0, "TMA alignment");
static_assert(OFF_BAR % 2 == 0, "mbarrier alignment");
static_assert(SMEM_BYTES <= 232448, "shared memory per CTA");

__device__ unsigned int d_status;

__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }
#if WFD_STRICT
// strict build: one rounded scalar operation per lane, never contracted (the reference has no FMA)
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return add2(mul2(a, b), c); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
// a - b written as the reference's -b + a
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return add2(neg2(b), a); }
#else
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// Negation and subtraction as one packed instruction each: b * -1 is exact, so b * -1 + a rounds
// once, like -b + a (a negated operand of the packed add would cost two scalar instructions).
__device__ __forceinline__ float2 neg2(float2 a) { return __fmul2_rn(a, make_float2(-1.0f, -1.0f)); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
#endif
__device__ __forceinline__ float2 sel2(bool c, float2 a, float2 b) { return c ? a : b; }
__device__ __forceinline__ float2 sqrt2(float2 a) { return make_float2(sqrtf(a.x), sqrtf(a.y)); }
__device__ __forceinline__ float2 div2(float2 a, float2 b) { return make_float2(a.x / b.x, a.y / b.y); }

#if WFD_STRICT
// 8-point staggered stencil c1(w4-w3) + c2(w5-w2) + c3(w6-w1) + c4(w7-w0), summed left to right:
// D+ with w = f(k-3..k+4), D- with w = f(k-4..k+3) (prop3DAcoIsoDenQ_DEO2_FDTD.h:846-864, :1113-1131)
__device__ __forceinline__ float2 st8(const Grid &g, float2 w0, float2 w1, float2 w2, float2 w3, float2 w4,
                                      float2 w5, float2 w6, float2 w7) {
    float2 s = mul2(bc2(g.c1), sub2(w4, w3));
    s = fma2(bc2(g.c2), sub2(w5, w2), s);
    s = fma2(bc2(g.c3), sub2(w6, w1), s);
    return fma2(bc2(g.c4), sub2(w7, w0), s);
}
#endif
// A derivative: the inverse spacing `id` times the stencil. The strict build multiplies the stencil
// sum (the reference's order); the fast build folds `id` into the four coefficients (one multiply
// fewer per derivative).
__device__ __forceinline__ float2 st8d(const Grid &g, float id, float2 w0, float2 w1, float2 w2, float2 w3, float2 w4,
                                       float2 w5, float2 w6, float2 w7) {
#if WFD_STRICT
    return mul2(bc2(id), st8(g, w0, w1, w2, w3, w4, w5, w6, w7));
#else
    float2 s = mul2(bc2(g.c1 * id), sub2(w4, w3));
    s = fma2(bc2(g.c2 * id), sub2(w5, w2), s);
    s = fma2(bc2(g.c3 * id), sub2(w6, w1), s);
    return fma2(bc2(g.c4 * id), sub2(w7, w0), s);
#endif
}
// the same along z for a cell pair from ten consecutive values v[0..9]: lane x takes v[o..o+7],
// lane y v[o+1..o+8]
__device__ __forceinline__ float2 st8zd(const Grid &g, float id, const float (&v)[10], int o) {
    auto w = [&](int i) { return make_float2(v[o + i], v[o + i + 1]); };
    return st8d(g, id, w(0), w(1), w(2), w(3), w(4), w(5), w(6), w(7));
}
__device__ __forceinline__ void load10(float (&v)[10], const float *p) {
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const float2 a = ld2(p + 2 * i);
        v[2 * i] = a.x;
        v[2 * i + 1] = a.y;
    }
}

__device__ __forceinline__ bool zok(const Grid &g, int z) { return z >= 0 && z < g.nz - 4 && (z >= 4 || g.fs); }
__device__ __forceinline__ bool yok(const Grid &g, int y) { return y >= 4 && y < g.ny - 4; }

// Pass-1 outputs of one cell pair (P = pCur, M = mCur derivatives through the material sandwich)
struct Out6 {
    float2 px, py, pz, mx, my, mz;
};

// Pass 1 at the cell pair with extended row er (y = y0-4+er) and extended column ec (z = z0-4+ec)
// of the lead plane. WHICH: 0 = all six outputs, 1 = y outputs only, 2 = z outputs only.
// ring[i] = ring slot of plane P-3+i. ok = the reference computes this cell's outputs.
template <int PHYS, int WHICH>
__device__ __forceinline__ Out6 pass1(const Grid &g, const float *const (&ring)[8], const float *mat, int er, int ec,
                                      bool ok, bool zero_xy) {
    const int off = (er + 3) * RZW + ec + 4;
    const float *cp = ring[3] + off;  // centre plane, this pair
    const bool need_x = WHICH == 0 || PHYS == TTI;
    const bool need_y = WHICH != 2 || PHYS == TTI;
    const bool need_z = WHICH != 1 || PHYS == TTI;
    const float2 zero = bc2(0.0f);
    float2 dPx = zero, dPy = zero, dPz = zero, dMx = zero, dMy = zero, dMz = zero;
    if (need_x) {
        dPx = st8d(g, g.idx, ld2(ring[0] + off), ld2(ring[1] + off), ld2(ring[2] + off), ld2(ring[3] + off),
                   ld2(ring[4] + off), ld2(ring[5] + off), ld2(ring[6] + off), ld2(ring[7] + off));
        const int o = off + RBOX;
        dMx = st8d(g, g.idx, ld2(ring[0] + o), ld2(ring[1] + o), ld2(ring[2] + o), ld2(ring[3] + o),
                   ld2(ring[4] + o), ld2(ring[5] + o), ld2(ring[6] + o), ld2(ring[7] + o));
    }
    if (need_y) {
        const float *p = cp;
        dPy = st8d(g, g.idy, ld2(p - 3 * RZW), ld2(p - 2 * RZW), ld2(p - RZW), ld2(p), ld2(p + RZW),
                   ld2(p + 2 * RZW), ld2(p + 3 * RZW), ld2(p + 4 * RZW));
        p = cp + RBOX;
        dMy = st8d(g, g.idy, ld2(p - 3 * RZW), ld2(p - 2 * RZW), ld2(p - RZW), ld2(p), ld2(p + RZW),
                   ld2(p + 2 * RZW), ld2(p + 3 * RZW), ld2(p + 4 * RZW));
    }
    if (need_z) {
        float v[10];
        load10(v, cp - 4);
        dPz = st8zd(g, g.idz, v, 1);
        load10(v, cp + RBOX - 4);
        dMz = st8zd(g, g.idz, v, 1);
    }
    if (zero_xy) {  // free-surface row kz = 0 (lane x): the x and y derivatives are zero
        dPx.x = 0.0f;
        dPy.x = 0.0f;
        dMx.x = 0.0f;
        dMy.x = 0.0f;
    }
    const int mo = er * MZW + ec;
    float2 bv = ld2(mat + MT_B * MBOX + mo);
    const float2 eps = ld2(mat + MT_E * MBOX + mo);
    // fast build, TTI: every output is a product with the buoyancy, so a zero buoyancy outside the
    // reference's range zeroes all six (the derivatives and materials are finite: TMA fills zeros)
    constexpr bool mask_b = !WFD_STRICT && PHYS == TTI;
    if (mask_b) bv = sel2(ok, bv, bc2(0.0f));
    const float2 eta = ld2(mat + MT_A * MBOX + mo), fv = ld2(mat + MT_F * MBOX + mo);
    const float2 one = bc2(1.0f), two = bc2(2.0f);
    Out6 o;
    if (PHYS == TTI) {
        // prop3DAcoTTIDenQ_DEO2_FDTD.h:885-976
        const float2 st = ld2(mat + MT_ST * MBOX + mo), ct = ld2(mat + MT_CT * MBOX + mo);
        const float2 sp = ld2(mat + MT_SP * MBOX + mo), cq = ld2(mat + MT_CP * MBOX + mo);
        const float2 stcp = mul2(st, cq);
        const float2 stsp = mul2(st, sp);
        const float2 eta2 = mul2(eta, eta);
        const float2 bvfv = mul2(bv, fv);
        const float2 g3P = fma2(ct, dPz, fma2(stsp, dPy, mul2(stcp, dPx)));
        const float2 g3M = fma2(ct, dMz, fma2(stsp, dMy, mul2(stcp, dMx)));
        const float2 tmpFE = mul2(mul2(bvfv, eta), sqrt2(sub2(one, eta2)));
        const float2 tmpP = fma2(tmpFE, g3M, mul2(mul2(neg2(bv), fma2(fv, eta2, mul2(two, eps))), g3P));
        const float2 tmpM = fma2(mul2(bvfv, eta2), g3M, mul2(tmpFE, g3P));
        const float2 tmpE = mul2(bv, fma2(two, eps, one));
        const float2 tmpF = mul2(bv, sub2(one, fv));
        o.px = fma2(stcp, tmpP, mul2(tmpE, dPx));
        o.py = fma2(stsp, tmpP, mul2(tmpE, dPy));
        o.pz = fma2(ct, tmpP, mul2(tmpE, dPz));
        o.mx = fma2(stcp, tmpM, mul2(tmpF, dMx));
        o.my = fma2(stsp, tmpM, mul2(tmpF, dMy));
        o.mz = fma2(ct, tmpM, mul2(tmpF, dMz));
    } else {
        // prop3DAcoVTIDenQ_DEO2_FDTD.h:945-957
        const float2 E = fma2(two, eps, one);
        const float2 BE = mul2(bv, E);
        const float2 BF1 = mul2(bv, sub2(one, fv));
        o.px = mul2(BE, dPx);
        o.py = mul2(BE, dPy);
        o.mx = mul2(BF1, dMx);
        o.my = mul2(BF1, dMy);
        if (WHICH != 1) {
            const float2 FA = mul2(fv, eta);
            const float2 FAA = mul2(FA, eta);
            const float2 SA2 = sqrt2(sub2(one, mul2(eta, eta)));
            o.pz = fma2(mul2(bv, mul2(FA, SA2)), dMz, mul2(mul2(bv, sub2(one, FAA)), dPz));
            o.mz = fma2(mul2(bv, add2(sub2(one, fv), FAA)), dMz, mul2(mul2(mul2(mul2(bv, fv), eta), SA2), dPz));
        } else {
            o.pz = zero;
            o.mz = zero;
        }
    }
    if (!mask_b) {
        const float2 z2 = zero;
        o.px = sel2(ok, o.px, z2);
        o.py = sel2(ok, o.py, z2);
        o.pz = sel2(ok, o.pz, z2);
        o.mx = sel2(ok, o.mx, z2);
        o.my = sel2(ok, o.my, z2);
        o.mz = sel2(ok, o.mz, z2);
    }
    return o;
}

// Register queues of phase PH = q & 7: the x outputs of lead plane P enter qx slot (PH+3)&7 and the
// D- x stencil of plane j = P-3 is formed over slots (PH+4)&7 .. (PH+3)&7; the y/z outputs of P
// enter slot (PH+3)&3 of qc (tile) and qh (halo), and those of plane j leave slot PH&3.
template <int PH>
__device__ __forceinline__ void queue_phase(const Grid &g, float2 (&qx)[8][2], float2 (&qc)[4][4], float2 (&qh)[4][2],
                                            const Out6 &c, float2 h0, float2 h1, float2 (&sx)[2],
                                            float2 (&cj)[4], float2 (&hj)[2]) {
    constexpr int N = (PH + 3) & 7;
    constexpr int N4 = (PH + 3) & 3;
    qx[N][0] = c.px;
    qx[N][1] = c.mx;
#pragma unroll
    for (int f = 0; f < 2; f++)
        sx[f] = st8d(g, g.idx, qx[(PH + 4) & 7][f], qx[(PH + 5) & 7][f], qx[(PH + 6) & 7][f], qx[(PH + 7) & 7][f],
                     qx[(PH + 0) & 7][f], qx[(PH + 1) & 7][f], qx[(PH + 2) & 7][f], qx[N][f]);
    qc[N4][0] = c.py;
    qc[N4][1] = c.pz;
    qc[N4][2] = c.my;
    qc[N4][3] = c.mz;
    qh[N4][0] = h0;
    qh[N4][1] = h1;
#pragma unroll
    for (int f = 0; f < 4; f++) cj[f] = qc[PH & 3][f];
    hj[0] = qh[PH & 3][0];
    hj[1] = qh[PH & 3][1];
}

// BATCH = false: one propagator object, tensor maps in the kernel parameters, static items.
// BATCH = true: many shots; each item names its shot, whose sizes, output pointers and tensor maps
// sit in a descriptor in global memory; CTAs take items from a shared counter.
template <int PHYS, bool LINEAR, bool BATCH, bool EPI = false>
__global__ void __launch_bounds__(NT, 1)
    k_aniso3d_tma(Grid g0, Fields F, const __grid_constant__ AnisoMaps M, int ntz0, int nty0, int nch0, int xchunk0,
                  const AnisoShotDesc *__restrict__ shots, const int *__restrict__ sel,
                  const int2 *__restrict__ items, int nitems, int *counter) {
    extern __shared__ __align__(1024) float sm[];
    float *TYs = sm + OFF_TY;  // [2][TYR][TZ]: y outputs of P then M
    float *TZs = sm + OFF_TZ;  // [2][TY][TZW]: z outputs of P then M
    uint64_t *rbar = reinterpret_cast<uint64_t *>(sm + OFF_BAR);
    uint64_t *mbar = rbar + NR;
    int *abort_flag = reinterpret_cast<int *>(mbar + NM);
    int *item_slot = abort_flag + 1;
    constexpr int nmat = PHYS == TTI ? 8 : 4;

    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < NR; s++) mbar_init(&rbar[s], 1);
        for (int s = 0; s < NM; s++) mbar_init(&mbar[s], 1);
        fence_mbar_init();
        *abort_flag = 0;
    }
    for (int i = tid; i < 2 * TYR * TZ + 2 * TY * TZW; i += NT) TYs[i] = 0.0f;
    __syncthreads();

    // this thread's tile pair (row, zp) and halo pair
    const int zp = tid & 15;
    const int row = tid >> 4;
    int h_er, h_ec, h_kind;  // kind 0: none, 1: y halo, 2: z halo
    if (tid < 112) {
        const int hr = tid >> 4;
        h_er = hr < 4 ? hr : hr + 16;
        h_ec = 4 + 2 * zp;
        h_kind = 1;
    } else if (tid >= 128 && tid < 192) {  // (warps 4-5: a warp holds one kind of halo task)
        const int u = tid - 128;
        const int hp = u & 3;
        h_er = 4 + (u >> 2);
        h_ec = hp < 2 ? 2 * hp : 36 + 2 * (hp - 2);
        h_kind = 2;
    } else {
        h_er = 4;
        h_ec = 4;
        h_kind = 0;
    }

    const long total = (long)ntz0 * nty0 * nch0;
    unsigned rseq = 0, mseq = 0;      // ring planes and stages of the items finished by this CTA
    unsigned r_issued = 0, m_issued = 0;  // issued by thread 0
    unsigned r_done = 0, m_done = 0;      // landed (waits that succeeded)

    for (long wstat = blockIdx.x;; wstat += gridDim.x) {
        Grid g = g0;
        const CUtensorMap *maps = M.m;
        float *out_pold = F.pold, *out_mold = F.mold, *out_pspace = F.pspace, *out_mspace = F.mspace;
        int ntz = ntz0, nty = nty0, xchunk = xchunk0;
        long w = wstat;
        if (BATCH) {
            if (tid == 0) *item_slot = atomicAdd(counter, 1);
            __syncthreads();
            const int wi = *item_slot;
            __syncthreads();
            if (wi >= nitems) break;
            const int2 it = items[wi];
            const AnisoShotDesc *d = shots + sel[it.x];
            g.nx = d->nx;
            g.ny = d->ny;
            g.nz = d->nz;
            g.sy = d->nz;
            g.sx = (long)d->ny * d->nz;
            g.n = g.nx * g.sx;
            maps = d->m;
            out_pold = d->pold;
            out_mold = d->mold;
            out_pspace = d->pspace;
            out_mspace = d->mspace;
            ntz = d->ntz;
            nty = d->nty;
            xchunk = d->xchunk;
            w = it.y;
        } else if (wstat >= total) {
            break;
        }
        const CUtensorMap *mP = maps + 0, *mM = maps + 1, *mB = maps + 2, *mE = maps + 3, *mA = maps + 4,
                          *mF = maps + 5, *mST = maps + 6, *mCT = maps + 7, *mSP = maps + 8, *mCP = maps + 9,
                          *mPO = maps + 10, *mMO = maps + 11, *mV = maps + 12, *mQ = maps + 13, *mBC = maps + 14;
        const int tzi = (int)(w % ntz);
        const int tyi = (int)((w / ntz) % nty);
        const int chi = (int)(w / ((long)ntz * nty));
        const int z0 = tzi * TZ, y0 = tyi * TY;
        const long xbeg = (long)chi * xchunk;
        const long xend = xbeg + xchunk < g.nx ? xbeg + xchunk : g.nx;
        const long jstart = xbeg - WARMUP;
        const int niter = (int)(xend - jstart);
        const int nplanes = niter + 7;  // ring planes jstart .. xend+6
        const bool top = z0 == 0 && g.fs;
        const int z = z0 + 2 * zp, y = y0 + row;
        const bool own = z < g.nz && y < g.ny;
        const int hz = z0 - 4 + h_ec, hy = y0 - 4 + h_er;

        auto issue_ring = [&](int rp, unsigned gidx) {
            uint64_t *bar = &rbar[gidx % NR];
            float *s = sm + OFF_RING + (gidx % NR) * R_SLOT;
            mbar_expect_tx(bar, 4u * R_SLOT);
            tma_load_3d(s, mP, bar, z0 - 8, y0 - 7, (int)(jstart + rp));
            tma_load_3d(s + RBOX, mM, bar, z0 - 8, y0 - 7, (int)(jstart + rp));
        };
        auto issue_stage = [&](int q, unsigned gidx) {
            uint64_t *bar = &mbar[gidx % NM];
            float *s = sm + OFF_MAT + (gidx % NM) * M_STAGE;
            float *c = s + NMAT * MBOX;
            mbar_expect_tx(bar, 4u * (nmat * MBOX + NCORE * CBOX));
            const int P = (int)(jstart + q + 3), j = (int)(jstart + q);
            tma_load_3d(s + MT_B * MBOX, mB, bar, z0 - 4, y0 - 4, P);
            tma_load_3d(s + MT_E * MBOX, mE, bar, z0 - 4, y0 - 4, P);
            tma_load_3d(s + MT_A * MBOX, mA, bar, z0 - 4, y0 - 4, P);
            tma_load_3d(s + MT_F * MBOX, mF, bar, z0 - 4, y0 - 4, P);
            if (PHYS == TTI) {
                tma_load_3d(s + MT_ST * MBOX, mST, bar, z0 - 4, y0 - 4, P);
                tma_load_3d(s + MT_CT * MBOX, mCT, bar, z0 - 4, y0 - 4, P);
                tma_load_3d(s + MT_SP * MBOX, mSP, bar, z0 - 4, y0 - 4, P);
                tma_load_3d(s + MT_CP * MBOX, mCP, bar, z0 - 4, y0 - 4, P);
            }
            tma_load_3d(c + C_PO * CBOX, mPO, bar, z0, y0, j);
            tma_load_3d(c + C_MO * CBOX, mMO, bar, z0, y0, j);
            tma_load_3d(c + C_V * CBOX, mV, bar, z0, y0, j);
            tma_load_3d(c + C_Q * CBOX, mQ, bar, z0, y0, j);
            tma_load_3d(c + C_B * CBOX, mBC, bar, z0, y0, j);
        };
        // antisymmetric image p[-k] = -p[k] (k = 1..3) above the free surface, in one ring plane
        auto image_plane = [&](unsigned gidx) {
            if (tid < 2 * 23) {
                float *s = sm + OFF_RING + (gidx % NR) * R_SLOT + (tid / 23) * RBOX + (3 + tid % 23) * RZW;
                // column of kz is kz + 8
                s[7] = -s[9];
                s[6] = -s[10];
                s[5] = -s[11];
            }
        };

        if (tid == ISSUER) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            const int nr0 = nplanes < 8 + DR ? nplanes : 8 + DR;
            for (int rp = 0; rp < nr0; rp++) issue_ring(rp, r_issued + rp);
            r_issued += nr0;
            const int nm0 = niter < DM ? niter : DM;
            for (int q = 0; q < nm0; q++) issue_stage(q, m_issued + q);
            m_issued += nm0;
        }
        // the first eight ring planes
        bool fail = false;
        for (int rp = 0; rp < 8 && rp < nplanes && !fail; rp++) {
            if (mbar_wait(&rbar[(rseq + rp) % NR], ((rseq + rp) / NR) & 1u)) r_done = rseq + rp + 1;
            else fail = true;
        }
        if (top)
            for (int rp = 0; rp < 8 && rp < nplanes; rp++) image_plane(rseq + rp);
        if (fail) {
            atomicExch(abort_flag, 1);
            atomicOr(&d_status, 1u);
        }
        __syncthreads();

        float2 qx[8][2], qc[4][4], qh[4][2];
#pragma unroll
        for (int i = 0; i < 8; i++) qx[i][0] = qx[i][1] = bc2(0.0f);
#pragma unroll
        for (int i = 0; i < 4; i++) {
#pragma unroll
            for (int f = 0; f < 4; f++) qc[i][f] = bc2(0.0f);
            qh[i][0] = qh[i][1] = bc2(0.0f);
        }

        bool stop = *abort_flag != 0;
        // ring slot of plane q (the oldest of the eight in use) and slot/parity of plane q + 7, kept
        // incrementally (no division by NR per plane)
        unsigned rs0 = rseq % NR;
        unsigned rw = (rseq + 7) % NR, rwpar = ((rseq + 7) / NR) & 1u;
        const bool yz_tile = yok(g, y) && zok(g, z), yz_halo = yok(g, hy) && zok(g, hz);
        for (int q = 0; q < niter && !stop; q++) {
            const long j = jstart + q;
            const long P = j + 3;
            if (tid == ISSUER) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (q + 8 + DR - 1 < nplanes && q >= 1) {
                    issue_ring(q + 8 + DR - 1, r_issued);
                    r_issued++;
                }
                if (q + DM < niter) {
                    issue_stage(q + DM, m_issued);
                    m_issued++;
                }
            }
            // the epilogue's inputs of plane j, loaded now so that their latency hides behind the waits
            // and pass 1 (born: dV, DP, DM; imaging: the image, DP, DM)
            float2 ea = bc2(0.0f), eb = bc2(0.0f), ec = bc2(0.0f);
            if (EPI && own && j >= xbeg) {
                const long k = j * g.sx + (long)y * g.nz + z;
                if (F.epi.born_dv) {
                    ea = __ldg(reinterpret_cast<const float2 *>(F.epi.born_dv + k));
                    eb = __ldg(reinterpret_cast<const float2 *>(F.epi.born_dp + k));
                    ec = __ldg(reinterpret_cast<const float2 *>(F.epi.born_dm + k));
                } else if (F.epi.img) {
                    ea = ld2(F.epi.img + k);
                    eb = __ldg(reinterpret_cast<const float2 *>(F.epi.img_dp + k));
                    ec = __ldg(reinterpret_cast<const float2 *>(F.epi.img_dm + k));
                }
            }
            bool ok_w = true;
            if (q >= 1 && q + 7 < nplanes) {
                const unsigned gi = rseq + q + 7;
                ok_w = mbar_wait(&rbar[rw], rwpar);
                if (ok_w) r_done = gi + 1;
                if (top && ok_w) image_plane(gi);
            }
            const unsigned ms = mseq + q;
            if (ok_w && mbar_wait(&mbar[ms % NM], (ms / NM) & 1u)) m_done = ms + 1;
            else ok_w = false;
            if (!ok_w) {
                atomicExch(abort_flag, 1);
                atomicOr(&d_status, 1u);
            }
            const float *ring[8];
            {
                const float *r0 = sm + OFF_RING + rs0 * R_SLOT;
#pragma unroll
                for (int i = 0; i < 8; i++) ring[i] = r0 + (rs0 + i >= NR ? (i - NR) * R_SLOT : i * R_SLOT);
            }
            const float *mat = sm + OFF_MAT + (ms % NM) * M_STAGE;
            const bool pin = P >= 4 && P < g.nx - 4;

            // pass 1 at the lead plane: the tile pair, then the halo pair
            const Out6 c = pass1<PHYS, 0>(g, ring, mat, row + 4, 4 + 2 * zp, pin && yz_tile, top && zp == 0);
            float2 h0 = bc2(0.0f), h1 = bc2(0.0f);
            // (the z-halo pairs above the free surface hold images, written by the tile pairs)
            if (h_kind == 1) {
                const Out6 h = pass1<PHYS, 1>(g, ring, mat, h_er, h_ec, pin && yz_halo, top && zp == 0);
                h0 = h.py;
                h1 = h.my;
            } else if (h_kind == 2 && !(top && h_ec < 4)) {
                const Out6 h = pass1<PHYS, 2>(g, ring, mat, h_er, h_ec, pin && yz_halo, false);
                h0 = h.pz;
                h1 = h.mz;
            }
            float2 sx[2], cj[4], hj[2];
            switch (q & 7) {
                case 0: queue_phase<0>(g, qx, qc, qh, c, h0, h1, sx, cj, hj); break;
                case 1: queue_phase<1>(g, qx, qc, qh, c, h0, h1, sx, cj, hj); break;
                case 2: queue_phase<2>(g, qx, qc, qh, c, h0, h1, sx, cj, hj); break;
                case 3: queue_phase<3>(g, qx, qc, qh, c, h0, h1, sx, cj, hj); break;
                case 4: queue_phase<4>(g, qx, qc, qh, c, h0, h1, sx, cj, hj); break;
                case 5: queue_phase<5>(g, qx, qc, qh, c, h0, h1, sx, cj, hj); break;
                case 6: queue_phase<6>(g, qx, qc, qh, c, h0, h1, sx, cj, hj); break;
                default: queue_phase<7>(g, qx, qc, qh, c, h0, h1, sx, cj, hj); break;
            }
            const bool pass2 = j >= xbeg;
            if (pass2) {
                // y/z outputs of plane j into shared memory
                st2(TYs + (row + 4) * TZ + 2 * zp, cj[0]);
                st2(TYs + TYR * TZ + (row + 4) * TZ + 2 * zp, cj[2]);
                st2(TZs + row * TZW + 4 + 2 * zp, cj[1]);
                st2(TZs + TY * TZW + row * TZW + 4 + 2 * zp, cj[3]);
                if (top && zp < 2) {
                    // symmetric image t[-k] = t[k-1] of the z outputs above the free surface
                    st2(TZs + row * TZW + 2 - 2 * zp, make_float2(cj[1].y, cj[1].x));
                    st2(TZs + TY * TZW + row * TZW + 2 - 2 * zp, make_float2(cj[3].y, cj[3].x));
                }
                if (h_kind == 1) {
                    st2(TYs + h_er * TZ + h_ec - 4, hj[0]);
                    st2(TYs + TYR * TZ + h_er * TZ + h_ec - 4, hj[1]);
                } else if (h_kind == 2 && !(top && h_ec < 4)) {
                    st2(TZs + (h_er - 4) * TZW + h_ec, hj[0]);
                    st2(TZs + TY * TZW + (h_er - 4) * TZW + h_ec, hj[1]);
                }
            }
            __syncthreads();
            if (pass2 && own) {
                // pass 2 at plane j (prop3DAcoTTIDenQ_DEO2_FDTD.h:1420-1421, VTI .h:1372-1378)
                const float *cs = mat + NMAT * MBOX;
                const int o = row * TZ + 2 * zp;
                float2 L[2];
#pragma unroll
                for (int f = 0; f < 2; f++) {
                    const float *ty = TYs + f * TYR * TZ + row * TZ + 2 * zp;
                    const float2 dy = st8d(g, g.idy, ld2(ty), ld2(ty + TZ), ld2(ty + 2 * TZ), ld2(ty + 3 * TZ),
                                           ld2(ty + 4 * TZ), ld2(ty + 5 * TZ), ld2(ty + 6 * TZ), ld2(ty + 7 * TZ));
                    float v[10];
                    load10(v, TZs + f * TY * TZW + row * TZW + 2 * zp);
                    const float2 dz = st8zd(g, g.idz, v, 0);
                    L[f] = add2(add2(sx[f], dy), dz);  // dx + dy + dz (sx[f] is dx)
                }
                const bool ok = j >= 4 && j < g.nx - 4 && yz_tile;
                if (top && zp == 0) {  // free-surface row: every derivative is zero
                    L[0].x = 0.0f + 0.0f + 0.0f;
                    L[1].x = 0.0f + 0.0f + 0.0f;
                }
                const float2 V = ld2(cs + C_V * CBOX + o), Q = ld2(cs + C_Q * CBOX + o), B = ld2(cs + C_B * CBOX + o);
                const float2 k2 = div2(mul2(mul2(bc2(g.dt2), V), V), B);
                const long k = j * g.sx + (long)y * g.nz + z;
                const int ro = (row + 7) * RZW + 8 + 2 * zp;
                // Born-V injection fused after the step (prop3DAcoTTIDenQ_DEO2_FDTD.h:423-452):
                // new += 2 dt^2 dV/V * DP (DM), every cell
                float2 bfac = bc2(0.0f);
                if (EPI && F.epi.born_dv) bfac = div2(mul2(bc2(2.0f * g.dt * g.dt), ea), V);
#pragma unroll
                for (int f = 0; f < 2; f++) {
                    const float2 pc = ld2(ring[0] + f * RBOX + ro);
                    const float2 po = ld2(cs + (f == 0 ? C_PO : C_MO) * CBOX + o);
                    const float2 t = sub2(sub2(mul2(k2, L[f]), mul2(Q, sub2(pc, po))), po);
                    const float2 np = add2(t, mul2(bc2(2.0f), pc));
                    float2 nv = ok ? np : po;
                    if (EPI && F.epi.born_dv) nv = add2(nv, mul2(bfac, f == 0 ? eb : ec));
                    st2((f == 0 ? out_pold : out_mold) + k, nv);
                    if (!LINEAR) {
                        float2 sp = ok ? L[f] : bc2(0.0f);
                        // ScaleSpatialDerivatives fused (.h:387-415): pSpace, mSpace *= V^2/B
                        if (EPI && F.epi.scale_space) sp = mul2(sp, div2(mul2(V, V), B));
                        st2((f == 0 ? out_pspace : out_mspace) + k, sp);
                    }
                }
                if (EPI && F.epi.img) {
                    // imaging condition fused after the step (.h:567-592): img += 2B/V^3 (DP pOld + DM
                    // mOld), pOld/mOld being this step's input pCur/mCur
                    const float2 pcp = ld2(ring[0] + ro), pcm = ld2(ring[0] + RBOX + ro);
                    const float2 fac = div2(mul2(bc2(2.0f), B), mul2(mul2(V, V), V));
                    st2(F.epi.img + k, add2(ea, mul2(fac, add2(mul2(eb, pcp), mul2(ec, pcm)))));
                }
                if (!BATCH && F.illum) {
                    // source illumination, every cell: sum += pCur^2 (separate IEEE multiply and add,
                    // as illumination.c:31-53 does)
                    const float2 pcp = ld2(ring[0] + ro);
                    float2 a = ld2(F.illum + k);
                    a.x = __fadd_rn(a.x, __fmul_rn(pcp.x, pcp.x));
                    a.y = __fadd_rn(a.y, __fmul_rn(pcp.y, pcp.y));
                    st2(F.illum + k, a);
                }
            }
            __syncthreads();
            if (*abort_flag) stop = true;
            rs0 = rs0 + 1 == NR ? 0u : rs0 + 1;
            rw = rw + 1 == NR ? 0u : rw + 1;
            rwpar ^= rw == 0 ? 1u : 0u;
        }
        rseq += nplanes;
        mseq += niter;
        if (stop) break;
    }
    if (*abort_flag && tid == ISSUER) {
        for (unsigned gi = r_done; gi < r_issued; gi++) mbar_wait(&rbar[gi % NR], (gi / NR) & 1u, 100000000ull);
        for (unsigned gi = m_done; gi < m_issued; gi++) mbar_wait(&mbar[gi % NM], (gi / NM) & 1u, 100000000ull);
    }
}

bool aniso_maps(const Grid &g, int phys, const Fields &F, CUtensorMap *m) {
    const float *srcs[15] = {F.pcur, F.mcur, F.b, F.eps, F.eta, F.f, F.st, F.ct, F.sp, F.cp,
                             F.pold, F.mold, F.v, F.q, F.b};
    for (int i = 0; i < 15; i++) {
        const float *src = srcs[i];
        if (phys != TTI && i >= 6 && i <= 9) src = F.b;  // unused by VTI: any valid map
        unsigned bz = i < 2 ? RZW : (i < 10 ? MZW : TZ);
        unsigned by = i < 2 ? RYH : (i < 10 ? MYH : TY);
        if (!make_tensor_map_3d(&m[i], src, g.nx, g.ny, g.nz, bz, by, 1)) return false;
    }
    return true;
}

template <int PHYS, bool LINEAR>
int aniso_grid_cap() {
    static int cap = 0;
    if (!cap) {
        for (auto kern : {k_aniso3d_tma<PHYS, LINEAR, false>, k_aniso3d_tma<PHYS, LINEAR, true>,
                          k_aniso3d_tma<PHYS, LINEAR, false, true>})
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_aniso3d_tma<PHYS, LINEAR, false>, NT, SMEM_BYTES);
        cap = sms * (per > 0 ? per : 1);
    }
    return cap;
}

template <int PHYS, bool LINEAR>
bool launch(const Grid &g, const Fields &F, cudaStream_t s) {
    AnisoMaps M;
    if (!aniso_maps(g, PHYS, F, M.m)) return false;
    const int grid_cap = aniso_grid_cap<PHYS, LINEAR>();
    const int ntz = (int)((g.nz + TZ - 1) / TZ);
    const int nty = (int)((g.ny + TY - 1) / TY);
    const long tiles = (long)ntz * nty;
    int best_nch = 1;
    double best_cost = 1e30;
    for (int nch = 1; nch <= 64 && nch <= g.nx / 16 + 1; nch++) {
        const long chunk = (g.nx + nch - 1) / nch;
        const long items = tiles * nch;
        const double waves = (double)((items + grid_cap - 1) / grid_cap);
        const double cost = waves * (double)(chunk + WARMUP * 0.6);
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
        k_aniso3d_tma<PHYS, LINEAR, false, true><<<grid, NT, SMEM_BYTES, s>>>(g, F, M, ntz, nty, nch, xchunk, nullptr,
                                                                              nullptr, nullptr, 0, nullptr);
    else
        k_aniso3d_tma<PHYS, LINEAR, false><<<grid, NT, SMEM_BYTES, s>>>(g, F, M, ntz, nty, nch, xchunk, nullptr,
                                                                        nullptr, nullptr, 0, nullptr);
    return true;
}

}  // namespace

bool fused_aniso3d_tma(const Grid &g, int phys, int linear, const Fields &F, cudaStream_t s) {
    if (g.ndim != 3 || g.nz % 4 != 0) return false;
    if (phys == TTI) return linear ? false : launch<TTI, false>(g, F, s);
    if (phys == VTI) return linear ? launch<VTI, true>(g, F, s) : launch<VTI, false>(g, F, s);
    return false;
}

bool aniso3d_tma_describe(const Grid &g, int phys, const Fields &F, int xchunk, AnisoShotDesc *d, TileInfo *t) {
    if (phys == VTI) return vti3d_tma_describe(g, F, xchunk, d, t);  // batched VTI uses the queue kernel
    if (g.ndim != 3 || g.nz % 4 != 0 || xchunk < 1 || phys != TTI) return false;
    if (d) {
        if (!aniso_maps(g, phys, F, d->m)) return false;
        d->pold = F.pold;
        d->mold = F.mold;
        d->pspace = F.pspace;
        d->mspace = F.mspace;
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
        t->grid_cap = aniso_grid_cap<TTI, false>();
    }
    return true;
}

void aniso3d_tma_batch(const Grid &gc, int phys, const AnisoShotDesc *shots, const int *sel, const int2 *items,
                       int nitems, int *counter, int grid, cudaStream_t s) {
    if (phys == TTI) {
        aniso_grid_cap<TTI, false>();
        k_aniso3d_tma<TTI, false, true><<<grid, NT, SMEM_BYTES, s>>>(gc, Fields{}, AnisoMaps{}, 0, 0, 0, 1, shots,
                                                                     sel, items, nitems, counter);
    } else {
        vti3d_tma_batch(gc, shots, sel, items, nitems, counter, grid, s);
    }
}

void aniso3d_set_pipeline_wait(unsigned long long ns) {
    const uint64_t v = ns;
    cudaMemcpyToSymbol(wfd_dev::d_pipeline_wait_ns, &v, sizeof(v));
}

unsigned aniso3d_status_and_clear() {
    unsigned v = 0, z = 0;
    cudaMemcpyFromSymbol(&v, d_status, sizeof(v));
    if (v) cudaMemcpyToSymbol(d_status, &z, sizeof(z));
    return v;
}

}  // namespace WFD_NS
