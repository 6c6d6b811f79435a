// Fused single-sweep 3D VTI step with TMA-staged tiles: both reference passes in one kernel
// (prop3DAcoVTIDenQ_DEO2_FDTD.h:326-376; pass 1 :945-957, update :1372-1378, linear :1697-1698).
// HBM traffic per cell: read pCur, mCur, pOld, mOld, V, B, eps, eta, f, Q; write pOld, mOld,
// pSpace, mSpace (56 B; 48 B for the linear step, which writes no pSpace/mSpace).
//
// VTI's pass-1 outputs on the halo need only y (rows above/below the tile) or z (columns beside
// it) derivatives, so, as in the isotropic kernel, the x derivative is formed from register queues
// on the tile and only the centre plane is staged with its halo. A CTA of 256 threads owns a (z,y)
// tile of 32 x 16 columns and sweeps a chunk of x planes. Per plane j one thread issues a group of
// TMA tile loads on one mbarrier, one plane ahead (2 stages, 102 KB, 2 CTAs per SM):
//   pCur(j), mCur(j) with halo (48 x 30 at z0-8, y0-7); b, eps, eta, f (j) with halo (40 x 24 at
//   z0-4, y0-4); pCur(j+7), mCur(j+7); b, eps, f (j+3); pOld, mOld, V, Q (j)  (32 x 16 each).
// A thread owns a pair of consecutive z cells of one row and keeps, per field, a register queue of
// pCur (planes j..j+7) and of the pass-1 x output (planes j-4..j+3); slot = plane mod 8, one code
// path per phase. The pass-1 y outputs of plane j on the 24 halo-extended rows (threads 0-95, one
// field, one quad, four rows sliding along y) and the z outputs on the 40 extended columns (threads
// 96-255, both fields, one quad each) go to shared memory; then every thread applies D- and the time
// update to its pair and stores pOld, mOld (and pSpace, mSpace). Arithmetic on float2 pairs with
// the packed FP32 instructions; the strict build uses separate IEEE multiply and add in the
// reference's order (bitwise equal to the reference). Region rules are selects; the free-surface
// images (antisymmetric pCur/mCur above kz = 0 in the z derivative, symmetric z outputs in D-) only
// in the top tile. Persistent CTAs loop over (tile, x-chunk) items; chunks start with 14 warm-up
// planes that only fill the queues (their groups load the queue boxes alone). Waits are bounded;
// on timeout the kernel records an error in a device status word and leaves. With an illumination
// sum attached (single objects), each cell's pCur^2 is added to it as the cell is updated.
// Requires nz % 4 == 0.
#include "wfd_kernels.h"
#include "wfd_tma.cuh"

namespace WFD_NS {
using namespace wfd;
using namespace wfd_dev;

namespace {

constexpr int TZ = 32, TY = 16, NT = 256;
constexpr int D = 1;       // prefetch distance in planes
constexpr int NS = D + 1;  // stages
constexpr int PZW = TZ + 16, PYH = TY + 14, PH_ = PZW * PYH;  // field halo box 48 x 30 at (z0-8, y0-7)
constexpr int MZW = TZ + 8, MYH = TY + 8, MH_ = MZW * MYH;    // material halo box 40 x 24 at (z0-4, y0-4)
constexpr int OS = TZ * TY;                                   // tile box 32 x 16
constexpr int TYR = TY + 8;                                   // y outputs: rows y0-4 .. y0+19
constexpr int TZW = TZ + 8;                                   // z outputs: columns z0-4 .. z0+35
// stage layout (floats)
constexpr int S_PH = 0, S_MH = S_PH + PH_, S_BH = S_MH + PH_, S_EH = S_BH + MH_, S_AH = S_EH + MH_,
              S_FH = S_AH + MH_, S_PN = S_FH + MH_, S_MN = S_PN + OS, S_BN = S_MN + OS, S_EN = S_BN + OS,
              S_FN = S_EN + OS, S_PO = S_FN + OS, S_MO = S_PO + OS, S_V = S_MO + OS, S_Q = S_V + OS,
              STAGE = S_Q + OS;
constexpr unsigned GROUP_BYTES = 4u * STAGE;
constexpr unsigned WARM_BYTES = 4u * 5 * OS;  // warm-up planes: pCur, mCur (j+7), b, eps, f (j+3)
constexpr int WARMUP = 14;
// The thread that issues the TMA copies: lane 0 of warp 7, a warp of halo z tasks (the lighter
// kind), so that the issue does not lengthen the busiest warps' planes.
constexpr int ISSUER = 224;
constexpr int OFF_TY = NS * STAGE;              // [2][TYR][TZ]
constexpr int OFF_TZ = OFF_TY + 2 * TYR * TZ;   // [2][TY][TZW]
constexpr int OFF_BAR = OFF_TZ + 2 * TY * TZW;
constexpr size_t SMEM_BYTES = (size_t)OFF_BAR * 4 + NS * 8 + 16;
static_assert(OFF_BAR % 2 == 0, "mbarrier alignment");
static_assert((STAGE * 4) % 128 == 0 && (PH_ * 4) % 128 == 0 && (MH_ * 4) % 128 == 0 && (OS * 4) % 128 == 0,
              "TMA destination alignment");

__device__ unsigned int d_status;

__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(float *p, float2 v) { *reinterpret_cast<float2 *>(p) = v; }
__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4 *>(p) = v; }
__device__ __forceinline__ float2 bc2(float s) { return make_float2(s, s); }
#if WFD_STRICT
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return make_float2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return add2(mul2(a, b), c); }
__device__ __forceinline__ float mul1(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add1(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
// a - b written as the reference's -b + a
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return add2(neg2(b), a); }
#else
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float mul1(float a, float b) { return a * b; }
__device__ __forceinline__ float add1(float a, float b) { return a + b; }
// Subtraction as one packed instruction: b * -1 is exact, so b * -1 + a rounds once, like -b + a (a
// negated operand of the packed add would cost two scalar instructions).
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
#endif
__device__ __forceinline__ float2 sqrt2(float2 a) { return make_float2(sqrtf(a.x), sqrtf(a.y)); }
__device__ __forceinline__ float2 div2(float2 a, float2 b) { return make_float2(a.x / b.x, a.y / b.y); }
__device__ __forceinline__ float at(const float4 &v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// 8-point staggered stencil c1(w4-w3) + c2(w5-w2) + c3(w6-w1) + c4(w7-w0), summed left to right:
// D+ with w = f(k-3..k+4), D- with w = f(k-4..k+3) (prop3DAcoIsoDenQ_DEO2_FDTD.h:846-864, :1113-1131)
__device__ __forceinline__ float2 st8(const Grid &g, float2 w0, float2 w1, float2 w2, float2 w3, float2 w4,
                                      float2 w5, float2 w6, float2 w7) {
    float2 s = mul2(bc2(g.c1), sub2(w4, w3));
    s = fma2(bc2(g.c2), sub2(w5, w2), s);
    s = fma2(bc2(g.c3), sub2(w6, w1), s);
    return fma2(bc2(g.c4), sub2(w7, w0), s);
}
__device__ __forceinline__ float st8s(const Grid &g, float w0, float w1, float w2, float w3, float w4, float w5,
                                      float w6, float w7) {
    float s = mul1(g.c1, add1(-w3, w4));
    s = add1(s, mul1(g.c2, add1(-w2, w5)));
    s = add1(s, mul1(g.c3, add1(-w1, w6)));
    return add1(s, mul1(g.c4, add1(-w0, w7)));
}

__device__ __forceinline__ bool y_in(const Grid &g, int y) { return y >= 4 && y < g.ny - 4; }
// cells of the pass-1 x/y outputs that the reference computes (free-surface row 0 holds zeros)
__device__ __forceinline__ bool xy_out_z(const Grid &g, int z) { return z < g.nz - 4 && (z >= 4 || (g.fs && z > 0)); }
// cells of the pass-1 z output and of the update
__device__ __forceinline__ bool z_out_z(const Grid &g, int z) { return z >= 0 && z < g.nz - 4 && (z >= 4 || g.fs); }

// Halo tasks of a plane: threads 0-95 form the pass-1 y outputs of one field on 4 extended rows
// and one quad (f = tid / 48; rows 4 ((tid % 48) >> 3) ..+3 of the 24 extended rows, quad tid & 7);
// threads 96-255 the z outputs of both fields on one tile row and one of the 10 extended-column
// quads (row (tid-96) / 10, quad (tid-96) % 10). Which cells the reference computes depends on x
// only through one flag, so the rest is a mask fixed for an item: bit 4 rr + m (y task, row
// r0+rr, cell m) or m (z task, cell m).
__device__ __forceinline__ unsigned ext_mask(const Grid &g, int tid, int z0, int y0) {
    unsigned mask = 0;
    if (tid < 96) {
        const int t = tid % 48, zz0 = z0 + 4 * (t & 7), r0 = (t >> 3) * 4;
#pragma unroll
        for (int rr = 0; rr < 4; rr++)
#pragma unroll
            for (int m = 0; m < 4; m++)
                if (y_in(g, y0 - 4 + r0 + rr) && xy_out_z(g, zz0 + m)) mask |= 1u << (4 * rr + m);
    } else {
        const int t = tid - 96, r = t / 10, zb = z0 - 4 + 4 * (t % 10);
#pragma unroll
        for (int m = 0; m < 4; m++)
            if (y_in(g, y0 + r) && z_out_z(g, zb + m)) mask |= 1u << m;
    }
    return mask;
}
__device__ __forceinline__ float2 keep2(unsigned mask, int bit, float2 v) {
    return make_float2((mask >> bit) & 1u ? v.x : 0.0f, (mask >> bit + 1) & 1u ? v.y : 0.0f);
}

// pass-1 y outputs of one field (`f`) on 4 extended rows r0..r0+3 (y = y0-4+r) and one quad zq of
// the centre plane, the 8-row window sliding along y: P: b*(1+2eps)*dy p; M: b*(1-f)*dy m
__device__ __forceinline__ void ext_y(const Grid &g, const unsigned em, const int f, const int zq, const int r0,
                                      const float *st, float *TYs) {
    const float *Fc = st + (f == 0 ? S_PH : S_MH);
    float4 w[11];
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = ld4(Fc + (r0 + i) * PZW + 8 + 4 * zq);
#pragma unroll
    for (int rr = 0; rr < 4; rr++) {
        const int r = r0 + rr;
        if (rr > 0)  // the window slides one row (row 30 would only feed the unused padding row 23)
            w[rr + 7] = r0 + rr + 7 < PYH ? ld4(Fc + (r0 + rr + 7) * PZW + 8 + 4 * zq) : make_float4(0.f, 0.f, 0.f, 0.f);
        const float4 b = ld4(st + S_BH + r * MZW + 4 + 4 * zq);
        const float4 e = ld4(st + (f == 0 ? S_EH : S_FH) + r * MZW + 4 + 4 * zq);
        float o[4];
#pragma unroll
        for (int m = 0; m < 4; m += 2) {
            const float2 s = st8(g, make_float2(at(w[rr], m), at(w[rr], m + 1)),
                                 make_float2(at(w[rr + 1], m), at(w[rr + 1], m + 1)),
                                 make_float2(at(w[rr + 2], m), at(w[rr + 2], m + 1)),
                                 make_float2(at(w[rr + 3], m), at(w[rr + 3], m + 1)),
                                 make_float2(at(w[rr + 4], m), at(w[rr + 4], m + 1)),
                                 make_float2(at(w[rr + 5], m), at(w[rr + 5], m + 1)),
                                 make_float2(at(w[rr + 6], m), at(w[rr + 6], m + 1)),
                                 make_float2(at(w[rr + 7], m), at(w[rr + 7], m + 1)));
            const float2 d = mul2(bc2(g.idy), s);
            const float2 bv = make_float2(at(b, m), at(b, m + 1)), ev = make_float2(at(e, m), at(e, m + 1));
            // prop3DAcoVTIDenQ_DEO2_FDTD.h:945-957: b*E (E = 1 + 2 eps) for P, b*(1 - f) for M
            const float2 k = f == 0 ? mul2(bv, fma2(bc2(2.0f), ev, bc2(1.0f))) : mul2(bv, sub2(bc2(1.0f), ev));
            const float2 t = keep2(em, 4 * rr + m, mul2(k, d));
            o[m] = t.x;
            o[m + 1] = t.y;
        }
        st4(TYs + f * TYR * TZ + r * TZ + 4 * zq, make_float4(o[0], o[1], o[2], o[3]));
    }
}

// pass-1 z outputs of both fields on tile row r and extended quad qi (column 4*qi is z = z0-4+4*qi);
// in the top tile the task of quad 1 also writes quad 0, the symmetric image t[-k] = t[k-1] above
// the free surface, and the task of quad 0 does nothing.
__device__ __forceinline__ void ext_z(const Grid &g, const unsigned em, const bool top, const int r, const int qi,
                                      const float *st, float *TZs) {
    if (top && qi == 0) return;
    const bool img = top && qi == 1;  // cells z = 0, 1, 2 reach above the free surface
    float d[2][4];                    // idz * D+z of p and m on the quad
#pragma unroll
    for (int f = 0; f < 2; f++) {
        const float *row = st + (f == 0 ? S_PH : S_MH) + (r + 7) * PZW;
        float v[12];
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float4 a = ld4(row + 4 * (qi + i));
            v[4 * i] = a.x, v[4 * i + 1] = a.y, v[4 * i + 2] = a.z, v[4 * i + 3] = a.w;
        }
#pragma unroll
        for (int m = 0; m < 4; m += 2) {
            auto win = [&](int i) { return make_float2(v[m + 1 + i], v[m + 2 + i]); };
            float2 sv = st8(g, win(0), win(1), win(2), win(3), win(4), win(5), win(6), win(7));
            if (img) {
                // antisymmetric image above the free surface, p[-j] = -p[j]; column of z is z + 8
                auto pm = [&](int jz) { return jz >= 0 ? row[jz + 8] : -row[-jz + 8]; };
                if (m == 0) {
                    sv.x = st8s(g, pm(-3), pm(-2), pm(-1), pm(0), pm(1), pm(2), pm(3), pm(4));
                    sv.y = st8s(g, pm(-2), pm(-1), pm(0), pm(1), pm(2), pm(3), pm(4), pm(5));
                } else {
                    sv.x = st8s(g, pm(-1), pm(0), pm(1), pm(2), pm(3), pm(4), pm(5), pm(6));
                }
            }
            const float2 dv = mul2(bc2(g.idz), sv);
            d[f][m] = dv.x;
            d[f][m + 1] = dv.y;
        }
    }
    const float4 b4 = ld4(st + S_BH + (r + 4) * MZW + 4 * qi);
    const float4 f4 = ld4(st + S_FH + (r + 4) * MZW + 4 * qi);
    const float4 a4 = ld4(st + S_AH + (r + 4) * MZW + 4 * qi);
    float op[4], om[4];
#pragma unroll
    for (int m = 0; m < 4; m += 2) {
        const float2 dPz = make_float2(d[0][m], d[0][m + 1]), dMz = make_float2(d[1][m], d[1][m + 1]);
        const float2 bv = make_float2(at(b4, m), at(b4, m + 1)), fv = make_float2(at(f4, m), at(f4, m + 1));
        const float2 eta = make_float2(at(a4, m), at(a4, m + 1));
        // prop3DAcoVTIDenQ_DEO2_FDTD.h:945-957
        const float2 one = bc2(1.0f);
        const float2 FA = mul2(fv, eta);
        const float2 FAA = mul2(FA, eta);
        const float2 SA2 = sqrt2(sub2(one, mul2(eta, eta)));
        const float2 tp = fma2(mul2(bv, mul2(FA, SA2)), dMz, mul2(mul2(bv, sub2(one, FAA)), dPz));
        const float2 tm = fma2(mul2(bv, add2(sub2(one, fv), FAA)), dMz, mul2(mul2(mul2(mul2(bv, fv), eta), SA2), dPz));
        const float2 kp = keep2(em, m, tp), km = keep2(em, m, tm);
        op[m] = kp.x;
        op[m + 1] = kp.y;
        om[m] = km.x;
        om[m + 1] = km.y;
    }
    float *tp = TZs + r * TZW + 4 * qi, *tm = TZs + TY * TZW + r * TZW + 4 * qi;
    st4(tp, make_float4(op[0], op[1], op[2], op[3]));
    st4(tm, make_float4(om[0], om[1], om[2], om[3]));
    if (img) {
        st4(tp - 4, make_float4(op[3], op[2], op[1], op[0]));
        st4(tm - 4, make_float4(om[3], om[2], om[1], om[0]));
    }
}

// Queue update of phase PH = q & 7 for the pair: pCur/mCur(j+7) enter qp slot (PH+7)&7, the pass-1
// x outputs at plane j+3 enter qt slot (PH+7)&7; returns the D- x stencils at plane j and pCur(j).
template <int PH>
__device__ __forceinline__ void queue_phase(const Grid &g, float2 (&qp)[8][2], float2 (&qt)[8][2], const float2 pn,
                                            const float2 mn, const float2 bn, const float2 en, const float2 fn,
                                            const bool okx0, const bool okx1, float2 (&sx)[2], float2 (&pc)[2]) {
    constexpr int N = (PH + 7) & 7;
    qp[N][0] = pn;
    qp[N][1] = mn;
    const float2 one = bc2(1.0f);
    // prop3DAcoVTIDenQ_DEO2_FDTD.h:945-957: b*E*dx p, b*(1-f)*dx m
    const float2 kp = mul2(bn, fma2(bc2(2.0f), en, one));
    const float2 km = mul2(bn, sub2(one, fn));
#pragma unroll
    for (int f = 0; f < 2; f++) {
        const float2 s = st8(g, qp[(PH + 0) & 7][f], qp[(PH + 1) & 7][f], qp[(PH + 2) & 7][f], qp[(PH + 3) & 7][f],
                             qp[(PH + 4) & 7][f], qp[(PH + 5) & 7][f], qp[(PH + 6) & 7][f], qp[N][f]);
        float2 t = mul2(f == 0 ? kp : km, mul2(bc2(g.idx), s));
        t.x = okx0 ? t.x : 0.0f;
        t.y = okx1 ? t.y : 0.0f;
        qt[N][f] = t;
    }
#pragma unroll
    for (int f = 0; f < 2; f++) {
        sx[f] = st8(g, qt[(PH + 0) & 7][f], qt[(PH + 1) & 7][f], qt[(PH + 2) & 7][f], qt[(PH + 3) & 7][f],
                    qt[(PH + 4) & 7][f], qt[(PH + 5) & 7][f], qt[(PH + 6) & 7][f], qt[N][f]);
        pc[f] = qp[PH][f];
    }
}

template <bool LINEAR, bool BATCH, bool EPI = false>
__global__ void __launch_bounds__(NT, 2)
    k_vti3d_tma(Grid g0, Fields F, const __grid_constant__ AnisoMaps M, int ntz0, int nty0, int nch0, int xchunk0,
                const AnisoShotDesc *__restrict__ shots, const int *__restrict__ sel, const int2 *__restrict__ items,
                int nitems, int *counter) {
    extern __shared__ __align__(1024) float sm[];
    float *TYs = sm + OFF_TY;
    float *TZs = sm + OFF_TZ;
    uint64_t *bars = reinterpret_cast<uint64_t *>(sm + OFF_BAR);
    int *abort_flag = reinterpret_cast<int *>(bars + NS);
    int *item_slot = abort_flag + 1;
    const int tid = threadIdx.x;
    if (tid == 0) {
        for (int s = 0; s < NS; s++) mbar_init(&bars[s], 1);
        fence_mbar_init();
        if (!BATCH)
            for (int i = 0; i < 15; i++) prefetch_tensor_map(&M.m[i]);
        *abort_flag = 0;
    }
    __syncthreads();

    const long total = (long)ntz0 * nty0 * nch0;
    unsigned gseq = 0;                  // groups consumed so far by this CTA
    unsigned out_from = 0, out_to = 0;  // groups issued but not yet consumed (issuing thread)
    const int zp = tid & 15, row = tid >> 4;

    for (long wstat = blockIdx.x;; wstat += gridDim.x) {
        Grid g = g0;
        const CUtensorMap *maps = M.m;
        float *o_po = F.pold, *o_mo = F.mold, *o_ps = F.pspace, *o_ms = F.mspace;
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
            o_po = d->pold;
            o_mo = d->mold;
            o_ps = d->pspace;
            o_ms = d->mspace;
            ntz = d->ntz;
            nty = d->nty;
            xchunk = d->xchunk;
            w = it.y;
        } else if (wstat >= total) {
            break;
        }
        const int tzi = (int)(w % ntz);
        const int tyi = (int)((w / ntz) % nty);
        const int chi = (int)(w / ((long)ntz * nty));
        const int z0 = tzi * TZ, y0 = tyi * TY;
        const int z = z0 + 2 * zp, y = y0 + row;
        const bool own = z < g.nz && y < g.ny;
        const long xbeg = (long)chi * xchunk;
        const long xend = xbeg + xchunk < g.nx ? xbeg + xchunk : g.nx;
        const long jstart = xbeg - WARMUP;
        const int ngroups = (int)(xend - jstart);
        const bool top = z0 == 0 && g.fs;
        const bool okxz0 = y_in(g, y) && xy_out_z(g, z), okxz1 = y_in(g, y) && xy_out_z(g, z + 1);
        const bool okz0 = y_in(g, y) && z_out_z(g, z), okz1 = y_in(g, y) && z_out_z(g, z + 1);
        const unsigned emask = ext_mask(g, tid, z0, y0);

        auto issue = [&](long jj, unsigned gs) {
            uint64_t *bar = &bars[gs % NS];
            float *s = sm + (gs % NS) * STAGE;
            const bool warm = jj < xbeg;
            mbar_expect_tx(bar, warm ? WARM_BYTES : GROUP_BYTES);
            tma_load_3d(s + S_PN, maps + 6, bar, z0, y0, (int)(jj + 7));
            tma_load_3d(s + S_MN, maps + 7, bar, z0, y0, (int)(jj + 7));
            tma_load_3d(s + S_BN, maps + 8, bar, z0, y0, (int)(jj + 3));
            tma_load_3d(s + S_EN, maps + 9, bar, z0, y0, (int)(jj + 3));
            tma_load_3d(s + S_FN, maps + 10, bar, z0, y0, (int)(jj + 3));
            if (!warm) {
                tma_load_3d(s + S_PH, maps + 0, bar, z0 - 8, y0 - 7, (int)jj);
                tma_load_3d(s + S_MH, maps + 1, bar, z0 - 8, y0 - 7, (int)jj);
                tma_load_3d(s + S_BH, maps + 2, bar, z0 - 4, y0 - 4, (int)jj);
                tma_load_3d(s + S_EH, maps + 3, bar, z0 - 4, y0 - 4, (int)jj);
                tma_load_3d(s + S_AH, maps + 4, bar, z0 - 4, y0 - 4, (int)jj);
                tma_load_3d(s + S_FH, maps + 5, bar, z0 - 4, y0 - 4, (int)jj);
                tma_load_3d(s + S_PO, maps + 11, bar, z0, y0, (int)jj);
                tma_load_3d(s + S_MO, maps + 12, bar, z0, y0, (int)jj);
                tma_load_3d(s + S_V, maps + 13, bar, z0, y0, (int)jj);
                tma_load_3d(s + S_Q, maps + 14, bar, z0, y0, (int)jj);
            }
        };
        if (tid == ISSUER) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            for (int q = 0; q < D && q < ngroups; q++) issue(jstart + q, gseq + q);
            out_from = gseq;
            out_to = gseq + (D < ngroups ? D : ngroups);
        }
        float2 qp[8][2], qt[8][2];
#pragma unroll
        for (int i = 0; i < 8; i++) qp[i][0] = qp[i][1] = qt[i][0] = qt[i][1] = bc2(0.0f);

        bool stop = false;
        for (int q = 0; q < ngroups; q++) {
            const long j = jstart + q;
            const unsigned gs = gseq + q;
            if (tid == ISSUER && q + D < ngroups) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                issue(j + D, gs + D);
                out_to = gs + D + 1;
            }
            // the epilogue's inputs of plane j, loaded now so that their latency hides behind the wait
            // and the pass-1 work (born: dV, DP, DM; imaging: the image, DP, DM)
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
            const bool landed = mbar_wait(&bars[gs % NS], (gs / NS) & 1u);
            if (!landed) {
                atomicExch(abort_flag, 1);
                atomicOr(&d_status, 1u);
            }
            // a group whose wait ran out may still be in flight: the drain below waits for it
            if (tid == ISSUER && landed) out_from = gs + 1;
            const float *st = sm + (gs % NS) * STAGE;
            float2 sx[2], pc[2];
            {
                const int o = row * TZ + 2 * zp;
                const float2 pn = ld2(st + S_PN + o), mn = ld2(st + S_MN + o);
                const float2 bn = ld2(st + S_BN + o), en = ld2(st + S_EN + o), fn = ld2(st + S_FN + o);
                const bool xin_a = j + 3 >= 4 && j + 3 < g.nx - 4;
                const bool k0 = xin_a && okxz0, k1 = xin_a && okxz1;
                switch (q & 7) {
                    case 0: queue_phase<0>(g, qp, qt, pn, mn, bn, en, fn, k0, k1, sx, pc); break;
                    case 1: queue_phase<1>(g, qp, qt, pn, mn, bn, en, fn, k0, k1, sx, pc); break;
                    case 2: queue_phase<2>(g, qp, qt, pn, mn, bn, en, fn, k0, k1, sx, pc); break;
                    case 3: queue_phase<3>(g, qp, qt, pn, mn, bn, en, fn, k0, k1, sx, pc); break;
                    case 4: queue_phase<4>(g, qp, qt, pn, mn, bn, en, fn, k0, k1, sx, pc); break;
                    case 5: queue_phase<5>(g, qp, qt, pn, mn, bn, en, fn, k0, k1, sx, pc); break;
                    case 6: queue_phase<6>(g, qp, qt, pn, mn, bn, en, fn, k0, k1, sx, pc); break;
                    default: queue_phase<7>(g, qp, qt, pn, mn, bn, en, fn, k0, k1, sx, pc); break;
                }
            }
            if (j >= xbeg) {
                const bool xin = j >= 4 && j < g.nx - 4;
                const unsigned em = xin ? emask : 0u;
                if (tid < 96) {  // 2 fields x 6 row groups x 8 quads
                    const int f = tid / 48, t = tid % 48;
                    ext_y(g, em, f, t & 7, (t >> 3) * 4, st, TYs);
                } else {  // 16 rows x 10 quads
                    const int t = tid - 96;
                    ext_z(g, em, top, t / 10, t % 10, st, TZs);
                }
                __syncthreads();
                if (own) {
                    // D- in y and z, the time update (prop3DAcoVTIDenQ_DEO2_FDTD.h:1372-1378)
                    const int o = row * TZ + 2 * zp;
                    float2 L[2];
#pragma unroll
                    for (int f = 0; f < 2; f++) {
                        const float *ty = TYs + f * TYR * TZ + row * TZ + 2 * zp;
                        const float2 sy = st8(g, ld2(ty), ld2(ty + TZ), ld2(ty + 2 * TZ), ld2(ty + 3 * TZ),
                                              ld2(ty + 4 * TZ), ld2(ty + 5 * TZ), ld2(ty + 6 * TZ), ld2(ty + 7 * TZ));
                        const float *tz = TZs + f * TY * TZW + row * TZW + 2 * zp;
                        float v[10];
#pragma unroll
                        for (int i = 0; i < 5; i++) {
                            const float2 a = ld2(tz + 2 * i);
                            v[2 * i] = a.x;
                            v[2 * i + 1] = a.y;
                        }
                        auto wz = [&](int i) { return make_float2(v[i], v[i + 1]); };
                        const float2 sz = st8(g, wz(0), wz(1), wz(2), wz(3), wz(4), wz(5), wz(6), wz(7));
                        L[f] = fma2(bc2(g.idz), sz, fma2(bc2(g.idy), sy, mul2(bc2(g.idx), sx[f])));
                    }
                    if (top && zp == 0) {  // free-surface row: every derivative is zero
                        L[0].x = 0.0f + 0.0f + 0.0f;
                        L[1].x = 0.0f + 0.0f + 0.0f;
                    }
                    const bool ok0 = xin && okz0, ok1 = xin && okz1;
                    const float2 V = ld2(st + S_V + o), Q = ld2(st + S_Q + o);
                    const float2 B = ld2(st + S_BH + (row + 4) * MZW + 4 + 2 * zp);
                    const float2 k2 = div2(mul2(mul2(bc2(g.dt2), V), V), B);
                    const long k = j * g.sx + (long)y * g.nz + z;
                    // Born-V injection fused after the step (prop3DAcoVTIDenQ_DEO2_FDTD.h:420-452):
                    // new += 2 dt^2 dV/V * DP (DM), every cell
                    float2 bfac = bc2(0.0f);
                    if (EPI && F.epi.born_dv) bfac = div2(mul2(bc2(2.0f * g.dt * g.dt), ea), V);
#pragma unroll
                    for (int f = 0; f < 2; f++) {
                        const float2 po = ld2(st + (f == 0 ? S_PO : S_MO) + o);
                        const float2 t = sub2(sub2(mul2(k2, L[f]), mul2(Q, sub2(pc[f], po))), po);
                        const float2 np = add2(t, mul2(bc2(2.0f), pc[f]));
                        float2 nv = make_float2(ok0 ? np.x : po.x, ok1 ? np.y : po.y);
                        if (EPI && F.epi.born_dv) nv = add2(nv, mul2(bfac, f == 0 ? eb : ec));
                        st2((f == 0 ? o_po : o_mo) + k, nv);
                        if (!LINEAR) {
                            float2 sp = make_float2(ok0 ? L[f].x : 0.0f, ok1 ? L[f].y : 0.0f);
                            // ScaleSpatialDerivatives fused (.h:384-407): pSpace, mSpace *= V^2/B
                            if (EPI && F.epi.scale_space) sp = mul2(sp, div2(mul2(V, V), B));
                            st2((f == 0 ? o_ps : o_ms) + k, sp);
                        }
                    }
                    if (EPI && F.epi.img) {
                        // imaging condition fused after the step (.h:564-589): img += 2B/V^3 (DP pOld +
                        // DM mOld), pOld/mOld being this step's input pCur/mCur
                        const float2 fac = div2(mul2(bc2(2.0f), B), mul2(mul2(V, V), V));
                        st2(F.epi.img + k, add2(ea, mul2(fac, add2(mul2(eb, pc[0]), mul2(ec, pc[1])))));
                    }
                    if (!BATCH && F.illum) {
                        // source illumination, every cell: sum += pCur^2 (separate IEEE multiply and
                        // add, as illumination.c:31-53 does)
                        float2 a = ld2(F.illum + k);
                        a.x = __fadd_rn(a.x, __fmul_rn(pc[0].x, pc[0].x));
                        a.y = __fadd_rn(a.y, __fmul_rn(pc[0].y, pc[0].y));
                        st2(F.illum + k, a);
                    }
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
    if (*abort_flag && tid == ISSUER) {
        for (unsigned gs = out_from; gs < out_to; gs++) mbar_wait(&bars[gs % NS], (gs / NS) & 1u, 100000000ull);
    }
}

bool vti_maps(const Grid &g, const Fields &F, CUtensorMap *m) {
    const float *src[15] = {F.pcur, F.mcur, F.b, F.eps, F.eta, F.f, F.pcur, F.mcur, F.b, F.eps, F.f,
                            F.pold, F.mold, F.v, F.q};
    for (int i = 0; i < 15; i++) {
        const unsigned bz = i < 2 ? PZW : (i < 6 ? MZW : TZ);
        const unsigned by = i < 2 ? PYH : (i < 6 ? MYH : TY);
        if (!make_tensor_map_3d(&m[i], src[i], g.nx, g.ny, g.nz, bz, by, 1)) return false;
    }
    return true;
}

template <bool LINEAR>
int vti_grid_cap() {
    static int cap = 0;
    if (!cap) {
        for (auto kern : {k_vti3d_tma<LINEAR, false>, k_vti3d_tma<LINEAR, true>, k_vti3d_tma<LINEAR, false, true>})
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
        int dev = 0, sms = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_vti3d_tma<LINEAR, false>, NT, SMEM_BYTES);
        cap = sms * (per > 0 ? per : 1);
    }
    return cap;
}

template <bool LINEAR>
bool launch(const Grid &g, const Fields &F, cudaStream_t s) {
    AnisoMaps M;
    if (!vti_maps(g, F, M.m)) return false;
    const int grid_cap = vti_grid_cap<LINEAR>();
    const int ntz = (int)((g.nz + TZ - 1) / TZ);
    const int nty = (int)((g.ny + TY - 1) / TY);
    const long tiles = (long)ntz * nty;
    int best_nch = 1;
    double best_cost = 1e30;
    for (int nch = 1; nch <= 64 && nch <= g.nx / 16 + 1; nch++) {
        const long chunk = (g.nx + nch - 1) / nch;
        const long items = tiles * nch;
        const double waves = (double)((items + grid_cap - 1) / grid_cap);
        const double cost = waves * (double)(chunk + WARMUP * 0.3);
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
            k_vti3d_tma<LINEAR, false, true><<<grid, NT, SMEM_BYTES, s>>>(g, F, M, ntz, nty, nch, xchunk, nullptr, nullptr, nullptr,
                                                           0, nullptr);
    else
            k_vti3d_tma<LINEAR, false><<<grid, NT, SMEM_BYTES, s>>>(g, F, M, ntz, nty, nch, xchunk, nullptr, nullptr, nullptr,
                                                           0, nullptr);
    return true;
}

}  // namespace

bool fused_vti3d_tma(const Grid &g, int linear, const Fields &F, cudaStream_t s) {
    if (g.ndim != 3 || g.nz % 4 != 0) return false;
    return linear ? launch<true>(g, F, s) : launch<false>(g, F, s);
}

bool vti3d_tma_describe(const Grid &g, const Fields &F, int xchunk, AnisoShotDesc *d, TileInfo *t) {
    if (g.ndim != 3 || g.nz % 4 != 0 || xchunk < 1) return false;
    if (d) {
        if (!vti_maps(g, F, d->m)) return false;
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
        t->grid_cap = vti_grid_cap<false>();
    }
    return true;
}

void vti3d_tma_batch(const Grid &gc, const AnisoShotDesc *shots, const int *sel, const int2 *items, int nitems,
                     int *counter, int grid, cudaStream_t s) {
    vti_grid_cap<false>();
    k_vti3d_tma<false, true><<<grid, NT, SMEM_BYTES, s>>>(gc, Fields{}, AnisoMaps{}, 0, 0, 0, 1, shots, sel, items,
                                                         nitems, counter);
}

void vti3d_set_pipeline_wait(unsigned long long ns) {
    const uint64_t v = ns;
    cudaMemcpyToSymbol(wfd_dev::d_pipeline_wait_ns, &v, sizeof(v));
}

unsigned vti3d_status_and_clear() {
    unsigned v = 0, z = 0;
    cudaMemcpyFromSymbol(&v, d_status, sizeof(v));
    if (v) cudaMemcpyToSymbol(d_status, &z, sizeof(z));
    return v;
}

}  // namespace WFD_NS
