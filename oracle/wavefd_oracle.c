/*
 * CPU restatement of WaveFD's single-step propagators -- TEST INFRASTRUCTURE ONLY (the checker).
 * See wavefd_oracle.h. References are to files of the WaveFD package (src/...).
 *
 * Semantics shared by every reference pass, restated once here:
 *  - a cell is "interior" when kx, ky, kz are all in [4, n-4);
 *  - with a free surface, rows kz = 0..3 with kx, ky interior are computed too
 *    (e.g. prop3DAcoIsoDenQ_DEO2_FDTD.h:896-1031 and :1162-1283);
 *  - every other cell of a derivative output is zero (the annulus zeroing at e.g. .h:801-838);
 *  - D+ at kz reads kz-3..kz+4 and, above the surface, the antisymmetric image p[-j] = -p[j];
 *    D- reads kz-4..kz+3 and the symmetric image t[-j] = t[j-1] (the hard-coded rows of
 *    propagatorStaticFunctions.h:80-160 and :230-310 are exactly these images);
 *  - in row kz = 0 the D+ x/y derivatives are literal zeros and every D- derivative is zero.
 */
#include "wavefd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define PI_ABSORB 3.1415926535897 /* absorb.h:12 */
#define FOR_XY(g)                                            \
    _Pragma("omp parallel for collapse(2) schedule(static)") \
    for (long x = 0; x < (g)->nx; x++)                       \
        for (long y = 0; y < (g)->ny; y++)

/* FP32 instantiation: the restatement pinned to the reference */
#define R float
#define SQRT sqrtf
#define G_T G
#define SFX(n) n
#define PUB(n) wfo_##n
#include "wfo_generic.inc"
#undef R
#undef SQRT
#undef G_T
#undef SFX
#undef PUB

/* FP64 instantiation: the same arithmetic in double precision */
#define R double
#define SQRT sqrt
#define G_T G64
#define SFX(n) n##_64
#define PUB(n) wfo64_##n
#include "wfo_generic.inc"
#undef R
#undef SQRT
#undef G_T
#undef SFX
#undef PUB


/* ------------------------------------------------------------------------------------------ */
/* absorb.h:23-75 (2D: log in float promoted to double, expf of the rounded value)            */
/* absorb.h:85-151 (3D: everything in float)                                                  */
void wfo_setup_q(const wfo_geom *w, long nsponge, float freqQ, float qMin, float qInterior, float *q) {
    const long nx = w->nx, ny = w->ndim == 3 ? w->ny : 1, nz = w->nz;
    if (freqQ < FLT_EPSILON) return; /* the reference exits the process here */
    if ((qMin < FLT_EPSILON) && (qInterior < FLT_EPSILON)) {
        memset(q, 0, 8); /* absorb.h:44 and :107 clear sizeof(float*) bytes only */
        return;
    }
    float *qprof = zalloc(nsponge);
    if (w->ndim == 2) {
        const double lqmin = logf(qMin);
        const double lqmax = logf(qInterior);
        for (long ks = 0; ks < nsponge; ks++) {
            const double dk = (double)ks / (double)(nsponge - 1);
            const double lq = lqmin + dk * (lqmax - lqmin);
            qprof[ks] = expf((float)lq);
        }
    } else {
        const float lqmin = logf(qMin);
        const float lqmax = logf(qInterior);
        for (long ks = 0; ks < nsponge; ks++) {
            const float dk = (float)ks / (float)(nsponge - 1);
            const float lq = lqmin + dk * (lqmax - lqmin);
            qprof[ks] = expf(lq);
        }
    }
    const float dt = w->dt;
    for (long x = 0; x < nx; x++)
        for (long y = 0; y < ny; y++)
            for (long z = 0; z < nz; z++) {
                const long ksx = x < nx - 1 - x ? x : nx - 1 - x;
                const long ksy = y < ny - 1 - y ? y : ny - 1 - y;
                const long ksz = w->fs ? (nz - 1 - z) : (z < nz - 1 - z ? z : nz - 1 - z);
                long ks = ksx < ksz ? ksx : ksz;
                if (w->ndim == 3 && ksy < ks) ks = ksy;
                const long k = (x * ny + y) * nz + z;
                q[k] = (float)((double)(dt * 2) * PI_ABSORB * (double)freqQ / (double)qInterior);
                if (ks < nsponge) q[k] = (float)((double)(dt * 2) * PI_ABSORB * (double)freqQ / (double)qprof[ks]);
            }
    free(qprof);
}


/* rotated D+ of the TTI Born/imaging helpers: 3D .h:2910-3166, 2D prop2DAcoTTIDenQ .h:1366-1530 */
static void tti_dplus(const G *g, const float *in, const float *sint, const float *cost, const float *sinp,
                      const float *cosp, float *o1, float *o2, float *o3) {
    FOR_XY(g) {
        for (long z = 0; z < g->nz; z++) {
            const long k = kof(g, x, y, z);
            const int r = region(g, x, y, z);
            if (!r) {
                o1[k] = 0;
                o2[k] = 0;
                o3[k] = 0;
                continue;
            }
            float dx, dy, dz;
            gradp(g, in, x, y, z, r, &dx, &dy, &dz);
            if (g->ndim == 3) {
                const float cosThetaCosPhi = cost[k] * cosp[k];
                const float cosThetaSinPhi = cost[k] * sinp[k];
                const float sinThetaCosPhi = sint[k] * cosp[k];
                o1[k] = cosThetaCosPhi * dx + cosThetaSinPhi * dy - sint[k] * dz;
                o2[k] = -sinp[k] * dx + cosp[k] * dy;
                o3[k] = sinThetaCosPhi * dx + sint[k] * sinp[k] * dy + cost[k] * dz;
            } else {
                o1[k] = cost[k] * dx - sint[k] * dz;
                o2[k] = 0;
                o3[k] = sint[k] * dx + cost[k] * dz;
            }
        }
    }
}

/* rotated D- with the back-rotation inside the stencil: 3D .h:3171-3661, 2D .h:1531-1719 */
static void tti_dminus(const G *g, const float *i1, const float *i2, const float *i3, const float *sint,
                       const float *cost, const float *sinp, const float *cosp, float *o1, float *o2,
                       float *o3) {
    const int nw = g->ndim == 3 ? 8 : 4;
    float *wt[8];
    for (int i = 0; i < nw; i++) wt[i] = zalloc(g->n);
    for (long k = 0; k < g->n; k++) {
        if (g->ndim == 3) {
            wt[0][k] = cost[k] * cosp[k] * i1[k]; /* G1, x */
            wt[1][k] = cost[k] * sinp[k] * i1[k]; /* G1, y */
            wt[2][k] = sint[k] * i1[k];           /* G1, z */
            wt[3][k] = sinp[k] * i2[k];           /* G2, x */
            wt[4][k] = cosp[k] * i2[k];           /* G2, y */
            wt[5][k] = sint[k] * cosp[k] * i3[k]; /* G3, x */
            wt[6][k] = sint[k] * sinp[k] * i3[k]; /* G3, y */
            wt[7][k] = cost[k] * i3[k];           /* G3, z */
        } else {
            wt[0][k] = cost[k] * i1[k];
            wt[1][k] = sint[k] * i1[k];
            wt[2][k] = sint[k] * i3[k];
            wt[3][k] = cost[k] * i3[k];
        }
    }
    FOR_XY(g) {
        for (long z = 0; z < g->nz; z++) {
            const long k = kof(g, x, y, z);
            const int r = region(g, x, y, z);
            if (!r || (r == 2 && z == 0)) {
                o1[k] = 0;
                o2[k] = 0;
                o3[k] = 0;
                continue;
            }
            if (g->ndim == 3) {
                o1[k] = g->idx * rawmx(g, wt[0], k) + g->idy * rawmy(g, wt[1], k) - g->idz * rawmz(g, wt[2], k, z);
                o2[k] = -g->idx * rawmx(g, wt[3], k) + g->idy * rawmy(g, wt[4], k);
                o3[k] = g->idx * rawmx(g, wt[5], k) + g->idy * rawmy(g, wt[6], k) + g->idz * rawmz(g, wt[7], k, z);
            } else {
                o1[k] = g->idx * rawmx(g, wt[0], k) - g->idz * rawmz(g, wt[1], k, z);
                o2[k] = 0;
                o3[k] = g->idx * rawmx(g, wt[2], k) + g->idz * rawmz(g, wt[3], k, z);
            }
        }
    }
    for (int i = 0; i < nw; i++) free(wt[i]);
}

/* gradient triple of the VEA helpers: plain D+ for VTI, rotated D+ for TTI */
static void vea_grad(const G *g, const wfo_geom *w, long tti, const float *in, const float *sint,
                     const float *cost, const float *sinp, const float *cosp, float *o[3]) {
    if (tti)
        tti_dplus(g, in, sint, cost, sinp, cosp, o[0], o[1], o[2]);
    else
        wfo_dplus(w, in, o[0], o[1], o[2]);
}

/* Born injection VEA: 3D VTI .h:457-551, 3D TTI .h:460-554, 2D VTI .h:383-472, 2D TTI .h:362-450 */
void wfo_born_vea(const wfo_geom *w, long tti, const float *v, const float *eps, const float *eta,
                  const float *b, const float *f, const float *sint, const float *cost, const float *sinp,
                  const float *cosp, const float *dv, const float *de, const float *da, const float *p,
                  const float *m, const float *dp, const float *dm, float *pcur, float *mcur) {
    G g = mk(w);
    (void)eps;
    float *tp1[3], *tm1[3], *tp2[3], *tm2[3];
    for (int i = 0; i < 3; i++) {
        tp1[i] = zalloc(g.n);
        tm1[i] = zalloc(g.n);
        tp2[i] = zalloc(g.n);
        tm2[i] = zalloc(g.n);
    }
    vea_grad(&g, w, tti, p, sint, cost, sinp, cosp, tp1);
    vea_grad(&g, w, tti, m, sint, cost, sinp, cosp, tm1);
    for (long k = 0; k < g.n; k++) {
        const float A = eta[k], B = b[k], F = f[k], dE = de[k], dA = da[k];
        tp2[0][k] = (+2 * B * dE) * tp1[0][k];
        tp2[1][k] = (+2 * B * dE) * tp1[1][k];
        tp2[2][k] = (-2 * B * F * A * dA) * tp1[2][k] + (dA * B * F * (1 - 2 * A * A) / sqrtf(1 - A * A)) * tm1[2][k];
        tm2[0][k] = 0;
        tm2[1][k] = 0;
        tm2[2][k] = (+2 * B * F * A * dA) * tm1[2][k] + (dA * B * F * (1 - 2 * A * A) / sqrtf(1 - A * A)) * tp1[2][k];
    }
    if (tti) {
        tti_dminus(&g, tp2[0], tp2[1], tp2[2], sint, cost, sinp, cosp, tp1[0], tp1[1], tp1[2]);
        tti_dminus(&g, tm2[0], tm2[1], tm2[2], sint, cost, sinp, cosp, tm1[0], tm1[1], tm1[2]);
    } else {
        dminus3(&g, tp2[0], tp2[1], tp2[2], tp1[0], tp1[1], tp1[2]);
        dminus3(&g, tm2[0], tm2[1], tm2[2], tm1[0], tm1[1], tm1[2]);
    }
    const float dt = g.dt;
    for (long k = 0; k < g.n; k++) {
        const float V = v[k], B = b[k], dV = dv[k];
        const float dt2v2OverB = dt * dt * V * V / B;
        const float factor = 2 * B * dV / (V * V * V);
        if (g.ndim == 3) {
            pcur[k] += dt2v2OverB * (factor * dp[k] + tp1[0][k] + tp1[1][k] + tp1[2][k]);
            mcur[k] += dt2v2OverB * (factor * dm[k] + tm1[0][k] + tm1[1][k] + tm1[2][k]);
        } else {
            pcur[k] += dt2v2OverB * (factor * dp[k] + tp1[0][k] + tp1[2][k]);
            mcur[k] += dt2v2OverB * (factor * dm[k] + tm1[0][k] + tm1[2][k]);
        }
    }
    for (int i = 0; i < 3; i++) {
        free(tp1[i]);
        free(tm1[i]);
        free(tp2[i]);
        free(tm2[i]);
    }
}

/* Imaging VEA: 3D VTI .h:730-787, 3D TTI .h:733-790, 2D VTI .h:629-690, 2D TTI .h:560-620 */
void wfo_image_vea(const wfo_geom *w, long tti, const float *v, const float *eps, const float *eta,
                   const float *b, const float *f, const float *sint, const float *cost, const float *sinp,
                   const float *cosp, const float *p, const float *m, const float *dp, const float *dm,
                   const float *pold, const float *mold, float *dv, float *de, float *da) {
    G g = mk(w);
    (void)eps;
    float *tp1[3], *tm1[3], *tp2[3], *tm2[3];
    for (int i = 0; i < 3; i++) {
        tp1[i] = zalloc(g.n);
        tm1[i] = zalloc(g.n);
        tp2[i] = zalloc(g.n);
        tm2[i] = zalloc(g.n);
    }
    vea_grad(&g, w, tti, p, sint, cost, sinp, cosp, tp1);
    vea_grad(&g, w, tti, m, sint, cost, sinp, cosp, tm1);
    vea_grad(&g, w, tti, pold, sint, cost, sinp, cosp, tp2);
    vea_grad(&g, w, tti, mold, sint, cost, sinp, cosp, tm2);
    for (long k = 0; k < g.n; k++) {
        const float V = v[k], A = eta[k], B = b[k], F = f[k];
        const float factor = 2 * B / (V * V * V);
        if (g.ndim == 3) {
            dv[k] += factor * (dp[k] * pold[k] + dm[k] * mold[k]);
            de[k] += (-2 * B * tp1[0][k] * tp2[0][k] - 2 * B * tp1[1][k] * tp2[1][k]);
        } else {
            dv[k] += factor * dp[k] * pold[k] + factor * dm[k] * mold[k];
            de[k] += -2 * B * tp1[0][k] * tp2[0][k];
        }
        const float partP = 2 * B * F * A * tp1[2][k] - (B * F * (1 - 2 * A * A) / sqrtf(1 - A * A)) * tm1[2][k];
        const float partM = 2 * B * F * A * tm1[2][k] + (B * F * (1 - 2 * A * A) / sqrtf(1 - A * A)) * tp1[2][k];
        if (g.ndim == 3)
            da[k] += (partP * tp2[2][k] - partM * tm2[2][k]);
        else
            da[k] += partP * tp2[2][k] - partM * tm2[2][k];
    }
    for (int i = 0; i < 3; i++) {
        free(tp1[i]);
        free(tm1[i]);
        free(tp2[i]);
        free(tm2[i]);
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Wavefield separation: 3D Iso .h:673-765, 3D VTI .h:606-725, 3D TTI .h:609-728, 2D Iso      */
/* .h:584-672. Per (x,y) column: zero-pad to nfft = 2nz, scale 1/nfft, transform with sign +1, */
/* zero bins [n/2+1, n) of the forward field and [kadj+1, kadj+n/2) of the adjoint field,      */
/* transform back with sign -1, accumulate 2B/V^3 * Re(a*b). Here in double precision.         */
static void dft(double *re, double *im, long n, int sign, double *wr, double *wi) {
    const double twopi = 6.283185307179586476925286766559;
    for (long k = 0; k < n; k++) {
        double sr = 0, si = 0;
        for (long j = 0; j < n; j++) {
            const long m = (j * k) % n;
            const double c = cos(twopi * (double)m / (double)n);
            const double s = sign * sin(twopi * (double)m / (double)n);
            sr += re[j] * c - im[j] * s;
            si += re[j] * s + im[j] * c;
        }
        wr[k] = sr;
        wi[k] = si;
    }
    memcpy(re, wr, sizeof(double) * (size_t)n);
    memcpy(im, wi, sizeof(double) * (size_t)n);
}

static void sep_column(long nz, long isfwi, const float *a, const float *bcol, double *out) {
    const long nfft = 2 * nz;
    const float scale = 1.0f / (float)nfft;
    const long kadj = isfwi ? 0 : nfft / 2;
    double *ar = calloc((size_t)nfft, sizeof(double)), *ai = calloc((size_t)nfft, sizeof(double));
    double *br = calloc((size_t)nfft, sizeof(double)), *bi = calloc((size_t)nfft, sizeof(double));
    double *wr = calloc((size_t)nfft, sizeof(double)), *wi = calloc((size_t)nfft, sizeof(double));
    for (long z = 0; z < nz; z++) {
        ar[z] = (double)(scale * a[z]);
        br[z] = (double)(scale * bcol[z]);
    }
    dft(ar, ai, nfft, +1, wr, wi);
    dft(br, bi, nfft, +1, wr, wi);
    for (long k = 1; k < nfft / 2; k++) {
        ar[nfft / 2 + k] = 0;
        ai[nfft / 2 + k] = 0;
        br[kadj + k] = 0;
        bi[kadj + k] = 0;
    }
    dft(ar, ai, nfft, -1, wr, wi);
    dft(br, bi, nfft, -1, wr, wi);
    for (long z = 0; z < nz; z++) out[z] = ar[z] * br[z] - ai[z] * bi[z];
    free(ar);
    free(ai);
    free(br);
    free(bi);
    free(wr);
    free(wi);
}

void wfo_image_wavefieldsep(const wfo_geom *w, long isfwi, const float *v, const float *b, const float *dp,
                            const float *pold, const float *dm, const float *mold, float *dv) {
    G g = mk(w);
    FOR_XY(&g) {
        double *rp = calloc((size_t)g.nz, sizeof(double)), *rm = calloc((size_t)g.nz, sizeof(double));
        const long k0 = kof(&g, x, y, 0);
        sep_column(g.nz, isfwi, dp + k0, pold + k0, rp);
        if (dm) sep_column(g.nz, isfwi, dm + k0, mold + k0, rm);
        for (long z = 0; z < g.nz; z++) {
            const long k = k0 + z;
            const double V = v[k], B = b[k];
            const double factor = 2 * B / (V * V * V);
            dv[k] = (float)((double)dv[k] + factor * (rp[z] + (dm ? rm[z] : 0.0)));
        }
        free(rp);
        free(rm);
    }
}

/* ------------------------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------------------------ */
/* Time interpolation between dtmod (fine, nm samples) and dtrec (coarse, nd samples) with nh
 * 8-tap filters h[k][0..7]; traces are contiguous in time, nslow traces. spacetime.cc:4-127:
 * the coarse index i runs over the helper calls (i, lo, hi) = (0,3,7), (1,2,7), (2,1,7),
 * (3..nd-5, 0,7), (nd-4,0,6), (nd-3,0,5), (nd-2,0,4); fine sample jk = i*nh + k (if < nm) pairs
 * with coarse samples i-3+l, l in [lo, hi]. Adjoint: m[jk] += h[k][l] d[i-3+l] (m zeroed first);
 * forward: d[i-3+l] += h[k][l] m[jk] (d zeroed first), in that loop order. Needs nd >= 7. */
#define WFO_INTERP(T, SUF)                                                                           \
    static void wfo_interp_calls_##SUF(long nd, long *ci, long *clo, long *chi, long *ncalls) {     \
        long n = 0;                                                                                  \
        ci[n] = 0, clo[n] = 3, chi[n++] = 7;                                                         \
        ci[n] = 1, clo[n] = 2, chi[n++] = 7;                                                         \
        ci[n] = 2, clo[n] = 1, chi[n++] = 7;                                                         \
        for (long i = 3; i < nd - 4; i++) ci[n] = i, clo[n] = 0, chi[n++] = 7;                       \
        ci[n] = nd - 4, clo[n] = 0, chi[n++] = 6;                                                    \
        ci[n] = nd - 3, clo[n] = 0, chi[n++] = 5;                                                    \
        ci[n] = nd - 2, clo[n] = 0, chi[n++] = 4;                                                    \
        *ncalls = n;                                                                                 \
    }                                                                                                \
    void wfo_interpadjoint_##SUF(const T *h, T *m, const T *d, long nh, long nm, long nd, long nslow) { \
        long *ci = malloc(sizeof(long) * (nd + 8)), *clo = malloc(sizeof(long) * (nd + 8)),         \
             *chi = malloc(sizeof(long) * (nd + 8)), nc;                                              \
        wfo_interp_calls_##SUF(nd, ci, clo, chi, &nc);                                               \
        for (long t = 0; t < nslow; t++) {                                                           \
            T *mt = m + t * nm;                                                                      \
            const T *dt = d + t * nd;                                                                \
            for (long j = 0; j < nm; j++) mt[j] = 0;                                                 \
            for (long c = 0; c < nc; c++)                                                            \
                for (long k = 0; k < nh; k++) {                                                      \
                    const long jk = ci[c] * nh + k;                                                  \
                    if (jk >= nm) continue;                                                          \
                    for (long l = clo[c]; l <= chi[c]; l++) mt[jk] += h[k * 8 + l] * dt[ci[c] - 3 + l]; \
                }                                                                                    \
        }                                                                                            \
        free(ci), free(clo), free(chi);                                                              \
    }                                                                                                \
    void wfo_interpforward_##SUF(const T *h, T *d, const T *m, long nh, long nd, long nm, long nslow) { \
        long *ci = malloc(sizeof(long) * (nd + 8)), *clo = malloc(sizeof(long) * (nd + 8)),         \
             *chi = malloc(sizeof(long) * (nd + 8)), nc;                                              \
        wfo_interp_calls_##SUF(nd, ci, clo, chi, &nc);                                               \
        for (long t = 0; t < nslow; t++) {                                                           \
            T *dt = d + t * nd;                                                                      \
            const T *mt = m + t * nm;                                                                \
            for (long i = 0; i < nd; i++) dt[i] = 0;                                                 \
            for (long c = 0; c < nc; c++)                                                            \
                for (long k = 0; k < nh; k++) {                                                      \
                    const long jk = ci[c] * nh + k;                                                  \
                    if (jk >= nm) continue;                                                          \
                    for (long l = clo[c]; l <= chi[c]; l++) dt[ci[c] - 3 + l] += h[k * 8 + l] * mt[jk]; \
                }                                                                                    \
        }                                                                                            \
        free(ci), free(clo), free(chi);                                                              \
    }
WFO_INTERP(float, float)
WFO_INTERP(double, double)

/* illumination.c:3-53: field = field^2 (accum NULL) or accum += field^2 */
void wfo_illum_float(float *accum, float *field, long n) {
    for (long i = 0; i < n; i++) {
        if (accum) accum[i] += field[i] * field[i];
        else field[i] = field[i] * field[i];
    }
}
