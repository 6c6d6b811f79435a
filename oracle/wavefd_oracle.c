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

typedef struct {
    int ndim, fs;
    long nx, ny, nz, sx, sy, n;
    float c1, c2, c3, c4, idx, idy, idz, dt;
} G;

static G mk(const wfo_geom *w) {
    G g;
    g.ndim = (int)w->ndim;
    g.fs = w->fs != 0;
    g.nx = w->nx;
    g.ny = w->ndim == 3 ? w->ny : 1;
    g.nz = w->nz;
    g.sy = g.nz;
    g.sx = g.ny * g.nz;
    g.n = g.nx * g.sx;
    /* prop3DAcoIsoDenQ_DEO2_FDTD.h:64-70: constants formed in double, stored as float */
    g.c1 = (float)(+1225.0 / 1024.0);
    g.c2 = (float)(-245.0 / 3072.0);
    g.c3 = (float)(+49.0 / 5120.0);
    g.c4 = (float)(-5.0 / 7168.0);
    g.idx = (float)(1.0 / (double)w->dx);
    g.idy = (float)(1.0 / (double)w->dy);
    g.idz = (float)(1.0 / (double)w->dz);
    g.dt = w->dt;
    return g;
}

static float *zalloc(long n) { return (float *)calloc((size_t)(n > 0 ? n : 1), sizeof(float)); }

/* 0 = not computed (zero output / no update), 1 = interior, 2 = free-surface row */
static inline int region(const G *g, long x, long y, long z) {
    if (x < 4 || x >= g->nx - 4) return 0;
    if (g->ndim == 3 && (y < 4 || y >= g->ny - 4)) return 0;
    if (z >= g->nz - 4) return 0;
    if (z >= 4) return 1;
    return g->fs ? 2 : 0;
}

static inline long kof(const G *g, long x, long y, long z) { return (x * g->ny + y) * g->nz + z; }

static inline float stp(const G *g, const float *f, long s) {
    return g->c1 * (-f[0] + f[s]) + g->c2 * (-f[-s] + f[2 * s]) + g->c3 * (-f[-2 * s] + f[3 * s]) +
           g->c4 * (-f[-3 * s] + f[4 * s]);
}
static inline float stm(const G *g, const float *f, long s) {
    return g->c1 * (-f[-s] + f[0]) + g->c2 * (-f[-2 * s] + f[s]) + g->c3 * (-f[-3 * s] + f[2 * s]) +
           g->c4 * (-f[-4 * s] + f[3 * s]);
}
static inline float imp(const float *col, long j) { return j >= 0 ? col[j] : -col[-j]; }
static inline float imm(const float *col, long j) { return j >= 0 ? col[j] : col[-j - 1]; }
static inline float stpz(const G *g, const float *col, long z) {
    return g->c1 * (-imp(col, z) + imp(col, z + 1)) + g->c2 * (-imp(col, z - 1) + imp(col, z + 2)) +
           g->c3 * (-imp(col, z - 2) + imp(col, z + 3)) + g->c4 * (-imp(col, z - 3) + imp(col, z + 4));
}
static inline float stmz(const G *g, const float *col, long z) {
    return g->c1 * (-imm(col, z - 1) + imm(col, z)) + g->c2 * (-imm(col, z - 2) + imm(col, z + 1)) +
           g->c3 * (-imm(col, z - 3) + imm(col, z + 2)) + g->c4 * (-imm(col, z - 4) + imm(col, z + 3));
}

/* D+ gradient of f at an active cell */
static inline void gradp(const G *g, const float *f, long x, long y, long z, int r, float *dx, float *dy,
                         float *dz) {
    const long k = kof(g, x, y, z);
    if (r == 2 && z == 0) {
        *dx = 0;
        *dy = 0;
    } else {
        *dx = g->idx * stp(g, f + k, g->sx);
        *dy = g->ndim == 3 ? g->idy * stp(g, f + k, g->sy) : 0.0f;
    }
    *dz = g->idz * stpz(g, f + k - z, z);
}

/* D- of three (possibly different) arrays along x, y, z at an active cell */
static inline void gradm3(const G *g, const float *fx, const float *fy, const float *fz, long x, long y,
                          long z, int r, float *dx, float *dy, float *dz) {
    const long k = kof(g, x, y, z);
    if (r == 2 && z == 0) {
        *dx = 0;
        *dy = 0;
        *dz = 0;
        return;
    }
    *dx = g->idx * stm(g, fx + k, g->sx);
    *dy = g->ndim == 3 ? g->idy * stm(g, fy + k, g->sy) : 0.0f;
    *dz = g->idz * stmz(g, fz + k - z, z);
}

/* raw (unscaled) D- stencils of one array */
static inline float rawmx(const G *g, const float *f, long k) { return stm(g, f + k, g->sx); }
static inline float rawmy(const G *g, const float *f, long k) { return stm(g, f + k, g->sy); }
static inline float rawmz(const G *g, const float *f, long k, long z) { return stmz(g, f + k - z, z); }

#define FOR_XY(g)                                            \
    _Pragma("omp parallel for collapse(2) schedule(static)") \
    for (long x = 0; x < (g)->nx; x++)                       \
        for (long y = 0; y < (g)->ny; y++)

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

/* ------------------------------------------------------------------------------------------ */
/* Iso: pass 1 prop3DAcoIsoDenQ_DEO2_FDTD.h:771-1033 (2D .h:678-861), pass 2 3D .h:1039-1284   */
/* (2D .h:867-1044); update line 3D .h:1152, 2D .h:943                                        */
void wfo_step_iso(const wfo_geom *w, const float *v, const float *b, const float *q, const float *pcur,
                  float *pold, float *pspace) {
    G g = mk(w);
    float *tx = zalloc(g.n), *ty = zalloc(g.n), *tz = zalloc(g.n);
    FOR_XY(&g) {
        for (long z = 0; z < g.nz; z++) {
            const long k = kof(&g, x, y, z);
            const int r = region(&g, x, y, z);
            if (!r) continue;
            float dx, dy, dz;
            gradp(&g, pcur, x, y, z, r, &dx, &dy, &dz);
            const float B = b[k];
            tx[k] = B * dx;
            ty[k] = B * dy;
            tz[k] = B * dz;
        }
    }
    const float dt2 = g.dt * g.dt;
    FOR_XY(&g) {
        for (long z = 0; z < g.nz; z++) {
            const long k = kof(&g, x, y, z);
            const int r = region(&g, x, y, z);
            if (!r) {
                pspace[k] = 0;
                continue;
            }
            float dx, dy, dz;
            gradm3(&g, tx, ty, tz, x, y, z, r, &dx, &dy, &dz);
            const float L = g.ndim == 3 ? dx + dy + dz : dx + dz;
            const float dt2V2_B = dt2 * v[k] * v[k] / b[k];
            pold[k] = dt2V2_B * L - q[k] * (pcur[k] - pold[k]) - pold[k] + 2 * pcur[k];
            pspace[k] = L;
        }
    }
    free(tx);
    free(ty);
    free(tz);
}

/* ------------------------------------------------------------------------------------------ */
/* VTI pass-1 sandwich: 3D prop3DAcoVTIDenQ_DEO2_FDTD.h:945-957, 2D prop2DAcoVTIDenQ_DEO2_FDTD.h:771-779 */
static inline void vti_sandwich(int ndim, float eps, float eta, float f, float b, float dPx, float dPy,
                                float dPz, float dMx, float dMy, float dMz, float *o) {
    const float E = 1 + 2 * eps;
    const float A = eta;
    const float F = f;
    const float B = b;
    if (ndim == 3) {
        const float SA2 = sqrtf(1 - A * A);
        o[0] = B * E * dPx;
        o[1] = B * E * dPy;
        o[2] = B * (1 - F * A * A) * dPz + B * (F * A * SA2) * dMz;
        o[3] = B * (1 - F) * dMx;
        o[4] = B * (1 - F) * dMy;
        o[5] = B * F * A * SA2 * dPz + B * (1 - F + F * A * A) * dMz;
    } else {
        o[0] = B * E * dPx;
        o[1] = 0;
        o[2] = B * (1 - F * A * A) * dPz + B * F * A * sqrtf(1 - A * A) * dMz;
        o[3] = B * (1 - F) * dMx;
        o[4] = 0;
        o[5] = B * F * A * sqrtf(1 - A * A) * dPz + B * (1 - F + F * A * A) * dMz;
    }
}

/* P/M pass 2 with the time update: 3D VTI .h:1231-1589 (update :1372-1378), linear .h:1594-1899;   */
/* 3D TTI .h:1274-1632 (update :1420-1421); 2D VTI .h:992-1247 / :1252-1480                          */
static void pm_update(const G *g, long linear, const float *t[6], const float *v, const float *b,
                      const float *q, const float *pcur, const float *mcur, float *pold, float *mold,
                      float *pspace, float *mspace) {
    const float dt2 = g->dt * g->dt;
    FOR_XY(g) {
        for (long z = 0; z < g->nz; z++) {
            const long k = kof(g, x, y, z);
            const int r = region(g, x, y, z);
            if (!r) {
                if (!linear) {
                    pspace[k] = 0;
                    mspace[k] = 0;
                }
                continue;
            }
            float dPx, dPy, dPz, dMx, dMy, dMz;
            gradm3(g, t[0], t[1], t[2], x, y, z, r, &dPx, &dPy, &dPz);
            gradm3(g, t[3], t[4], t[5], x, y, z, r, &dMx, &dMy, &dMz);
            const float LP = g->ndim == 3 ? dPx + dPy + dPz : dPx + dPz;
            const float LM = g->ndim == 3 ? dMx + dMy + dMz : dMx + dMz;
            const float dt2V2_B = dt2 * v[k] * v[k] / b[k];
            if (!linear) {
                pspace[k] = LP;
                mspace[k] = LM;
            }
            pold[k] = dt2V2_B * LP - q[k] * (pcur[k] - pold[k]) - pold[k] + 2 * pcur[k];
            mold[k] = dt2V2_B * LM - q[k] * (mcur[k] - mold[k]) - mold[k] + 2 * mcur[k];
        }
    }
}

void wfo_step_vti(const wfo_geom *w, long linear, const float *v, const float *eps, const float *eta,
                  const float *b, const float *f, const float *q, const float *pcur, const float *mcur,
                  float *pold, float *mold, float *pspace, float *mspace) {
    G g = mk(w);
    float *t[6];
    for (int i = 0; i < 6; i++) t[i] = zalloc(g.n);
    FOR_XY(&g) {
        for (long z = 0; z < g.nz; z++) {
            const long k = kof(&g, x, y, z);
            const int r = region(&g, x, y, z);
            if (!r) continue;
            float dPx, dPy, dPz, dMx, dMy, dMz, o[6];
            gradp(&g, pcur, x, y, z, r, &dPx, &dPy, &dPz);
            gradp(&g, mcur, x, y, z, r, &dMx, &dMy, &dMz);
            vti_sandwich(g.ndim, eps[k], eta[k], f[k], b[k], dPx, dPy, dPz, dMx, dMy, dMz, o);
            for (int i = 0; i < 6; i++) t[i][k] = o[i];
        }
    }
    pm_update(&g, linear, (const float **)t, v, b, q, pcur, mcur, pold, mold, pspace, mspace);
    for (int i = 0; i < 6; i++) free(t[i]);
}

/* ------------------------------------------------------------------------------------------ */
/* TTI. 3D pass 1 prop3DAcoTTIDenQ_DEO2_FDTD.h:796-1255 (interior :885-976); 2D pass 1        */
/* prop2DAcoTTIDenQ_DEO2_FDTD.h:672-992; 2D pass 2 with the back-rotation inside the D- stencil */
/* prop2DAcoTTIDenQ_DEO2_FDTD.h:997-1361                                                       */
void wfo_step_tti(const wfo_geom *w, const float *v, const float *eps, const float *eta, const float *b,
                  const float *f, const float *q, const float *sint, const float *cost, const float *sinp,
                  const float *cosp, const float *pcur, const float *mcur, float *pold, float *mold,
                  float *pspace, float *mspace) {
    G g = mk(w);
    float *t[6];
    for (int i = 0; i < 6; i++) t[i] = zalloc(g.n);
    FOR_XY(&g) {
        for (long z = 0; z < g.nz; z++) {
            const long k = kof(&g, x, y, z);
            const int r = region(&g, x, y, z);
            if (!r) continue;
            float dpdx, dpdy, dpdz, dmdx, dmdy, dmdz;
            gradp(&g, pcur, x, y, z, r, &dpdx, &dpdy, &dpdz);
            gradp(&g, mcur, x, y, z, r, &dmdx, &dmdy, &dmdz);
            if (g.ndim == 3) {
                const float sinThetaCosPhi = sint[k] * cosp[k];
                const float sinThetaSinPhi = sint[k] * sinp[k];
                const float fieldEta2 = eta[k] * eta[k];
                const float fieldBuoyVsVp = b[k] * f[k];
                const float g3P = sinThetaCosPhi * dpdx + sinThetaSinPhi * dpdy + cost[k] * dpdz;
                const float g3M = sinThetaCosPhi * dmdx + sinThetaSinPhi * dmdy + cost[k] * dmdz;
                const float tmpFE = fieldBuoyVsVp * eta[k] * sqrtf(1 - fieldEta2);
                const float tmpP = -b[k] * (2 * eps[k] + f[k] * fieldEta2) * g3P + tmpFE * g3M;
                const float tmpM = tmpFE * g3P + fieldBuoyVsVp * fieldEta2 * g3M;
                const float tmpE = b[k] * (1 + 2 * eps[k]);
                const float tmpF = b[k] * (1 - f[k]);
                t[0][k] = tmpE * dpdx + sinThetaCosPhi * tmpP;
                t[1][k] = tmpE * dpdy + sinThetaSinPhi * tmpP;
                t[2][k] = tmpE * dpdz + cost[k] * tmpP;
                t[3][k] = tmpF * dmdx + sinThetaCosPhi * tmpM;
                t[4][k] = tmpF * dmdy + sinThetaSinPhi * tmpM;
                t[5][k] = tmpF * dmdz + cost[k] * tmpM;
            } else {
                const float dPG1 = cost[k] * dpdx - sint[k] * dpdz;
                const float dPG3 = sint[k] * dpdx + cost[k] * dpdz;
                const float dMG1 = cost[k] * dmdx - sint[k] * dmdz;
                const float dMG3 = sint[k] * dmdx + cost[k] * dmdz;
                const float E = 1 + 2 * eps[k];
                const float A = eta[k];
                const float F = f[k];
                const float B = b[k];
                t[0][k] = B * E * dPG1;
                t[2][k] = B * (1 - F * A * A) * dPG3 + B * F * A * sqrtf(1 - A * A) * dMG3;
                t[3][k] = B * (1 - F) * dMG1;
                t[5][k] = B * F * A * sqrtf(1 - A * A) * dPG3 + B * (1 - F + F * A * A) * dMG3;
            }
        }
    }
    if (g.ndim == 3) {
        pm_update(&g, 0, (const float **)t, v, b, q, pcur, mcur, pold, mold, pspace, mspace);
    } else {
        /* weighted terms cos*G1, sin*G1, sin*G3, cos*G3 for P and M */
        float *wt[8];
        for (int i = 0; i < 8; i++) wt[i] = zalloc(g.n);
        for (long k = 0; k < g.n; k++) {
            wt[0][k] = cost[k] * t[0][k];
            wt[1][k] = sint[k] * t[0][k];
            wt[2][k] = sint[k] * t[2][k];
            wt[3][k] = cost[k] * t[2][k];
            wt[4][k] = cost[k] * t[3][k];
            wt[5][k] = sint[k] * t[3][k];
            wt[6][k] = sint[k] * t[5][k];
            wt[7][k] = cost[k] * t[5][k];
        }
        const float dt2 = g.dt * g.dt;
        FOR_XY(&g) {
            for (long z = 0; z < g.nz; z++) {
                const long k = kof(&g, x, y, z);
                const int r = region(&g, x, y, z);
                if (!r) {
                    pspace[k] = 0;
                    mspace[k] = 0;
                    continue;
                }
                float dPG1 = 0, dPG3 = 0, dMG1 = 0, dMG3 = 0;
                if (!(r == 2 && z == 0)) {
                    dPG1 = g.idx * rawmx(&g, wt[0], k) - g.idz * rawmz(&g, wt[1], k, z);
                    dPG3 = g.idx * rawmx(&g, wt[2], k) + g.idz * rawmz(&g, wt[3], k, z);
                    dMG1 = g.idx * rawmx(&g, wt[4], k) - g.idz * rawmz(&g, wt[5], k, z);
                    dMG3 = g.idx * rawmx(&g, wt[6], k) + g.idz * rawmz(&g, wt[7], k, z);
                }
                const float dt2V2_B = dt2 * v[k] * v[k] / b[k];
                pspace[k] = dPG1 + dPG3;
                mspace[k] = dMG1 + dMG3;
                pold[k] = dt2V2_B * pspace[k] - q[k] * (pcur[k] - pold[k]) - pold[k] + 2 * pcur[k];
                mold[k] = dt2V2_B * mspace[k] - q[k] * (mcur[k] - mold[k]) - mold[k] + 2 * mcur[k];
            }
        }
        for (int i = 0; i < 8; i++) free(wt[i]);
    }
    for (int i = 0; i < 6; i++) free(t[i]);
}

/* ------------------------------------------------------------------------------------------ */
/* scaleSpatialDerivatives: 3D Iso .h:269-291, VTI .h:384-407, TTI .h:387-415, 2D Iso .h:222-239 */
void wfo_scale(const wfo_geom *w, const float *v, const float *b, float *pspace, float *mspace) {
    G g = mk(w);
    for (long k = 0; k < g.n; k++) {
        const float v2OverB = v[k] * v[k] / b[k];
        pspace[k] *= v2OverB;
        if (mspace) mspace[k] *= v2OverB;
    }
}

/* propagatorStaticFunctions.h:10-161 (2D D+), :317-528 (3D D+) */
void wfo_dplus(const wfo_geom *w, const float *in, float *outx, float *outy, float *outz) {
    G g = mk(w);
    FOR_XY(&g) {
        for (long z = 0; z < g.nz; z++) {
            const long k = kof(&g, x, y, z);
            const int r = region(&g, x, y, z);
            float dx = 0, dy = 0, dz = 0;
            if (r) gradp(&g, in, x, y, z, r, &dx, &dy, &dz);
            outx[k] = dx;
            if (g.ndim == 3) outy[k] = dy;
            outz[k] = dz;
        }
    }
}

/* propagatorStaticFunctions.h:167-311 (2D D-), :534-738 (3D D-) */
void wfo_dminus(const wfo_geom *w, const float *in, float *outx, float *outy, float *outz) {
    G g = mk(w);
    FOR_XY(&g) {
        for (long z = 0; z < g.nz; z++) {
            const long k = kof(&g, x, y, z);
            const int r = region(&g, x, y, z);
            float dx = 0, dy = 0, dz = 0;
            if (r) gradm3(&g, in, in, in, x, y, z, r, &dx, &dy, &dz);
            outx[k] = dx;
            if (g.ndim == 3) outy[k] = dy;
            outz[k] = dz;
        }
    }
}

/* D- along x/y/z of three different arrays, zero outside the active region */
static void dminus3(const G *g, const float *fx, const float *fy, const float *fz, float *ox, float *oy,
                    float *oz) {
    FOR_XY(g) {
        for (long z = 0; z < g->nz; z++) {
            const long k = kof(g, x, y, z);
            const int r = region(g, x, y, z);
            float dx = 0, dy = 0, dz = 0;
            if (r) gradm3(g, fx, fy, fz, x, y, z, r, &dx, &dy, &dz);
            ox[k] = dx;
            oy[k] = dy;
            oz[k] = dz;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* Born injection, Iso: 3D .h:305-334 (V), .h:351-417 (VB), .h:434-498 (B);                    */
/* 2D prop2DAcoIsoDenQ_DEO2_FDTD.h:253-280 (V) and the 2D VB/B forms that follow it            */
void wfo_born_iso(const wfo_geom *w, long which, const float *v, const float *b, const float *dv,
                  const float *db, const float *p, const float *dp, float *pcur) {
    G g = mk(w);
    const float dt = g.dt;
    if (which == 0) {
        for (long k = 0; k < g.n; k++) {
            const float V = v[k], B = b[k], dV = dv[k];
            if (g.ndim == 3) {
                const float dt2v2OverB = dt * dt * V * V / B;
                const float factorV = 2 * B * dV / (V * V * V);
                pcur[k] += dt2v2OverB * dp[k] * factorV;
            } else {
                const float factor = 2 * dt * dt * dV / V;
                pcur[k] += factor * dp[k];
            }
        }
        return;
    }
    float *t1[3], *t2[3];
    for (int i = 0; i < 3; i++) {
        t1[i] = zalloc(g.n);
        t2[i] = zalloc(g.n);
    }
    wfo_dplus(w, p, t1[0], t1[1], t1[2]);
    for (long k = 0; k < g.n; k++) {
        const float dB = db[k];
        for (int i = 0; i < 3; i++) t2[i][k] = dB * t1[i][k];
    }
    dminus3(&g, t2[0], t2[1], t2[2], t1[0], t1[1], t1[2]);
    for (long k = 0; k < g.n; k++) {
        const float V = v[k], B = b[k], dB = db[k];
        if (g.ndim == 3) {
            const float dt2v2OverB = dt * dt * V * V / B;
            const float factorB = -dB / (V * V);
            if (which == 1) {
                const float dV = dv[k];
                const float factorV = 2 * B * dV / (V * V * V);
                pcur[k] += dt2v2OverB * (dp[k] * (factorV + factorB) + t1[0][k] + t1[1][k] + t1[2][k]);
            } else {
                pcur[k] += dt2v2OverB * (dp[k] * factorB + t1[0][k] + t1[1][k] + t1[2][k]);
            }
        } else {
            const float V2 = V * V;
            const float dt2v2OverB = dt * dt * V2 / B;
            if (which == 1) {
                const float dV = dv[k];
                pcur[k] += dt2v2OverB * (dp[k] / V2 * (2 * B * dV / V - dB) + t1[0][k] + t1[2][k]);
            } else {
                const float factorB = -dB / V2;
                pcur[k] += dt2v2OverB * (dp[k] * factorB + t1[0][k] + t1[2][k]);
            }
        }
    }
    for (int i = 0; i < 3; i++) {
        free(t1[i]);
        free(t2[i]);
    }
}

/* Born injection V, VTI/TTI 2D/3D: 3D VTI .h:420-452, 3D TTI .h:423-452 */
void wfo_born_aniso_v(const wfo_geom *w, const float *v, const float *dv, const float *dp, const float *dm,
                      float *pcur, float *mcur) {
    G g = mk(w);
    const float dt = g.dt;
    for (long k = 0; k < g.n; k++) {
        const float V = v[k], dV = dv[k];
        const float factor = 2 * dt * dt * dV / V;
        pcur[k] += factor * dp[k];
        mcur[k] += factor * dm[k];
    }
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

/* ------------------------------------------------------------------------------------------ */
/* Imaging, Iso: 3D .h:518-546 (V), .h:563-656 (VB, B); 2D prop2DAcoIsoDenQ_DEO2_FDTD.h V/VB/B */
void wfo_image_iso(const wfo_geom *w, long which, const float *v, const float *b, const float *p,
                   const float *dp, const float *pold, float *dv, float *db) {
    G g = mk(w);
    float *t1[3] = {0, 0, 0}, *t2[3] = {0, 0, 0};
    if (which != 0) {
        for (int i = 0; i < 3; i++) {
            t1[i] = zalloc(g.n);
            t2[i] = zalloc(g.n);
        }
        wfo_dplus(w, p, t1[0], t1[1], t1[2]);
        wfo_dplus(w, pold, t2[0], t2[1], t2[2]);
    }
    for (long k = 0; k < g.n; k++) {
        const float V = v[k], B = b[k];
        if (which == 0 || which == 1) {
            const float factorV = +2 * B / (V * V * V);
            dv[k] += factorV * dp[k] * pold[k];
        }
        if (which != 0) {
            const float factorB = -1 / (V * V);
            if (g.ndim == 3)
                db[k] += factorB * dp[k] * pold[k] - t1[0][k] * t2[0][k] - t1[1][k] * t2[1][k] - t1[2][k] * t2[2][k];
            else
                db[k] += factorB * dp[k] * pold[k] - t1[0][k] * t2[0][k] - t1[2][k] * t2[2][k];
        }
    }
    for (int i = 0; i < 3; i++) {
        free(t1[i]);
        free(t2[i]);
    }
}

/* Imaging V, VTI/TTI: 3D VTI .h:564-589, 3D TTI .h:567-592, 2D VTI .h:473-500 */
void wfo_image_aniso_v(const wfo_geom *w, const float *v, const float *b, const float *dp, const float *dm,
                       const float *pold, const float *mold, float *dv) {
    G g = mk(w);
    for (long k = 0; k < g.n; k++) {
        const float V = v[k], B = b[k];
        const float factor = 2 * B / (V * V * V);
        dv[k] += factor * (dp[k] * pold[k] + dm[k] * mold[k]);
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
void wfo_inject(float *field, const float *data, long it, long nt, const long *iu, const long *ir,
                const float *c, long n) {
    for (long i = 0; i < n; i++) field[iu[i] - 1] += c[i] * data[(ir[i] - 1) * nt + it - 1];
}

void wfo_extract(float *data, const float *field, long it, long nt, const long *iu, const long *ir,
                 const float *c, long n) {
    for (long i = 0; i < n; i++) data[(ir[i] - 1) * nt + it - 1] += c[i] * field[iu[i] - 1];
}

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
