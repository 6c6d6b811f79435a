/*
 * CPU restatement of WaveFD's single-step acoustic propagators -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the checker the CUDA path is compared against; nothing in the product links it.
 * Every function restates one reference routine (file:line cited at its definition) with the
 * same per-cell floating-point expression trees, so that when compiled with IEEE semantics
 * (-fno-fast-math -ffp-contract=off) it is bit-identical (up to the sign of zero) to the
 * reference compiled the same way. The control structure is the project's own: one generic
 * first-derivative routine with the free-surface image rules, composed per physics.
 *
 * Layout: k = (kx*ny + ky)*nz + kz (z fastest); 2D uses ny = 1.
 */
#ifndef WAVEFD_ORACLE_H
#define WAVEFD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    long ndim; /* 2 or 3 */
    long fs;   /* free surface at kz = 0 */
    long nx, ny, nz;
    float dx, dy, dz, dt;
} wfo_geom;

/* absorb.h:23-75 (2D) and :85-151 (3D) */
void wfo_setup_q(const wfo_geom *g, long nsponge, float freqQ, float qMin, float qInterior, float *q);

/* time steps: the caller swaps (pcur,pold) afterwards, as the reference does internally */
void wfo_step_iso(const wfo_geom *g, const float *v, const float *b, const float *q,
                  const float *pcur, float *pold, float *pspace);
void wfo_step_vti(const wfo_geom *g, long linear, const float *v, const float *eps, const float *eta,
                  const float *b, const float *f, const float *q, const float *pcur, const float *mcur,
                  float *pold, float *mold, float *pspace, float *mspace);
void wfo_step_tti(const wfo_geom *g, const float *v, const float *eps, const float *eta, const float *b,
                  const float *f, const float *q, const float *sint, const float *cost, const float *sinp,
                  const float *cosp, const float *pcur, const float *mcur, float *pold, float *mold,
                  float *pspace, float *mspace);

/* scaleSpatialDerivatives: mspace may be NULL (Iso) */
void wfo_scale(const wfo_geom *g, const float *v, const float *b, float *pspace, float *mspace);

/* standalone staggered derivatives (propagatorStaticFunctions.h); outy ignored in 2D */
void wfo_dplus(const wfo_geom *g, const float *in, float *outx, float *outy, float *outz);
void wfo_dminus(const wfo_geom *g, const float *in, float *outx, float *outy, float *outz);

/* Born injection */
void wfo_born_iso(const wfo_geom *g, long which /*0=V,1=VB,2=B*/, const float *v, const float *b,
                  const float *dv, const float *db, const float *p, const float *dp, float *pcur);
void wfo_born_aniso_v(const wfo_geom *g, const float *v, const float *dv, const float *dp, const float *dm,
                      float *pcur, float *mcur);
void wfo_born_vea(const wfo_geom *g, long tti, const float *v, const float *eps, const float *eta,
                  const float *b, const float *f, const float *sint, const float *cost, const float *sinp,
                  const float *cosp, const float *dv, const float *de, const float *da, const float *p,
                  const float *m, const float *dp, const float *dm, float *pcur, float *mcur);

/* imaging conditions */
void wfo_image_iso(const wfo_geom *g, long which /*0=V,1=VB,2=B*/, const float *v, const float *b,
                   const float *p, const float *dp, const float *pold, float *dv, float *db);
void wfo_image_aniso_v(const wfo_geom *g, const float *v, const float *b, const float *dp, const float *dm,
                       const float *pold, const float *mold, float *dv);
void wfo_image_vea(const wfo_geom *g, long tti, const float *v, const float *eps, const float *eta,
                   const float *b, const float *f, const float *sint, const float *cost, const float *sinp,
                   const float *cosp, const float *p, const float *m, const float *dp, const float *dm,
                   const float *pold, const float *mold, float *dv, float *de, float *da);
/* wavefield separation (dm/mold NULL for Iso); transforms in double precision */
void wfo_image_wavefieldsep(const wfo_geom *g, long isfwi, const float *v, const float *b,
                            const float *dp, const float *pold, const float *dm, const float *mold,
                            float *dv);

/* spacetime.cc:144-162 / :184-204 on a flat, already-ordered point list (1-based iu, ir) */
void wfo_inject(float *field, const float *data, long it, long nt, const long *iu, const long *ir,
                const float *c, long n);
void wfo_extract(float *data, const float *field, long it, long nt, const long *iu, const long *ir,
                 const float *c, long n);

/* spacetime.cc:4-127 time interpolation (h: nh x 8 filters, row-major), nslow traces; nd >= 7 */
void wfo_interpadjoint_float(const float *h, float *m, const float *d, long nh, long nm, long nd, long nslow);
void wfo_interpforward_float(const float *h, float *d, const float *m, long nh, long nd, long nm, long nslow);
void wfo_interpadjoint_double(const double *h, double *m, const double *d, long nh, long nm, long nd, long nslow);
void wfo_interpforward_double(const double *h, double *d, const double *m, long nh, long nd, long nm, long nslow);

/* illumination.c:3-53 (float): field = field^2 when accum is NULL, else accum += field^2 */
void wfo_illum_float(float *accum, float *field, long n);

/* FP64 rerun: the time steps, scaling, standalone D+/D-, Born injection and imaging conditions
 * (V, VB, B for Iso; V for VTI/TTI) and injection/extraction above, evaluated in double precision
 * on double arrays (wfo_generic.inc instantiated with double). */
void wfo64_step_iso(const wfo_geom *g, const double *v, const double *b, const double *q,
                    const double *pcur, double *pold, double *pspace);
void wfo64_step_vti(const wfo_geom *g, long linear, const double *v, const double *eps, const double *eta,
                    const double *b, const double *f, const double *q, const double *pcur,
                    const double *mcur, double *pold, double *mold, double *pspace, double *mspace);
void wfo64_step_tti(const wfo_geom *g, const double *v, const double *eps, const double *eta,
                    const double *b, const double *f, const double *q, const double *sint,
                    const double *cost, const double *sinp, const double *cosp, const double *pcur,
                    const double *mcur, double *pold, double *mold, double *pspace, double *mspace);
void wfo64_scale(const wfo_geom *g, const double *v, const double *b, double *pspace, double *mspace);
void wfo64_dplus(const wfo_geom *g, const double *in, double *outx, double *outy, double *outz);
void wfo64_dminus(const wfo_geom *g, const double *in, double *outx, double *outy, double *outz);
void wfo64_born_iso(const wfo_geom *g, long which, const double *v, const double *b, const double *dv,
                    const double *db, const double *p, const double *dp, double *pcur);
void wfo64_born_aniso_v(const wfo_geom *g, const double *v, const double *dv, const double *dp,
                        const double *dm, double *pcur, double *mcur);
void wfo64_image_iso(const wfo_geom *g, long which, const double *v, const double *b, const double *p,
                     const double *dp, const double *pold, double *dv, double *db);
void wfo64_image_aniso_v(const wfo_geom *g, const double *v, const double *b, const double *dp,
                         const double *dm, const double *pold, const double *mold, double *dv);
void wfo64_inject(double *field, const double *data, long it, long nt, const long *iu, const long *ir,
                  const double *c, long n);
void wfo64_extract(double *data, const double *field, long it, long nt, const long *iu, const long *ir,
                   const double *c, long n);

#ifdef __cplusplus
}
#endif

#endif
