/*
 * WaveFD-B200: the C ABI of the B200 (sm_100a) propagator library.
 *
 * Part 1 declares the drop-in surface: the same extern "C" names, argument lists and meaning as
 * the reference's shared libraries, so that WaveFD's Julia ccall layer (or any other binding)
 * can load this library in their place. Each block cites the reference file it replaces.
 * Contract kept from the reference: calls are synchronous and return nothing; the object owns
 * every array; getters return pointers the caller reads and writes between calls (here CUDA
 * managed memory, so host code may dereference them); objects are not re-entrant.
 *
 * Part 2 declares add-on entry points that the reference does not have (status reporting,
 * asynchronous stepping, device-resident source/receiver tables).
 *
 * Memory layout everywhere: k = (kx*ny + ky)*nz + kz, i.e. a column-major (nz,ny,nx) Julia array.
 */
#ifndef WAVEFD_B200_H
#define WAVEFD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================================== */
/* Part 1: drop-in surface                                                                  */
/* ======================================================================================== */

/* ---- src/prop3DAcoIsoDenQ_DEO2_FDTD.cc:6-140 ---- */
void *Prop3DAcoIsoDenQ_DEO2_FDTD_alloc(long fs, long nthread, long nx, long ny, long nz, long nsponge, float dx,
                                       float dy, float dz, float dt, long nbx, long nby, long nbz);
void Prop3DAcoIsoDenQ_DEO2_FDTD_free(void *p);
void Prop3DAcoIsoDenQ_DEO2_FDTD_SetupDtOmegaInvQ(void *p, float freqQ, float qMin, float qInterior);
void Prop3DAcoIsoDenQ_DEO2_FDTD_TimeStep(void *p);
void Prop3DAcoIsoDenQ_DEO2_FDTD_ScaleSpatialDerivatives(void *p);
void Prop3DAcoIsoDenQ_DEO2_FDTD_ForwardBornInjection_V(void *p, float *dVel, float *wavefieldDP);
void Prop3DAcoIsoDenQ_DEO2_FDTD_ForwardBornInjection_VB(void *p, float *dVel, float *dBuoy, float *wavefieldP,
                                                        float *wavefieldDP);
void Prop3DAcoIsoDenQ_DEO2_FDTD_ForwardBornInjection_B(void *p, float *dBuoy, float *wavefieldP, float *wavefieldDP);
void Prop3DAcoIsoDenQ_DEO2_FDTD_AdjointBornAccumulation_V(void *p, float *dVel, float *wavefieldDP);
void Prop3DAcoIsoDenQ_DEO2_FDTD_AdjointBornAccumulation_VB(void *p, float *dVel, float *dBuoy, float *wavefieldP,
                                                           float *wavefieldDP);
void Prop3DAcoIsoDenQ_DEO2_FDTD_AdjointBornAccumulation_B(void *p, float *dBuoy, float *wavefieldP,
                                                          float *wavefieldDP);
void Prop3DAcoIsoDenQ_DEO2_FDTD_AdjointBornAccumulation_wavefieldsep(void *p, float *dVel, float *wavefieldDP,
                                                                     const long isFWI);
long Prop3DAcoIsoDenQ_DEO2_FDTD_getNx(void *p);
long Prop3DAcoIsoDenQ_DEO2_FDTD_getNy(void *p);
long Prop3DAcoIsoDenQ_DEO2_FDTD_getNz(void *p);
float *Prop3DAcoIsoDenQ_DEO2_FDTD_getV(void *p);
float *Prop3DAcoIsoDenQ_DEO2_FDTD_getB(void *p);
float *Prop3DAcoIsoDenQ_DEO2_FDTD_getDtOmegaInvQ(void *p);
float *Prop3DAcoIsoDenQ_DEO2_FDTD_getPSpace(void *p);
float *Prop3DAcoIsoDenQ_DEO2_FDTD_getPCur(void *p);
float *Prop3DAcoIsoDenQ_DEO2_FDTD_getPOld(void *p);

/* ---- src/prop3DAcoVTIDenQ_DEO2_FDTD.cc:6-157 (getDtOmegaInvQ is an addition) ---- */
void *Prop3DAcoVTIDenQ_DEO2_FDTD_alloc(long fs, long nthread, long nx, long ny, long nz, long nsponge, float dx,
                                       float dy, float dz, float dt, long nbx, long nby, long nbz);
void Prop3DAcoVTIDenQ_DEO2_FDTD_free(void *p);
void Prop3DAcoVTIDenQ_DEO2_FDTD_SetupDtOmegaInvQ(void *p, float freqQ, float qMin, float qInterior);
void Prop3DAcoVTIDenQ_DEO2_FDTD_TimeStepLinear(void *p);
void Prop3DAcoVTIDenQ_DEO2_FDTD_TimeStep(void *p);
void Prop3DAcoVTIDenQ_DEO2_FDTD_ScaleSpatialDerivatives(void *p);
void Prop3DAcoVTIDenQ_DEO2_FDTD_ForwardBornInjection_V(void *p, float *dVel, float *wavefieldDP, float *wavefieldDM);
void Prop3DAcoVTIDenQ_DEO2_FDTD_ForwardBornInjection_VEA(void *p, float *dVel, float *dEps, float *dEta,
                                                         float *wavefieldP, float *wavefieldM, float *wavefieldDP,
                                                         float *wavefieldDM);
void Prop3DAcoVTIDenQ_DEO2_FDTD_AdjointBornAccumulation_V(void *p, float *dVel, float *wavefieldDP,
                                                          float *wavefieldDM);
void Prop3DAcoVTIDenQ_DEO2_FDTD_AdjointBornAccumulation_wavefieldsep_V(void *p, float *dVel, float *wavefieldDP,
                                                                       float *wavefieldDM, const long isFWI);
void Prop3DAcoVTIDenQ_DEO2_FDTD_AdjointBornAccumulation_VEA(void *p, float *dVel, float *dEps, float *dEta,
                                                            float *wavefieldP, float *wavefieldM,
                                                            float *wavefieldDP, float *wavefieldDM);
long Prop3DAcoVTIDenQ_DEO2_FDTD_getNx(void *p);
long Prop3DAcoVTIDenQ_DEO2_FDTD_getNy(void *p);
long Prop3DAcoVTIDenQ_DEO2_FDTD_getNz(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getV(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getEps(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getEta(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getB(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getF(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getDtOmegaInvQ(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getPSpace(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getMSpace(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getPCur(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getPOld(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getMCur(void *p);
float *Prop3DAcoVTIDenQ_DEO2_FDTD_getMOld(void *p);

/* ---- src/prop3DAcoTTIDenQ_DEO2_FDTD.cc:6-180 ---- */
void *Prop3DAcoTTIDenQ_DEO2_FDTD_alloc(long fs, long nthread, long nx, long ny, long nz, long nsponge, float dx,
                                       float dy, float dz, float dt, long nbx, long nby, long nbz);
void Prop3DAcoTTIDenQ_DEO2_FDTD_free(void *p);
void Prop3DAcoTTIDenQ_DEO2_FDTD_SetupDtOmegaInvQ(void *p, float freqQ, float qMin, float qInterior);
void Prop3DAcoTTIDenQ_DEO2_FDTD_TimeStep(void *p);
void Prop3DAcoTTIDenQ_DEO2_FDTD_ScaleSpatialDerivatives(void *p);
void Prop3DAcoTTIDenQ_DEO2_FDTD_ForwardBornInjection_V(void *p, float *dVel, float *wavefieldDP, float *wavefieldDM);
void Prop3DAcoTTIDenQ_DEO2_FDTD_ForwardBornInjection_VEA(void *p, float *dVel, float *dEps, float *dEta,
                                                         float *wavefieldP, float *wavefieldM, float *wavefieldDP,
                                                         float *wavefieldDM);
void Prop3DAcoTTIDenQ_DEO2_FDTD_AdjointBornAccumulation_V(void *p, float *dVel, float *wavefieldDP,
                                                          float *wavefieldDM);
void Prop3DAcoTTIDenQ_DEO2_FDTD_AdjointBornAccumulation_wavefieldsep_V(void *p, float *dVel, float *wavefieldDP,
                                                                       float *wavefieldDM, const long isFWI);
void Prop3DAcoTTIDenQ_DEO2_FDTD_AdjointBornAccumulation_VEA(void *p, float *dVel, float *dEps, float *dEta,
                                                            float *wavefieldP, float *wavefieldM,
                                                            float *wavefieldDP, float *wavefieldDM);
long Prop3DAcoTTIDenQ_DEO2_FDTD_getNx(void *p);
long Prop3DAcoTTIDenQ_DEO2_FDTD_getNy(void *p);
long Prop3DAcoTTIDenQ_DEO2_FDTD_getNz(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getV(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getEps(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getEta(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getSinTheta(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getCosTheta(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getSinPhi(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getCosPhi(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getB(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getF(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getDtOmegaInvQ(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getPSpace(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getMSpace(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getPCur(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getPOld(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getMCur(void *p);
float *Prop3DAcoTTIDenQ_DEO2_FDTD_getMOld(void *p);

/* ---- src/prop2DAcoIsoDenQ_DEO2_FDTD.cc:6-131 ---- */
void *Prop2DAcoIsoDenQ_DEO2_FDTD_alloc(long fs, long nthread, long nx, long nz, long nsponge, float dx, float dz,
                                       float dt, long nbx, long nbz);
void Prop2DAcoIsoDenQ_DEO2_FDTD_free(void *p);
void Prop2DAcoIsoDenQ_DEO2_FDTD_SetupDtOmegaInvQ(void *p, float freqQ, float qMin, float qInterior);
void Prop2DAcoIsoDenQ_DEO2_FDTD_TimeStep(void *p);
void Prop2DAcoIsoDenQ_DEO2_FDTD_ScaleSpatialDerivatives(void *p);
void Prop2DAcoIsoDenQ_DEO2_FDTD_ForwardBornInjection_V(void *p, float *dVel, float *wavefieldDP);
void Prop2DAcoIsoDenQ_DEO2_FDTD_ForwardBornInjection_VB(void *p, float *dVel, float *dBuoy, float *wavefieldP,
                                                        float *wavefieldDP);
void Prop2DAcoIsoDenQ_DEO2_FDTD_ForwardBornInjection_B(void *p, float *dBuoy, float *wavefieldP, float *wavefieldDP);
void Prop2DAcoIsoDenQ_DEO2_FDTD_AdjointBornAccumulation_V(void *p, float *dVel, float *wavefieldDP);
void Prop2DAcoIsoDenQ_DEO2_FDTD_AdjointBornAccumulation_VB(void *p, float *dVel, float *dBuoy, float *wavefieldP,
                                                           float *wavefieldDP);
void Prop2DAcoIsoDenQ_DEO2_FDTD_AdjointBornAccumulation_B(void *p, float *dBuoy, float *wavefieldP,
                                                          float *wavefieldDP);
void Prop2DAcoIsoDenQ_DEO2_FDTD_AdjointBornAccumulation_wavefieldsep(void *p, float *dVel, float *wavefieldDP,
                                                                     const long isFWI);
long Prop2DAcoIsoDenQ_DEO2_FDTD_getNx(void *p);
long Prop2DAcoIsoDenQ_DEO2_FDTD_getNz(void *p);
float *Prop2DAcoIsoDenQ_DEO2_FDTD_getV(void *p);
float *Prop2DAcoIsoDenQ_DEO2_FDTD_getB(void *p);
float *Prop2DAcoIsoDenQ_DEO2_FDTD_getDtOmegaInvQ(void *p);
float *Prop2DAcoIsoDenQ_DEO2_FDTD_getPSpace(void *p);
float *Prop2DAcoIsoDenQ_DEO2_FDTD_getPCur(void *p);
float *Prop2DAcoIsoDenQ_DEO2_FDTD_getPOld(void *p);

/* ---- src/prop2DAcoVTIDenQ_DEO2_FDTD.cc:6-176 ---- */
void *Prop2DAcoVTIDenQ_DEO2_FDTD_alloc(long fs, long nthread, long nx, long nz, long nsponge, float dx, float dz,
                                       float dt, long nbx, long nbz);
void Prop2DAcoVTIDenQ_DEO2_FDTD_free(void *p);
void Prop2DAcoVTIDenQ_DEO2_FDTD_SetupDtOmegaInvQ(void *p, float freqQ, float qMin, float qInterior);
void Prop2DAcoVTIDenQ_DEO2_FDTD_TimeStepLinear(void *p);
void Prop2DAcoVTIDenQ_DEO2_FDTD_TimeStep(void *p);
void Prop2DAcoVTIDenQ_DEO2_FDTD_ScaleSpatialDerivatives(void *p);
void Prop2DAcoVTIDenQ_DEO2_FDTD_ForwardBornInjection_V(void *p, float *dVel, float *wavefieldDP, float *wavefieldDM);
void Prop2DAcoVTIDenQ_DEO2_FDTD_ForwardBornInjection_VEA(void *p, float *dVel, float *dEps, float *dEta,
                                                         float *wavefieldP, float *wavefieldM, float *wavefieldDP,
                                                         float *wavefieldDM);
void Prop2DAcoVTIDenQ_DEO2_FDTD_AdjointBornAccumulation_V(void *p, float *dVel, float *wavefieldDP,
                                                          float *wavefieldDM);
void Prop2DAcoVTIDenQ_DEO2_FDTD_AdjointBornAccumulation_wavefieldsep_V(void *p, float *dVel, float *wavefieldDP,
                                                                       float *wavefieldDM, const long isFWI);
void Prop2DAcoVTIDenQ_DEO2_FDTD_AdjointBornAccumulation_VEA(void *p, float *dVel, float *dEps, float *dEta,
                                                            float *wavefieldP, float *wavefieldM,
                                                            float *wavefieldDP, float *wavefieldDM);
long Prop2DAcoVTIDenQ_DEO2_FDTD_getNx(void *p);
long Prop2DAcoVTIDenQ_DEO2_FDTD_getNz(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getV(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getEps(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getEta(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getB(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getF(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getDtOmegaInvQ(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getPSpace(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getMSpace(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getPCur(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getPOld(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getMCur(void *p);
float *Prop2DAcoVTIDenQ_DEO2_FDTD_getMOld(void *p);
/* src/prop2DAcoVTIDenQ_DEO2_FDTD.cc:158-176 */
void Prop2DAcoVTIDenQ_DEO2_FDTD_applyFirstDerivatives2D_PlusHalf(
    const long freeSurface, const long nx, const long nz, const long nthread, const float c8_1, const float c8_2,
    const float c8_3, const float c8_4, const float invDx, const float invDz, const float *inX, const float *inZ,
    float *outX, float *outZ, const long BX_2D, const long BZ_2D);

/* ---- src/prop2DAcoTTIDenQ_DEO2_FDTD.cc:6-161 ---- */
void *Prop2DAcoTTIDenQ_DEO2_FDTD_alloc(long fs, long nthread, long nx, long nz, long nsponge, float dx, float dz,
                                       float dt, long nbx, long nbz);
void Prop2DAcoTTIDenQ_DEO2_FDTD_free(void *p);
void Prop2DAcoTTIDenQ_DEO2_FDTD_SetupDtOmegaInvQ(void *p, float freqQ, float qMin, float qInterior);
void Prop2DAcoTTIDenQ_DEO2_FDTD_TimeStep(void *p);
void Prop2DAcoTTIDenQ_DEO2_FDTD_ScaleSpatialDerivatives(void *p);
void Prop2DAcoTTIDenQ_DEO2_FDTD_ForwardBornInjection_V(void *p, float *dVel, float *wavefieldDP, float *wavefieldDM);
void Prop2DAcoTTIDenQ_DEO2_FDTD_ForwardBornInjection_VEA(void *p, float *dVel, float *dEps, float *dEta,
                                                         float *wavefieldP, float *wavefieldM, float *wavefieldDP,
                                                         float *wavefieldDM);
void Prop2DAcoTTIDenQ_DEO2_FDTD_AdjointBornAccumulation_V(void *p, float *dVel, float *wavefieldDP,
                                                          float *wavefieldDM);
void Prop2DAcoTTIDenQ_DEO2_FDTD_AdjointBornAccumulation_wavefieldsep_V(void *p, float *dVel, float *wavefieldDP,
                                                                       float *wavefieldDM, const long isFWI);
void Prop2DAcoTTIDenQ_DEO2_FDTD_AdjointBornAccumulation_VEA(void *p, float *dVel, float *dEps, float *dEta,
                                                            float *wavefieldP, float *wavefieldM,
                                                            float *wavefieldDP, float *wavefieldDM);
long Prop2DAcoTTIDenQ_DEO2_FDTD_getNx(void *p);
long Prop2DAcoTTIDenQ_DEO2_FDTD_getNz(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getV(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getEps(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getEta(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getSinTheta(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getCosTheta(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getB(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getF(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getDtOmegaInvQ(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getPSpace(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getMSpace(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getPCur(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getPOld(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getMCur(void *p);
float *Prop2DAcoTTIDenQ_DEO2_FDTD_getMOld(void *p);

/* ---- src/spacetime.cc:132-204 (and src/spacetime.jl:793-808 for the point types) ---- */
typedef struct SourcePoint32 {
    long iu;  /* 1-based linear grid index */
    long ir;  /* 1-based trace index */
    float c;  /* weight */
} SourcePoint32;
typedef struct SourcePoint64 {
    long iu;
    long ir;
    double c;
} SourcePoint64;
void injectdata_float(float *field, float *data, size_t it, size_t nt, SourcePoint32 **partitions,
                      size_t npartitions, long *npoints_per_partition, size_t nthreads);
void injectdata_double(double *field, double *data, size_t it, size_t nt, SourcePoint64 **partitions,
                       size_t npartitions, long *npoints_per_partition, size_t nthreads);
void extractdata_float(float *data, float *field, SourcePoint32 **partitions, size_t npartitions,
                       long *npoints_per_partition, size_t it, size_t nt, size_t nthreads);
void extractdata_double(double *data, double *field, SourcePoint64 **partitions, size_t npartitions,
                        long *npoints_per_partition, size_t it, size_t nt, size_t nthreads);

/* ---- src/spacetime.cc:228-330: time interpolation dtmod <-> dtrec (filters from interpfilters,
 * src/spacetime.jl:333-360; nh pointers to 8 taps each; traces contiguous in time; nd >= 7) ---- */
void interpadjoint_1d_float(float **h, float *m, float *d, size_t nh, size_t nm, size_t nd);
void interpadjoint_1d_double(double **h, double *m, double *d, size_t nh, size_t nm, size_t nd);
void interpforward_1d_float(float **h, float *d, float *m, size_t nh, size_t nd, size_t nm);
void interpforward_1d_double(double **h, double *d, double *m, size_t nh, size_t nd, size_t nm);
void interpadjoint_nd_float(float **h, float *m, float *d, size_t nh, size_t nm, size_t nd, size_t nslow,
                            size_t nthreads);
void interpadjoint_nd_double(double **h, double *m, double *d, size_t nh, size_t nm, size_t nd, size_t nslow,
                             size_t nthreads);
void interpforward_nd_float(float **h, float *d, float *m, size_t nh, size_t nd, size_t nm, size_t nslow,
                            size_t nthreads);
void interpforward_nd_double(double **h, double *d, double *m, size_t nh, size_t nd, size_t nm, size_t nslow,
                             size_t nthreads);

/* ---- src/illumination.c:3-53 (libillumination): field = field^2; accum += field^2 ---- */
void srcillum_helper_float(float *field_ginsu, size_t n, int nthreads);
void srcillum_helper_double(double *field_ginsu, size_t n, int nthreads);
void illum_accumulate_float(float *field_ginsu_accum, float *field_ginsu, size_t n, int nthreads);
void illum_accumulate_double(double *field_ginsu_accum, double *field_ginsu, size_t n, int nthreads);

/* ======================================================================================== */
/* Part 2: add-on entry points (no counterpart in the reference)                            */
/* ======================================================================================== */

/* status codes */
#define WFD_OK 0
#define WFD_ERR_CUDA 1
#define WFD_ERR_ALLOC 2
#define WFD_ERR_ARG 3
#define WFD_ERR_UNSUPPORTED 4
#define WFD_ERR_TIMEOUT 5
#define WFD_ERR_IO 6

/* last error of calls that have no object (alloc, spacetime), and of a given object */
int WFD_LastError(void);
const char *WFD_LastErrorMessage(void);
int WFD_Prop_Status(void *p);
const char *WFD_Prop_Message(void *p);

/* Failure-detection hook (no counterpart in the reference): the limit, in ns, of the waits of the TMA
 * step kernels for their tile loads (default 2 s; 0 restores it). A wait that runs out makes the
 * kernel record a timeout in its device status word, let its copies in flight land and leave; the
 * object then reports WFD_ERR_TIMEOUT. Tests shorten the limit to make a wait run out. Device-wide
 * and synchronous; not for use while other work runs. */
int WFD_Debug_SetPipelineWait(unsigned long long ns);

/* 1 = bitwise-parity kernels (IEEE order, no FMA), 0 = fast kernels (default) */
int WFD_Prop_SetStrict(void *p, int strict);
/* 1 = fused single-sweep step kernels where available (default), 0 = the two-pass kernels */
int WFD_Prop_SetFused(void *p, int fused);
/* enqueue nsteps time steps (linear != 0: TimeStepLinear) without host synchronisation */
int WFD_Prop_TimeStepAsync(void *p, long nsteps, int linear);
int WFD_Prop_Synchronize(void *p);
/* move every array of the object to device memory (after host writes through the getters) */
int WFD_Prop_Prefetch(void *p);
/* the object's CUDA stream (a cudaStream_t) */
void *WFD_Prop_Stream(void *p);
/* kernels the last time step launched: 1 = fused single-sweep kernel, 2 = the two passes (one more
 * when a source illumination sum is attached and the step kernel does not accumulate it itself);
 * after WFD_Prop_Run, the launches per step of its loop (step kernels, the injection unless the step
 * kernel applied it, the extraction) */
int WFD_Prop_StepKernels(void *p);
/* kernels launched by the last WFD_Prop_Run (one for a 2D Iso loop run as a single cooperative launch) */
long WFD_Prop_RunLaunches(void *p);
/* No counterpart in the reference as one call: TimeStep followed by ForwardBornInjection_V
 * (WFD_Prop_TimeStepBorn) or by AdjointBornAccumulation_V (WFD_Prop_TimeStepImage), with the
 * reference's arithmetic for each (prop3DAcoIsoDenQ_DEO2_FDTD.h:305-334 / :518-546,
 * prop3DAcoVTIDenQ_DEO2_FDTD.h:420-452 / :564-589, prop3DAcoTTIDenQ_DEO2_FDTD.h:423-452 / :567-592).
 * The 3D step kernels apply them to each cell as they write it, so the fields cross HBM once; 2D
 * objects run the separate kernels after the step. The imaging condition's pOld/mOld are the
 * step's input pCur/mCur, as they are after the reference's TimeStep. wavefieldDM is required for
 * VTI/TTI, ignored for Iso. linear != 0 (VTI only): the step is TimeStepLinear, as the reference's
 * adjoint propagation uses. Device or managed arrays only; asynchronous on the object's stream. */
int WFD_Prop_TimeStepBorn(void *p, const float *dVel, const float *wavefieldDP, const float *wavefieldDM);
int WFD_Prop_TimeStepImage(void *p, float *dVel, const float *wavefieldDP, const float *wavefieldDM, int linear);
/* No counterpart in the reference as one call: TimeStep followed by ScaleSpatialDerivatives (3D Iso
 * .h:269-291, VTI .h:384-407, TTI .h:387-415): the 3D step kernels write pSpace (mSpace) already
 * multiplied by V^2/B. Asynchronous on the object's stream. */
int WFD_Prop_TimeStepScaled(void *p);
/* Source illumination fused into the time step: with a device sum attached (ncells floats), every
 * later step adds pCur^2 (the field the step reads) to it, as illum_accumulate_float would; the 3D
 * Iso, VTI and TTI step kernels (nz a multiple of 4) do it in place of a separate pass. NULL
 * detaches. */
int WFD_Prop_SetIllumination(void *p, float *accum);
/* nsteps time steps of the object (TimeStep, then injection into pCur at time index it, then
 * extraction of pCur at it, it = it0, it0+1, ...; either table may be NULL), with every pair of steps
 * replayed from one CUDA graph when use_graph != 0; indices beyond nt are skipped. A 2D Iso object
 * (fused kernels, no illumination sum, at most 1024 source groups) runs the whole loop as one
 * cooperative launch instead, with a grid-wide barrier between steps (bounded: a barrier that waits
 * longer than 2 s returns WFD_ERR_TIMEOUT). Enqueued on the object's stream; returns after the
 * launches are complete. */
int WFD_Prop_Run(void *p, long nsteps, long it0, void *src_table, const float *wavelet, void *rec_table,
                 float *traces, long nt, int use_graph);
/* device-resident source/receiver tables built from a flat point list (grouped by written
 * location, contributions accumulated in list order, as the reference does partition-wise) */
void *WFD_Points_Create(const SourcePoint32 *points, long npoints, int by_receiver);
void WFD_Points_Free(void *table);
long WFD_Points_Groups(void *table);
/* field[iu-1] += c * data[(ir-1)*nt + it-1] on the device; data column-major (nt, ntraces) */
int WFD_Inject(void *table, float *field, const float *data, long it, long nt, void *stream);
/* data[(ir-1)*nt + it-1] += c * field[iu-1] on the device */
int WFD_Extract(void *table, float *data, const float *field, long it, long nt, void *stream);

/* Time interpolation on device arrays (the arithmetic of interpforward_nd_float (forward != 0:
 * out = nd x nslow coarse from in = nm x nslow fine) or interpadjoint_nd_float), h = nh x 8 taps
 * in device memory, asynchronous on `stream`. */
int WFD_Interp(int forward, const float *h, float *out, const float *in, long nh, long nm, long nd, long nslow,
               void *stream);
/* Receiver extraction streamed into the forward time interpolation: at fine step it (1-based, of
 * nm) each receiver trace's sample (field values through a WFD_Points_Create(..., 1) table) is
 * added into the coarse traces (nd x ntraces, zeroed by the caller before the first step) with
 * the taps h (device, nh x 8); after the last step the coarse traces equal extractdata into a fine
 * buffer followed by interpforward_nd_float, bit for bit, with no fine buffer. */
int WFD_ExtractInterp(void *table, float *coarse, const float *field, const float *h, long nh, long it, long nm,
                      long nd, void *stream);

/* Source illumination for the time loop: accum[i] += field[i]^2 on device arrays (the arithmetic of
 * illum_accumulate_float), asynchronous on `stream`. */
int WFD_IllumAccumulate(float *accum, const float *field, long n, void *stream);

/* Snapshot files: saved forward fields on disk with an offsets/lengths index, the role of
 * Compressor/compressedwrite/compressedread! (src/compressedio.jl:1-137) for the plain FP32
 * fallback and for codec codes. Layout: a header ("WFDSNAP1", version, flags, nfields, slot bytes,
 * data offset, then per field offset and length, -1 = never written; a multiple of 4096 bytes)
 * and field i's payload at data offset + i * slot (slot = max_bytes rounded up to 4096). Writes and
 * reads of device arrays are stream-ordered and asynchronous (device staging, pinned staging, a
 * worker thread doing pwrite/pread); a write's source may be overwritten as soon as later work on
 * `stream` runs. I/O errors (short writes: "wrote X of Y bytes of field i in <path>") are
 * WFD_ERR_IO, reported by the call that sees them (the next Write/Read/Sync/Close). */
#define WFD_SNAP_READ 1   /* open an existing file (nfields, max_bytes come from its header) */
#define WFD_SNAP_HOST 2   /* payloads are host memory: pwrite/pread only, no CUDA call */
#define WFD_SNAP_DIRECT 4 /* O_DIRECT for payloads where the file system allows it */
#define WFD_SNAP_CODEC 8  /* recorded in the header: the payloads are codec codes */
void *WFD_Snap_Open(const char *path, long nfields, long max_bytes, int flags);
int WFD_Snap_Write(void *f, long ifield, const void *src, long nbytes, void *stream);
/* start reading field ifield into a staging slot (a later Read of it only waits) */
int WFD_Snap_Prefetch(void *f, long ifield);
int WFD_Snap_Read(void *f, long ifield, void *dst, long nbytes, void *stream);
long WFD_Snap_Length(void *f, long ifield);
long WFD_Snap_NumFields(void *f);
int WFD_Snap_Flags(void *f);
/* wait for every transfer, then write the header (index) */
int WFD_Snap_Sync(void *f);
int WFD_Snap_Close(void *f);

/* Batched shots (no counterpart in the reference, whose Ginsu is exported but not defined,
 * src/WaveFD.jl:52). A batch advances many 3D objects made by the *_alloc calls above (uneven sizes;
 * Iso, VTI and TTI mixed; same dx, dy, dz, dt, free surface and strict/fast mode; nz a multiple of 4)
 * with one persistent launch per physics class per time step; each object's arrays are bitwise
 * those of stepping it alone, and its getters and pointer swap stay valid. The objects must outlive
 * the batch. Returns NULL on error (WFD_LastError). */
void *WFD_Batch_Create(void *const *props, long nprops);
void WFD_Batch_Free(void *batch);
int WFD_Batch_Status(void *batch);
const char *WFD_Batch_Message(void *batch);
/* Sources and receivers of shot i (its points, 1-based iu into that object's grid and ir into the
 * traces) with device-resident wavelet and traces, column-major (nt, ntraces). Each step injects
 * the wavelet at the current time index into pCur after the step, then extracts pCur into the
 * traces, as WFD_Inject / WFD_Extract do; time indices beyond nt are skipped. nsrc = nrec = 0 clears. */
int WFD_Batch_SetAcquisition(void *batch, long shot, const SourcePoint32 *src, long nsrc, const float *wavelet,
                             const SourcePoint32 *rec, long nrec, float *traces, long nt);
/* Explicit plan: x-chunk length target (the tiles' extent along the sweep; 0 = whole nx), item order
 * (0 = longest first, 1 = shots interleaved), class launches concurrent (1) or serial (0). */
int WFD_Batch_Plan(void *batch, long xchunk_target, int order, int concurrent);
/* Autotune the plan by timing candidate launches (reps each) on the batch's own arrays; the arrays
 * the trial launches overwrite are saved first and restored after (a temporary device copy). */
int WFD_Batch_Tune(void *batch, int reps);
/* Advance every shot nsteps time steps, injecting/extracting at time indices it0, it0+1, ...;
 * use_graph != 0 replays a captured two-step CUDA graph. Asynchronous on the batch's stream, which
 * is ordered after, and before, work on the objects' own streams. */
int WFD_Batch_Run(void *batch, long nsteps, long it0, int use_graph);
int WFD_Batch_Synchronize(void *batch);
void *WFD_Batch_Stream(void *batch);
/* info[0..15]: per class (Iso, VTI, TTI) {shots, items, CTAs, x-chunk target}; mode (0 concurrent);
 * item orders (bit per class); kernels per step; tuned. */
int WFD_Batch_Info(void *batch, long *info, long ninfo);
/* Ginsu window of a survey array: shot[x,y,z] = survey[x0+x, y0+y, z0+z] (indices clamped to the
 * survey), and the scatter-add of a shot image back into the survey image. Device arrays, (nz,ny,nx)
 * z-fastest; asynchronous on `stream`. */
int WFD_Ginsu_Crop(const float *survey, long snx, long sny, long snz, long x0, long y0, long z0, float *shot,
                   long nx, long ny, long nz, void *stream);
int WFD_Ginsu_Accumulate(float *survey, long snx, long sny, long snz, long x0, long y0, long z0, const float *shot,
                         long nx, long ny, long nz, void *stream);

/* Learned wavefield codec (no counterpart in the reference's arithmetic; it takes the role of
 * CvxCompress in src/compressedio.jl:1-137, which compresses the saved forward fields). A 3D conv
 * autoencoder (4^3/s4 1->16, 2^3/s2 16->32, and back), BF16 weights, FP32 accumulation: each 8^3
 * block becomes 32 BF16 values and one FP32 scale. Device arrays, (nz,ny,nx) z-fastest; latent
 * buffers hold WFD_Codec_LatentBytes bytes. Encode/decode are asynchronous on `stream`. */
long WFD_Codec_NumParams(void);
long WFD_Codec_LatentBytes(long nx, long ny, long nz);
void *WFD_Codec_Create(unsigned seed);
void WFD_Codec_Free(void *codec);
/* FP32 master weights (host arrays of WFD_Codec_NumParams floats); SetWeights resets Adam's moments */
int WFD_Codec_SetWeights(void *codec, const float *w, long n);
int WFD_Codec_GetWeights(void *codec, float *w, long n);
int WFD_Codec_Encode(void *codec, const float *field, long nx, long ny, long nz, void *latent, void *stream);
int WFD_Codec_Decode(void *codec, const void *latent, long nx, long ny, long nz, float *field, void *stream);
/* Encode/decode engine: 0 = mma.sync, 1 = tcgen05 tensor cores (UMMA with the accumulators in tensor
 * memory), 2 = encode on mma.sync and decode on tcgen05 (the default: the faster kernel of each
 * direction). The kernels read each other's codes. WFD_ERR_UNSUPPORTED when the tcgen05 kernels cannot
 * be launched here. WAVEFD_B200_CODEC=mma or =tcgen05 selects engine 0 or 1 at creation. */
int WFD_Codec_SetEngine(void *codec, int engine);
int WFD_Codec_Engine(void *codec);
/* CTAs launched by the encode (0: mma.sync, 2: tcgen05) and decode (1: mma.sync, 3: tcgen05) kernels */
int WFD_Codec_Grid(void *codec, int kernel);
/* Synchronises the device; WFD_ERR_TIMEOUT (and clears it) when a tcgen05 completion wait of an
 * encode or decode ran out (bounded at 2 s), else WFD_OK. */
int WFD_Codec_Status(void *codec);
/* training: n 8^3 blocks at device origins[3*i..] (x, y, z) gathered in the codec's cell order and
 * scaled by their max |value| (scales optional); one Adam step on a device batch of blocks
 * (*loss, host, receives the batch's mean squared error before the step); the gradient of that
 * loss without a step (host arrays grad[NumParams], *loss) */
int WFD_Codec_GatherBlocks(const float *field, long nx, long ny, long nz, const int *origins, long n, float *blocks,
                           float *scales, void *stream);
int WFD_Codec_TrainStep(void *codec, const float *blocks, long n, float lr, float *loss, void *stream);
int WFD_Codec_Gradient(void *codec, const float *blocks, long n, float *grad, float *loss);

/* No counterpart in the reference. The wavefield-separation imaging condition (the arithmetic of
 * AdjointBornAccumulation_wavefieldsep / _wavefieldsep_V) for callers that cannot call cudaMalloc:
 * it allocates no memory. Every array must already be device or managed memory (nx*ny*nz floats,
 * z fastest; ny = 1 for 2D; wavefieldDM and mOld both NULL for the isotropic case); dVel is
 * accumulated. Its FFT scratch is a fixed 160 KiB device array inside the library, so nz is
 * limited to 2048 (larger nz returns WFD_ERR_ARG). The first call on each device looks up that
 * array's device address; make that first call before any stream capture, and do not use the
 * entry point across a cudaDeviceReset. The image must be on the current device. All calls share
 * the array (it keeps the tables of the last FFT length): calls that overlap on the GPU race. The
 * arithmetic is the fast build's, or the bitwise-parity build's when WAVEFD_B200_STRICT=1 (as for
 * new propagator objects). Work is enqueued on `stream` (a cudaStream_t, NULL for the default
 * stream) without host synchronisation. Returns a WFD_* status. */
int WFD_AdjointBornAccumulation_wavefieldsep_NoAlloc(long nx, long ny, long nz, long isFWI, const float *v,
                                                     const float *b, const float *wavefieldDP, const float *pOld,
                                                     const float *wavefieldDM, const float *mOld, float *dVel,
                                                     void *stream);

#ifdef __cplusplus
}
#endif

#endif /* WAVEFD_B200_H */
