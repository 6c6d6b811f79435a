// Launch interface of the CUDA kernels. Each kernel translation unit is compiled twice (see
// wfd_common.cuh); the dispatcher picks wfd_strict (bitwise parity with the reference) or
// wfd_fast (FMA contraction, approximate division) per propagator object.
#pragma once

#include <cuda_runtime.h>

#include "wfd_common.cuh"

namespace wfd {

// Model and wavefield arrays of one propagator object (device-accessible pointers).
struct Fields {
    float *v, *b, *q, *eps, *eta, *f, *st, *ct, *sp, *cp;
    float *pcur, *pold, *pspace, *mcur, *mold, *mspace;
};

// Scratch of the unfused passes (the reference's tmp arrays), device memory.
struct Scratch {
    float *t[12];
};

}  // namespace wfd

#define WFD_DECLARE_LAUNCHERS(NS)                                                                        \
    namespace NS {                                                                                       \
    /* unfused reference pass structure */                                                               \
    void pass1(const wfd::Grid &g, int phys, const wfd::Fields &F, const wfd::Scratch &S, cudaStream_t s); \
    void pass2(const wfd::Grid &g, int phys, int linear, const wfd::Fields &F, const wfd::Scratch &S,    \
               cudaStream_t s);                                                                          \
    /* fused single-sweep steps; return false when the geometry is not handled */                        \
    bool fused_step(const wfd::Grid &g, int phys, int linear, const wfd::Fields &F, cudaStream_t s);     \
    void scale(const wfd::Grid &g, const wfd::Fields &F, bool two, cudaStream_t s);                      \
    void dplus(const wfd::Grid &g, const float *in, float *ox, float *oy, float *oz, cudaStream_t s);    \
    void dplus3(const wfd::Grid &g, const float *inx, const float *iny, const float *inz, float *ox,     \
                float *oy, float *oz, cudaStream_t s);                                                   \
    bool fused_iso3d(const wfd::Grid &g, const wfd::Fields &F, cudaStream_t s);                          \
    bool fused_iso3d_tma(const wfd::Grid &g, const wfd::Fields &F, cudaStream_t s);                      \
    bool fused_aniso3d_tma(const wfd::Grid &g, int phys, int linear, const wfd::Fields &F, cudaStream_t s); \
    unsigned iso3d_status_and_clear();                                                                   \
    unsigned aniso3d_status_and_clear();                                                                 \
    unsigned fused_status_and_clear();                                                                   \
    void dminus3(const wfd::Grid &g, const float *fx, const float *fy, const float *fz, float *ox,       \
                 float *oy, float *oz, cudaStream_t s);                                                  \
    void tti_dplus(const wfd::Grid &g, const wfd::Fields &F, const float *in, float *o1, float *o2,      \
                   float *o3, cudaStream_t s);                                                           \
    void tti_dminus(const wfd::Grid &g, const wfd::Fields &F, const float *i1, const float *i2,          \
                    const float *i3, float *o1, float *o2, float *o3, cudaStream_t s);                   \
    void born_iso(const wfd::Grid &g, int which, const wfd::Fields &F, const float *dv, const float *db, \
                  const float *dp, const float *const *lap, cudaStream_t s);                            \
    void born_iso_scaleb(const wfd::Grid &g, const float *db, const float *const *t1, float *const *t2,  \
                         cudaStream_t s);                                                                \
    void born_aniso_v(const wfd::Grid &g, const wfd::Fields &F, const float *dv, const float *dp,        \
                      const float *dm, cudaStream_t s);                                                  \
    void born_vea_sandwich(const wfd::Grid &g, const wfd::Fields &F, const float *de, const float *da,   \
                           const float *const *tp1, const float *const *tm1, float *const *tp2,          \
                           float *const *tm2, cudaStream_t s);                                           \
    void born_vea_final(const wfd::Grid &g, const wfd::Fields &F, const float *dv, const float *dp,      \
                        const float *dm, const float *const *lp, const float *const *lm, cudaStream_t s); \
    void image_iso(const wfd::Grid &g, int which, const wfd::Fields &F, const float *dp,                 \
                   const float *const *t1, const float *const *t2, float *dv, float *db, cudaStream_t s); \
    void image_aniso_v(const wfd::Grid &g, const wfd::Fields &F, const float *dp, const float *dm,       \
                       float *dv, cudaStream_t s);                                                       \
    void image_vea(const wfd::Grid &g, const wfd::Fields &F, const float *dp, const float *dm,           \
                   const float *const *tp1, const float *const *tm1, const float *const *tp2,            \
                   const float *const *tm2, float *dv, float *de, float *da, cudaStream_t s);            \
    void image_wavefieldsep(const wfd::Grid &g, long isfwi, const wfd::Fields &F, const float *dp,       \
                            const float *dm, float *dv, float2 *work, long ncols_per_pass,               \
                            cudaStream_t s);                                                             \
    void image_wavefieldsep_tables(const wfd::Grid &g, long isfwi, const wfd::Fields &F, const float *dp, \
                                   const float *dm, float *dv, const float2 *tables, int m,              \
                                   cudaStream_t s);                                                      \
    }

WFD_DECLARE_LAUNCHERS(wfd_fast)
WFD_DECLARE_LAUNCHERS(wfd_strict)
