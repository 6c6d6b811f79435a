// Launch interface of the CUDA kernels. Each kernel translation unit is compiled twice (see
// wfd_common.cuh); the dispatcher picks wfd_strict (bitwise parity with the reference) or
// wfd_fast (FMA contraction, approximate division) per propagator object.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "wfd_common.cuh"

namespace wfd {

// Model and wavefield arrays of one propagator object (device-accessible pointers).
// A source injection that a step kernel applies to the field it writes (graph-replayed time loops,
// where the time index sits in device memory): new field[key[g]] += c[j] * wav[other[j] * nt + it-1]
// for j = start[g] .. start[g+1]-1 in order, each product and sum rounded (IEEE), it = *d_it,
// nothing when it is outside 1..nt. ngroups = 0: no injection in the step kernel.
struct StepInject {
    long ngroups;
    const long *key, *start, *other;
    const float *c, *wav;
    long nt;
    const long *d_it;
};

// Work fused into the end of a 3D step (single objects; a null pointer turns it off), each cell as
// the reference computes it, so that the arrays cross HBM once:
// * born: ForwardBornInjection_V applied to the new fields right after the step (3D Iso
//   prop3DAcoIsoDenQ_DEO2_FDTD.h:305-334: p += dt^2 V^2/B DP (2B dV/V^3); VTI/TTI .h:420-452 /
//   :423-452: p += 2 dt^2 dV/V DP, m += 2 dt^2 dV/V DM);
// * image: AdjointBornAccumulation_V right after the step, whose pOld/mOld are the step's input
//   pCur/mCur (3D Iso .h:518-546: img += 2B/V^3 DP pOld; VTI/TTI .h:564-589 / :567-592:
//   img += 2B/V^3 (DP pOld + DM mOld)).
// * scale_space: ScaleSpatialDerivatives right after the step (3D Iso .h:269-291, VTI .h:384-407, TTI
//   .h:387-415): pSpace (and mSpace) written already multiplied by V^2/B.
struct StepEpilogue {
    const float *born_dv, *born_dp, *born_dm;
    float *img;
    const float *img_dp, *img_dm;
    int scale_space;
};

// Receiver extraction inside a persistent time loop: data[key[g]*nt + it-1] += c[j] * field[other[j]]
// for j = start[g] .. start[g+1]-1 in order, each product and sum rounded (IEEE).
struct RunExtract {
    long ngroups;
    const long *key, *start, *other;
    const float *c;
    float *data;
    long nt;
};

struct Fields {
    float *v, *b, *q, *eps, *eta, *f, *st, *ct, *sp, *cp;
    float *pcur, *pold, *pspace, *mcur, *mold, *mspace;
    float *illum;  // source illumination sum (sum over steps of pCur^2), or nullptr
    StepInject inj;
    StepEpilogue epi;
};

// Scratch of the unfused passes (the reference's tmp arrays), device memory.
struct Scratch {
    float *t[12];
};

// Tensor maps of the TMA step kernels, passed by value (single object) or held in a shot descriptor.
struct IsoMaps {
    CUtensorMap m[7];  // pCur halo box, pCur tile, B halo box, B tile, pOld, V, Q
};
struct AnisoMaps {
    CUtensorMap m[15];  // pCur, mCur (ring boxes), b, eps, eta, f, st, ct, sp, cp (halo boxes), pOld, mOld, V, Q, b
};

// One shot of a batched launch (device memory, read by the kernel per work item): its sizes, the
// arrays the kernel stores to, its tensor maps and its x-chunk length. A work item is (shot,
// local item) with local item = (chunk * nty + tile_y) * ntz + tile_z.
struct alignas(64) IsoShotDesc {
    CUtensorMap m[7];
    float *pold, *pspace;
    int nx, ny, nz, ntz, nty, xchunk;
};
struct alignas(64) AnisoShotDesc {
    CUtensorMap m[15];
    float *pold, *mold, *pspace, *mspace;
    int nx, ny, nz, ntz, nty, xchunk;
};

// Tile geometry and capacity of a TMA step kernel, for the batch planner.
struct TileInfo {
    int tz, ty;      // (z, y) cross-section of a tile
    int warmup;      // planes swept before the first output plane of an x-chunk
    int grid_cap;    // resident CTAs on this device (SMs x CTAs per SM)
};

}  // namespace wfd

#define WFD_DECLARE_LAUNCHERS(NS)                                                                        \
    namespace NS {                                                                                       \
    /* unfused reference pass structure */                                                               \
    void pass1(const wfd::Grid &g, int phys, const wfd::Fields &F, const wfd::Scratch &S, cudaStream_t s); \
    void pass2(const wfd::Grid &g, int phys, int linear, const wfd::Fields &F, const wfd::Scratch &S,    \
               cudaStream_t s);                                                                          \
    /* fused single-sweep steps; 0 when the geometry is not handled, else flags: 1 stepped, 2 F.illum \
       accumulated inside the step kernel, 4 F.inj applied inside the step kernel, 8 F.epi applied  \
       inside the step kernel */                                                                         \
    int fused_step(const wfd::Grid &g, int phys, int linear, const wfd::Fields &F, cudaStream_t s);      \
    void scale(const wfd::Grid &g, const wfd::Fields &F, bool two, cudaStream_t s);                      \
    void dplus3(const wfd::Grid &g, const float *inx, const float *iny, const float *inz, float *ox,     \
                float *oy, float *oz, cudaStream_t s);                                                   \
    bool fused_iso3d(const wfd::Grid &g, const wfd::Fields &F, cudaStream_t s);                          \
    bool fused_iso2d(const wfd::Grid &g, const wfd::Fields &F, cudaStream_t s);                          \
    bool fused_aniso2d(const wfd::Grid &g, int phys, int linear, const wfd::Fields &F, cudaStream_t s);  \
    /* whole 2D Iso time loop in one cooperative launch: 0 launched, -1 not available, 1 launch error */ \
    int iso2d_run(const wfd::Grid &g, const wfd::Fields &F, long nsteps, long it0, const wfd::RunExtract &ex, \
                  unsigned *sync_words, cudaStream_t s);                                                 \
    /* the same for 2D VTI and TTI (phys), the tiles shared out over the co-resident CTAs */           \
    int aniso2d_run(const wfd::Grid &g, int phys, const wfd::Fields &F, long nsteps, long it0,          \
                    const wfd::RunExtract &ex, unsigned *sync_words, cudaStream_t s);                    \
    bool fused_iso3d_tma(const wfd::Grid &g, const wfd::Fields &F, cudaStream_t s);                      \
    bool fused_aniso3d_tma(const wfd::Grid &g, int phys, int linear, const wfd::Fields &F, cudaStream_t s); \
    bool fused_vti3d_tma(const wfd::Grid &g, int linear, const wfd::Fields &F, cudaStream_t s);         \
    bool vti3d_tma_describe(const wfd::Grid &g, const wfd::Fields &F, int xchunk, wfd::AnisoShotDesc *d, \
                            wfd::TileInfo *t);                                                           \
    void vti3d_tma_batch(const wfd::Grid &gc, const wfd::AnisoShotDesc *shots, const int *sel,          \
                         const int2 *items, int nitems, int *counter, int grid, cudaStream_t s);        \
    unsigned vti3d_status_and_clear();                                                                   \
    unsigned iso3d_status_and_clear();                                                                   \
    /* batched launches over many shots (descriptors and items in device memory) */                     \
    bool iso3d_tma_describe(const wfd::Grid &g, const wfd::Fields &F, int xchunk, wfd::IsoShotDesc *d,   \
                            wfd::TileInfo *t);                                                           \
    void iso3d_tma_batch(const wfd::Grid &gc, const wfd::IsoShotDesc *shots, const int *sel,            \
                         const int2 *items, int nitems, int *counter, int grid, cudaStream_t s);        \
    bool aniso3d_tma_describe(const wfd::Grid &g, int phys, const wfd::Fields &F, int xchunk,           \
                              wfd::AnisoShotDesc *d, wfd::TileInfo *t);                                  \
    void aniso3d_tma_batch(const wfd::Grid &gc, int phys, const wfd::AnisoShotDesc *shots,              \
                           const int *sel, const int2 *items, int nitems, int *counter, int grid,       \
                           cudaStream_t s);                                                              \
    unsigned aniso3d_status_and_clear();                                                                 \
    unsigned fused_status_and_clear();                                                                   \
    void iso3d_set_pipeline_wait(unsigned long long ns);                                                 \
    void vti3d_set_pipeline_wait(unsigned long long ns);                                                 \
    void aniso3d_set_pipeline_wait(unsigned long long ns);                                               \
    void fused_set_pipeline_wait(unsigned long long ns);                                                 \
    void born_iso_v(const wfd::Grid &g, const wfd::Fields &F, const float *dv, const float *dp,          \
                    cudaStream_t s);                                                                     \
    void born_aniso_v(const wfd::Grid &g, const wfd::Fields &F, const float *dv, const float *dp,        \
                      const float *dm, cudaStream_t s);                                                  \
    void image_iso_v(const wfd::Grid &g, const wfd::Fields &F, const float *dp, float *dv,              \
                     cudaStream_t s);                                                                    \
    void image_aniso_v(const wfd::Grid &g, const wfd::Fields &F, const float *dp, const float *dm,       \
                       float *dv, cudaStream_t s);                                                       \
    /* the VB/B and VEA Born injections and imaging conditions with the gradient triples and their D-  \
       formed per cell (t: 3 scratch arrays for born_iso_fused, 6 for born_vea_fused) */                 \
    void born_iso_fused(const wfd::Grid &g, int which, const wfd::Fields &F, const float *dv,            \
                        const float *db, const float *P, const float *dp, float *const *t, cudaStream_t s); \
    void image_iso_fused(const wfd::Grid &g, int which, const wfd::Fields &F, const float *dp,          \
                         const float *P, float *dv, float *db, cudaStream_t s);                          \
    void born_vea_fused(const wfd::Grid &g, bool rot, const wfd::Fields &F, const float *dv,             \
                        const float *de, const float *da, const float *P, const float *M, const float *dp, \
                        const float *dm, float *const *t, cudaStream_t s);                              \
    void image_vea_fused(const wfd::Grid &g, bool rot, const wfd::Fields &F, const float *dp,            \
                         const float *dm, const float *P, const float *M, float *dv, float *de, float *da, \
                         cudaStream_t s);                                                                \
    void image_wavefieldsep(const wfd::Grid &g, long isfwi, const wfd::Fields &F, const float *dp,       \
                            const float *dm, float *dv, float2 *work, long ncols_per_pass,               \
                            cudaStream_t s);                                                             \
    void image_wavefieldsep_tables(const wfd::Grid &g, long isfwi, const wfd::Fields &F, const float *dp, \
                                   const float *dm, float *dv, const float2 *tables, int m,              \
                                   cudaStream_t s);                                                      \
    }

WFD_DECLARE_LAUNCHERS(wfd_fast)
WFD_DECLARE_LAUNCHERS(wfd_strict)
