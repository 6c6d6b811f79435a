// The drop-in C ABI: the exact `extern "C"` symbols and signatures of the reference's propagator
// libraries (src/prop{2D,3D}Aco{Iso,VTI,TTI}DenQ_DEO2_FDTD.cc), declared in
// include/wavefd_b200.h, plus the add-on WFD_* entry points of this package.
//
// Drop-in calls keep the reference's contract: void, synchronous, arrays reached through the
// getters (here CUDA managed memory, so a host caller writes them in place), the object owns
// every array and is not re-entrant.
#include <string.h>

#include <string>

#include "wfd_prop.h"

using wfd::Prop;

namespace {

Prop *P(void *p) { return reinterpret_cast<Prop *>(p); }

// Host code may have written the managed arrays it reached through getters since the object's last
// device call; move those back before the kernels run (the kernels would also fault them in on
// demand). Only the arrays whose getters were called, and not an array whose getter has come before
// every one of the last two device calls: that is a time loop passing the pointer on (the reference's
// loop asks for pCur each step), where a prefetch walks the whole array for nothing (0.43 ms for a
// 537 MB array on a B200). Pages that host code does write in such a loop still move back, on demand.
void before_device(Prop *p) { wfd::prefetch_touched(p, p->stream); }

float *getter(void *p, int f) {
    P(p)->host_touched |= 1u << f;
    return P(p)->field[f];
}

}  // namespace

namespace wfd {

void prefetch_touched(Prop *p, cudaStream_t s) {
    const unsigned mask = p->host_touched;
    p->host_touched = 0;
    const size_t bytes = sizeof(float) * (size_t)p->ncells();
    for (int f = 0; f < F_COUNT; f++) {
        if (!(mask >> f & 1u)) {
            p->touch_streak[f] = 0;
            continue;
        }
        const bool again = p->touch_streak[f] >= 2;
        if (p->touch_streak[f] < 255) p->touch_streak[f]++;
        if (again || !p->field[f]) continue;
#if CUDART_VERSION >= 13000
        cudaMemLocation loc{cudaMemLocationTypeDevice, p->device};
        cudaMemPrefetchAsync(p->field[f], bytes, loc, 0, s);
#else
        cudaMemPrefetchAsync(p->field[f], bytes, p->device, s);
#endif
    }
}

}  // namespace wfd

#define WFD_COMMON(NAME)                                                                                   \
    extern "C" void NAME##_free(void *p) { wfd::prop_destroy(P(p)); }                                     \
    extern "C" void NAME##_SetupDtOmegaInvQ(void *p, float freqQ, float qMin, float qInterior) {          \
        wfd::prop_setup_q(P(p), freqQ, qMin, qInterior);                                                   \
    }                                                                                                      \
    extern "C" void NAME##_TimeStep(void *p) {                                                             \
        before_device(P(p));                                                                               \
        wfd::prop_step(P(p), false, true);                                                                 \
    }                                                                                                      \
    extern "C" void NAME##_ScaleSpatialDerivatives(void *p) {                                              \
        before_device(P(p));                                                                               \
        wfd::prop_scale(P(p));                                                                             \
    }                                                                                                      \
    extern "C" long NAME##_getNx(void *p) { return P(p)->nx; }                                             \
    extern "C" long NAME##_getNz(void *p) { return P(p)->nz; }                                             \
    extern "C" float *NAME##_getV(void *p) { return getter(p, wfd::F_V); }                                 \
    extern "C" float *NAME##_getB(void *p) { return getter(p, wfd::F_B); }                                 \
    extern "C" float *NAME##_getDtOmegaInvQ(void *p) { return getter(p, wfd::F_Q); }                       \
    extern "C" float *NAME##_getPSpace(void *p) { return getter(p, wfd::F_PSPACE); }                       \
    extern "C" float *NAME##_getPCur(void *p) { return getter(p, wfd::F_PCUR); }                           \
    extern "C" float *NAME##_getPOld(void *p) { return getter(p, wfd::F_POLD); }

#define WFD_ANISO(NAME)                                                                                    \
    extern "C" float *NAME##_getEps(void *p) { return getter(p, wfd::F_EPS); }                             \
    extern "C" float *NAME##_getEta(void *p) { return getter(p, wfd::F_ETA); }                             \
    extern "C" float *NAME##_getF(void *p) { return getter(p, wfd::F_F); }                                 \
    extern "C" float *NAME##_getMSpace(void *p) { return getter(p, wfd::F_MSPACE); }                       \
    extern "C" float *NAME##_getMCur(void *p) { return getter(p, wfd::F_MCUR); }                           \
    extern "C" float *NAME##_getMOld(void *p) { return getter(p, wfd::F_MOLD); }                           \
    extern "C" void NAME##_ForwardBornInjection_V(void *p, float *dVel, float *wavefieldDP, float *wavefieldDM) { \
        before_device(P(p));                                                                               \
        float *a[3] = {dVel, wavefieldDP, wavefieldDM};                                                    \
        wfd::prop_born(P(p), "V", a, 3);                                                                   \
    }                                                                                                      \
    extern "C" void NAME##_ForwardBornInjection_VEA(void *p, float *dVel, float *dEps, float *dEta,        \
                                                    float *wavefieldP, float *wavefieldM, float *wavefieldDP, \
                                                    float *wavefieldDM) {                                  \
        before_device(P(p));                                                                               \
        float *a[7] = {dVel, dEps, dEta, wavefieldP, wavefieldM, wavefieldDP, wavefieldDM};                \
        wfd::prop_born(P(p), "VEA", a, 7);                                                                 \
    }                                                                                                      \
    extern "C" void NAME##_AdjointBornAccumulation_V(void *p, float *dVel, float *wavefieldDP,             \
                                                     float *wavefieldDM) {                                 \
        before_device(P(p));                                                                               \
        float *a[3] = {dVel, wavefieldDP, wavefieldDM};                                                    \
        wfd::prop_image(P(p), "V", a, 3, 0);                                                               \
    }                                                                                                      \
    extern "C" void NAME##_AdjointBornAccumulation_wavefieldsep_V(void *p, float *dVel, float *wavefieldDP, \
                                                                  float *wavefieldDM, const long isFWI) {  \
        before_device(P(p));                                                                               \
        float *a[3] = {dVel, wavefieldDP, wavefieldDM};                                                    \
        wfd::prop_image(P(p), "wavefieldsep_V", a, 3, isFWI);                                              \
    }                                                                                                      \
    extern "C" void NAME##_AdjointBornAccumulation_VEA(void *p, float *dVel, float *dEps, float *dEta,     \
                                                       float *wavefieldP, float *wavefieldM,               \
                                                       float *wavefieldDP, float *wavefieldDM) {           \
        before_device(P(p));                                                                               \
        float *a[7] = {dVel, dEps, dEta, wavefieldP, wavefieldM, wavefieldDP, wavefieldDM};                \
        wfd::prop_image(P(p), "VEA", a, 7, 0);                                                             \
    }

#define WFD_ISO_BORN(NAME)                                                                                 \
    extern "C" void NAME##_ForwardBornInjection_V(void *p, float *dVel, float *wavefieldDP) {              \
        before_device(P(p));                                                                               \
        float *a[2] = {dVel, wavefieldDP};                                                                 \
        wfd::prop_born(P(p), "V", a, 2);                                                                   \
    }                                                                                                      \
    extern "C" void NAME##_ForwardBornInjection_VB(void *p, float *dVel, float *dBuoy, float *wavefieldP,  \
                                                   float *wavefieldDP) {                                   \
        before_device(P(p));                                                                               \
        float *a[4] = {dVel, dBuoy, wavefieldP, wavefieldDP};                                              \
        wfd::prop_born(P(p), "VB", a, 4);                                                                  \
    }                                                                                                      \
    extern "C" void NAME##_ForwardBornInjection_B(void *p, float *dBuoy, float *wavefieldP, float *wavefieldDP) { \
        before_device(P(p));                                                                               \
        float *a[3] = {dBuoy, wavefieldP, wavefieldDP};                                                    \
        wfd::prop_born(P(p), "B", a, 3);                                                                   \
    }                                                                                                      \
    extern "C" void NAME##_AdjointBornAccumulation_V(void *p, float *dVel, float *wavefieldDP) {           \
        before_device(P(p));                                                                               \
        float *a[2] = {dVel, wavefieldDP};                                                                 \
        wfd::prop_image(P(p), "V", a, 2, 0);                                                               \
    }                                                                                                      \
    extern "C" void NAME##_AdjointBornAccumulation_VB(void *p, float *dVel, float *dBuoy, float *wavefieldP, \
                                                      float *wavefieldDP) {                                \
        before_device(P(p));                                                                               \
        float *a[4] = {dVel, dBuoy, wavefieldP, wavefieldDP};                                              \
        wfd::prop_image(P(p), "VB", a, 4, 0);                                                              \
    }                                                                                                      \
    extern "C" void NAME##_AdjointBornAccumulation_B(void *p, float *dBuoy, float *wavefieldP,             \
                                                     float *wavefieldDP) {                                 \
        before_device(P(p));                                                                               \
        float *a[3] = {dBuoy, wavefieldP, wavefieldDP};                                                    \
        wfd::prop_image(P(p), "B", a, 3, 0);                                                               \
    }                                                                                                      \
    extern "C" void NAME##_AdjointBornAccumulation_wavefieldsep(void *p, float *dVel, float *wavefieldDP,  \
                                                                const long isFWI) {                        \
        before_device(P(p));                                                                               \
        float *a[2] = {dVel, wavefieldDP};                                                                 \
        wfd::prop_image(P(p), "wavefieldsep", a, 2, isFWI);                                                \
    }

#define WFD_LINEAR(NAME)                                                                                   \
    extern "C" void NAME##_TimeStepLinear(void *p) {                                                       \
        before_device(P(p));                                                                               \
        wfd::prop_step(P(p), true, true);                                                                  \
    }

// ---- 3D ----------------------------------------------------------------------------------------------
#define WFD_ALLOC3(NAME, PHYS)                                                                             \
    extern "C" void *NAME##_alloc(long fs, long nthread, long nx, long ny, long nz, long nsponge, float dx, \
                                  float dy, float dz, float dt, long nbx, long nby, long nbz) {            \
        return wfd::prop_create(3, PHYS, fs, nthread, nx, ny, nz, nsponge, dx, dy, dz, dt, nbx, nby, nbz); \
    }                                                                                                      \
    extern "C" long NAME##_getNy(void *p) { return P(p)->ny; }

#define WFD_ALLOC2(NAME, PHYS)                                                                             \
    extern "C" void *NAME##_alloc(long fs, long nthread, long nx, long nz, long nsponge, float dx, float dz, \
                                  float dt, long nbx, long nbz) {                                          \
        return wfd::prop_create(2, PHYS, fs, nthread, nx, 1, nz, nsponge, dx, 1.0f, dz, dt, nbx, 1, nbz);  \
    }

// prop3DAcoIsoDenQ_DEO2_FDTD.cc:6-140
WFD_ALLOC3(Prop3DAcoIsoDenQ_DEO2_FDTD, wfd::ISO)
WFD_COMMON(Prop3DAcoIsoDenQ_DEO2_FDTD)
WFD_ISO_BORN(Prop3DAcoIsoDenQ_DEO2_FDTD)

// prop3DAcoVTIDenQ_DEO2_FDTD.cc:6-157 (getDtOmegaInvQ is an addition here)
WFD_ALLOC3(Prop3DAcoVTIDenQ_DEO2_FDTD, wfd::VTI)
WFD_COMMON(Prop3DAcoVTIDenQ_DEO2_FDTD)
WFD_ANISO(Prop3DAcoVTIDenQ_DEO2_FDTD)
WFD_LINEAR(Prop3DAcoVTIDenQ_DEO2_FDTD)

// prop3DAcoTTIDenQ_DEO2_FDTD.cc:6-180
WFD_ALLOC3(Prop3DAcoTTIDenQ_DEO2_FDTD, wfd::TTI)
WFD_COMMON(Prop3DAcoTTIDenQ_DEO2_FDTD)
WFD_ANISO(Prop3DAcoTTIDenQ_DEO2_FDTD)
extern "C" float *Prop3DAcoTTIDenQ_DEO2_FDTD_getSinTheta(void *p) { return getter(p, wfd::F_ST); }
extern "C" float *Prop3DAcoTTIDenQ_DEO2_FDTD_getCosTheta(void *p) { return getter(p, wfd::F_CT); }
extern "C" float *Prop3DAcoTTIDenQ_DEO2_FDTD_getSinPhi(void *p) { return getter(p, wfd::F_SP); }
extern "C" float *Prop3DAcoTTIDenQ_DEO2_FDTD_getCosPhi(void *p) { return getter(p, wfd::F_CP); }

// ---- 2D ----------------------------------------------------------------------------------------------
// prop2DAcoIsoDenQ_DEO2_FDTD.cc:6-131
WFD_ALLOC2(Prop2DAcoIsoDenQ_DEO2_FDTD, wfd::ISO)
WFD_COMMON(Prop2DAcoIsoDenQ_DEO2_FDTD)
WFD_ISO_BORN(Prop2DAcoIsoDenQ_DEO2_FDTD)

// prop2DAcoVTIDenQ_DEO2_FDTD.cc:6-176
WFD_ALLOC2(Prop2DAcoVTIDenQ_DEO2_FDTD, wfd::VTI)
WFD_COMMON(Prop2DAcoVTIDenQ_DEO2_FDTD)
WFD_ANISO(Prop2DAcoVTIDenQ_DEO2_FDTD)
WFD_LINEAR(Prop2DAcoVTIDenQ_DEO2_FDTD)

// prop2DAcoTTIDenQ_DEO2_FDTD.cc:6-161
WFD_ALLOC2(Prop2DAcoTTIDenQ_DEO2_FDTD, wfd::TTI)
WFD_COMMON(Prop2DAcoTTIDenQ_DEO2_FDTD)
WFD_ANISO(Prop2DAcoTTIDenQ_DEO2_FDTD)
extern "C" float *Prop2DAcoTTIDenQ_DEO2_FDTD_getSinTheta(void *p) { return getter(p, wfd::F_ST); }
extern "C" float *Prop2DAcoTTIDenQ_DEO2_FDTD_getCosTheta(void *p) { return getter(p, wfd::F_CT); }

// prop2DAcoVTIDenQ_DEO2_FDTD.cc:158-176: the standalone 2D D+ with caller-provided coefficients
extern "C" void Prop2DAcoVTIDenQ_DEO2_FDTD_applyFirstDerivatives2D_PlusHalf(
    const long freeSurface, const long nx, const long nz, const long nthread, const float c8_1, const float c8_2,
    const float c8_3, const float c8_4, const float invDx, const float invDz, const float *inX, const float *inZ,
    float *outX, float *outZ, const long BX_2D, const long BZ_2D) {
    (void)nthread;
    (void)BX_2D;
    (void)BZ_2D;
    wfd::apply_dplus2d(freeSurface != 0, nx, nz, c8_1, c8_2, c8_3, c8_4, invDx, invDz, inX, inZ, outX, outZ);
}
