// The reference's own time-step passes instantiated with Type = double -- TEST INFRASTRUCTURE ONLY.
//
// The pass functions of src/prop{2D,3D}Aco{Iso,VTI,TTI}DenQ_DEO2_FDTD.h are static member
// templates on the arithmetic type; the reference instantiates them with float. This harness calls
// the same templates with double from the same call sequence as each class's timeStep() (e.g.
// prop3DAcoIsoDenQ_DEO2_FDTD.h:247-261), which makes the reference's FP64 rerun. The caller owns
// every array (double, layout k = (kx*ny + ky)*nz + kz) including the six pass-1 scratch arrays,
// and swaps (pcur, pold) and (mcur, mold) after each step as timeStep() does.
//
// Constants as the constructors form them (prop3DAcoIsoDenQ_DEO2_FDTD.h:64-70), but kept in double:
// c8 = {1225/1024, -245/3072, 49/5120, -5/7168}, inverse spacings 1/d of the FP32 spacings.
//
// Built by oracle/Makefile (target ref64) from the headers where they lie; one translation unit per
// propagator header (REF64_UNIT selects it), since the headers are not meant to share a unit.
#include <stddef.h>

#if REF64_UNIT == 1
#include "prop3DAcoIsoDenQ_DEO2_FDTD.h"
#elif REF64_UNIT == 2
#include "prop3DAcoVTIDenQ_DEO2_FDTD.h"
#elif REF64_UNIT == 3
#include "prop3DAcoTTIDenQ_DEO2_FDTD.h"
#elif REF64_UNIT == 4
#include "prop2DAcoIsoDenQ_DEO2_FDTD.h"
#elif REF64_UNIT == 5
#include "prop2DAcoVTIDenQ_DEO2_FDTD.h"
#elif REF64_UNIT == 6
#include "prop2DAcoTTIDenQ_DEO2_FDTD.h"
#endif

namespace {
// several reference passes take non-const pointers to arrays they only read
template <class T>
T *nc(const T *p) { return const_cast<T *>(p); }
const double C1 = +1225.0 / 1024.0, C2 = -245.0 / 3072.0, C3 = +49.0 / 5120.0, C4 = -5.0 / 7168.0;
const long NTHREAD = 1;  // the result does not depend on it; the caller's process runs the loops
}  // namespace

extern "C" {

#if REF64_UNIT == 1
// prop3DAcoIsoDenQ_DEO2_FDTD.h:247-261
void ref64_step_iso3d(long fs, long nx, long ny, long nz, float dx, float dy, float dz, float dt, const double *v,
                      const double *b, const double *q, const double *pcur, double *pold, double *pspace,
                      double *t0, double *t1, double *t2) {
    const double idx = 1.0 / (double)dx, idy = 1.0 / (double)dy, idz = 1.0 / (double)dz;
    Prop3DAcoIsoDenQ_DEO2_FDTD::applyFirstDerivatives3D_PlusHalf_Sandwich_Isotropic<double>(
        fs, nx, ny, nz, NTHREAD, C1, C2, C3, C4, idx, idy, idz, pcur, pcur, pcur, b, t0, t1, t2, 8, 8, nz);
    Prop3DAcoIsoDenQ_DEO2_FDTD::applyFirstDerivatives3D_MinusHalf_TimeUpdate_Nonlinear_Isotropic<double>(
        fs, nx, ny, nz, NTHREAD, C1, C2, C3, C4, idx, idy, idz, (double)dt, t0, t1, t2, v, b, q, pcur, pspace, pold,
        8, 8, nz);
}
#elif REF64_UNIT == 2
// prop3DAcoVTIDenQ_DEO2_FDTD.h:326-376 (linear: timeStepLinear, no pSpace/mSpace)
void ref64_step_vti3d(long fs, long linear, long nx, long ny, long nz, float dx, float dy, float dz, float dt,
                      const double *v, const double *eps, const double *eta, const double *b, const double *f,
                      const double *q, const double *pcur, const double *mcur, double *pold, double *mold,
                      double *pspace, double *mspace, double *t0, double *t1, double *t2, double *t3, double *t4,
                      double *t5) {
    typedef Prop3DAcoVTIDenQ_DEO2_FDTD P;
    const double idx = 1.0 / (double)dx, idy = 1.0 / (double)dy, idz = 1.0 / (double)dz;
    P::applyFirstDerivatives3D_PlusHalf_Sandwich<double>(fs, nx, ny, nz, NTHREAD, C1, C2, C3, C4, idx, idy, idz, nc(pcur), nc(pcur), nc(pcur), nc(mcur), nc(mcur), nc(mcur), nc(eps), nc(eta), nc(f), nc(b), t0, t1, t2, t3, t4, t5, 8, 8, nz);
    if (linear)
        P::applyFirstDerivatives3D_MinusHalf_TimeUpdate_Linear<double>(fs, nx, ny, nz, NTHREAD, C1, C2, C3, C4, idx, idy, idz, (double)dt, t0, t1, t2, t3, t4, t5, nc(v), nc(b), nc(q), nc(pcur), nc(mcur), pold, mold, 8, 8, nz);
    else
        P::applyFirstDerivatives3D_MinusHalf_TimeUpdate_Nonlinear<double>(fs, nx, ny, nz, NTHREAD, C1, C2, C3, C4, idx, idy, idz, (double)dt, t0, t1, t2, t3, t4, t5, nc(v), nc(b), nc(q), nc(pcur), nc(mcur), pspace, mspace, pold, mold, 8, 8, nz);
}
#elif REF64_UNIT == 3
// prop3DAcoTTIDenQ_DEO2_FDTD.h:359-385
void ref64_step_tti3d(long fs, long nx, long ny, long nz, float dx, float dy, float dz, float dt, const double *v,
                      const double *eps, const double *eta, const double *b, const double *f, const double *q,
                      const float *st, const float *ct, const float *sp, const float *cp, const double *pcur,
                      const double *mcur, double *pold, double *mold, double *pspace, double *mspace, double *t0,
                      double *t1, double *t2, double *t3, double *t4, double *t5) {
    typedef Prop3DAcoTTIDenQ_DEO2_FDTD P;
    const double idx = 1.0 / (double)dx, idy = 1.0 / (double)dy, idz = 1.0 / (double)dz;
    P::applyRotationSandwichRotation_TTI_FirstDerivatives3D_PlusHalf_TwoFields<double>(fs, nx, ny, nz, NTHREAD, C1, C2, C3, C4, idx, idy, idz, nc(pcur), nc(mcur), nc(st), nc(ct), nc(sp), nc(cp), nc(eps), nc(eta), nc(f), nc(b), t0, t1, t2, t3, t4, t5, 8, 8, nz);
    P::applyFirstDerivatives3D_MinusHalf_TimeUpdate_Nonlinear<double>(fs, nx, ny, nz, NTHREAD, C1, C2, C3, C4, idx, idy, idz, (double)dt, t0, t1, t2, t3, t4, t5, nc(v), nc(b), nc(q), nc(pcur), nc(mcur), pspace, mspace, pold, mold, 8, 8, nz);
}
#elif REF64_UNIT == 4
// prop2DAcoIsoDenQ_DEO2_FDTD.h:200-214
void ref64_step_iso2d(long fs, long nx, long nz, float dx, float dz, float dt, const double *v, const double *b,
                      const double *q, const double *pcur, double *pold, double *pspace, double *t0, double *t1) {
    typedef Prop2DAcoIsoDenQ_DEO2_FDTD P;
    const double idx = 1.0 / (double)dx, idz = 1.0 / (double)dz;
    P::applyFirstDerivatives2D_PlusHalf_Sandwich<double>(fs, nx, nz, NTHREAD, C1, C2, C3, C4, idx, idz, nc(pcur), nc(pcur), nc(b), t0, t1, 8, nz);
    P::applyFirstDerivatives2D_MinusHalf_TimeUpdate_Nonlinear<double>(fs, nx, nz, NTHREAD, C1, C2, C3, C4, idx, idz, (double)dt, t0, t1, nc(v), nc(b), nc(q), nc(pcur), pspace, pold, 8, nz);
}
#elif REF64_UNIT == 5
// prop2DAcoVTIDenQ_DEO2_FDTD.h:263-317
void ref64_step_vti2d(long fs, long linear, long nx, long nz, float dx, float dz, float dt, const double *v,
                      const double *eps, const double *eta, const double *b, const double *f, const double *q,
                      const double *pcur, const double *mcur, double *pold, double *mold, double *pspace,
                      double *mspace, double *t0, double *t1, double *t2, double *t3) {
    typedef Prop2DAcoVTIDenQ_DEO2_FDTD P;
    const double idx = 1.0 / (double)dx, idz = 1.0 / (double)dz;
    P::applyFirstDerivatives2D_PlusHalf_Sandwich<double>(fs, nx, nz, NTHREAD, C1, C2, C3, C4, idx, idz, nc(pcur), nc(pcur), nc(mcur), nc(mcur), nc(eps), nc(eta), nc(f), nc(b), t0, t1, t2, t3, 8, nz);
    if (linear)
        P::applyFirstDerivatives2D_MinusHalf_TimeUpdate_Linear<double>(fs, nx, nz, NTHREAD, C1, C2, C3, C4, idx, idz, (double)dt, t0, t1, t2, t3, nc(v), nc(b), nc(q), nc(pcur), nc(mcur), pold, mold, 8, nz);
    else
        P::applyFirstDerivatives2D_MinusHalf_TimeUpdate_Nonlinear<double>(fs, nx, nz, NTHREAD, C1, C2, C3, C4, idx, idz, (double)dt, t0, t1, t2, t3, nc(v), nc(b), nc(q), nc(pcur), nc(mcur), pspace, mspace, pold, mold, 8, nz);
}
#elif REF64_UNIT == 6
// prop2DAcoTTIDenQ_DEO2_FDTD.h:271-296
void ref64_step_tti2d(long fs, long nx, long nz, float dx, float dz, float dt, const double *v, const double *eps,
                      const double *eta, const double *b, const double *f, const double *q, const float *st,
                      const float *ct, const double *pcur, const double *mcur, double *pold, double *mold,
                      double *pspace, double *mspace, double *t0, double *t1, double *t2, double *t3) {
    typedef Prop2DAcoTTIDenQ_DEO2_FDTD P;
    const double idx = 1.0 / (double)dx, idz = 1.0 / (double)dz;
    P::applyFirstDerivatives2D_TTI_PlusHalf_Sandwich<double>(fs, nx, nz, NTHREAD, C1, C2, C3, C4, idx, idz, nc(pcur), nc(pcur), nc(mcur), nc(mcur), nc(st), nc(ct), nc(eps), nc(eta), nc(f), nc(b), t0, t1, t2, t3, 8, nz);
    P::applyFirstDerivatives2D_TTI_MinusHalf_TimeUpdate_Nonlinear<double>(fs, nx, nz, NTHREAD, C1, C2, C3, C4, idx, idz, (double)dt, t0, t1, t2, t3, nc(st), nc(ct), nc(v), nc(b), nc(q), nc(pcur), nc(mcur), pspace, mspace, pold, mold, 8, nz);
}
#endif

}  // extern "C"
