// Add-on entry points of the C ABI (status, modes, asynchronous stepping, prefetch).
#include <string>

#include "wavefd_b200.h"
#include "wfd_prop.h"

using wfd::Prop;

namespace {
Prop *P(void *p) { return reinterpret_cast<Prop *>(p); }
thread_local std::string t_msg;
}  // namespace

extern "C" int WFD_LastError(void) { return wfd::global_error(nullptr); }

extern "C" const char *WFD_LastErrorMessage(void) {
    wfd::global_error(&t_msg);
    return t_msg.c_str();
}

extern "C" int WFD_Debug_SetPipelineWait(unsigned long long ns) {
    const unsigned long long v = ns ? ns : 2000000000ull;
    if (cudaDeviceSynchronize() != cudaSuccess) return WFD_ERR_CUDA;
    wfd_fast::fused_set_pipeline_wait(v);
    wfd_strict::fused_set_pipeline_wait(v);
    return cudaDeviceSynchronize() == cudaSuccess ? WFD_OK : WFD_ERR_CUDA;
}

extern "C" int WFD_Prop_Status(void *p) { return p ? P(p)->status : WFD_ERR_ARG; }

extern "C" const char *WFD_Prop_Message(void *p) { return p ? P(p)->message.c_str() : "null object"; }

extern "C" int WFD_Prop_SetStrict(void *p, int strict) {
    if (!p) return WFD_ERR_ARG;
    P(p)->strict = strict != 0;
    return WFD_OK;
}

extern "C" int WFD_Prop_SetFused(void *p, int fused) {
    if (!p) return WFD_ERR_ARG;
    P(p)->fused = fused != 0;
    return WFD_OK;
}

extern "C" int WFD_Prop_TimeStepAsync(void *p, long nsteps, int linear) {
    if (!p || nsteps < 0) return WFD_ERR_ARG;
    if (linear && P(p)->phys != wfd::VTI) return wfd::prop_fail(P(p), WFD_ERR_UNSUPPORTED, "linear step is VTI only");
    for (long i = 0; i < nsteps; i++) {
        int rc = wfd::prop_step(P(p), linear != 0, false);
        if (rc) return rc;
    }
    return WFD_OK;
}

// a time step followed by the Born-V injection or the V imaging condition, fused into the step kernel
// where it applies them (3D); asynchronous on the object's stream, device or managed arrays only
extern "C" int WFD_Prop_TimeStepBorn(void *p, const float *dVel, const float *wavefieldDP, const float *wavefieldDM) {
    if (!p || !dVel || !wavefieldDP) return WFD_ERR_ARG;
    const bool aniso = P(p)->phys != wfd::ISO;
    if (aniso && !wavefieldDM) return WFD_ERR_ARG;
    for (const float *a : {dVel, wavefieldDP, aniso ? wavefieldDM : dVel})
        if (!wfd::device_accessible(a)) return wfd::prop_fail(P(p), WFD_ERR_ARG, "device or managed arrays expected");
    wfd::StepEpilogue e{};
    e.born_dv = dVel;
    e.born_dp = wavefieldDP;
    e.born_dm = aniso ? wavefieldDM : nullptr;
    return wfd::prop_step_epilogue(P(p), e, false);
}

extern "C" int WFD_Prop_TimeStepImage(void *p, float *dVel, const float *wavefieldDP, const float *wavefieldDM,
                                      int linear) {
    if (!p || !dVel || !wavefieldDP) return WFD_ERR_ARG;
    if (linear && P(p)->phys != wfd::VTI) return wfd::prop_fail(P(p), WFD_ERR_UNSUPPORTED, "linear step is VTI only");
    const bool aniso = P(p)->phys != wfd::ISO;
    if (aniso && !wavefieldDM) return WFD_ERR_ARG;
    for (const float *a : {(const float *)dVel, wavefieldDP, aniso ? wavefieldDM : (const float *)dVel})
        if (!wfd::device_accessible(a)) return wfd::prop_fail(P(p), WFD_ERR_ARG, "device or managed arrays expected");
    wfd::StepEpilogue e{};
    e.img = dVel;
    e.img_dp = wavefieldDP;
    e.img_dm = aniso ? wavefieldDM : nullptr;
    return wfd::prop_step_epilogue(P(p), e, linear != 0);
}

extern "C" int WFD_Prop_TimeStepScaled(void *p) {
    if (!p) return WFD_ERR_ARG;
    wfd::StepEpilogue e{};
    e.scale_space = 1;
    return wfd::prop_step_epilogue(P(p), e, false);
}

extern "C" int WFD_Prop_Synchronize(void *p) { return p ? wfd::prop_sync(P(p)) : WFD_ERR_ARG; }

extern "C" int WFD_Prop_Prefetch(void *p) {
    if (!p) return WFD_ERR_ARG;
    Prop *q = P(p);
    q->host_touched = 0;
    const size_t bytes = sizeof(float) * (size_t)q->ncells();
    for (int f = 0; f < wfd::F_COUNT; f++) {
        if (!q->field[f]) continue;
#if CUDART_VERSION >= 13000
        cudaMemLocation loc{cudaMemLocationTypeDevice, q->device};
        cudaMemPrefetchAsync(q->field[f], bytes, loc, 0, q->stream);
#else
        cudaMemPrefetchAsync(q->field[f], bytes, q->device, q->stream);
#endif
    }
    return wfd::prop_sync(q);
}

extern "C" void *WFD_Prop_Stream(void *p) { return p ? (void *)P(p)->stream : nullptr; }

extern "C" int WFD_Prop_StepKernels(void *p) { return p ? P(p)->step_kernels : WFD_ERR_ARG; }

extern "C" long WFD_Prop_RunLaunches(void *p) { return p ? P(p)->run_launches : -1; }

extern "C" int WFD_Prop_SetIllumination(void *p, float *accum) {
    if (!p) return WFD_ERR_ARG;
    if (accum && !wfd::device_accessible(accum)) return WFD_ERR_ARG;
    P(p)->illum = accum;
    return WFD_OK;
}
