// Propagator object behind the reference's C ABI.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "wavefd_b200.h"
#include "wfd_kernels.h"

namespace wfd {

enum FieldId {
    F_V = 0, F_B, F_Q, F_EPS, F_ETA, F_F, F_ST, F_CT, F_SP, F_CP,
    F_PCUR, F_POLD, F_PSPACE, F_MCUR, F_MOLD, F_MSPACE,
    F_COUNT
};

// Status codes (WFD_OK, WFD_ERR_*) are the add-on API's, from the public header.

struct Prop {
    int ndim = 3;
    int phys = ISO;
    bool fs = true;
    long nx = 0, ny = 1, nz = 0, nsponge = 0, nthread = 1;
    long nbx = 0, nby = 0, nbz = 0;
    float dx = 0, dy = 0, dz = 0, dt = 0;
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool strict = false;     // bitwise parity kernels instead of the FMA build
    bool fused = true;       // single-sweep kernels where available
    float *field[F_COUNT] = {};
    float *tmp[12] = {};     // scratch of the unfused passes (the reference's tmp arrays)
    float *stage[7] = {};    // device copies of host arrays given to Born/imaging calls (first use)
    float2 *work = nullptr;  // FFT workspace of the wavefield-separation condition
    float *illum = nullptr;  // caller's source illumination sum (device), accumulated by every step
    long work_cols = 0;
    int status = WFD_OK;
    std::string message;
    long steps = 0;
    unsigned host_touched = 0;  // bit f: the getter of field f was called since the last device call
    unsigned char touch_streak[F_COUNT] = {};  // device calls in a row preceded by that getter
    int step_kernels = 0;  // kernels launched by the last time step (1 fused, 2 unfused)
    long run_launches = 0; // kernels launched by the last WFD_Prop_Run
    StepInject inj{};      // a source injection for the step kernel to apply (WFD_Prop_Run), or none
    StepEpilogue epi{};    // Born injection / imaging condition to apply right after the next step, or none
    bool inject_done = false;  // the last step kernel applied `inj`

    long ncells() const { return nx * ny * nz; }
    Grid grid() const;
    Fields fields() const;
    Scratch scratch() const;
};

Prop *prop_create(int ndim, int phys, long fs, long nthread, long nx, long ny, long nz, long nsponge, float dx,
                  float dy, float dz, float dt, long nbx, long nby, long nbz);
void prop_destroy(Prop *p);
void prop_setup_q(Prop *p, float freqQ, float qMin, float qInterior);
int prop_step(Prop *p, bool linear, bool sync);
// one step followed by ForwardBornInjection_V (e.born_*) or AdjointBornAccumulation_V (e.img*), fused
// into the step kernel where it can apply them, else as the separate kernels after it; asynchronous
int prop_step_epilogue(Prop *p, const StepEpilogue &e, bool linear);
int prop_scale(Prop *p);
int prop_born(Prop *p, const char *variant, float *const *args, int nargs);
int prop_image(Prop *p, const char *variant, float *const *args, int nargs, long isfwi);
int prop_sync(Prop *p);
int prop_fail(Prop *p, int code, const std::string &msg);
bool ensure_scratch(Prop *p, int count);

// process-wide error slot for calls that have no object (alloc)
void set_global_error(int code, const std::string &msg);
int global_error(std::string *msg);

// standalone 2D D+ with caller constants (prop2DAcoVTIDenQ_DEO2_FDTD.cc:158-176)
void apply_dplus2d(bool fs, long nx, long nz, float c1, float c2, float c3, float c4, float invDx, float invDz,
                   const float *inX, const float *inZ, float *outX, float *outZ);

// move the arrays of the object whose getters were called since its last device call (managed
// memory that host code may have written) back to its device, and clear that record
void prefetch_touched(Prop *p, cudaStream_t s);

// sum[i] += field[i]^2 on the device (wfd_illum.cu)
void illum_accumulate(float *sum, const float *field, long n, cudaStream_t s);

// true when the pointer can be dereferenced by kernels (device or managed memory)
bool device_accessible(const void *ptr);

}  // namespace wfd
