// Propagator objects: allocation (managed memory behind the getters), the Q/sponge profile,
// and dispatch of the time step, Born injection and imaging conditions to the kernels.
#include "wfd_prop.h"
#include "wfd_alloc.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

namespace wfd {

namespace {
std::mutex g_err_mu;
int g_err_code = WFD_OK;
std::string g_err_msg;

bool uses(int phys, int ndim, int f) {
    switch (f) {
        case F_V: case F_B: case F_Q: case F_PCUR: case F_POLD: case F_PSPACE: return true;
        case F_EPS: case F_ETA: case F_F: case F_MCUR: case F_MOLD: case F_MSPACE: return phys != ISO;
        case F_ST: case F_CT: return phys == TTI;
        case F_SP: case F_CP: return phys == TTI && ndim == 3;
        default: return false;
    }
}
}  // namespace

// ---- allocation fault injector (wfd_alloc.h) ----------------------------------------------------
namespace {
std::atomic<long> g_alloc_count{0};
thread_local const char *t_injected = "";

long fail_at() {
    static const long n = [] {
        const char *e = getenv("WAVEFD_B200_FAIL_ALLOC");
        return e && *e ? strtol(e, nullptr, 10) : 0L;
    }();
    return n;
}
}  // namespace

bool alloc_should_fail() {
    const long n = fail_at();
    if (n <= 0) return false;
    const bool fail = g_alloc_count.fetch_add(1) + 1 == n;
    t_injected = fail ? " (injected: WAVEFD_B200_FAIL_ALLOC)" : "";
    return fail;
}

const char *alloc_injected_note() { return t_injected; }

void set_global_error(int code, const std::string &msg) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_err_code = code;
    g_err_msg = msg;
}

int global_error(std::string *msg) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    if (msg) *msg = g_err_msg;
    return g_err_code;
}

int prop_fail(Prop *p, int code, const std::string &msg) {
    if (p) {
        p->status = code;
        p->message = msg;
    }
    set_global_error(code, msg);
    return code;
}

static int check_cuda(Prop *p, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return WFD_OK;
    return prop_fail(p, WFD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

Grid Prop::grid() const {
    Grid g;
    g.ndim = ndim;
    g.fs = fs ? 1 : 0;
    g.nx = nx;
    g.ny = ndim == 3 ? ny : 1;
    g.nz = nz;
    g.sy = nz;
    g.sx = g.ny * nz;
    g.n = g.nx * g.sx;
    // prop3DAcoIsoDenQ_DEO2_FDTD.h:64-70: formed in double, stored in float members
    g.c1 = (float)(+1225.0 / 1024.0);
    g.c2 = (float)(-245.0 / 3072.0);
    g.c3 = (float)(+49.0 / 5120.0);
    g.c4 = (float)(-5.0 / 7168.0);
    g.idx = (float)(1.0 / (double)dx);
    g.idy = (float)(1.0 / (double)dy);
    g.idz = (float)(1.0 / (double)dz);
    g.dt = dt;
    g.dt2 = dt * dt;
    return g;
}

Fields Prop::fields() const {
    Fields F;
    F.v = field[F_V];
    F.b = field[F_B];
    F.q = field[F_Q];
    F.eps = field[F_EPS];
    F.eta = field[F_ETA];
    F.f = field[F_F];
    F.st = field[F_ST];
    F.ct = field[F_CT];
    F.sp = field[F_SP];
    F.cp = field[F_CP];
    F.pcur = field[F_PCUR];
    F.pold = field[F_POLD];
    F.pspace = field[F_PSPACE];
    F.mcur = field[F_MCUR];
    F.mold = field[F_MOLD];
    F.mspace = field[F_MSPACE];
    F.illum = illum;
    F.inj = inj;
    F.epi = epi;
    return F;
}

Scratch Prop::scratch() const {
    Scratch S;
    for (int i = 0; i < 12; i++) S.t[i] = tmp[i];
    return S;
}

bool ensure_scratch(Prop *p, int count) {
    const size_t bytes = sizeof(float) * (size_t)p->ncells();
    for (int i = 0; i < count && i < 12; i++) {
        if (p->tmp[i]) continue;
        cudaError_t e = wfd::dMalloc(&p->tmp[i], bytes);
        if (e != cudaSuccess) {
            p->tmp[i] = nullptr;
            prop_fail(p, WFD_ERR_ALLOC,
                      std::string("scratch allocation failed: ") + cudaGetErrorString(e) + alloc_injected_note());
            return false;
        }
        cudaMemsetAsync(p->tmp[i], 0, bytes, p->stream);
    }
    return true;
}

Prop *prop_create(int ndim, int phys, long fs, long nthread, long nx, long ny, long nz, long nsponge, float dx,
                  float dy, float dz, float dt, long nbx, long nby, long nbz) {
    if (nx <= 8 || nz <= 8 || (ndim == 3 && ny <= 8)) {
        set_global_error(WFD_ERR_ARG, "grid must exceed 8 cells per axis");
        return nullptr;
    }
    Prop *p = new Prop();
    p->ndim = ndim;
    p->phys = phys;
    p->fs = fs > 0;  // prop3DAcoIsoDenQ_DEO2_FDTD.cc:19
    p->nthread = nthread;
    p->nx = nx;
    p->ny = ndim == 3 ? ny : 1;
    p->nz = nz;
    p->nsponge = nsponge;
    p->dx = dx;
    p->dy = ndim == 3 ? dy : 1.0f;
    p->dz = dz;
    p->dt = dt;
    p->nbx = nbx;
    p->nby = nby;
    p->nbz = nbz;
    const char *mode = getenv("WAVEFD_B200_STRICT");
    p->strict = mode && mode[0] == '1';
    const char *fz = getenv("WAVEFD_B200_UNFUSED");
    p->fused = !(fz && fz[0] == '1');
    cudaGetDevice(&p->device);
    // the arrays first, then the stream (an allocation failure is reported before any other call)
    const size_t bytes = sizeof(float) * (size_t)p->ncells();
    for (int f = 0; f < F_COUNT; f++) {
        if (!uses(phys, ndim, f)) continue;
        cudaError_t e = wfd::dMallocManaged(&p->field[f], bytes, cudaMemAttachGlobal);
        if (e != cudaSuccess) {
            set_global_error(WFD_ERR_ALLOC, std::string("managed allocation failed: ") + cudaGetErrorString(e) +
                                                alloc_injected_note());
            prop_destroy(p);
            return nullptr;
        }
    }
    if (cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_global_error(WFD_ERR_CUDA, "stream creation failed");
        prop_destroy(p);
        return nullptr;
    }
    p->own_stream = true;
    for (int f = 0; f < F_COUNT; f++) {
        if (!p->field[f]) continue;
#if CUDART_VERSION >= 13000
        cudaMemLocation loc{cudaMemLocationTypeDevice, p->device};
        cudaMemAdvise(p->field[f], bytes, cudaMemAdviseSetPreferredLocation, loc);
#else
        cudaMemAdvise(p->field[f], bytes, cudaMemAdviseSetPreferredLocation, p->device);
#endif
        // the reference zero-fills every array at construction (numaFirstTouch, .h:94-205)
        cudaMemsetAsync(p->field[f], 0, bytes, p->stream);
    }
    if (cudaStreamSynchronize(p->stream) != cudaSuccess) {
        set_global_error(WFD_ERR_CUDA, "initialisation failed");
        prop_destroy(p);
        return nullptr;
    }
    return p;
}

void prop_destroy(Prop *p) {
    if (!p) return;
    if (p->stream) cudaStreamSynchronize(p->stream);
    for (int f = 0; f < F_COUNT; f++)
        if (p->field[f]) cudaFree(p->field[f]);
    for (int i = 0; i < 12; i++)
        if (p->tmp[i]) cudaFree(p->tmp[i]);
    for (int i = 0; i < 7; i++)
        if (p->stage[i]) cudaFree(p->stage[i]);
    if (p->work) cudaFree(p->work);
    if (p->own_stream && p->stream) cudaStreamDestroy(p->stream);
    delete p;
}

// ---------------------------------------------------------------------------------------------
// Q/sponge profile (absorb.h:23-75 for 2D, :85-151 for 3D). The nsponge-long profile is formed
// on the host with the same libm calls and precision as the reference; the grid is filled on
// the device from the table {value(ksponge) for ksponge < nsponge, interior value}.
__global__ void k_fill_q(Grid g, long nsponge, const float *__restrict__ table, float *q) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    const long z = k % g.nz;
    const long r = k / g.nz;
    const long y = r % g.ny;
    const long x = r / g.ny;
    const long ksx = x < g.nx - 1 - x ? x : g.nx - 1 - x;
    const long ksz = g.fs ? (g.nz - 1 - z) : (z < g.nz - 1 - z ? z : g.nz - 1 - z);
    long ks = ksx < ksz ? ksx : ksz;
    if (g.ndim == 3) {
        const long ksy = y < g.ny - 1 - y ? y : g.ny - 1 - y;
        if (ksy < ks) ks = ksy;
    }
    q[k] = table[ks < nsponge ? ks : nsponge];
}

void prop_setup_q(Prop *p, float freqQ, float qMin, float qInterior) {
    if (freqQ < FLT_EPSILON) {
        // absorb.h:35-40 (and :97-102): the reference reports and terminates the process
        char msg[1000];
        snprintf(msg, sizeof(msg), "Error -- freqQ [%f] is too small!\n", freqQ);
        const char *noexit = getenv("WAVEFD_B200_NO_EXIT");
        if (noexit && noexit[0] == '1') {
            prop_fail(p, WFD_ERR_ARG, msg);
            return;
        }
        perror(msg);
        exit(EXIT_FAILURE);
    }
    if ((qMin < FLT_EPSILON) && (qInterior < FLT_EPSILON)) {
        // absorb.h:42-46: warning, then a memset of sizeof(float*) bytes only
        printf("Warning -- qMin and qMax unphysical, dtOmegaInvQ set to zero!\n");
        cudaMemsetAsync(p->field[F_Q], 0, 8, p->stream);
        cudaStreamSynchronize(p->stream);
        return;
    }
    const long ns = p->nsponge > 0 ? p->nsponge : 0;
    std::vector<float> table((size_t)ns + 1);
    const double PI = 3.1415926535897;  // absorb.h:12
    const float dt = p->dt;
    std::vector<float> qprof((size_t)(ns > 0 ? ns : 1));
    if (p->ndim == 2) {
        const double lqmin = logf(qMin);
        const double lqmax = logf(qInterior);
        for (long k = 0; k < ns; k++) {
            const double dk = (double)k / (double)(ns - 1);
            const double lq = lqmin + dk * (lqmax - lqmin);
            qprof[k] = expf((float)lq);
        }
    } else {
        const float lqmin = logf(qMin);
        const float lqmax = logf(qInterior);
        for (long k = 0; k < ns; k++) {
            const float dk = (float)k / (float)(ns - 1);
            const float lq = lqmin + dk * (lqmax - lqmin);  // host code is built with -ffp-contract=off
            qprof[k] = expf(lq);
        }
    }
    for (long k = 0; k < ns; k++) table[k] = (float)((double)(dt * 2) * PI * (double)freqQ / (double)qprof[k]);
    table[ns] = (float)((double)(dt * 2) * PI * (double)freqQ / (double)qInterior);
    float *dtable = nullptr;
    if (check_cuda(p, wfd::dMallocAsync(&dtable, sizeof(float) * table.size(), p->stream), "q table")) return;
    cudaMemcpyAsync(dtable, table.data(), sizeof(float) * table.size(), cudaMemcpyHostToDevice, p->stream);
    Grid g = p->grid();
    k_fill_q<<<(unsigned)((g.n + 255) / 256), 256, 0, p->stream>>>(g, ns, dtable, p->field[F_Q]);
    cudaFreeAsync(dtable, p->stream);
    check_cuda(p, cudaStreamSynchronize(p->stream), "SetupDtOmegaInvQ");
}

// ---------------------------------------------------------------------------------------------
int prop_sync(Prop *p) {
    if (int rc = check_cuda(p, cudaStreamSynchronize(p->stream), "synchronize")) return rc;
    // device status words of the TMA kernels: a bounded wait that ran out
    if (wfd_fast::fused_status_and_clear() | wfd_strict::fused_status_and_clear())
        return prop_fail(p, WFD_ERR_TIMEOUT, "a fused step kernel timed out waiting for its tile loads");
    return WFD_OK;
}

int prop_step(Prop *p, bool linear, bool sync) {
    Grid g = p->grid();
    Fields F = p->fields();
    // the step kernels read the epilogue's arrays 16 (Iso) or 8 bytes at a time: arrays at other
    // alignments take the separate kernels after the step
    auto a16 = [](const void *q) { return (reinterpret_cast<uintptr_t>(q) & 15u) == 0; };
    const StepEpilogue &pe = p->epi;
    if (!(a16(pe.born_dv) && a16(pe.born_dp) && a16(pe.born_dm) && a16(pe.img) && a16(pe.img_dp) &&
          a16(pe.img_dm)))
        F.epi = StepEpilogue{};
    bool done = false, illum_done = false, epi_done = false;
    p->inject_done = false;
    if (p->fused) {
        const int r = p->strict ? wfd_strict::fused_step(g, p->phys, linear, F, p->stream)
                                : wfd_fast::fused_step(g, p->phys, linear, F, p->stream);
        done = (r & 1) != 0;
        illum_done = (r & 2) != 0;
        p->inject_done = (r & 4) != 0;
        epi_done = (r & 8) != 0;
    }
    if (!done) {
        if (!ensure_scratch(p, p->phys == ISO ? 3 : 6)) return p->status;
        Scratch S = p->scratch();
        if (p->strict) {
            wfd_strict::pass1(g, p->phys, F, S, p->stream);
            wfd_strict::pass2(g, p->phys, linear, F, S, p->stream);
        } else {
            wfd_fast::pass1(g, p->phys, F, S, p->stream);
            wfd_fast::pass2(g, p->phys, linear, F, S, p->stream);
        }
    }
    // the illumination of pCur (read-only during the step) when the step kernel did not add it
    if (p->illum && !illum_done) illum_accumulate(p->illum, p->field[F_PCUR], p->ncells(), p->stream);
    const bool epi_wanted = p->epi.born_dv || p->epi.img || p->epi.scale_space;
    p->step_kernels = (done ? 1 : 2) + (p->illum && !illum_done ? 1 : 0);
    if (int rc = check_cuda(p, cudaGetLastError(), "time step launch")) return rc;
    // pointer swap (prop3DAcoIsoDenQ_DEO2_FDTD.h:258-260)
    std::swap(p->field[F_PCUR], p->field[F_POLD]);
    std::swap(p->field[F_MCUR], p->field[F_MOLD]);
    p->steps++;
    if (epi_wanted && !epi_done) {
        // the step kernel did not apply them: the separate kernels on the swapped fields (the new
        // field is pCur, the step's input is pOld), as the reference's calls after TimeStep
        Fields Fs = p->fields();
        const StepEpilogue &e = p->epi;
        const bool iso = p->phys == ISO;
        if (e.scale_space) {
            if (p->strict) wfd_strict::scale(g, Fs, !iso, p->stream);
            else wfd_fast::scale(g, Fs, !iso, p->stream);
            p->step_kernels++;
        }
        if (e.born_dv) {
            if (iso) {
                if (p->strict) wfd_strict::born_iso_v(g, Fs, e.born_dv, e.born_dp, p->stream);
                else wfd_fast::born_iso_v(g, Fs, e.born_dv, e.born_dp, p->stream);
            } else if (p->strict) {
                wfd_strict::born_aniso_v(g, Fs, e.born_dv, e.born_dp, e.born_dm, p->stream);
            } else {
                wfd_fast::born_aniso_v(g, Fs, e.born_dv, e.born_dp, e.born_dm, p->stream);
            }
            p->step_kernels++;
        }
        if (e.img) {
            if (iso) {
                if (p->strict) wfd_strict::image_iso_v(g, Fs, e.img_dp, e.img, p->stream);
                else wfd_fast::image_iso_v(g, Fs, e.img_dp, e.img, p->stream);
            } else if (p->strict) {
                wfd_strict::image_aniso_v(g, Fs, e.img_dp, e.img_dm, e.img, p->stream);
            } else {
                wfd_fast::image_aniso_v(g, Fs, e.img_dp, e.img_dm, e.img, p->stream);
            }
            p->step_kernels++;
        }
        if (int rc = check_cuda(p, cudaGetLastError(), "Born/imaging launch")) return rc;
    }
    if (sync) return prop_sync(p);
    return WFD_OK;
}

int prop_step_epilogue(Prop *p, const StepEpilogue &e, bool linear) {
    p->epi = e;
    const int rc = prop_step(p, linear, false);
    p->epi = StepEpilogue{};
    return rc;
}

int prop_scale(Prop *p) {
    Grid g = p->grid();
    Fields F = p->fields();
    if (p->strict) wfd_strict::scale(g, F, p->phys != ISO, p->stream);
    else wfd_fast::scale(g, F, p->phys != ISO, p->stream);
    if (int rc = check_cuda(p, cudaGetLastError(), "scale launch")) return rc;
    return prop_sync(p);
}

}  // namespace wfd
