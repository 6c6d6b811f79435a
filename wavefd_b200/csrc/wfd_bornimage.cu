// Born injection and imaging-condition entry points, composed from the unfused kernels in the
// reference's order (e.g. prop3DAcoIsoDenQ_DEO2_FDTD.h:351-417, prop3DAcoTTIDenQ_DEO2_FDTD.h:460-554).
//
// Caller arrays may live anywhere: device or managed pointers are used in place; plain host
// pointers (the Julia arrays of the drop-in path) are staged through device buffers, inputs
// copied in and accumulated images copied back, inside the call.
#include <string.h>

#include <string>
#include <vector>

#include "wfd_prop.h"
#include "wfd_alloc.h"

namespace wfd {

bool device_accessible(const void *ptr) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

namespace {

struct Staged {
    float *user = nullptr;
    float *dev = nullptr;
    bool copied = false;
};

class Stager {
  public:
    explicit Stager(Prop *p) : p_(p) {}
    // map a caller array of ncells floats; copy host contents in. Host arrays go through the
    // object's staging buffers, allocated on first use and kept for its later calls.
    float *in(float *user) {
        Staged s;
        s.user = user;
        if (!user) return nullptr;
        if (device_accessible(user)) {
            s.dev = user;
        } else {
            if (next_ >= (int)(sizeof(p_->stage) / sizeof(p_->stage[0]))) {
                ok_ = false;
                return nullptr;
            }
            const size_t bytes = sizeof(float) * (size_t)p_->ncells();
            if (!p_->stage[next_] && wfd::dMalloc(&p_->stage[next_], bytes) != cudaSuccess) {
                p_->stage[next_] = nullptr;
                ok_ = false;
                return nullptr;
            }
            s.dev = p_->stage[next_++];
            cudaMemcpyAsync(s.dev, user, bytes, cudaMemcpyHostToDevice, p_->stream);
            s.copied = true;
        }
        v_.push_back(s);
        return s.dev;
    }
    // copy accumulated outputs back to their host arrays
    void writeback(float *dev) {
        for (auto &s : v_)
            if (s.dev == dev && s.copied)
                cudaMemcpyAsync(s.user, s.dev, sizeof(float) * (size_t)p_->ncells(), cudaMemcpyDeviceToHost,
                                p_->stream);
    }
    bool ok() const { return ok_; }

  private:
    Prop *p_;
    std::vector<Staged> v_;
    int next_ = 0;
    bool ok_ = true;
};

struct K {
    bool strict;
#define WFD_DISPATCH(fn)                                                      \
    template <class... A>                                                     \
    void fn(A... a) const {                                                   \
        if (strict) wfd_strict::fn(a...);                                     \
        else wfd_fast::fn(a...);                                              \
    }
    WFD_DISPATCH(born_iso_v)
    WFD_DISPATCH(born_aniso_v)
    WFD_DISPATCH(image_iso_v)
    WFD_DISPATCH(image_aniso_v)
    WFD_DISPATCH(image_wavefieldsep)
    WFD_DISPATCH(born_iso_fused)
    WFD_DISPATCH(image_iso_fused)
    WFD_DISPATCH(born_vea_fused)
    WFD_DISPATCH(image_vea_fused)
#undef WFD_DISPATCH
};

int finish(Prop *p, const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) return prop_fail(p, WFD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return WFD_OK;
}

}  // namespace

int prop_born(Prop *p, const char *variant, float *const *args, int nargs) {
    const K k{p->strict};
    const Grid g = p->grid();
    const Fields F = p->fields();
    Stager st(p);
    std::vector<float *> a(nargs);
    for (int i = 0; i < nargs; i++) a[i] = st.in(args[i]);
    if (!st.ok()) return prop_fail(p, WFD_ERR_ALLOC, "staging allocation failed");
    float **t = p->tmp;
    if (p->phys == ISO) {
        if (!strcmp(variant, "V")) {
            k.born_iso_v(g, F, a[0], a[1], p->stream);
        } else {
            const bool vb = !strcmp(variant, "VB");
            float *dv = vb ? a[0] : nullptr, *db = vb ? a[1] : a[0], *P = vb ? a[2] : a[1], *DP = vb ? a[3] : a[2];
            if (!ensure_scratch(p, 3)) return p->status;
            k.born_iso_fused(g, vb ? 1 : 2, F, dv, db, P, DP, t, p->stream);
        }
    } else if (!strcmp(variant, "V")) {
        k.born_aniso_v(g, F, a[0], a[1], a[2], p->stream);
    } else {  // VEA: dV, dEps, dEta, P, M, DP, DM
        if (!ensure_scratch(p, 6)) return p->status;
        k.born_vea_fused(g, p->phys == TTI, F, a[0], a[1], a[2], a[3], a[4], a[5], a[6], t, p->stream);
    }
    return finish(p, "ForwardBornInjection");
}

int prop_image(Prop *p, const char *variant, float *const *args, int nargs, long isfwi) {
    const K k{p->strict};
    const Grid g = p->grid();
    const Fields F = p->fields();
    Stager st(p);
    std::vector<float *> a(nargs);
    for (int i = 0; i < nargs; i++) a[i] = st.in(args[i]);
    if (!st.ok()) return prop_fail(p, WFD_ERR_ALLOC, "staging allocation failed");
    float **t = p->tmp;
    std::vector<float *> outs;
    if (!strncmp(variant, "wavefieldsep", 12)) {
        const long ncols = g.nx * g.ny;
        const long nfft = 2 * g.nz;
        if (!p->work) {
            long cols = ncols < 4096 ? ncols : 4096;
            if (wfd::dMalloc(&p->work, sizeof(float2) * (size_t)cols * (size_t)nfft * 2) != cudaSuccess)
                return prop_fail(p, WFD_ERR_ALLOC, "FFT workspace allocation failed");
            p->work_cols = cols;
        }
        float *dm = p->phys == ISO ? nullptr : a[2];
        k.image_wavefieldsep(g, isfwi, F, a[1], (const float *)dm, a[0], p->work, p->work_cols, p->stream);
        outs.push_back(a[0]);
    } else if (p->phys == ISO) {
        if (!strcmp(variant, "V")) {
            k.image_iso_v(g, F, a[1], a[0], p->stream);
            outs.push_back(a[0]);
        } else {
            const bool vb = !strcmp(variant, "VB");
            float *dv = vb ? a[0] : nullptr, *db = vb ? a[1] : a[0], *P = vb ? a[2] : a[1], *DP = vb ? a[3] : a[2];
            k.image_iso_fused(g, vb ? 1 : 2, F, DP, P, dv, db, p->stream);
            if (dv) outs.push_back(dv);
            outs.push_back(db);
        }
    } else if (!strcmp(variant, "V")) {
        k.image_aniso_v(g, F, a[1], a[2], a[0], p->stream);
        outs.push_back(a[0]);
    } else {  // VEA: dV, dEps, dEta, P, M, DP, DM
        k.image_vea_fused(g, p->phys == TTI, F, a[5], a[6], a[3], a[4], a[0], a[1], a[2], p->stream);
        outs.push_back(a[0]);
        outs.push_back(a[1]);
        outs.push_back(a[2]);
    }
    for (float *o : outs) st.writeback(o);
    return finish(p, "AdjointBornAccumulation");
}

void apply_dplus2d(bool fs, long nx, long nz, float c1, float c2, float c3, float c4, float invDx, float invDz,
                   const float *inX, const float *inZ, float *outX, float *outZ) {
    Prop tmp;  // carries the stream and the geometry only
    tmp.ndim = 2;
    tmp.nx = nx;
    tmp.ny = 1;
    tmp.nz = nz;
    if (cudaStreamCreateWithFlags(&tmp.stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_global_error(WFD_ERR_CUDA, "stream creation failed");
        return;
    }
    {
        Stager st(&tmp);
        float *ix = st.in(const_cast<float *>(inX));
        float *iz = st.in(const_cast<float *>(inZ));
        float *ox = st.in(outX);
        float *oz = st.in(outZ);
        if (st.ok()) {
            Grid g{};
            g.ndim = 2;
            g.fs = fs ? 1 : 0;
            g.nx = nx;
            g.ny = 1;
            g.nz = nz;
            g.sy = nz;
            g.sx = nz;
            g.n = nx * nz;
            g.c1 = c1;
            g.c2 = c2;
            g.c3 = c3;
            g.c4 = c4;
            g.idx = invDx;
            g.idy = 1.0f;
            g.idz = invDz;
            wfd_strict::dplus3(g, ix, ix, iz, ox, ox, oz, tmp.stream);
            st.writeback(ox);
            st.writeback(oz);
        } else {
            set_global_error(WFD_ERR_ALLOC, "staging allocation failed");
        }
    }
    cudaError_t e = cudaStreamSynchronize(tmp.stream);
    if (e != cudaSuccess) set_global_error(WFD_ERR_CUDA, cudaGetErrorString(e));
    for (float *&b : tmp.stage) {
        if (b) cudaFree(b);
        b = nullptr;
    }
    cudaStreamDestroy(tmp.stream);
    tmp.stream = nullptr;
}

}  // namespace wfd
