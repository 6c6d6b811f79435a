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
    WFD_DISPATCH(dplus)
    WFD_DISPATCH(dminus3)
    WFD_DISPATCH(tti_dplus)
    WFD_DISPATCH(tti_dminus)
    WFD_DISPATCH(born_iso)
    WFD_DISPATCH(born_iso_scaleb)
    WFD_DISPATCH(born_aniso_v)
    WFD_DISPATCH(born_vea_sandwich)
    WFD_DISPATCH(born_vea_final)
    WFD_DISPATCH(image_iso)
    WFD_DISPATCH(image_aniso_v)
    WFD_DISPATCH(image_vea)
    WFD_DISPATCH(image_wavefieldsep)
#undef WFD_DISPATCH
};

int finish(Prop *p, const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) return prop_fail(p, WFD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    return WFD_OK;
}

// gradient triple for the VEA helpers: plain D+ for VTI, rotated D+ for TTI
void vea_grad(const K &k, Prop *p, const Grid &g, const Fields &F, const float *in, float *const *o) {
    if (p->phys == TTI) k.tti_dplus(g, F, in, o[0], o[1], o[2], p->stream);
    else k.dplus(g, in, o[0], o[1], o[2], p->stream);
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
            k.born_iso(g, 0, F, a[0], (const float *)nullptr, a[1], (const float *const *)nullptr, p->stream);
        } else {
            const bool vb = !strcmp(variant, "VB");
            float *dv = vb ? a[0] : nullptr, *db = vb ? a[1] : a[0], *P = vb ? a[2] : a[1], *DP = vb ? a[3] : a[2];
            if (!ensure_scratch(p, 6)) return p->status;
            k.dplus(g, P, t[0], t[1], t[2], p->stream);
            k.born_iso_scaleb(g, db, (const float *const *)t, t + 3, p->stream);
            k.dminus3(g, t[3], t[4], t[5], t[0], t[1], t[2], p->stream);
            k.born_iso(g, vb ? 1 : 2, F, dv, db, DP, (const float *const *)t, p->stream);
        }
    } else if (!strcmp(variant, "V")) {
        k.born_aniso_v(g, F, a[0], a[1], a[2], p->stream);
    } else {  // VEA: dV, dEps, dEta, P, M, DP, DM
        if (!ensure_scratch(p, 12)) return p->status;
        vea_grad(k, p, g, F, a[3], t);
        vea_grad(k, p, g, F, a[4], t + 3);
        k.born_vea_sandwich(g, F, a[1], a[2], (const float *const *)t, (const float *const *)(t + 3), t + 6, t + 9,
                            p->stream);
        if (p->phys == TTI) {
            k.tti_dminus(g, F, t[6], t[7], t[8], t[0], t[1], t[2], p->stream);
            k.tti_dminus(g, F, t[9], t[10], t[11], t[3], t[4], t[5], p->stream);
        } else {
            k.dminus3(g, t[6], t[7], t[8], t[0], t[1], t[2], p->stream);
            k.dminus3(g, t[9], t[10], t[11], t[3], t[4], t[5], p->stream);
        }
        k.born_vea_final(g, F, a[0], a[5], a[6], (const float *const *)t, (const float *const *)(t + 3), p->stream);
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
            k.image_iso(g, 0, F, a[1], (const float *const *)nullptr, (const float *const *)nullptr, a[0],
                        (float *)nullptr, p->stream);
            outs.push_back(a[0]);
        } else {
            const bool vb = !strcmp(variant, "VB");
            float *dv = vb ? a[0] : nullptr, *db = vb ? a[1] : a[0], *P = vb ? a[2] : a[1], *DP = vb ? a[3] : a[2];
            if (!ensure_scratch(p, 6)) return p->status;
            k.dplus(g, P, t[0], t[1], t[2], p->stream);
            k.dplus(g, F.pold, t[3], t[4], t[5], p->stream);
            k.image_iso(g, vb ? 1 : 2, F, DP, (const float *const *)t, (const float *const *)(t + 3), dv, db,
                        p->stream);
            if (dv) outs.push_back(dv);
            outs.push_back(db);
        }
    } else if (!strcmp(variant, "V")) {
        k.image_aniso_v(g, F, a[1], a[2], a[0], p->stream);
        outs.push_back(a[0]);
    } else {  // VEA: dV, dEps, dEta, P, M, DP, DM
        if (!ensure_scratch(p, 12)) return p->status;
        vea_grad(k, p, g, F, a[3], t);
        vea_grad(k, p, g, F, a[4], t + 3);
        vea_grad(k, p, g, F, F.pold, t + 6);
        vea_grad(k, p, g, F, F.mold, t + 9);
        k.image_vea(g, F, a[5], a[6], (const float *const *)t, (const float *const *)(t + 3),
                    (const float *const *)(t + 6), (const float *const *)(t + 9), a[0], a[1], a[2], p->stream);
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
