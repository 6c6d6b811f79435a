// Selection of the fused single-sweep step kernels by physics and dimension.
#include "wfd_kernels.h"

namespace WFD_NS {
using namespace wfd;

int fused_step(const Grid &g, int phys, int linear, const Fields &F, cudaStream_t s) {
    Fields Fn = F;
    Fn.illum = nullptr;      // the TMA-staged Iso, VTI and TTI kernels accumulate the illumination
    Fn.inj.ngroups = 0;      // themselves; only the 2D Iso kernel applies a source injection itself
    Fn.epi = StepEpilogue{};  // and only the TMA-staged 3D kernels apply the Born/imaging epilogue
    Fields Fl = Fn;
    Fl.illum = F.illum;
    Fields Fe = Fl;
    Fe.epi = F.epi;
    const int lit = F.illum ? 2 : 0;
    const int ept = (F.epi.born_dv || F.epi.img || F.epi.scale_space) ? 8 : 0;
    if (g.ndim == 3 && phys == ISO) {
        // TMA-staged kernel when the tensor maps can be encoded (nz*4 a multiple of 16 bytes),
        // else the variant that stages its tiles with ordinary loads
        if (fused_iso3d_tma(g, Fe, s)) return 1 | lit | ept;
        return fused_iso3d(g, Fn, s) ? 1 : 0;
    }
    if (g.ndim == 3 && phys == VTI) {
        // the VTI kernel with x-direction register queues, else the ring-staged kernel TTI uses
        if (fused_vti3d_tma(g, linear, Fe, s)) return 1 | lit | ept;
        return fused_aniso3d_tma(g, phys, linear, Fn, s) ? 1 : 0;
    }
    if (g.ndim == 3 && phys == TTI) return fused_aniso3d_tma(g, phys, linear, Fe, s) ? 1 | lit | ept : 0;
    if (g.ndim == 2 && phys == ISO) {
        Fields Fi = Fn;
        Fi.inj = F.inj;
        return fused_iso2d(g, Fi, s) ? 1 | (F.inj.ngroups ? 4 : 0) : 0;
    }
    if (g.ndim == 2) return fused_aniso2d(g, phys, linear, Fn, s) ? 1 : 0;
    return 0;
}

// limit of the tile-load waits of every TMA step kernel (test hook)
void fused_set_pipeline_wait(unsigned long long ns) {
    iso3d_set_pipeline_wait(ns);
    vti3d_set_pipeline_wait(ns);
    aniso3d_set_pipeline_wait(ns);
}

// timeout flags of every fused kernel, cleared on read
unsigned fused_status_and_clear() {
    return iso3d_status_and_clear() | aniso3d_status_and_clear() | vti3d_status_and_clear();
}

}  // namespace WFD_NS
