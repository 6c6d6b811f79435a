// Selection of the fused single-sweep step kernels by physics and dimension.
#include "wfd_kernels.h"

namespace WFD_NS {
using namespace wfd;

bool fused_step(const Grid &g, int phys, int linear, const Fields &F, cudaStream_t s) {
    (void)linear;
    if (g.ndim == 3 && phys == ISO) {
        // TMA-staged kernel when the tensor maps can be encoded (nz*4 a multiple of 16 bytes),
        // else the variant that stages its tiles with ordinary loads
        if (fused_iso3d_tma(g, F, s)) return true;
        return fused_iso3d(g, F, s);
    }
    return false;
}

}  // namespace WFD_NS
