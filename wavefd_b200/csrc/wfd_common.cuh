// Shared device definitions for the WaveFD-B200 kernels.
//
// Every kernel source is compiled twice: once with IEEE order of operations (-fmad=false,
// IEEE division and square root; namespace wfd_strict) and once for speed (FMA contraction,
// approximate division; namespace wfd_fast). Expressions are written in the reference's
// evaluation order, so the strict build reproduces the reference's FP32 results bit for bit.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#ifndef WFD_STRICT
#define WFD_STRICT 0
#endif

#if WFD_STRICT
#define WFD_NS wfd_strict
#else
#define WFD_NS wfd_fast
#endif

namespace wfd {

// Geometry and stencil constants, passed by value to every kernel.
// Layout k = (kx*ny + ky)*nz + kz; 2D uses ny = 1.
struct Grid {
    int ndim;
    int fs;
    long nx, ny, nz;
    long sx, sy;  // strides of x and y
    long n;       // cells
    float c1, c2, c3, c4;
    float idx, idy, idz;
    float dt, dt2;
};

enum Physics { ISO = 0, VTI = 1, TTI = 2 };

// Region of a cell in every reference pass: 0 = outside (derivative outputs are zero, fields
// are not updated), 1 = interior [4, n-4) in every axis, 2 = free-surface row kz in 0..3.
__host__ __device__ __forceinline__ int region(const Grid &g, long x, long y, long z) {
    if (x < 4 || x >= g.nx - 4) return 0;
    if (g.ndim == 3 && (y < 4 || y >= g.ny - 4)) return 0;
    if (z >= g.nz - 4) return 0;
    if (z >= 4) return 1;
    return g.fs ? 2 : 0;
}

}  // namespace wfd
