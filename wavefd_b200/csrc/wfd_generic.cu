// Unfused kernels: the reference's pass structure on the GPU, one thread per cell.
//
// These serve the Born-injection and imaging-condition entry points (which the reference
// builds from standalone D+/D- passes and pointwise loops) and act as the unfused time step
// for geometries the fused kernels do not take. Per-cell arithmetic follows the reference's
// expression trees; see the file:line notes at each kernel.
#include "wfd_kernels.h"

namespace WFD_NS {
using namespace wfd;

namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(long n) { return (unsigned)((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ void cell_xyz(const Grid &g, long k, long &x, long &y, long &z) {
    z = k % g.nz;
    const long r = k / g.nz;
    y = r % g.ny;
    x = r / g.ny;
}

// D+ at f[0] along stride s reads f[-3s..4s]; D- reads f[-4s..3s]
// (prop3DAcoIsoDenQ_DEO2_FDTD.h:846-864 and :1113-1131).
__device__ __forceinline__ float stp(const Grid &g, const float *__restrict__ f, long s) {
    return g.c1 * (-f[0] + f[s]) + g.c2 * (-f[-s] + f[2 * s]) + g.c3 * (-f[-2 * s] + f[3 * s]) +
           g.c4 * (-f[-3 * s] + f[4 * s]);
}
__device__ __forceinline__ float stm(const Grid &g, const float *__restrict__ f, long s) {
    return g.c1 * (-f[-s] + f[0]) + g.c2 * (-f[-2 * s] + f[s]) + g.c3 * (-f[-3 * s] + f[2 * s]) +
           g.c4 * (-f[-4 * s] + f[3 * s]);
}
// free-surface images above kz = 0: antisymmetric for D+ inputs, symmetric for D- inputs
// (the hard-coded rows of propagatorStaticFunctions.h:80-160 and :230-310)
__device__ __forceinline__ float imp(const float *__restrict__ col, long j) { return j >= 0 ? col[j] : -col[-j]; }
__device__ __forceinline__ float imm(const float *__restrict__ col, long j) { return j >= 0 ? col[j] : col[-j - 1]; }
__device__ __forceinline__ float stpz(const Grid &g, const float *__restrict__ col, long z) {
    return g.c1 * (-imp(col, z) + imp(col, z + 1)) + g.c2 * (-imp(col, z - 1) + imp(col, z + 2)) +
           g.c3 * (-imp(col, z - 2) + imp(col, z + 3)) + g.c4 * (-imp(col, z - 3) + imp(col, z + 4));
}
__device__ __forceinline__ float stmz(const Grid &g, const float *__restrict__ col, long z) {
    return g.c1 * (-imm(col, z - 1) + imm(col, z)) + g.c2 * (-imm(col, z - 2) + imm(col, z + 1)) +
           g.c3 * (-imm(col, z - 3) + imm(col, z + 2)) + g.c4 * (-imm(col, z - 4) + imm(col, z + 3));
}

// Weighted D- terms w(j) * f(j) (TTI back-rotation inside the stencil,
// prop2DAcoTTIDenQ_DEO2_FDTD.h:1060-1118, prop3DAcoTTIDenQ_DEO2_FDTD.h:3293-3347)
struct T1 {
    const float *__restrict__ w;
    const float *__restrict__ f;
    __device__ __forceinline__ float operator()(long j) const { return w[j] * f[j]; }
};
struct T2 {
    const float *__restrict__ w1;
    const float *__restrict__ w2;
    const float *__restrict__ f;
    __device__ __forceinline__ float operator()(long j) const { return w1[j] * w2[j] * f[j]; }
};
template <class T>
__device__ __forceinline__ float stm_t(const Grid &g, const T &t, long k, long s) {
    return g.c1 * (-t(k - s) + t(k)) + g.c2 * (-t(k - 2 * s) + t(k + s)) + g.c3 * (-t(k - 3 * s) + t(k + 2 * s)) +
           g.c4 * (-t(k - 4 * s) + t(k + 3 * s));
}
template <class T>
__device__ __forceinline__ float stmz_t(const Grid &g, const T &t, long k0, long z) {
    auto m = [&](long j) { return t(k0 + (j >= 0 ? j : -j - 1)); };
    return g.c1 * (-m(z - 1) + m(z)) + g.c2 * (-m(z - 2) + m(z + 1)) + g.c3 * (-m(z - 3) + m(z + 2)) +
           g.c4 * (-m(z - 4) + m(z + 3));
}

__device__ __forceinline__ void gradp(const Grid &g, const float *__restrict__ f, long k, long z, int r,
                                      float &dx, float &dy, float &dz) {
    if (r == 2 && z == 0) {
        dx = 0.0f;
        dy = 0.0f;
    } else {
        dx = g.idx * stp(g, f + k, g.sx);
        dy = g.ndim == 3 ? g.idy * stp(g, f + k, g.sy) : 0.0f;
    }
    dz = g.idz * stpz(g, f + k - z, z);
}

__device__ __forceinline__ void gradm3(const Grid &g, const float *__restrict__ fx, const float *__restrict__ fy,
                                       const float *__restrict__ fz, long k, long z, int r, float &dx, float &dy,
                                       float &dz) {
    if (r == 2 && z == 0) {
        dx = 0.0f;
        dy = 0.0f;
        dz = 0.0f;
        return;
    }
    dx = g.idx * stm(g, fx + k, g.sx);
    dy = g.ndim == 3 ? g.idy * stm(g, fy + k, g.sy) : 0.0f;
    dz = g.idz * stmz(g, fz + k - z, z);
}

// ---------------------------------------------------------------------------------------------
// Pass 1: D+ and the material sandwich.
// Iso: prop3DAcoIsoDenQ_DEO2_FDTD.h:841-893; VTI: prop3DAcoVTIDenQ_DEO2_FDTD.h:945-957 and
// prop2DAcoVTIDenQ_DEO2_FDTD.h:771-779; TTI: prop3DAcoTTIDenQ_DEO2_FDTD.h:885-976 and
// prop2DAcoTTIDenQ_DEO2_FDTD.h:672-760.
template <int PHYS>
__global__ void __launch_bounds__(kThreads) k_pass1(Grid g, Fields F, Scratch S) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    long x, y, z;
    cell_xyz(g, k, x, y, z);
    const int r = region(g, x, y, z);
    const int nout = PHYS == ISO ? 3 : 6;
    if (!r) {
        for (int i = 0; i < nout; i++) S.t[i][k] = 0.0f;
        return;
    }
    float dPx, dPy, dPz;
    gradp(g, F.pcur, k, z, r, dPx, dPy, dPz);
    if (PHYS == ISO) {
        const float B = F.b[k];
        S.t[0][k] = B * dPx;
        S.t[1][k] = B * dPy;
        S.t[2][k] = B * dPz;
        return;
    }
    float dMx, dMy, dMz;
    gradp(g, F.mcur, k, z, r, dMx, dMy, dMz);
    if (PHYS == VTI) {
        const float E = 1 + 2 * F.eps[k];
        const float A = F.eta[k];
        const float Fv = F.f[k];
        const float B = F.b[k];
        if (g.ndim == 3) {
            const float SA2 = sqrtf(1 - A * A);
            S.t[0][k] = B * E * dPx;
            S.t[1][k] = B * E * dPy;
            S.t[2][k] = B * (1 - Fv * A * A) * dPz + B * (Fv * A * SA2) * dMz;
            S.t[3][k] = B * (1 - Fv) * dMx;
            S.t[4][k] = B * (1 - Fv) * dMy;
            S.t[5][k] = B * Fv * A * SA2 * dPz + B * (1 - Fv + Fv * A * A) * dMz;
        } else {
            S.t[0][k] = B * E * dPx;
            S.t[1][k] = 0.0f;
            S.t[2][k] = B * (1 - Fv * A * A) * dPz + B * Fv * A * sqrtf(1 - A * A) * dMz;
            S.t[3][k] = B * (1 - Fv) * dMx;
            S.t[4][k] = 0.0f;
            S.t[5][k] = B * Fv * A * sqrtf(1 - A * A) * dPz + B * (1 - Fv + Fv * A * A) * dMz;
        }
        return;
    }
    // TTI
    if (g.ndim == 3) {
        const float sinThetaCosPhi = F.st[k] * F.cp[k];
        const float sinThetaSinPhi = F.st[k] * F.sp[k];
        const float eta = F.eta[k];
        const float eps = F.eps[k];
        const float fv = F.f[k];
        const float bv = F.b[k];
        const float cosT = F.ct[k];
        const float fieldEta2 = eta * eta;
        const float fieldBuoyVsVp = bv * fv;
        const float g3P = sinThetaCosPhi * dPx + sinThetaSinPhi * dPy + cosT * dPz;
        const float g3M = sinThetaCosPhi * dMx + sinThetaSinPhi * dMy + cosT * dMz;
        const float tmpFE = fieldBuoyVsVp * eta * sqrtf(1 - fieldEta2);
        const float tmpP = -bv * (2 * eps + fv * fieldEta2) * g3P + tmpFE * g3M;
        const float tmpM = tmpFE * g3P + fieldBuoyVsVp * fieldEta2 * g3M;
        const float tmpE = bv * (1 + 2 * eps);
        const float tmpF = bv * (1 - fv);
        S.t[0][k] = tmpE * dPx + sinThetaCosPhi * tmpP;
        S.t[1][k] = tmpE * dPy + sinThetaSinPhi * tmpP;
        S.t[2][k] = tmpE * dPz + cosT * tmpP;
        S.t[3][k] = tmpF * dMx + sinThetaCosPhi * tmpM;
        S.t[4][k] = tmpF * dMy + sinThetaSinPhi * tmpM;
        S.t[5][k] = tmpF * dMz + cosT * tmpM;
    } else {
        const float cosT = F.ct[k], sinT = F.st[k];
        const float dPG1 = cosT * dPx - sinT * dPz;
        const float dPG3 = sinT * dPx + cosT * dPz;
        const float dMG1 = cosT * dMx - sinT * dMz;
        const float dMG3 = sinT * dMx + cosT * dMz;
        const float E = 1 + 2 * F.eps[k];
        const float A = F.eta[k];
        const float Fv = F.f[k];
        const float B = F.b[k];
        S.t[0][k] = B * E * dPG1;
        S.t[1][k] = 0.0f;
        S.t[2][k] = B * (1 - Fv * A * A) * dPG3 + B * Fv * A * sqrtf(1 - A * A) * dMG3;
        S.t[3][k] = B * (1 - Fv) * dMG1;
        S.t[4][k] = 0.0f;
        S.t[5][k] = B * Fv * A * sqrtf(1 - A * A) * dPG3 + B * (1 - Fv + Fv * A * A) * dMG3;
    }
}

// Pass 2: D- and the second-order time update with the Q term.
// Iso 3D .h:1108-1159 (update :1152), 2D .h:943; VTI 3D .h:1372-1378 (linear .h:1697-1698);
// TTI 3D .h:1420-1421; TTI 2D with the back-rotation in the stencil .h:1055-1135.
template <int PHYS, bool LINEAR>
__global__ void __launch_bounds__(kThreads) k_pass2(Grid g, Fields F, Scratch S) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    long x, y, z;
    cell_xyz(g, k, x, y, z);
    const int r = region(g, x, y, z);
    if (!r) {
        if (!LINEAR) {
            F.pspace[k] = 0.0f;
            if (PHYS != ISO) F.mspace[k] = 0.0f;
        }
        return;
    }
    const float V = F.v[k];
    const float dt2V2_B = g.dt2 * V * V / F.b[k];
    const float Q = F.q[k];
    if (PHYS == ISO) {
        float dx, dy, dz;
        gradm3(g, S.t[0], S.t[1], S.t[2], k, z, r, dx, dy, dz);
        const float L = g.ndim == 3 ? dx + dy + dz : dx + dz;
        const float pc = F.pcur[k], po = F.pold[k];
        F.pold[k] = dt2V2_B * L - Q * (pc - po) - po + 2 * pc;
        F.pspace[k] = L;
        return;
    }
    float LP, LM;
    if (PHYS == TTI && g.ndim == 2) {
        float dPG1 = 0.0f, dPG3 = 0.0f, dMG1 = 0.0f, dMG3 = 0.0f;
        if (!(r == 2 && z == 0)) {
            const long k0 = k - z;
            dPG1 = g.idx * stm_t(g, T1{F.ct, S.t[0]}, k, g.sx) - g.idz * stmz_t(g, T1{F.st, S.t[0]}, k0, z);
            dPG3 = g.idx * stm_t(g, T1{F.st, S.t[2]}, k, g.sx) + g.idz * stmz_t(g, T1{F.ct, S.t[2]}, k0, z);
            dMG1 = g.idx * stm_t(g, T1{F.ct, S.t[3]}, k, g.sx) - g.idz * stmz_t(g, T1{F.st, S.t[3]}, k0, z);
            dMG3 = g.idx * stm_t(g, T1{F.st, S.t[5]}, k, g.sx) + g.idz * stmz_t(g, T1{F.ct, S.t[5]}, k0, z);
        }
        LP = dPG1 + dPG3;
        LM = dMG1 + dMG3;
    } else {
        float dPx, dPy, dPz, dMx, dMy, dMz;
        gradm3(g, S.t[0], S.t[1], S.t[2], k, z, r, dPx, dPy, dPz);
        gradm3(g, S.t[3], S.t[4], S.t[5], k, z, r, dMx, dMy, dMz);
        LP = g.ndim == 3 ? dPx + dPy + dPz : dPx + dPz;
        LM = g.ndim == 3 ? dMx + dMy + dMz : dMx + dMz;
    }
    if (!LINEAR) {
        F.pspace[k] = LP;
        F.mspace[k] = LM;
    }
    const float pc = F.pcur[k], po = F.pold[k];
    const float mc = F.mcur[k], mo = F.mold[k];
    F.pold[k] = dt2V2_B * LP - Q * (pc - po) - po + 2 * pc;
    F.mold[k] = dt2V2_B * LM - Q * (mc - mo) - mo + 2 * mc;
}

// scaleSpatialDerivatives (3D Iso .h:269-291; VTI .h:384-407; TTI .h:387-415)
__global__ void __launch_bounds__(kThreads) k_scale(Grid g, Fields F, int two) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    const float v2OverB = F.v[k] * F.v[k] / F.b[k];
    F.pspace[k] *= v2OverB;
    if (two) F.mspace[k] *= v2OverB;
}

// standalone D+ / D- (propagatorStaticFunctions.h:10-738)
__global__ void __launch_bounds__(kThreads) k_dplus(Grid g, const float *__restrict__ inx,
                                                    const float *__restrict__ iny, const float *__restrict__ inz,
                                                    float *ox, float *oy, float *oz) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    long x, y, z;
    cell_xyz(g, k, x, y, z);
    const int r = region(g, x, y, z);
    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    if (r) {
        if (r == 2 && z == 0) {
            dx = 0.0f;
            dy = 0.0f;
        } else {
            dx = g.idx * stp(g, inx + k, g.sx);
            dy = g.ndim == 3 ? g.idy * stp(g, iny + k, g.sy) : 0.0f;
        }
        dz = g.idz * stpz(g, inz + k - z, z);
    }
    ox[k] = dx;
    if (g.ndim == 3) oy[k] = dy;
    oz[k] = dz;
}

// ---------------------------------------------------------------------------------------------
// Born injection V, Iso: 3D .h:305-334, 2D .h:253-280 (a different expression)
struct Ptr3 {
    const float *p[3];
};
struct MPtr3 {
    float *p[3];
};
__global__ void __launch_bounds__(kThreads) k_born_iso_v(Grid g, Fields F, const float *__restrict__ dv,
                                                         const float *__restrict__ dp) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    const float V = F.v[k], B = F.b[k];
    const float dt = g.dt;
    const float dV = dv[k];
    if (g.ndim == 3) {
        const float dt2v2OverB = dt * dt * V * V / B;
        const float factorV = 2 * B * dV / (V * V * V);
        F.pcur[k] += dt2v2OverB * dp[k] * factorV;
    } else {
        const float factor = 2 * dt * dt * dV / V;
        F.pcur[k] += factor * dp[k];
    }
}

// Born injection V for VTI/TTI (3D VTI .h:420-452; 3D TTI .h:423-452; 2D alike)
__global__ void __launch_bounds__(kThreads) k_born_aniso_v(Grid g, Fields F, const float *__restrict__ dv,
                                                           const float *__restrict__ dp,
                                                           const float *__restrict__ dm) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    const float V = F.v[k], dV = dv[k];
    const float factor = 2 * g.dt * g.dt * dV / V;
    F.pcur[k] += factor * dp[k];
    F.mcur[k] += factor * dm[k];
}

// ---------------------------------------------------------------------------------------------
// Imaging conditions. Iso V: 3D .h:518-546 and the 2D form.
__global__ void __launch_bounds__(kThreads) k_image_iso_v(Grid g, Fields F, const float *__restrict__ dp, float *dv) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    const float V = F.v[k], B = F.b[k];
    const float factorV = +2 * B / (V * V * V);
    dv[k] += factorV * dp[k] * F.pold[k];
}

// VTI/TTI V (3D VTI .h:564-589; 3D TTI .h:567-592; 2D alike)
__global__ void __launch_bounds__(kThreads) k_image_aniso_v(Grid g, Fields F, const float *__restrict__ dp,
                                                            const float *__restrict__ dm, float *dv) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    const float V = F.v[k], B = F.b[k];
    const float factor = 2 * B / (V * V * V);
    dv[k] += factor * (dp[k] * F.pold[k] + dm[k] * F.mold[k]);
}


// ---------------------------------------------------------------------------------------------
// The VB/B and VEA Born injections and imaging conditions: the gradient triples and their D- are
// formed per cell in registers, not passed through scratch arrays (the reference's tmp arrays),
// each value by the reference's operations (applyFirstDerivatives3D_PlusHalf / MinusHalf,
// propagatorStaticFunctions.h:10-738, and the rotated forms of the TTI helpers, 3D TTI
// .h:2910-3661, 2D .h:1366-1719). Born VB/B: 2 launches and 3 scratch arrays
// (from 4 launches and 6); Born VEA: 2 launches and 6 (from 6 and 12); imaging VB/B and VEA: 1
// launch and no scratch (from 3 and 5).

// gradient triple at cell k, zero outside the interior: D+ (as k_dplus writes it) or, rotated, its
// TTI form (3D .h:2910-3166; 2D .h:1366-1530); 2D leaves o[1] zero
template <bool ROT>
__device__ __forceinline__ void grad_at(const Grid &g, const Fields &F, const float *__restrict__ in, long k, long z,
                                        int r, float (&o)[3]) {
    o[0] = 0.0f;
    o[1] = 0.0f;
    o[2] = 0.0f;
    if (!r) return;
    float dx, dy, dz;
    gradp(g, in, k, z, r, dx, dy, dz);
    if (!ROT) {
        o[0] = dx;
        o[1] = dy;
        o[2] = dz;
        return;
    }
    const float st = F.st[k], ct = F.ct[k];
    if (g.ndim == 3) {
        const float sp = F.sp[k], cp = F.cp[k];
        const float cosThetaCosPhi = ct * cp;
        const float cosThetaSinPhi = ct * sp;
        const float sinThetaCosPhi = st * cp;
        o[0] = cosThetaCosPhi * dx + cosThetaSinPhi * dy - st * dz;
        o[1] = -sp * dx + cp * dy;
        o[2] = sinThetaCosPhi * dx + st * sp * dy + ct * dz;
    } else {
        o[0] = ct * dx - st * dz;
        o[2] = st * dx + ct * dz;
    }
}

// D- triple at cell k, zero outside the interior and on kz = 0 under a free surface: plain, or
// rotated with the back-rotation inside the stencil (3D .h:3171-3661; 2D .h:1531-1719)
template <bool ROT>
__device__ __forceinline__ void dminus_at(const Grid &g, const Fields &F, const float *__restrict__ i1,
                                          const float *__restrict__ i2, const float *__restrict__ i3, long k, long z,
                                          int r, float (&o)[3]) {
    o[0] = 0.0f;
    o[1] = 0.0f;
    o[2] = 0.0f;
    if (!ROT) {
        if (r) gradm3(g, i1, i2, i3, k, z, r, o[0], o[1], o[2]);
        return;
    }
    if (!r || (r == 2 && z == 0)) return;
    const long k0 = k - z;
    if (g.ndim == 3) {
        o[0] = g.idx * stm_t(g, T2{F.ct, F.cp, i1}, k, g.sx) + g.idy * stm_t(g, T2{F.ct, F.sp, i1}, k, g.sy) -
               g.idz * stmz_t(g, T1{F.st, i1}, k0, z);
        o[1] = -g.idx * stm_t(g, T1{F.sp, i2}, k, g.sx) + g.idy * stm_t(g, T1{F.cp, i2}, k, g.sy);
        o[2] = g.idx * stm_t(g, T2{F.st, F.cp, i3}, k, g.sx) + g.idy * stm_t(g, T2{F.st, F.sp, i3}, k, g.sy) +
               g.idz * stmz_t(g, T1{F.ct, i3}, k0, z);
    } else {
        o[0] = g.idx * stm_t(g, T1{F.ct, i1}, k, g.sx) - g.idz * stmz_t(g, T1{F.st, i1}, k0, z);
        o[2] = g.idx * stm_t(g, T1{F.st, i3}, k, g.sx) + g.idz * stmz_t(g, T1{F.ct, i3}, k0, z);
    }
}

// Born VB/B, first launch: t = dB * D+ P (3D Iso .h:353-381)
__global__ void __launch_bounds__(kThreads) k_born_iso_b1(Grid g, Fields F, const float *__restrict__ db,
                                                          const float *__restrict__ P, MPtr3 t) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    long x, y, z;
    cell_xyz(g, k, x, y, z);
    float d[3];
    grad_at<false>(g, F, P, k, z, region(g, x, y, z), d);
    const float dB = db[k];
    t.p[0][k] = dB * d[0];
    if (g.ndim == 3) t.p[1][k] = dB * d[1];
    t.p[2][k] = dB * d[2];
}

// Born VB/B, second launch: D- of t and the update of pCur (3D .h:383-416 / .h:466-497; 2D alike)
__global__ void __launch_bounds__(kThreads) k_born_iso_b2(Grid g, int which, Fields F, const float *__restrict__ dv,
                                                          const float *__restrict__ db, const float *__restrict__ dp,
                                                          Ptr3 t) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    long x, y, z;
    cell_xyz(g, k, x, y, z);
    float L[3];
    dminus_at<false>(g, F, t.p[0], t.p[1], t.p[2], k, z, region(g, x, y, z), L);
    const float V = F.v[k], B = F.b[k];
    const float dt = g.dt;
    const float dB = db[k];
    if (g.ndim == 3) {
        const float dt2v2OverB = dt * dt * V * V / B;
        const float factorB = -dB / (V * V);
        if (which == 1) {
            const float dV = dv[k];
            const float factorV = 2 * B * dV / (V * V * V);
            F.pcur[k] += dt2v2OverB * (dp[k] * (factorV + factorB) + L[0] + L[1] + L[2]);
        } else {
            F.pcur[k] += dt2v2OverB * (dp[k] * factorB + L[0] + L[1] + L[2]);
        }
    } else {
        const float V2 = V * V;
        const float dt2v2OverB = dt * dt * V2 / B;
        if (which == 1) {
            const float dV = dv[k];
            F.pcur[k] += dt2v2OverB * (dp[k] / V2 * (2 * B * dV / V - dB) + L[0] + L[2]);
        } else {
            const float factorB = -dB / V2;
            F.pcur[k] += dt2v2OverB * (dp[k] * factorB + L[0] + L[2]);
        }
    }
}

// imaging VB/B in one launch: D+ of P and of pOld at the cell (3D Iso .h:563-656; 2D alike)
__global__ void __launch_bounds__(kThreads) k_image_iso_b(Grid g, int which, Fields F, const float *__restrict__ dp,
                                                          const float *__restrict__ P, float *dv, float *db) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    long x, y, z;
    cell_xyz(g, k, x, y, z);
    const int r = region(g, x, y, z);
    float a[3], b[3];
    grad_at<false>(g, F, P, k, z, r, a);
    grad_at<false>(g, F, F.pold, k, z, r, b);
    const float V = F.v[k], B = F.b[k];
    const float po = F.pold[k];
    if (which == 1) {
        const float factorV = +2 * B / (V * V * V);
        dv[k] += factorV * dp[k] * po;
    }
    const float factorB = -1 / (V * V);
    if (g.ndim == 3)
        db[k] += factorB * dp[k] * po - a[0] * b[0] - a[1] * b[1] - a[2] * b[2];
    else
        db[k] += factorB * dp[k] * po - a[0] * b[0] - a[2] * b[2];
}

// Born VEA, first launch: the gradient triples of P and M and the sandwich into tp2, tm2 (3D VTI
// .h:480-511; 3D TTI .h:481-512; 2D alike)
template <bool ROT>
__global__ void __launch_bounds__(kThreads) k_born_vea_1(Grid g, Fields F, const float *__restrict__ de,
                                                         const float *__restrict__ da, const float *__restrict__ P,
                                                         const float *__restrict__ M, MPtr3 tp2, MPtr3 tm2) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    long x, y, z;
    cell_xyz(g, k, x, y, z);
    const int r = region(g, x, y, z);
    float tp1[3], tm1[3];
    grad_at<ROT>(g, F, P, k, z, r, tp1);
    grad_at<ROT>(g, F, M, k, z, r, tm1);
    const float A = F.eta[k], B = F.b[k], Fv = F.f[k], dE = de[k], dA = da[k];
    tp2.p[0][k] = (+2 * B * dE) * tp1[0];
    if (g.ndim == 3) tp2.p[1][k] = (+2 * B * dE) * tp1[1];
    tp2.p[2][k] = (-2 * B * Fv * A * dA) * tp1[2] + (dA * B * Fv * (1 - 2 * A * A) / sqrtf(1 - A * A)) * tm1[2];
    tm2.p[0][k] = 0.0f;
    if (g.ndim == 3) tm2.p[1][k] = 0.0f;
    tm2.p[2][k] = (+2 * B * Fv * A * dA) * tm1[2] + (dA * B * Fv * (1 - 2 * A * A) / sqrtf(1 - A * A)) * tp1[2];
}

// Born VEA, second launch: D- of tp2 and tm2 and the update of pCur, mCur (3D VTI .h:513-548;
// 3D TTI .h:514-551; 2D alike)
template <bool ROT>
__global__ void __launch_bounds__(kThreads) k_born_vea_2(Grid g, Fields F, const float *__restrict__ dv,
                                                         const float *__restrict__ dp, const float *__restrict__ dm,
                                                         Ptr3 tp2, Ptr3 tm2) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    long x, y, z;
    cell_xyz(g, k, x, y, z);
    const int r = region(g, x, y, z);
    float lp[3], lm[3];
    dminus_at<ROT>(g, F, tp2.p[0], tp2.p[1], tp2.p[2], k, z, r, lp);
    dminus_at<ROT>(g, F, tm2.p[0], tm2.p[1], tm2.p[2], k, z, r, lm);
    const float V = F.v[k], B = F.b[k], dV = dv[k];
    const float dt2v2OverB = g.dt * g.dt * V * V / B;
    const float factor = 2 * B * dV / (V * V * V);
    if (g.ndim == 3) {
        F.pcur[k] += dt2v2OverB * (factor * dp[k] + lp[0] + lp[1] + lp[2]);
        F.mcur[k] += dt2v2OverB * (factor * dm[k] + lm[0] + lm[1] + lm[2]);
    } else {
        F.pcur[k] += dt2v2OverB * (factor * dp[k] + lp[0] + lp[2]);
        F.mcur[k] += dt2v2OverB * (factor * dm[k] + lm[0] + lm[2]);
    }
}

// imaging VEA in one launch: the gradient triples of P, M, pOld and mOld at the cell (3D VTI
// .h:730-787; 3D TTI .h:733-790; 2D alike)
template <bool ROT>
__global__ void __launch_bounds__(kThreads) k_image_vea_f(Grid g, Fields F, const float *__restrict__ dp,
                                                          const float *__restrict__ dm, const float *__restrict__ P,
                                                          const float *__restrict__ M, float *dv, float *de,
                                                          float *da) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= g.n) return;
    long x, y, z;
    cell_xyz(g, k, x, y, z);
    const int r = region(g, x, y, z);
    float tp1[3], tm1[3], tp2[3], tm2[3];
    grad_at<ROT>(g, F, P, k, z, r, tp1);
    grad_at<ROT>(g, F, M, k, z, r, tm1);
    grad_at<ROT>(g, F, F.pold, k, z, r, tp2);
    grad_at<ROT>(g, F, F.mold, k, z, r, tm2);
    const float V = F.v[k], A = F.eta[k], B = F.b[k], Fv = F.f[k];
    const float factor = 2 * B / (V * V * V);
    if (g.ndim == 3) {
        dv[k] += factor * (dp[k] * F.pold[k] + dm[k] * F.mold[k]);
        de[k] += (-2 * B * tp1[0] * tp2[0] - 2 * B * tp1[1] * tp2[1]);
    } else {
        dv[k] += factor * dp[k] * F.pold[k] + factor * dm[k] * F.mold[k];
        de[k] += -2 * B * tp1[0] * tp2[0];
    }
    const float partP = 2 * B * Fv * A * tp1[2] - (B * Fv * (1 - 2 * A * A) / sqrtf(1 - A * A)) * tm1[2];
    const float partM = 2 * B * Fv * A * tm1[2] + (B * Fv * (1 - 2 * A * A) / sqrtf(1 - A * A)) * tp1[2];
    da[k] += (partP * tp2[2] - partM * tm2[2]);
}

Ptr3 p3(const float *const *a) { return Ptr3{{a[0], a[1], a[2]}}; }
MPtr3 m3(float *const *a) { return MPtr3{{a[0], a[1], a[2]}}; }

}  // namespace

// ---------------------------------------------------------------------------------------------
void pass1(const Grid &g, int phys, const Fields &F, const Scratch &S, cudaStream_t s) {
    const unsigned nb = blocks_for(g.n);
    if (phys == ISO) k_pass1<ISO><<<nb, kThreads, 0, s>>>(g, F, S);
    else if (phys == VTI) k_pass1<VTI><<<nb, kThreads, 0, s>>>(g, F, S);
    else k_pass1<TTI><<<nb, kThreads, 0, s>>>(g, F, S);
}

void pass2(const Grid &g, int phys, int linear, const Fields &F, const Scratch &S, cudaStream_t s) {
    const unsigned nb = blocks_for(g.n);
    if (phys == ISO) k_pass2<ISO, false><<<nb, kThreads, 0, s>>>(g, F, S);
    else if (phys == VTI && linear) k_pass2<VTI, true><<<nb, kThreads, 0, s>>>(g, F, S);
    else if (phys == VTI) k_pass2<VTI, false><<<nb, kThreads, 0, s>>>(g, F, S);
    else k_pass2<TTI, false><<<nb, kThreads, 0, s>>>(g, F, S);
}

void scale(const Grid &g, const Fields &F, bool two, cudaStream_t s) {
    k_scale<<<blocks_for(g.n), kThreads, 0, s>>>(g, F, two ? 1 : 0);
}

void dplus3(const Grid &g, const float *inx, const float *iny, const float *inz, float *ox, float *oy, float *oz,
            cudaStream_t s) {
    k_dplus<<<blocks_for(g.n), kThreads, 0, s>>>(g, inx, iny, inz, ox, oy, oz);
}

void born_iso_v(const Grid &g, const Fields &F, const float *dv, const float *dp, cudaStream_t s) {
    k_born_iso_v<<<blocks_for(g.n), kThreads, 0, s>>>(g, F, dv, dp);
}

void born_aniso_v(const Grid &g, const Fields &F, const float *dv, const float *dp, const float *dm,
                  cudaStream_t s) {
    k_born_aniso_v<<<blocks_for(g.n), kThreads, 0, s>>>(g, F, dv, dp, dm);
}

void image_iso_v(const Grid &g, const Fields &F, const float *dp, float *dv, cudaStream_t s) {
    k_image_iso_v<<<blocks_for(g.n), kThreads, 0, s>>>(g, F, dp, dv);
}

void image_aniso_v(const Grid &g, const Fields &F, const float *dp, const float *dm, float *dv, cudaStream_t s) {
    k_image_aniso_v<<<blocks_for(g.n), kThreads, 0, s>>>(g, F, dp, dm, dv);
}

void born_iso_fused(const Grid &g, int which, const Fields &F, const float *dv, const float *db, const float *P,
                    const float *dp, float *const *t, cudaStream_t s) {
    k_born_iso_b1<<<blocks_for(g.n), kThreads, 0, s>>>(g, F, db, P, m3(t));
    k_born_iso_b2<<<blocks_for(g.n), kThreads, 0, s>>>(g, which, F, dv, db, dp, p3(t));
}

void image_iso_fused(const Grid &g, int which, const Fields &F, const float *dp, const float *P, float *dv, float *db,
                     cudaStream_t s) {
    k_image_iso_b<<<blocks_for(g.n), kThreads, 0, s>>>(g, which, F, dp, P, dv, db);
}

void born_vea_fused(const Grid &g, bool rot, const Fields &F, const float *dv, const float *de, const float *da,
                    const float *P, const float *M, const float *dp, const float *dm, float *const *t,
                    cudaStream_t s) {
    const unsigned nb = blocks_for(g.n);
    if (rot) {
        k_born_vea_1<true><<<nb, kThreads, 0, s>>>(g, F, de, da, P, M, m3(t), m3(t + 3));
        k_born_vea_2<true><<<nb, kThreads, 0, s>>>(g, F, dv, dp, dm, p3(t), p3(t + 3));
    } else {
        k_born_vea_1<false><<<nb, kThreads, 0, s>>>(g, F, de, da, P, M, m3(t), m3(t + 3));
        k_born_vea_2<false><<<nb, kThreads, 0, s>>>(g, F, dv, dp, dm, p3(t), p3(t + 3));
    }
}

void image_vea_fused(const Grid &g, bool rot, const Fields &F, const float *dp, const float *dm, const float *P,
                     const float *M, float *dv, float *de, float *da, cudaStream_t s) {
    if (rot) k_image_vea_f<true><<<blocks_for(g.n), kThreads, 0, s>>>(g, F, dp, dm, P, M, dv, de, da);
    else k_image_vea_f<false><<<blocks_for(g.n), kThreads, 0, s>>>(g, F, dp, dm, P, M, dv, de, da);
}

}  // namespace WFD_NS
