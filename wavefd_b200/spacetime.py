"""Host-side source/receiver machinery of the path (src/spacetime.jl, src/wavelet.jl restated).

* `hickscoeffs` / `linearcoeffs`: interpolation weights and 1-based grid indices of off-grid
  points (src/spacetime.jl:812-1013), with the free-surface reflection and the deletion of
  out-of-bounds and |c| < eps points;
* `source_blocking` / `receiver_blocking` (src/spacetime.jl:1087-1129);
* `injectdata` / `extractdata`: the spacetime.cc C ABI of the CUDA library;
* `ricker` / `causal_ricker` (src/wavelet.jl:150-155, :173-181).

Indices follow the reference exactly (same Float64 arithmetic). The Kaiser window uses
numpy's modified Bessel function I0 where the reference uses SpecialFunctions.besseli, so the
weights agree to rounding, not bit for bit; the GPU consumes whatever table it is given, exactly.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .abi import SourcePoint32, SpacetimeABI

SOURCEPOINT32 = np.dtype({"names": ["iu", "ir", "c"], "formats": ["<i8", "<i8", "<f4"], "offsets": [0, 8, 16],
                          "itemsize": 24})


def kaiser(b, r, x):
    """src/spacetime.jl:678: I0(b*sqrt(1-(x/r)^2))/I0(b), zero outside |x| <= r."""
    x = np.asarray(x, dtype=np.float32)
    arg = np.float32(b) * np.sqrt(np.float32(1) - (x / np.float32(r)) ** 2).astype(np.float32)
    out = (np.i0(arg.astype(np.float64)) / np.i0(np.float64(np.float32(b)))).astype(np.float32)
    return np.where(np.abs(x) > r, np.float32(0), out).astype(np.float32)


def _sinc(x):
    x = np.asarray(x, dtype=np.float32)
    return np.sinc(x.astype(np.float64)).astype(np.float32)


def _hicks1d(alpha, b=6.42, r=4):
    a = np.arange(1, 2 * r + 1) - r
    xx = (a - np.float32(alpha)).astype(np.float32)
    return (kaiser(b, r, xx) * _sinc(xx)).astype(np.float32)


def _reflect(ci, iz_first, fs_index):
    # src/spacetime.jl:900-913: fold the weights above the free surface back with a sign flip
    if iz_first == fs_index - 3:
        ci[4] -= ci[2]
        ci[5] -= ci[1]
        ci[6] -= ci[0]
    if iz_first == fs_index - 2:
        ci[3] -= ci[1]
        ci[4] -= ci[0]
    if iz_first == fs_index - 1:
        ci[2] -= ci[0]


def _finish(iz, iy, ix, ir, c, nz, ny, nx, T):
    keep = (iz >= 1) & (iz <= nz) & (ix >= 1) & (ix <= nx)
    if iy is not None:
        keep &= (iy >= 1) & (iy <= ny)
    keep &= ~(np.abs(c) < np.finfo(T).eps)
    iz, ix, ir, c = iz[keep], ix[keep], ir[keep], c[keep]
    if iy is not None:
        iy = iy[keep]
        iu = iz + (iy - 1) * nz + (ix - 1) * nz * ny
    else:
        iu = iz + (ix - 1) * nz
    pts = np.zeros(len(c), SOURCEPOINT32)
    pts["iu"], pts["ir"], pts["c"] = iu, ir, c
    return pts


def hickscoeffs(dz, dx, z0, x0, nz, nx, z, x, fs_index=1, zstagger=0.0, xstagger=0.0, dy=None, y0=None, ny=None,
                y=None, ystagger=0.0):
    """2D (src/spacetime.jl:812-865) or, with dy/y0/ny/y, 3D (:867-925) Hicks weights, FP32."""
    T = np.float32
    three = dy is not None
    dz, dx = float(np.float32(dz)), float(np.float32(dx))
    dyf = float(np.float32(dy)) if three else None
    r, l = 4, 8
    z, x = np.atleast_1d(np.asarray(z, np.float64)), np.atleast_1d(np.asarray(x, np.float64))
    yv = np.atleast_1d(np.asarray(y, np.float64)) if three else None
    IZ, IY, IX, IR, C = [], [], [], [], []
    for i in range(len(z)):
        iz_mid = int(np.floor((z[i] - z0) / dz)) + 1
        ix_mid = int(np.floor((x[i] - x0) / dx)) + 1
        az = T((z[i] - (z0 + (iz_mid - 1 + zstagger) * dz)) / dz)
        ax = T((x[i] - (x0 + (ix_mid - 1 + xstagger) * dx)) / dx)
        fz, fx = _hicks1d(az), _hicks1d(ax)
        if three:
            iy_mid = int(np.floor((yv[i] - y0) / dyf)) + 1
            ay = T((yv[i] - (y0 + (iy_mid - 1 + ystagger) * dyf)) / dyf)
            fy = _hicks1d(ay)
            ci = (fz[:, None, None] * fy[None, :, None] * fx[None, None, :]).astype(T)  # [iz, iy, ix]
            _reflect(ci, iz_mid - r + 1, fs_index)
            kz, ky, kx = np.meshgrid(np.arange(1, l + 1), np.arange(1, l + 1), np.arange(1, l + 1), indexing="ij")
            # Julia order: ix outer, iy, iz inner
            order = np.lexsort((kz.ravel(), ky.ravel(), kx.ravel()))
            IZ.append((iz_mid - r + kz.ravel())[order])
            IY.append((iy_mid - r + ky.ravel())[order])
            IX.append((ix_mid - r + kx.ravel())[order])
            C.append(ci.ravel()[order])
        else:
            ci = (fz[:, None] * fx[None, :]).astype(T)
            _reflect(ci, iz_mid - r + 1, fs_index)
            kz, kx = np.meshgrid(np.arange(1, l + 1), np.arange(1, l + 1), indexing="ij")
            order = np.lexsort((kz.ravel(), kx.ravel()))
            IZ.append((iz_mid - r + kz.ravel())[order])
            IX.append((ix_mid - r + kx.ravel())[order])
            C.append(ci.ravel()[order])
        IR.append(np.full(C[-1].shape, i + 1))
    cat = lambda a: np.concatenate(a) if a else np.zeros(0, np.int64)
    return _finish(cat(IZ), cat(IY) if three else None, cat(IX), cat(IR), np.concatenate(C).astype(T) if C else
                   np.zeros(0, T), nz, ny, nx, T)


def linearcoeffs(dz, dx, z0, x0, nz, nx, z, x, fs_index=1, dy=None, y0=None, ny=None, y=None):
    """2D (src/spacetime.jl:927-966) or 3D (:968-1013) bilinear/trilinear weights."""
    T = np.float32
    three = dy is not None
    dz, dx = float(np.float32(dz)), float(np.float32(dx))
    z, x = np.atleast_1d(np.asarray(z, np.float64)), np.atleast_1d(np.asarray(x, np.float64))
    IZ, IY, IX, IR, C = [], [], [], [], []
    for i in range(len(z)):
        kx = int(np.floor((x[i] - x0) / dx)) + 1
        kz = int(np.floor((z[i] - z0) / dz)) + 1
        rx = (x[i] - (x0 + dx * (kx - 1))) / dx
        rz = (z[i] - (z0 + dz * (kz - 1))) / dz
        if three:
            dyf = float(np.float32(dy))
            yy = float(np.atleast_1d(y)[i])
            ky = int(np.floor((yy - y0) / dyf)) + 1
            ry = (yy - (y0 + dyf * (ky - 1))) / dyf
            for _ix in (0, 1):
                for _iy in (0, 1):
                    for _iz in (0, 1):
                        w = ((rx if _ix else 1.0 - rx) * (ry if _iy else 1.0 - ry) * (rz if _iz else 1.0 - rz))
                        if kz == fs_index and _iz == 0:
                            w = 0.0
                        IZ.append(kz + _iz)
                        IY.append(ky + _iy)
                        IX.append(kx + _ix)
                        IR.append(i + 1)
                        C.append(T(w))
        else:
            for _ix in (0, 1):
                for _iz in (0, 1):
                    w = (rx if _ix else 1.0 - rx) * (rz if _iz else 1.0 - rz)
                    if kz == fs_index and _iz == 0:
                        w = 0.0
                    IZ.append(kz + _iz)
                    IX.append(kx + _ix)
                    IR.append(i + 1)
                    C.append(T(w))
    a = lambda v: np.asarray(v, np.int64)
    return _finish(a(IZ), a(IY) if three else None, a(IX), a(IR), np.asarray(C, T), nz, ny, nx, T)


def blocking(points, key, nthreads):
    """src/spacetime.jl:1087-1129: stable sort by key, then partitions with no key shared."""
    pts = points[np.argsort(points[key], kind="stable")]
    n = len(pts)
    npart = min(nthreads, n)
    if npart < 1:
        raise ValueError(f"max(nthreads, length(points)) must be greater than zero, nthreads={nthreads}, "
                         f"length(points)={n}")
    nominal, r = divmod(n, npart)
    if r > 0:
        nominal += 1
    parts = [[] for _ in range(npart)]
    ip, counter = 0, 1
    keys = pts[key]
    for i in range(n):
        if counter <= nominal or (i > 0 and keys[i] == keys[i - 1]):
            parts[ip].append(i)
            counter += 1
        else:
            ip += 1
            if ip >= len(parts):
                parts.append([])
            parts[ip].append(i)
            counter = 1
    return [np.ascontiguousarray(pts[idx]) for idx in parts if idx]


def source_blocking(points, nthreads=8):
    return blocking(points, "iu", nthreads)


def receiver_blocking(points, nthreads=8):
    return blocking(points, "ir", nthreads)


def _partition_args(partitions):
    ptrs = (ctypes.POINTER(SourcePoint32) * len(partitions))(
        *[p.ctypes.data_as(ctypes.POINTER(SourcePoint32)) for p in partitions])
    counts = (ctypes.c_long * len(partitions))(*[len(p) for p in partitions])
    return ptrs, counts


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def injectdata(field, partitions, data, it, nthreads=8, lib=None):
    """field[iu] += c * data[it, ir] (1-based it; data shaped (ntraces, nt) C order = Julia (nt, ntraces))."""
    from . import _lib
    st = SpacetimeABI(lib or _lib.library())
    ptrs, counts = _partition_args(partitions)
    nt = data.shape[-1]
    st.injectdata_float(_fp(field), _fp(data), it, nt, ptrs, len(partitions), counts, nthreads)


def extractdata(data, field, it, partitions, nthreads=8, lib=None):
    from . import _lib
    st = SpacetimeABI(lib or _lib.library())
    ptrs, counts = _partition_args(partitions)
    nt = data.shape[-1]
    st.extractdata_float(_fp(data), _fp(field), ptrs, len(partitions), counts, it, nt, nthreads)


# ---- wavelets (src/wavelet.jl) --------------------------------------------------------------------
def ricker(t, f=15.0, a=1.0):
    """src/wavelet.jl:150-155 without phase shift or taper."""
    t = np.asarray(t, np.float64)
    return (a * (1.0 - 2.0 * (np.pi * f * t) ** 2) * np.exp(-(np.pi * f * t) ** 2)).astype(np.float32)


def causal_ricker(t, f=15.0, a=1.0, tol=1e-4):
    """src/wavelet.jl:173-181: the Ricker centred on mean(t), shifted to start where |w| > tol*a."""
    t = np.asarray(t, np.float64)
    wav = ricker(t - t.mean(), f, a)
    idx = int(np.nonzero(np.abs(wav) > tol * a)[0][0])
    out = np.zeros_like(wav)
    out[: len(wav) - idx] = wav[idx:]
    return out


def interpfilters(dtmod, dtrec, mode=0, dtype=np.float32):
    """src/spacetime.jl:333-360: nh = dtrec/dtmod 8-tap sinc filters (nh x 8) mapping dtmod <-> dtrec;
    mode 0 preserves amplitude in the forward operator (fine -> coarse), mode 1 in the adjoint. The
    8x8 solve runs in float64 and is rounded to `dtype` (Julia solves in the element type, so the
    taps agree to rounding; the interpolation kernels consume whatever taps they are given exactly)."""
    n = int(round(dtrec / dtmod))
    if abs(n * dtmod - dtrec) / dtrec > 1e-6:
        raise ValueError(f"dtrec/dtmod must be an integer (n={n}, dtrec={dtrec}, dtmod={dtmod})")
    d = dtmod / dtrec * np.arange(n)
    fmax = 0.066 + 0.265 * np.log(8.0)
    j = np.arange(1, 9)
    a = np.sinc((j - 1) * fmax)
    A = np.array([[a[abs(r - c)] for c in range(8)] for r in range(8)])
    h = np.stack([np.linalg.solve(A, np.sinc((4 - j + d[i]) * fmax)) for i in range(n)])
    if mode == 0:
        h = h / n
    return np.ascontiguousarray(h.astype(dtype))


def interp(lib_abi, forward, h, inp, nout):
    """Run a library's interpforward_nd / interpadjoint_nd on traces (ntraces, nin) -> (ntraces, nout)."""
    h = np.ascontiguousarray(h)
    T = "double" if h.dtype == np.float64 else "float"
    ct = ctypes.c_double if T == "double" else ctypes.c_float
    rows = (ctypes.POINTER(ct) * len(h))(*[h[k].ctypes.data_as(ctypes.POINTER(ct)) for k in range(len(h))])
    inp = np.ascontiguousarray(inp, dtype=h.dtype)
    ntr, nin = inp.shape
    out = np.zeros((ntr, nout), dtype=h.dtype)
    p = lambda a: a.ctypes.data_as(ctypes.POINTER(ct))
    if forward:
        getattr(lib_abi, f"interpforward_nd_{T}")(rows, p(out), p(inp), len(h), nout, nin, ntr, 8)
    else:
        getattr(lib_abi, f"interpadjoint_nd_{T}")(rows, p(out), p(inp), len(h), nout, nin, ntr, 8)
    return out
