"""Seeded synthetic earth models and acquisition geometry for the benchmark workloads.

Stand-ins for field data (none is available offline), with the shapes and value ranges of the
workloads: 8 flat velocity layers 1500-4500 m/s plus a Gaussian-smoothed random perturbation
(+-5 %, 200 m correlation length), Gardner density, Q from 50-200 in smooth random blocks with the
reference's log ramp to qMin inside the sponge (absorb.h:85-151), and for VTI/TTI layered-plus-
random epsilon/eta and smooth random tilt/azimuth. Arrays are torch tensors shaped (nx, ny, nz)
(C order, z fastest), generated on `device`.
"""
from __future__ import annotations

import math

import numpy as np
import torch


def _gauss_smooth(x, sigma_cells):
    for ax, n in enumerate(x.shape):
        if n < 2:
            continue
        k = torch.fft.rfftfreq(n, device=x.device)
        g = torch.exp(-2.0 * (math.pi * sigma_cells * k) ** 2)
        gs = [1] * x.dim()
        gs[ax] = -1
        x = torch.fft.irfft(torch.fft.rfft(x, dim=ax) * g.reshape(gs), n=n, dim=ax)
    return x


def _smooth_noise(shape, sigma_cells, gen, device):
    x = torch.randn(shape, generator=gen, device=device, dtype=torch.float32)
    for ax, n in enumerate(shape):
        if n < 2:
            continue
        k = torch.fft.rfftfreq(n, device=device)
        g = torch.exp(-2.0 * (math.pi * sigma_cells * k) ** 2)
        gs = [1] * len(shape)
        gs[ax] = -1
        x = torch.fft.irfft(torch.fft.rfft(x, dim=ax) * g.reshape(gs), n=n, dim=ax)
    return x / x.abs().max().clamp_min(1e-12)


def _layers(nz, lo, hi, nlayers, device):
    li = (torch.arange(nz, device=device) * nlayers) // nz
    return lo + (hi - lo) * li.float() / max(nlayers - 1, 1)


def earth_model(shape, physics="iso", seed=1, d=10.0, dt=0.0005, nsponge=40, freqQ=5.0, qmin=0.1, fs=True,
                q_blocks=True, device="cuda"):
    """Returns a dict of tensors named like the propagator getters (V, B, DtOmegaInvQ, Eps, ...)."""
    nx, ny, nz = shape
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    corr = 200.0 / d
    v = _layers(nz, 1500.0, 4500.0, 8, device).reshape(1, 1, nz).expand(nx, ny, nz).clone()
    v *= 1.0 + 0.05 * _smooth_noise(shape, corr, gen, device)
    rho = (0.31 * v.pow(0.25)).clamp(1.0, 2.5)  # Gardner, g/cc
    m = {"V": v, "B": 1.0 / rho}
    # Q: uniform 50-200 per 32^3 block, smoothed; log ramp to qmin in the sponge
    if q_blocks:
        bs = 32
        nb = (max(1, -(-nx // bs)), max(1, -(-ny // bs)), max(1, -(-nz // bs)))
        qb = 50.0 + 150.0 * torch.rand(nb, generator=gen, device=device)
        q = qb.repeat_interleave(bs, 0).repeat_interleave(bs, 1).repeat_interleave(bs, 2)[:nx, :ny, :nz]
        q = _gauss_smooth(q.float(), 4.0).clamp(50.0, 200.0)
    else:
        q = torch.full(shape, 100.0, device=device)
    ix = torch.arange(nx, device=device)
    iy = torch.arange(ny, device=device)
    iz = torch.arange(nz, device=device)
    ksx = torch.minimum(ix, nx - 1 - ix).reshape(nx, 1, 1)
    ksy = torch.minimum(iy, ny - 1 - iy).reshape(1, ny, 1)
    ksz = (nz - 1 - iz) if fs else torch.minimum(iz, nz - 1 - iz)
    ks = torch.minimum(torch.minimum(ksx, ksy), ksz.reshape(1, 1, nz)).float()
    ramp = torch.exp(math.log(qmin) + ks / (nsponge - 1) * (torch.log(q) - math.log(qmin)))
    q = torch.where(ks < nsponge, ramp, q)
    m["DtOmegaInvQ"] = (dt * 2.0 * math.pi * freqQ) / q
    if physics in ("vti", "tti"):
        m["Eps"] = (_layers(nz, 0.0, 0.25, 8, device).reshape(1, 1, nz) + 0.05 * (1 + _smooth_noise(shape, corr, gen, device)) / 2).clamp(0, 0.3)
        m["Eta"] = (_layers(nz, 0.0, 0.12, 8, device).reshape(1, 1, nz) + 0.03 * (1 + _smooth_noise(shape, corr, gen, device)) / 2).clamp(0, 0.15)
        m["F"] = torch.full(shape, 0.85, device=device)
    if physics == "tti":
        th = (math.pi / 8) * (1 + _smooth_noise(shape, corr, gen, device))  # 0..45 degrees
        ph = math.pi * (1 + _smooth_noise(shape, corr, gen, device))  # 0..360 degrees
        m["SinTheta"], m["CosTheta"] = torch.sin(th), torch.cos(th)
        m["SinPhi"], m["CosPhi"] = torch.sin(ph), torch.cos(ph)
    return {k: t.to(torch.float32).contiguous() for k, t in m.items()}


def surface_receivers(shape, nrx, nry, nsponge, depth_index=2):
    """On-grid receiver points (weights collapse to 1, as hickscoeffs gives on grid) on a
    nrx x nry grid at the given depth, inside the sponge. Returns a SourcePoint32 array."""
    from .spacetime import SOURCEPOINT32
    nx, ny, nz = shape
    xs = np.round(np.linspace(nsponge, nx - 1 - nsponge, nrx)).astype(np.int64)
    ys = np.round(np.linspace(nsponge, ny - 1 - nsponge, nry)).astype(np.int64)
    gx, gy = np.meshgrid(xs, ys, indexing="ij")
    iz = depth_index + 1
    iu = iz + gy.ravel() * nz + gx.ravel() * nz * ny  # 1-based linear index of (z, y, x)
    pts = np.zeros(iu.size, SOURCEPOINT32)
    pts["iu"] = iu
    pts["ir"] = np.arange(1, iu.size + 1)
    pts["c"] = 1.0
    return pts


def center_source(shape, d, depth=2.5):
    """Hicks-interpolated point source near the surface at the centre of the model (off grid)."""
    from .spacetime import hickscoeffs
    nx, ny, nz = shape
    return hickscoeffs(d, d, 0.0, 0.0, nz, nx, [depth * d], [(nx // 2 + 0.5) * d], dy=d, y0=0.0, ny=ny,
                       y=[(ny // 2 + 0.5) * d])


def surface_acquisition_2d(shape, d, depth=1.0):
    """2D: a Hicks source at the centre of the top row and on-grid receivers on every surface cell
    (depth index 2). shape = (nx, nz). Returns (sources, receivers) SourcePoint32 arrays."""
    from .spacetime import SOURCEPOINT32, hickscoeffs
    nx, nz = shape
    src = hickscoeffs(d, d, 0.0, 0.0, nz, nx, [depth * d], [(nx // 2) * d])
    iu = 3 + np.arange(nx) * nz  # 1-based (z index 2, x)
    rec = np.zeros(nx, SOURCEPOINT32)
    rec["iu"] = iu
    rec["ir"] = np.arange(1, nx + 1)
    rec["c"] = 1.0
    return src, rec
