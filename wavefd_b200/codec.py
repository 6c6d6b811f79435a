"""Learned compression of saved forward wavefields (the role CvxCompress plays in the reference's
src/compressedio.jl:1-137), on the GPU.

`WavefieldCodec` wraps the CUDA codec of libwavefd_b200 (wfd_codec.cu): a 3D conv autoencoder with
BF16 weights and FP32 accumulation that turns each 8^3 block into 32 BF16 values and a scale, with
the 1 % worst-coded blocks kept raw. Its weights are trained here, on the GPU, by the library's own
forward/backward kernels and Adam, on 32^3 patches of wavefields the propagators themselves generate
(`propagated_snapshots`, `training_blocks`, `train`).

    codec = WavefieldCodec(seed=0)
    blocks = training_blocks(snapshots, npatches=2048, seed=0)
    history = train(codec, blocks, steps=1500)
    code = codec.empty_code(shape)            # device buffer, codec.code_bytes(shape) bytes
    codec.encode(field, shape, code)          # field: device tensor (nx, ny, nz)
    codec.decode(code, shape, out)
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_float, c_int, c_long, c_uint, c_void_p

import numpy as np

from . import _lib

_declared = False


def _L():
    global _declared
    lib = _lib.library()
    if not _declared:
        def fn(name, restype, argtypes):
            f = getattr(lib, name)
            f.restype = restype
            f.argtypes = argtypes
        fn("WFD_Codec_NumParams", c_long, [])
        fn("WFD_Codec_LatentBytes", c_long, [c_long, c_long, c_long])
        fn("WFD_Codec_Create", c_void_p, [c_uint])
        fn("WFD_Codec_Free", None, [c_void_p])
        fn("WFD_Codec_SetWeights", c_int, [c_void_p, POINTER(c_float), c_long])
        fn("WFD_Codec_GetWeights", c_int, [c_void_p, POINTER(c_float), c_long])
        fn("WFD_Codec_Encode", c_int, [c_void_p, c_void_p, c_long, c_long, c_long, c_void_p, c_void_p])
        fn("WFD_Codec_Decode", c_int, [c_void_p, c_void_p, c_long, c_long, c_long, c_void_p, c_void_p])
        fn("WFD_Codec_RawBlocks", c_long, [c_void_p, c_long, c_long, c_long])
        fn("WFD_Codec_SetEngine", c_int, [c_void_p, c_int])
        fn("WFD_Codec_Engine", c_int, [c_void_p])
        fn("WFD_Codec_Grid", c_int, [c_void_p, c_int])
        fn("WFD_Codec_Status", c_int, [c_void_p])
        fn("WFD_Codec_GatherBlocks", c_int, [c_void_p, c_long, c_long, c_long, c_void_p, c_long, c_void_p, c_void_p,
                                             c_void_p])
        fn("WFD_Codec_TrainStep", c_int, [c_void_p, c_void_p, c_long, c_float, POINTER(c_float), c_void_p])
        fn("WFD_Codec_Gradient", c_int, [c_void_p, c_void_p, c_long, POINTER(c_float), POINTER(c_float)])
        _declared = True
    return lib


def _dp(t):
    """Device address of a tensor for the C ABI, which takes dense row-major arrays."""
    if t is None:
        return None
    if not t.is_contiguous():
        raise ValueError("the codec takes contiguous tensors (call .contiguous())")
    return c_void_p(t.data_ptr())


def _check(rc, what):
    if rc != 0:
        raise _lib.WaveFDError(f"{what} failed (status {rc}): {_L().WFD_LastErrorMessage().decode()}")


class WavefieldCodec:
    def __init__(self, seed: int = 0):
        self.c = _L().WFD_Codec_Create(seed)
        if not self.c:
            raise _lib.WaveFDError("WFD_Codec_Create failed: " + _L().WFD_LastErrorMessage().decode())
        self.nparams = int(_L().WFD_Codec_NumParams())

    # -- weights ------------------------------------------------------------------------------------
    @property
    def params(self) -> np.ndarray:
        w = np.empty(self.nparams, np.float32)
        _check(_L().WFD_Codec_GetWeights(self.c, w.ctypes.data_as(POINTER(c_float)), self.nparams), "GetWeights")
        return w

    @params.setter
    def params(self, w):
        w = np.ascontiguousarray(w, np.float32)
        _check(_L().WFD_Codec_SetWeights(self.c, w.ctypes.data_as(POINTER(c_float)), w.size), "SetWeights")

    def save(self, path):
        np.save(path, self.params)

    def load(self, path):
        self.params = np.load(path)

    # -- coding -------------------------------------------------------------------------------------
    @staticmethod
    def code_bytes(shape) -> int:
        nx, ny, nz = shape
        return int(_L().WFD_Codec_LatentBytes(nx, ny, nz))

    def empty_code(self, shape, device="cuda"):
        import torch
        return torch.empty(self.code_bytes(shape), dtype=torch.uint8, device=device)

    def encode(self, field, shape, code, stream=None):
        nx, ny, nz = shape
        _check(_L().WFD_Codec_Encode(self.c, _dp(field), nx, ny, nz, _dp(code), stream), "Encode")

    def decode(self, code, shape, out, stream=None):
        nx, ny, nz = shape
        _check(_L().WFD_Codec_Decode(self.c, _dp(code), nx, ny, nz, _dp(out), stream), "Decode")

    def raw_blocks(self, code, shape) -> int:
        nx, ny, nz = shape
        return int(_L().WFD_Codec_RawBlocks(_dp(code), nx, ny, nz))

    _ENGINES = ("mma.sync", "tcgen05", "mixed")

    @property
    def engine(self) -> str:
        """"mma.sync", "tcgen05" (UMMA with the accumulators in tensor memory) or "mixed" (encode on
        mma.sync, decode on tcgen05: the default, the faster kernel of each direction)."""
        return self._ENGINES[_L().WFD_Codec_Engine(self.c)]

    @engine.setter
    def engine(self, name: str):
        _check(_L().WFD_Codec_SetEngine(self.c, self._ENGINES.index(name)), "SetEngine")

    def grids(self):
        """CTAs launched by each coding kernel."""
        names = ("encode mma.sync", "decode mma.sync", "encode tcgen05", "decode tcgen05")
        return {n: int(_L().WFD_Codec_Grid(self.c, i)) for i, n in enumerate(names)}

    def status(self):
        """Synchronises the device; raises if a tensor-core completion wait ran out."""
        _check(_L().WFD_Codec_Status(self.c), "Status")

    # -- training -----------------------------------------------------------------------------------
    def train_step(self, blocks, lr: float) -> float:
        """One Adam step on a device batch of normalised blocks (n, 512); returns the batch loss."""
        loss = c_float(0.0)
        _check(_L().WFD_Codec_TrainStep(self.c, _dp(blocks), blocks.shape[0], lr, ctypes.byref(loss), None),
               "TrainStep")
        return float(loss.value)

    def gradient(self, blocks):
        """(gradient of the mean squared error over the blocks, the loss), without a step."""
        g = np.empty(self.nparams, np.float32)
        loss = c_float(0.0)
        _check(_L().WFD_Codec_Gradient(self.c, _dp(blocks), blocks.shape[0], g.ctypes.data_as(POINTER(c_float)),
                                       ctypes.byref(loss)), "Gradient")
        return g, float(loss.value)

    def free(self):
        if self.c:
            _L().WFD_Codec_Free(self.c)
            self.c = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def gather_blocks(field, shape, origins):
    """Blocks of `field` at int32 device origins (n, 3) in the codec's cell order, each divided by its
    max |value|; returns (blocks (n, 512), scales (n,)) device tensors."""
    import torch
    nx, ny, nz = shape
    n = origins.shape[0]
    blocks = torch.empty((n, 512), device=field.device)
    scales = torch.empty(n, device=field.device)
    _check(_L().WFD_Codec_GatherBlocks(_dp(field), nx, ny, nz, _dp(origins.contiguous()), n, _dp(blocks),
                                       _dp(scales), None), "GatherBlocks")
    return blocks, scales


def training_blocks(snapshots, npatches=2048, seed=0, min_rel=1e-3, return_scales=False):
    """Normalised 8^3 blocks of random 32^3 patches (unaligned) of the snapshots, keeping blocks whose
    max |value| is at least min_rel of their snapshot's max. snapshots: list of device (nx, ny, nz).
    With return_scales, also each block's max |value| relative to its snapshot's max."""
    import torch
    rng = np.random.default_rng(seed)
    out, rel = [], []
    per = max(1, npatches // max(1, len(snapshots)))
    for f in snapshots:
        nx, ny, nz = f.shape
        px = rng.integers(0, max(1, nx - 32), per)
        py = rng.integers(0, max(1, ny - 32), per)
        pz = rng.integers(0, max(1, nz - 32), per)
        o = np.stack([px, py, pz], 1)[:, None, :] + 8 * np.stack(np.meshgrid(np.arange(4), np.arange(4), np.arange(4),
                                                                             indexing="ij"), -1).reshape(1, 64, 3)
        org = torch.from_numpy(o.reshape(-1, 3).astype(np.int32)).to(f.device)
        b, s = gather_blocks(f, (nx, ny, nz), org)
        fmax = float(f.abs().max())
        keep = s >= min_rel * fmax
        out.append(b[keep])
        rel.append(s[keep] / fmax)
    if return_scales:
        return torch.cat(out), torch.cat(rel)
    return torch.cat(out)


def train(codec: WavefieldCodec, blocks, steps=1500, batch=2048, lr=2e-3, lr_final=2e-4, seed=0, log_every=0,
          sample_weights=None):
    """Adam on minibatches of the blocks, learning rate decayed geometrically; returns the loss history.
    sample_weights (one per block) draws minibatches with those relative probabilities, e.g. the
    blocks' amplitudes, so that the normalised loss stands for the error in the field itself."""
    import torch
    gen = torch.Generator(device=blocks.device)
    gen.manual_seed(seed)
    hist = []
    decay = (lr_final / lr) ** (1.0 / max(1, steps - 1))
    for it in range(steps):
        if sample_weights is not None:
            idx = torch.multinomial(sample_weights, batch, replacement=True, generator=gen)
        else:
            idx = torch.randint(0, blocks.shape[0], (batch,), generator=gen, device=blocks.device)
        loss = codec.train_step(blocks[idx].contiguous(), lr * decay ** it)
        hist.append(loss)
        if log_every and it % log_every == 0:
            print(f"codec step {it}: loss {loss:.3e}", flush=True)
    return hist


def propagated_snapshots(shape, physics="iso", seed=0, nt=600, every=20, start=100, d=10.0, dt=0.0005, fpeak=12.0,
                         nsponge=20):
    """Forward wavefields that the propagators themselves generate: a seeded synthetic earth model, a
    Hicks-interpolated Ricker point source at a random position near the surface, and every `every`
    steps after `start` the scaled spatial derivative field (pSpace after ScaleSpatialDerivatives, the
    second time derivative of p that Born imaging saves). Returns device tensors (nx, ny, nz)."""
    import torch

    from . import props, synthetic
    from .abi import SourcePoint32
    from .spacetime import causal_ricker, hickscoeffs
    nx, ny, nz = shape
    cls = {"iso": props.Prop3DAcoIsoDenQ_DEO2_FDTD, "vti": props.Prop3DAcoVTIDenQ_DEO2_FDTD,
           "tti": props.Prop3DAcoTTIDenQ_DEO2_FDTD}[physics]
    p = cls(nz=nz, ny=ny, nx=nx, nsponge=nsponge, dz=d, dy=d, dx=d, dt=dt, freesurface=True)
    model = synthetic.earth_model(shape, physics, seed=seed, d=d, dt=dt, nsponge=nsponge, device="cuda")
    import ctypes as ct
    for k, t in model.items():
        ptr = ct.cast(getattr(p.abi, "get" + k)(p.p), ct.c_void_p).value
        dst = torch.as_tensor(_CAI(ptr, shape), device="cuda")
        dst.copy_(t)
    torch.cuda.synchronize()
    p.prefetch()
    rng = np.random.default_rng(seed)
    sx, sy = rng.uniform(0.3, 0.7, 2)
    src = hickscoeffs(d, d, 0.0, 0.0, nz, nx, [rng.uniform(2.0, 8.0) * d], [sx * nx * d], dy=d, y0=0.0, ny=ny,
                      y=[sy * ny * d])
    lib = _lib.library()
    tab = lib.WFD_Points_Create(src.ctypes.data_as(ct.POINTER(SourcePoint32)), len(src), 0)
    wav = torch.from_numpy(causal_ricker(dt * np.arange(nt), f=fpeak).astype(np.float32)).cuda()
    stream = ct.c_void_p(p.stream())
    out = []
    torch.cuda.synchronize()
    for it in range(1, nt + 1):
        p.step_async(1)
        pc = ct.c_void_p(ct.cast(p.abi.getPCur(p.p), ct.c_void_p).value)
        _check(lib.WFD_Inject(tab, pc, c_void_p(wav.data_ptr()), it, nt, stream), "Inject")
        if it >= start and it % every == 0:
            p.synchronize()
            props.scale_spatial_derivatives(p)
            ptr = ct.cast(p.abi.getPSpace(p.p), ct.c_void_p).value
            out.append(torch.as_tensor(_CAI(ptr, shape), device="cuda").clone())
    p.synchronize()
    lib.WFD_Points_Free(tab)
    props.free(p)
    return out


class _CAI:
    def __init__(self, ptr, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (ptr, False), "version": 3,
                                         "strides": None}


def train_on_propagated(codec: WavefieldCodec, shape=(96, 96, 96), physics=("iso", "vti", "tti"), seeds=(11, 12),
                        nt=700, every=25, npatches=4096, steps=16000, batch=2048, lr=2e-3, log_every=0,
                        weight_power=1.5):
    """Train the codec on wavefields the propagators generate: for each physics and seed a synthetic
    earth model and a randomly placed source (`propagated_snapshots`), then `train` on random 32^3
    patches of all snapshots, drawing blocks with probability proportional to their relative
    amplitude ** weight_power. Returns (loss history, number of training blocks)."""
    snaps = []
    for ph in physics:
        for sd in seeds:
            snaps += propagated_snapshots(shape, ph, seed=sd, nt=nt, every=every)
    blocks, rel = training_blocks(snaps, npatches=npatches, seed=seeds[0], return_scales=True)
    del snaps
    w = rel ** weight_power if weight_power else None
    hist = train(codec, blocks, steps=steps, batch=batch, lr=lr, log_every=log_every, sample_weights=w)
    return hist, int(blocks.shape[0])
