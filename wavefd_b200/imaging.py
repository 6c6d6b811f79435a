"""Born (linearised) imaging of one shot on the GPU, with the saved forward wavefield kept either in
the learned codec's compressed form or uncompressed.

This is the reference's workflow around the propagators (JetPackWaveFD drives WaveFD this way, and
src/compressedio.jl:1-137 is its snapshot store): a forward run from the source saves the scaled
spatial-derivative fields (pSpace, mSpace after ScaleSpatialDerivatives) every `every` steps; an
adjoint run from the receivers back-propagates the recorded data and, at each saved step,
accumulates the standard imaging condition (AdjointBornAccumulation_V) with the saved fields. Both are
fused into the step kernels: the forward steps that save a snapshot write pSpace/mSpace already
scaled (WFD_Prop_TimeStepScaled), and the adjoint steps at saved time indices accumulate the image
as they step (WFD_Prop_TimeStepImage).

Snapshot stores:
  CodecStore   -- the learned codec (wfd_codec.cu), codes resident in device memory;
  HostStore    -- uncompressed FP32 in pinned host memory, copies overlapped with the propagation
                  (device staging ring + a copy stream, prefetch one snapshot ahead); the store for
                  shots whose saved fields do not fit in device memory;
  DeviceStore  -- uncompressed FP32 in device memory (exact reference for small shots);
  DiskStore    -- uncompressed FP32 in a snapshot file on disk (wavefd_b200/snapio.py: offsets/
                  lengths index, staging and a worker thread in the library), the fallback when
                  the saved fields fit neither in device nor in host memory.
"""
from __future__ import annotations

import ctypes as ct
import time

import numpy as np

from . import _lib, props, synthetic
from .abi import SourcePoint32
from .codec import _CAI

_CLASSES = {"iso": props.Prop3DAcoIsoDenQ_DEO2_FDTD, "vti": props.Prop3DAcoVTIDenQ_DEO2_FDTD,
            "tti": props.Prop3DAcoTTIDenQ_DEO2_FDTD}


def _field(prop, name, shape):
    import torch
    ptr = ct.cast(getattr(prop.abi, "get" + name)(prop.p), ct.c_void_p).value
    return torch.as_tensor(_CAI(ptr, shape), device="cuda")


class _PCur:
    """pCur of an object across its pointer swaps, without a getter call per step (a getter marks the
    object's managed arrays as touched by the host, which makes the next drop-in call move them)."""

    def __init__(self, prop):
        self.a = ct.cast(prop.abi.getPCur(prop.p), ct.c_void_p).value
        self.b = ct.cast(prop.abi.getPOld(prop.p), ct.c_void_p).value
        self.n = 0

    def step(self):
        self.n += 1
        return ct.c_void_p(self.b if self.n & 1 else self.a)


class DeviceStore:
    def __init__(self, shape, nsnap, nfields):
        import torch
        self.buf = torch.empty((nsnap, nfields) + tuple(shape), device="cuda")

    def put(self, k, fields, stream):
        import torch
        with torch.cuda.stream(stream):  # behind the step that wrote the fields
            for i, f in enumerate(fields):
                self.buf[k, i].copy_(f, non_blocking=True)

    def get(self, k, stream):
        return [self.buf[k, i] for i in range(self.buf.shape[1])]

    def nbytes(self):
        return self.buf.numel() * 4


class CodecStore:
    def __init__(self, codec, shape, nsnap, nfields):
        import torch
        self.codec, self.shape = codec, tuple(shape)
        nb = codec.code_bytes(shape)
        self.codes = torch.empty((nsnap, nfields, nb), dtype=torch.uint8, device="cuda")
        self.out = [torch.empty(self.shape, device="cuda") for _ in range(nfields)]

    def put(self, k, fields, stream):
        for i, f in enumerate(fields):
            self.codec.encode(f, self.shape, self.codes[k, i], stream)

    def get(self, k, stream):
        for i in range(len(self.out)):
            self.codec.decode(self.codes[k, i], self.shape, self.out[i], stream)
        return self.out

    def nbytes(self):
        return self.codes.numel()

    def raw_blocks(self, k, i=0):
        return self.codec.raw_blocks(self.codes[k, i], self.shape)


class HostStore:
    """Pinned host snapshots. A put copies the fields into a device staging slot on the propagation
    stream (so the next time step may overwrite pSpace) and then to the host on a copy stream; a get
    (the adjoint asks for snapshots in decreasing order) waits for its slot and starts the host-to-
    device copy of the next one, so the copies overlap the propagation both ways."""

    def __init__(self, shape, nsnap, nfields, ring=2):
        import torch
        self.shape, self.nf, self.ring = tuple(shape), nfields, ring
        self.host = torch.empty((nsnap, nfields) + self.shape, pin_memory=True)
        self.stage = torch.empty((ring, nfields) + self.shape, device="cuda")
        self.copy = torch.cuda.Stream()
        self.free_ev = [None] * ring   # the slot's last reader or copy is done after this event
        self.ready_ev = [None] * ring  # the slot holds snapshot slot_k after this event
        self.slot_k = [None] * ring

    def put(self, k, fields, stream):
        import torch
        s = k % self.ring
        if self.free_ev[s] is not None:
            stream.wait_event(self.free_ev[s])
        with torch.cuda.stream(stream):
            for i, f in enumerate(fields):
                self.stage[s, i].copy_(f, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(stream)
        self.copy.wait_event(ev)
        with torch.cuda.stream(self.copy):
            self.host[k].copy_(self.stage[s], non_blocking=True)
        fe = torch.cuda.Event()
        fe.record(self.copy)
        self.free_ev[s] = fe
        self.slot_k[s] = None

    def _fetch(self, k):
        import torch
        s = k % self.ring
        if self.free_ev[s] is not None:
            self.copy.wait_event(self.free_ev[s])
        with torch.cuda.stream(self.copy):
            self.stage[s].copy_(self.host[k], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(self.copy)
        self.ready_ev[s] = ev
        self.slot_k[s] = k

    def get(self, k, stream):
        s = k % self.ring
        if self.slot_k[s] != k:
            self._fetch(k)
        stream.wait_event(self.ready_ev[s])
        if k - 1 >= 0 and self.slot_k[(k - 1) % self.ring] != k - 1:
            self._fetch(k - 1)
        return [self.stage[s, i] for i in range(self.nf)]

    def release(self, k, stream):
        import torch
        ev = torch.cuda.Event()
        ev.record(stream)
        self.free_ev[k % self.ring] = ev

    def nbytes(self):
        return self.host.numel() * 4


class DiskStore:
    """Uncompressed snapshots in a snapshot file: field i of snapshot k is file field k * nfields + i.
    A put writes (device staging on the propagation stream, so the next step may overwrite pSpace;
    the disk write runs behind it); a get reads snapshot k into the store's device arrays on the
    adjoint stream and starts reading snapshot k - 1 (the adjoint asks in decreasing order)."""

    def __init__(self, shape, nsnap, nfields, path, direct=False, keep=False):
        import torch
        from .snapio import SnapshotFile
        self.shape, self.nf, self.path, self.keep = tuple(shape), nfields, str(path), keep
        self.field_bytes = int(np.prod(self.shape)) * 4
        self.file = SnapshotFile(self.path, "w", nsnap * nfields, self.field_bytes, direct=direct)
        self.out = [torch.empty(self.shape, device="cuda") for _ in range(nfields)]
        self.nsnap = nsnap

    def put(self, k, fields, stream):
        for i, f in enumerate(fields):
            self.file.write(k * self.nf + i, f, stream)

    def get(self, k, stream):
        for i in range(self.nf):
            self.file.read(k * self.nf + i, self.out[i], stream)
        if k - 1 >= 0:
            for i in range(self.nf):
                self.file.prefetch((k - 1) * self.nf + i)
        return self.out

    def nbytes(self):
        return self.nsnap * self.nf * self.field_bytes

    def close(self):
        import os
        self.file.close()
        if not self.keep and os.path.exists(self.path):
            os.remove(self.path)


def make_shot(physics, shape, seed=0, d=10.0, dt=0.0005, nsponge=40, fpeak=12.0, nt=1000, nrec=(32, 32),
              perturbation=True, horizons=(0.15, 0.9)):
    """Seeded shot: the earth model (device tensors), a Hicks source at the centre near the surface, a
    surface receiver grid, the causal Ricker wavelet, and the Born velocity perturbation (+-2 % on 20
    horizons between the given fractions of the depth, sparse) used as the reflectivity of the data."""
    import torch
    from .spacetime import causal_ricker
    model = synthetic.earth_model(shape, physics, seed=seed, d=d, dt=dt, nsponge=nsponge, device="cuda")
    src = synthetic.center_source(shape, d)
    rec = synthetic.surface_receivers(shape, nrec[0], nrec[1], min(nsponge, shape[0] // 4))
    wav = torch.from_numpy(causal_ricker(dt * np.arange(nt), f=fpeak).astype(np.float32)).cuda()
    dv = None
    if perturbation:
        nx, ny, nz = shape
        rng = np.random.default_rng(seed + 1000)
        dv = torch.zeros(shape, device="cuda")
        for z in np.linspace(nz * horizons[0], nz * horizons[1], 20).astype(int):
            mask = torch.from_numpy((rng.random((nx, ny)) < 0.1).astype(np.float32)).cuda()
            dv[:, :, z] = mask * model["V"][:, :, z] * float(rng.choice([-0.02, 0.02]))
    return dict(model=model, src=src, rec=rec, wavelet=wav, dv=dv, shape=tuple(shape), d=d, dt=dt, nsponge=nsponge,
                nt=nt, physics=physics)


def _new_prop(shot):
    nx, ny, nz = shot["shape"]
    d = shot["d"]
    p = _CLASSES[shot["physics"]](nz=nz, ny=ny, nx=nx, nsponge=shot["nsponge"], dz=d, dy=d, dx=d, dt=shot["dt"],
                                  freesurface=True)
    for k, t in shot["model"].items():
        _field(p, k, shot["shape"]).copy_(t)
    return p


def born_data(shot):
    """Linearised (Born) data of the shot's velocity perturbation at the receivers: the background
    wavefield's scaled derivative field drives ForwardBornInjection_V into a second propagator."""
    import torch
    shape, nt = shot["shape"], shot["nt"]
    lib = _lib.library()
    p0, p1 = _new_prop(shot), _new_prop(shot)
    torch.cuda.synchronize()
    p0.prefetch()
    p1.prefetch()
    tsrc = lib.WFD_Points_Create(shot["src"].ctypes.data_as(ct.POINTER(SourcePoint32)), len(shot["src"]), 0)
    trec = lib.WFD_Points_Create(shot["rec"].ctypes.data_as(ct.POINTER(SourcePoint32)), len(shot["rec"]), 1)
    data = torch.zeros(len(shot["rec"]) * nt, device="cuda")
    mtype = getattr(props, p1.NAME + "_Model_V")()
    wf = {"pspace": _field(p0, "PSpace", shape)}
    if shot["physics"] != "iso":
        wf["mspace"] = _field(p0, "MSpace", shape)
    c0, c1 = _PCur(p0), _PCur(p1)
    for it in range(1, nt + 1):
        p0.step_async(1)
        _lib.check(lib.WFD_Inject(tsrc, c0.step(), ct.c_void_p(shot["wavelet"].data_ptr()), it, nt,
                                  ct.c_void_p(p0.stream())), "inject")
        p0.synchronize()
        props.scale_spatial_derivatives(p0)
        props.propagateforward(p1)
        props.forwardBornInjection(p1, mtype, {"v": shot["dv"]}, wf)
        _lib.check(lib.WFD_Extract(trec, ct.c_void_p(data.data_ptr()), c1.step(), it, nt, ct.c_void_p(p1.stream())),
                   "extract")
        p1.synchronize()
    lib.WFD_Points_Free(tsrc)
    lib.WFD_Points_Free(trec)
    props.free(p0)
    props.free(p1)
    return data


def born_image(shot, data, store, every=4, nt=None):
    """Adjoint Born image of the shot's data with the forward fields kept in `store`; returns
    (image, seconds) with the forward and the adjoint run each timed on the device."""
    import torch
    shape = shot["shape"]
    nt = nt or shot["nt"]
    lib = _lib.library()
    aniso = shot["physics"] != "iso"
    fwd, adj = _new_prop(shot), _new_prop(shot)
    torch.cuda.synchronize()
    fwd.prefetch()
    adj.prefetch()
    tsrc = lib.WFD_Points_Create(shot["src"].ctypes.data_as(ct.POINTER(SourcePoint32)), len(shot["src"]), 0)
    tadj = lib.WFD_Points_Create(shot["rec"].ctypes.data_as(ct.POINTER(SourcePoint32)), len(shot["rec"]), 0)
    image = torch.zeros(shape, device="cuda")
    fs = torch.cuda.ExternalStream(fwd.stream())
    as_ = torch.cuda.ExternalStream(adj.stream())
    f_space = [_field(fwd, "PSpace", shape)] + ([_field(fwd, "MSpace", shape)] if aniso else [])
    fcur, acur = _PCur(fwd), _PCur(adj)
    props.scale_spatial_derivatives(adj)  # the device call after the getters (moves the arrays once)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    linear = shot["physics"] == "vti"
    fp, ap = ct.c_void_p(fwd.p), ct.c_void_p(adj.p)
    for it in range(1, nt + 1):
        if it % every == 0:
            # TimeStep with ScaleSpatialDerivatives fused into the step kernel (3D)
            _lib.check(lib.WFD_Prop_TimeStepScaled(fp), "scaled step", fwd.p)
        else:
            fwd.step_async(1)
        _lib.check(lib.WFD_Inject(tsrc, fcur.step(), ct.c_void_p(shot["wavelet"].data_ptr()), it, shot["nt"],
                                  ct.c_void_p(fwd.stream())), "inject")
        if it % every == 0:
            store.put(it // every - 1, f_space, fs)
    fwd.synchronize()
    for it in range(nt, 0, -1):
        # self-adjoint steps: TimeStep (Iso, TTI), TimeStepLinear (VTI), as propagateadjoint does; at a
        # saved step the imaging condition (AdjointBornAccumulation_V, which reads the step's input
        # fields) is fused into the step kernel
        if it % every == 0:
            k = it // every - 1
            f = store.get(k, as_)
            dm = ct.c_void_p(f[1].data_ptr()) if aniso else None
            _lib.check(lib.WFD_Prop_TimeStepImage(ap, ct.c_void_p(image.data_ptr()), ct.c_void_p(f[0].data_ptr()),
                                                  dm, int(linear)), "imaging step", adj.p)
            if hasattr(store, "release"):
                store.release(k, as_)
        else:
            adj.step_async(1, linear=linear)
        _lib.check(lib.WFD_Inject(tadj, acur.step(), ct.c_void_p(data.data_ptr()), it, shot["nt"],
                                  ct.c_void_p(adj.stream())), "inject adjoint")
    adj.synchronize()
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    lib.WFD_Points_Free(tsrc)
    lib.WFD_Points_Free(tadj)
    props.free(fwd)
    props.free(adj)
    return image, secs


class _StateArrays:
    """The two pressure arrays (and two m arrays) of an object, fixed across its pointer swaps, and the
    object's step count: after n steps pCur is the second array when n is odd, else the first."""

    def __init__(self, prop, shape, aniso):
        names = [("PCur", "POld")] + ([("MCur", "MOld")] if aniso else [])
        self.pairs = [(_field(prop, a, shape), _field(prop, b, shape)) for a, b in names]
        self.n = 0

    def save(self):
        return [(a.clone(), b.clone()) for a, b in self.pairs], self.n

    def restore(self, saved, stream):
        """Set the object to the saved state (its pCur/pOld/mCur/mOld values), whatever the parity of
        the steps taken since: the arrays are exchanged when the parities differ."""
        import torch
        arrays, n = saved
        swap = (self.n - n) & 1
        with torch.cuda.stream(stream):
            for (a, b), (sa, sb) in zip(self.pairs, arrays):
                a.copy_(sb if swap else sa, non_blocking=True)
                b.copy_(sa if swap else sb, non_blocking=True)


def born_image_checkpointed(shot, data, every=4, seg=200, nt=None, learned=None):
    """Adjoint Born image with exact FP32 forward fields held on the device by recomputation: the
    forward run keeps the full state (pCur, pOld, mCur, mOld) every `seg` steps; the adjoint run goes
    through the record segment by segment from the end, recomputing each segment's forward fields
    from its checkpoint into device memory (seg / every snapshots) before back-propagating over it.
    One forward pass more than storing every snapshot, for seg / every snapshots of memory instead
    of nt / every. Returns (image, seconds, learned image or None): with a snapshot store `learned`
    (filled during the same forward run) the adjoint run also accumulates the image of the learned
    fields, through the same adjoint wavefield, so that the two images differ only by the stored
    fields (the timing then includes that second imaging condition)."""
    import torch
    shape = shot["shape"]
    nt = nt or shot["nt"]
    lib = _lib.library()
    aniso = shot["physics"] != "iso"
    linear = shot["physics"] == "vti"
    fwd, rec, adj = _new_prop(shot), _new_prop(shot), _new_prop(shot)
    torch.cuda.synchronize()
    for p in (fwd, rec, adj):
        p.prefetch()
    tsrc = lib.WFD_Points_Create(shot["src"].ctypes.data_as(ct.POINTER(SourcePoint32)), len(shot["src"]), 0)
    tadj = lib.WFD_Points_Create(shot["rec"].ctypes.data_as(ct.POINTER(SourcePoint32)), len(shot["rec"]), 0)
    image = torch.zeros(shape, device="cuda")
    image_l = torch.zeros(shape, device="cuda") if learned is not None else None
    fs, rs, as_ = (torch.cuda.ExternalStream(p.stream()) for p in (fwd, rec, adj))
    f_space = [_field(fwd, "PSpace", shape)] + ([_field(fwd, "MSpace", shape)] if aniso else [])
    r_space = [_field(rec, "PSpace", shape)] + ([_field(rec, "MSpace", shape)] if aniso else [])
    fstate, rstate = _StateArrays(fwd, shape, aniso), _StateArrays(rec, shape, aniso)
    fcur, rcur, acur = _PCur(fwd), _PCur(rec), _PCur(adj)
    props.scale_spatial_derivatives(adj)
    mtype = getattr(props, adj.NAME + "_Model_V")()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    fp, rp, ap = ct.c_void_p(fwd.p), ct.c_void_p(rec.p), ct.c_void_p(adj.p)
    wav = ct.c_void_p(shot["wavelet"].data_ptr())

    def fstep(p, pp, cur, state, it):
        """forward step `it` of object p with the source injection (the scaled step at saved steps)"""
        if it % every == 0:
            _lib.check(lib.WFD_Prop_TimeStepScaled(pp), "scaled step", p.p)
        else:
            p.step_async(1)
        state.n += 1
        _lib.check(lib.WFD_Inject(tsrc, cur.step(), wav, it, shot["nt"], ct.c_void_p(p.stream())), "inject")

    # forward: checkpoints every seg steps (the state after step k * seg), learned snapshots if any
    nseg = (nt + seg - 1) // seg
    checkpoints = []
    for it in range(1, nt + 1):
        if (it - 1) % seg == 0:
            with torch.cuda.stream(fs):
                checkpoints.append(fstate.save())
        fstep(fwd, fp, fcur, fstate, it)
        if learned is not None and it % every == 0:
            learned.put(it // every - 1, f_space, fs)
    fwd.synchronize()
    snaps = {}
    for s in range(nseg - 1, -1, -1):
        lo, hi = s * seg + 1, min((s + 1) * seg, nt)
        # recompute the segment's forward fields from its checkpoint
        rstate.restore(checkpoints[s], rs)
        snaps.clear()
        for it in range(lo, hi + 1):
            fstep(rec, rp, rcur, rstate, it)
            if it % every == 0:
                with torch.cuda.stream(rs):
                    snaps[it // every - 1] = [t.clone() for t in r_space]
        rec.synchronize()
        for it in range(hi, lo - 1, -1):
            if it % every == 0:
                k = it // every - 1
                e = snaps[k]
                dm = ct.c_void_p(e[1].data_ptr()) if aniso else None
                _lib.check(lib.WFD_Prop_TimeStepImage(ap, ct.c_void_p(image.data_ptr()), ct.c_void_p(e[0].data_ptr()),
                                                      dm, int(linear)), "imaging step", adj.p)
                if learned is not None:
                    f = learned.get(k, as_)
                    wf = {"pspace": f[0]}
                    if aniso:
                        wf["mspace"] = f[1]
                    adj.synchronize()
                    props.adjointBornAccumulation(adj, mtype, props.ImagingConditionStandard(), {"v": image_l}, wf)
            else:
                adj.step_async(1, linear=linear)
            _lib.check(lib.WFD_Inject(tadj, acur.step(), ct.c_void_p(data.data_ptr()), it, shot["nt"],
                                      ct.c_void_p(adj.stream())), "inject adjoint")
        adj.synchronize()
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    snaps.clear()
    del checkpoints
    lib.WFD_Points_Free(tsrc)
    lib.WFD_Points_Free(tadj)
    for p in (fwd, rec, adj):
        props.free(p)
    return image, secs, image_l
