"""Batched shots: many 3D propagator objects advanced together on one GPU.

The reference has no batching: `Ginsu` is exported (src/WaveFD.jl:52) but not defined, and its tile
knobs (nbx, nby, nbz; tilesize(), src/prop3DAcoIsoDenQ_DEO2_FDTD.jl:159-185) are per object. Here a
`ShotBatch` takes objects made by the usual constructors (uneven sizes; Iso, VTI and TTI mixed) and
advances all of them with one persistent launch per physics class per time step; the time loop
(steps, source injection, receiver extraction) is a CUDA graph of two steps replayed. Every
object's arrays end bitwise equal to stepping it alone, and its getters stay valid.

    batch = ShotBatch([prop_a, prop_b, ...])
    batch.set_acquisition(0, src_points, wavelet, rec_points, traces, nt)   # device arrays
    batch.tune()                    # pick x-chunk length, item order and launch mode by timing
    batch.run(nt, it0=1)            # all shots, all steps
    batch.synchronize()

`ginsu_crop` / `ginsu_accumulate` cut a shot window out of a survey array and add a shot image back.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_int, c_long, c_void_p

import numpy as np

from . import _lib
from .abi import SourcePoint32

_declared = False


def _L():
    global _declared
    lib = _lib.library()
    if not _declared:
        def fn(name, restype, argtypes):
            f = getattr(lib, name)
            f.restype = restype
            f.argtypes = argtypes
        fn("WFD_Batch_Create", c_void_p, [POINTER(c_void_p), c_long])
        fn("WFD_Batch_Free", None, [c_void_p])
        fn("WFD_Batch_Status", c_int, [c_void_p])
        fn("WFD_Batch_Message", ctypes.c_char_p, [c_void_p])
        fn("WFD_Batch_SetAcquisition", c_int, [c_void_p, c_long, POINTER(SourcePoint32), c_long, c_void_p,
                                               POINTER(SourcePoint32), c_long, c_void_p, c_long])
        fn("WFD_Batch_Plan", c_int, [c_void_p, c_long, c_int, c_int])
        fn("WFD_Batch_Tune", c_int, [c_void_p, c_int])
        fn("WFD_Batch_Run", c_int, [c_void_p, c_long, c_long, c_int])
        fn("WFD_Batch_Synchronize", c_int, [c_void_p])
        fn("WFD_Batch_Stream", c_void_p, [c_void_p])
        fn("WFD_Batch_Info", c_int, [c_void_p, POINTER(c_long), c_long])
        fn("WFD_Ginsu_Crop", c_int, [c_void_p, c_long, c_long, c_long, c_long, c_long, c_long, c_void_p, c_long,
                                     c_long, c_long, c_void_p])
        fn("WFD_Ginsu_Accumulate", c_int, [c_void_p, c_long, c_long, c_long, c_long, c_long, c_long, c_void_p,
                                           c_long, c_long, c_long, c_void_p])
        _declared = True
    return lib


def _addr(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        if hasattr(a, "is_contiguous") and not a.is_contiguous():
            raise ValueError("the C ABI takes contiguous arrays (call .contiguous())")
        return c_void_p(a.data_ptr())
    if isinstance(a, int):
        return c_void_p(a)
    raise TypeError("device arrays (torch tensors) or raw device addresses expected")


def _points(pts):
    if pts is None or len(pts) == 0:
        return None, 0
    arr = np.ascontiguousarray(pts)
    return arr.ctypes.data_as(POINTER(SourcePoint32)), len(arr), arr


class ShotBatch:
    """Advance many propagator objects (wavefd_b200.props classes) together."""

    def __init__(self, props):
        lib = _L()
        self.props = list(props)
        handles = (c_void_p * len(self.props))(*[p.p for p in self.props])
        self.b = lib.WFD_Batch_Create(handles, len(self.props))
        if not self.b:
            raise _lib.WaveFDError(f"WFD_Batch_Create failed: {lib.WFD_LastErrorMessage().decode()}")
        self._keep = {}

    def _check(self, rc, what):
        if rc != 0:
            msg = _L().WFD_Batch_Message(self.b).decode()
            raise _lib.WaveFDError(f"{what} failed (status {rc}): {msg}")

    def set_acquisition(self, shot, src_points, wavelet, rec_points, traces, nt):
        """Sources (SourcePoint32 array, ir into the wavelet's columns) and receivers of one shot;
        wavelet and traces are device tensors, column-major (nt, ntraces) i.e. torch shape (ntraces, nt)."""
        s = _points(src_points)
        r = _points(rec_points)
        rc = _L().WFD_Batch_SetAcquisition(self.b, shot, s[0], s[1], _addr(wavelet), r[0], r[1], _addr(traces), nt)
        self._keep[shot] = (wavelet, traces)
        self._check(rc, "set_acquisition")

    def plan(self, xchunk_target=128, order=0, concurrent=True):
        self._check(_L().WFD_Batch_Plan(self.b, xchunk_target, order, 1 if concurrent else 0), "plan")

    def tune(self, reps=2):
        self._check(_L().WFD_Batch_Tune(self.b, reps), "tune")

    def run(self, nsteps, it0=1, graph=True):
        self._check(_L().WFD_Batch_Run(self.b, nsteps, it0, 1 if graph else 0), "run")

    def synchronize(self):
        self._check(_L().WFD_Batch_Synchronize(self.b), "synchronize")

    def stream(self):
        return _L().WFD_Batch_Stream(self.b)

    def info(self):
        a = (c_long * 16)()
        self._check(_L().WFD_Batch_Info(self.b, a, 16), "info")
        v = list(a)
        classes = {}
        for i, name in enumerate(("iso", "vti", "tti")):
            classes[name] = dict(shots=v[4 * i], items=v[4 * i + 1], ctas=v[4 * i + 2], xchunk_target=v[4 * i + 3],
                                 order=(v[13] >> i) & 1)
        return dict(classes=classes, concurrent=v[12] == 0, kernels_per_step=v[14], tuned=bool(v[15]))

    def free(self):
        if self.b:
            _L().WFD_Batch_Free(self.b)
            self.b = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def ginsu_crop(survey, survey_shape, origin, shot, shot_shape, stream=None):
    """shot[x,y,z] = survey[x0+x, y0+y, z0+z] (indices clamped to the survey); shapes (nx, ny, nz)."""
    snx, sny, snz = survey_shape
    x0, y0, z0 = origin
    nx, ny, nz = shot_shape
    rc = _L().WFD_Ginsu_Crop(_addr(survey), snx, sny, snz, x0, y0, z0, _addr(shot), nx, ny, nz, stream)
    if rc:
        raise _lib.WaveFDError(f"ginsu_crop failed (status {rc})")


def ginsu_accumulate(survey, survey_shape, origin, shot, shot_shape, stream=None):
    """survey[x0+x, y0+y, z0+z] += shot[x,y,z] where inside the survey."""
    snx, sny, snz = survey_shape
    x0, y0, z0 = origin
    nx, ny, nz = shot_shape
    rc = _L().WFD_Ginsu_Accumulate(_addr(survey), snx, sny, snz, x0, y0, z0, _addr(shot), nx, ny, nz, stream)
    if rc:
        raise _lib.WaveFDError(f"ginsu_accumulate failed (status {rc})")
