"""Loader of the CUDA library (wavefd_b200/lib/libwavefd_b200.so).

There is no CPU fallback: if the library is missing, importing the propagators raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_int, c_long, c_void_p

from .abi import SourcePoint32

HERE = os.path.dirname(os.path.abspath(__file__))
# WAVEFD_B200_LIB selects another build of the same library (e.g. a tuning variant)
LIB_PATH = os.environ.get("WAVEFD_B200_LIB") or os.path.join(HERE, "lib", "libwavefd_b200.so")

_lib = None


class WaveFDError(RuntimeError):
    pass


def library() -> ctypes.CDLL:
    """The loaded CUDA library; raises WaveFDError if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise WaveFDError(f"CUDA library not built: {LIB_PATH} (run python -m wavefd_b200.build)")
        lib = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_LOCAL)
        _declare(lib)
        _lib = lib
    return _lib


def _declare(lib):
    def fn(name, restype, argtypes):
        f = getattr(lib, name)
        f.restype = restype
        f.argtypes = argtypes

    fn("WFD_LastError", c_int, [])
    fn("WFD_LastErrorMessage", ctypes.c_char_p, [])
    fn("WFD_Prop_Status", c_int, [c_void_p])
    fn("WFD_Prop_Message", ctypes.c_char_p, [c_void_p])
    fn("WFD_Prop_SetStrict", c_int, [c_void_p, c_int])
    fn("WFD_Prop_SetFused", c_int, [c_void_p, c_int])
    fn("WFD_Prop_TimeStepAsync", c_int, [c_void_p, c_long, c_int])
    fn("WFD_Prop_Synchronize", c_int, [c_void_p])
    fn("WFD_Prop_Prefetch", c_int, [c_void_p])
    fn("WFD_Prop_Stream", c_void_p, [c_void_p])
    fn("WFD_Prop_StepKernels", c_int, [c_void_p])
    fn("WFD_Prop_RunLaunches", c_long, [c_void_p])
    fn("WFD_Prop_TimeStepBorn", c_int, [c_void_p, c_void_p, c_void_p, c_void_p])
    fn("WFD_Prop_TimeStepImage", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int])
    fn("WFD_Prop_TimeStepScaled", c_int, [c_void_p])
    fn("WFD_Debug_SetPipelineWait", c_int, [ctypes.c_ulonglong])
    fn("WFD_Points_Create", c_void_p, [POINTER(SourcePoint32), c_long, c_int])
    fn("WFD_Points_Free", None, [c_void_p])
    fn("WFD_Points_Groups", c_long, [c_void_p])
    fn("WFD_Inject", c_int, [c_void_p, c_void_p, c_void_p, c_long, c_long, c_void_p])
    fn("WFD_Extract", c_int, [c_void_p, c_void_p, c_void_p, c_long, c_long, c_void_p])
    fn("WFD_Prop_SetIllumination", c_int, [c_void_p, c_void_p])
    fn("WFD_Prop_Run", c_int, [c_void_p, c_long, c_long, c_void_p, c_void_p, c_void_p, c_void_p, c_long, c_int])
    fn("WFD_IllumAccumulate", c_int, [c_void_p, c_void_p, c_long, c_void_p])
    fn("WFD_Snap_Open", c_void_p, [ctypes.c_char_p, c_long, c_long, c_int])
    fn("WFD_Snap_Write", c_int, [c_void_p, c_long, c_void_p, c_long, c_void_p])
    fn("WFD_Snap_Prefetch", c_int, [c_void_p, c_long])
    fn("WFD_Snap_Read", c_int, [c_void_p, c_long, c_void_p, c_long, c_void_p])
    fn("WFD_Snap_Length", c_long, [c_void_p, c_long])
    fn("WFD_Snap_NumFields", c_long, [c_void_p])
    fn("WFD_Snap_Flags", c_int, [c_void_p])
    fn("WFD_Snap_Sync", c_int, [c_void_p])
    fn("WFD_Snap_Close", c_int, [c_void_p])
    fn("WFD_Interp", c_int, [c_int, c_void_p, c_void_p, c_void_p, c_long, c_long, c_long, c_long, c_void_p])
    fn("WFD_ExtractInterp", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_long, c_long, c_long, c_long,
                                     c_void_p])


def check(status: int, what: str = "call", obj=None):
    if status != 0:
        lib = library()
        msg = lib.WFD_Prop_Message(obj).decode() if obj else lib.WFD_LastErrorMessage().decode()
        raise WaveFDError(f"{what} failed (status {status}): {msg}")
