"""Python mirror of WaveFD's Julia propagator API (src/prop{2D,3D}Aco{Iso,VTI,TTI}DenQ_DEO2_FDTD.jl).

Same constructor keywords and defaults, same operations, same argument dictionaries:

    prop = Prop3DAcoIsoDenQ_DEO2_FDTD(nz=..., ny=..., nx=..., dz=10, dy=10, dx=10, dt=0.0005)
    V(prop)[:] = ...; B(prop)[:] = ...
    propagateforward(prop)                      # one time step, pointers swapped inside
    forwardBornInjection(prop, Prop3DAcoIsoDenQ_DEO2_FDTD_Model_V(), {"v": dv}, {"pspace": dp})
    adjointBornAccumulation(prop, Prop3DAcoIsoDenQ_DEO2_FDTD_Model_V(), ImagingConditionStandard(),
                            {"v": img}, {"pspace": dp})
    free(prop)

Getters return numpy views of the library's managed arrays shaped (nx, ny, nz) (3D) or (nx, nz)
(2D), C order -- the same memory as Julia's column-major (nz, ny, nx) view. Julia's `!` suffix is
dropped from function names.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from .abi import PROPAGATORS, PropagatorABI

_f32p = ctypes.POINTER(ctypes.c_float)


class ImagingCondition:
    pass


class ImagingConditionStandard(ImagingCondition):
    pass


class ImagingConditionWaveFieldSeparationFWI(ImagingCondition):
    pass


class ImagingConditionWaveFieldSeparationRTM(ImagingCondition):
    pass


class ImagingConditionWaveFieldSeparationMIX(ImagingCondition):
    pass


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"]:
            raise TypeError("float32 C-contiguous arrays expected")
        return a.ctypes.data_as(_f32p)
    if hasattr(a, "data_ptr"):  # torch tensor on the device
        return ctypes.cast(ctypes.c_void_p(a.data_ptr()), _f32p)
    raise TypeError(f"unsupported array type {type(a)}")


class _Propagator:
    NAME = ""

    def __init__(self, *, nz=0, ny=0, nx=0, nsponge=60, nbz=512, nby=8, nbx=8, dz=5.0, dy=8.0, dx=5.0, dt=0.001,
                 nthreads=None, freesurface=True, freqQ=5.0, qMin=0.1, qInterior=100.0, lib=None):
        ndim = PROPAGATORS[self.NAME][0]
        nthreads = os.cpu_count() if nthreads is None else nthreads
        nz, ny, nx, nsponge, nbz, nby, nbx, nthreads = (int(round(v)) for v in (nz, ny, nx, nsponge, nbz, nby, nbx,
                                                                                 nthreads))
        # the Julia constructors' @asserts (e.g. prop3DAcoIsoDenQ_DEO2_FDTD.jl:25-32)
        assert nx > 0
        if ndim == 3:
            assert ny > 0
        assert nz > 0
        assert nsponge > 0
        assert nthreads > 0
        if ndim == 3:
            assert nbx > 0 and nby > 0 and nbz > 0
        self.abi = PropagatorABI(lib if lib is not None else _lib.library(), self.NAME)
        self.ndim = ndim
        self.physics = PROPAGATORS[self.NAME][1]
        fs = 1 if freesurface else 0
        f32 = np.float32
        if ndim == 3:
            self.p = self.abi.alloc(fs, nthreads, nx, ny, nz, nsponge, f32(dx), f32(dy), f32(dz), f32(dt), nbx, nby, nbz)
        else:
            self.p = self.abi.alloc(fs, nthreads, nx, nz, nsponge, f32(dx), f32(dz), f32(dt), nbx, nbz)
        if not self.p:
            raise _lib.WaveFDError("alloc failed: " + _lib.library().WFD_LastErrorMessage().decode())
        self.abi.SetupDtOmegaInvQ(self.p, f32(freqQ), f32(qMin), f32(qInterior))

    # -- object -------------------------------------------------------------------------------
    def shape(self):
        if self.ndim == 3:
            return (self.abi.getNx(self.p), self.abi.getNy(self.p), self.abi.getNz(self.p))
        return (self.abi.getNx(self.p), self.abi.getNz(self.p))

    def field(self, name):
        ptr = getattr(self.abi, "get" + name)(self.p)
        return np.ctypeslib.as_array(ptr, shape=self.shape())

    def __repr__(self):
        return f"{self.NAME} -- shape (x[,y],z) {self.shape()}"

    # -- add-ons ------------------------------------------------------------------------------
    def set_strict(self, on=True):
        _lib.check(_lib.library().WFD_Prop_SetStrict(self.p, int(bool(on))), "SetStrict", self.p)

    def set_fused(self, on=True):
        _lib.check(_lib.library().WFD_Prop_SetFused(self.p, int(bool(on))), "SetFused", self.p)

    def step_async(self, nsteps=1, linear=False):
        _lib.check(_lib.library().WFD_Prop_TimeStepAsync(self.p, nsteps, int(bool(linear))), "TimeStepAsync", self.p)

    def synchronize(self):
        _lib.check(_lib.library().WFD_Prop_Synchronize(self.p), "Synchronize", self.p)

    def prefetch(self):
        _lib.check(_lib.library().WFD_Prop_Prefetch(self.p), "Prefetch", self.p)

    def stream(self):
        return _lib.library().WFD_Prop_Stream(self.p)

    def status(self):
        return _lib.library().WFD_Prop_Status(self.p)


def _make(name, doc):
    cls = type(name, (_Propagator,), {"NAME": name, "__doc__": doc})
    return cls


Prop2DAcoIsoDenQ_DEO2_FDTD = _make("Prop2DAcoIsoDenQ_DEO2_FDTD", "2D variable-density visco-acoustic isotropic.")
Prop2DAcoVTIDenQ_DEO2_FDTD = _make("Prop2DAcoVTIDenQ_DEO2_FDTD", "2D variable-density visco-acoustic VTI.")
Prop2DAcoTTIDenQ_DEO2_FDTD = _make("Prop2DAcoTTIDenQ_DEO2_FDTD", "2D variable-density visco-acoustic TTI.")
Prop3DAcoIsoDenQ_DEO2_FDTD = _make("Prop3DAcoIsoDenQ_DEO2_FDTD", "3D variable-density visco-acoustic isotropic.")
Prop3DAcoVTIDenQ_DEO2_FDTD = _make("Prop3DAcoVTIDenQ_DEO2_FDTD", "3D variable-density visco-acoustic VTI.")
Prop3DAcoTTIDenQ_DEO2_FDTD = _make("Prop3DAcoTTIDenQ_DEO2_FDTD", "3D variable-density visco-acoustic TTI.")

ALL = [Prop2DAcoIsoDenQ_DEO2_FDTD, Prop2DAcoVTIDenQ_DEO2_FDTD, Prop2DAcoTTIDenQ_DEO2_FDTD,
       Prop3DAcoIsoDenQ_DEO2_FDTD, Prop3DAcoVTIDenQ_DEO2_FDTD, Prop3DAcoTTIDenQ_DEO2_FDTD]

# model-space types (e.g. prop3DAcoIsoDenQ_DEO2_FDTD.jl:63-66, prop3DAcoVTIDenQ_DEO2_FDTD.jl:70-72)
_MODEL_TYPES = {}
for _cls in ALL:
    for _v in PROPAGATORS[_cls.NAME][3]:
        _t = type(f"{_cls.NAME}_Model_{_v}", (), {"variant": _v, "propagator": _cls.NAME})
        globals()[_t.__name__] = _t
        _MODEL_TYPES[_t.__name__] = _t


# -- getters (Julia: V(prop) etc.) --------------------------------------------------------------
def _getter(name):
    def g(prop):
        return prop.field(name)
    g.__name__ = name
    return g


for _n in ("V", "B", "DtOmegaInvQ", "PSpace", "PCur", "POld", "Eps", "Eta", "F", "MSpace", "MCur", "MOld",
           "SinTheta", "CosTheta", "SinPhi", "CosPhi"):
    globals()[_n] = _getter(_n)


def size(prop):
    """(nz[, ny], nx) as in Julia's size(prop)."""
    return tuple(reversed(prop.shape()))


def free(prop):
    if prop.p:
        prop.abi.free(prop.p)
        prop.p = None


def propagateforward(prop):
    prop.abi.TimeStep(prop.p)
    _raise_on_status(prop, "TimeStep")


def propagateforward_linear(prop):
    prop.abi.TimeStepLinear(prop.p)
    _raise_on_status(prop, "TimeStepLinear")


def propagateadjoint(prop):
    # self-adjoint: Iso/TTI use TimeStep, VTI uses TimeStepLinear (prop3DAcoVTIDenQ_DEO2_FDTD.jl:65)
    if prop.physics == "vti":
        propagateforward_linear(prop)
    else:
        propagateforward(prop)


def scale_spatial_derivatives(prop):
    prop.abi.ScaleSpatialDerivatives(prop.p)
    _raise_on_status(prop, "ScaleSpatialDerivatives")


def _raise_on_status(prop, what):
    st = prop.status()
    if st != 0:
        raise _lib.WaveFDError(f"{what} failed: " + _lib.library().WFD_Prop_Message(prop.p).decode())


def forwardBornInjection(prop, modeltype, dmodel, wavefields):
    v = modeltype.variant
    fn = getattr(prop.abi, "ForwardBornInjection_" + v)
    if prop.physics == "iso":
        args = {"V": (dmodel.get("v"), wavefields.get("pspace")),
                "VB": (dmodel.get("v"), dmodel.get("b"), wavefields.get("pold"), wavefields.get("pspace")),
                "B": (dmodel.get("b"), wavefields.get("pold"), wavefields.get("pspace"))}[v]
    elif v == "V":
        args = (dmodel["v"], wavefields["pspace"], wavefields["mspace"])
    else:
        args = (dmodel["v"], dmodel["ϵ"], dmodel["η"], wavefields["pold"], wavefields["mold"], wavefields["pspace"],
                wavefields["mspace"])
    fn(prop.p, *[_ptr(a) for a in args])
    _raise_on_status(prop, "ForwardBornInjection")


def adjointBornAccumulation(prop, modeltype, imagingcondition, dmodel, wavefields):
    v = modeltype.variant
    if isinstance(imagingcondition, ImagingConditionWaveFieldSeparationMIX):
        # Standard into the "all_*" images, RTM separation into "rtm_*" (prop3DAcoIsoDenQ_DEO2_FDTD.jl:131-150)
        keys = {"V": ("v",), "VB": ("v", "b"), "B": ("b",), "VEA": ("v", "ϵ", "η")}[v]
        adjointBornAccumulation(prop, modeltype, ImagingConditionStandard(), {k: dmodel["all_" + k] for k in keys},
                                wavefields)
        adjointBornAccumulation(prop, modeltype, ImagingConditionWaveFieldSeparationRTM(),
                                {k: dmodel["rtm_" + k] for k in keys}, wavefields)
        return
    if not isinstance(imagingcondition, ImagingConditionStandard):
        if v != "V":
            raise TypeError("wavefield separation is defined for the velocity-only model space")
        isfwi = 1 if isinstance(imagingcondition, ImagingConditionWaveFieldSeparationFWI) else 0
        if prop.physics == "iso":
            prop.abi.AdjointBornAccumulation_wavefieldsep(prop.p, _ptr(dmodel["v"]), _ptr(wavefields["pspace"]), isfwi)
        else:
            prop.abi.AdjointBornAccumulation_wavefieldsep_V(prop.p, _ptr(dmodel["v"]), _ptr(wavefields["pspace"]),
                                                            _ptr(wavefields["mspace"]), isfwi)
        _raise_on_status(prop, "AdjointBornAccumulation")
        return
    fn = getattr(prop.abi, "AdjointBornAccumulation_" + v)
    if prop.physics == "iso":
        args = {"V": (dmodel.get("v"), wavefields.get("pspace")),
                "VB": (dmodel.get("v"), dmodel.get("b"), wavefields.get("pold"), wavefields.get("pspace")),
                "B": (dmodel.get("b"), wavefields.get("pold"), wavefields.get("pspace"))}[v]
    elif v == "V":
        args = (dmodel["v"], wavefields["pspace"], wavefields["mspace"])
    else:
        args = (dmodel["v"], dmodel["ϵ"], dmodel["η"], wavefields["pold"], wavefields["mold"], wavefields["pspace"],
                wavefields["mspace"])
    fn(prop.p, *[_ptr(a) for a in args])
    _raise_on_status(prop, "AdjointBornAccumulation")
