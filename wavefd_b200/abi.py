"""ctypes description of WaveFD's propagator C ABI (the boundary this package sits behind).

The table below restates the `extern "C"` surface of the reference shared libraries
(src/prop{2D,3D}Aco{Iso,VTI,TTI}DenQ_DEO2_FDTD.cc and src/spacetime.cc:144-204) as the
Julia `ccall` sites bind it (e.g. src/prop3DAcoIsoDenQ_DEO2_FDTD.jl:36-128). The same
binding drives any library exporting those names: the CUDA build of this package, or a
CPU build of the reference used as a checker.
"""
from __future__ import annotations

import ctypes
from ctypes import POINTER, c_float, c_long, c_size_t, c_void_p

_f32p = POINTER(c_float)

# name -> (ndim, physics, getters, born variants, imaging variants, has TimeStepLinear)
PROPAGATORS = {
    "Prop2DAcoIsoDenQ_DEO2_FDTD": (2, "iso", ("V", "B", "DtOmegaInvQ", "PSpace", "PCur", "POld"),
                                   ("V", "VB", "B"), ("V", "VB", "B", "wavefieldsep"), False),
    "Prop3DAcoIsoDenQ_DEO2_FDTD": (3, "iso", ("V", "B", "DtOmegaInvQ", "PSpace", "PCur", "POld"),
                                   ("V", "VB", "B"), ("V", "VB", "B", "wavefieldsep"), False),
    "Prop2DAcoVTIDenQ_DEO2_FDTD": (2, "vti", ("V", "Eps", "Eta", "B", "F", "DtOmegaInvQ", "PSpace", "MSpace",
                                              "PCur", "POld", "MCur", "MOld"),
                                   ("V", "VEA"), ("V", "wavefieldsep_V", "VEA"), True),
    # the reference's 3D VTI library exports no DtOmegaInvQ getter (prop3DAcoVTIDenQ_DEO2_FDTD.cc:94-157)
    "Prop3DAcoVTIDenQ_DEO2_FDTD": (3, "vti", ("V", "Eps", "Eta", "B", "F", "PSpace", "MSpace",
                                              "PCur", "POld", "MCur", "MOld"),
                                   ("V", "VEA"), ("V", "wavefieldsep_V", "VEA"), True),
    "Prop2DAcoTTIDenQ_DEO2_FDTD": (2, "tti", ("V", "Eps", "Eta", "SinTheta", "CosTheta", "B", "F", "DtOmegaInvQ",
                                              "PSpace", "MSpace", "PCur", "POld", "MCur", "MOld"),
                                   ("V", "VEA"), ("V", "wavefieldsep_V", "VEA"), False),
    "Prop3DAcoTTIDenQ_DEO2_FDTD": (3, "tti", ("V", "Eps", "Eta", "SinTheta", "CosTheta", "SinPhi", "CosPhi", "B",
                                              "F", "DtOmegaInvQ", "PSpace", "MSpace", "PCur", "POld", "MCur", "MOld"),
                                   ("V", "VEA"), ("V", "wavefieldsep_V", "VEA"), False),
}


def _born_args(physics: str, variant: str):
    if physics == "iso":
        return {"V": 2, "VB": 4, "B": 3}[variant]
    return {"V": 3, "VEA": 7}[variant]


def _image_args(physics: str, variant: str):
    if physics == "iso":
        return {"V": 2, "VB": 4, "B": 3, "wavefieldsep": 2}[variant]
    return {"V": 3, "wavefieldsep_V": 3, "VEA": 7}[variant]


class PropagatorABI:
    """Typed handles to one propagator's exports in a loaded shared library."""

    def __init__(self, lib: ctypes.CDLL, name: str):
        if name not in PROPAGATORS:
            raise KeyError(f"unknown propagator {name}")
        self.name = name
        self.ndim, self.physics, self.getters, self.born, self.images, self.has_linear = PROPAGATORS[name]
        self.lib = lib
        fn = self._fn
        if self.ndim == 3:
            fn("alloc", c_void_p, [c_long, c_long, c_long, c_long, c_long, c_long,
                                   c_float, c_float, c_float, c_float, c_long, c_long, c_long])
            fn("getNy", c_long, [c_void_p])
        else:
            fn("alloc", c_void_p, [c_long, c_long, c_long, c_long, c_long,
                                   c_float, c_float, c_float, c_long, c_long])
        fn("free", None, [c_void_p])
        fn("SetupDtOmegaInvQ", None, [c_void_p, c_float, c_float, c_float])
        fn("TimeStep", None, [c_void_p])
        if self.has_linear:
            fn("TimeStepLinear", None, [c_void_p])
        fn("ScaleSpatialDerivatives", None, [c_void_p])
        fn("getNx", c_long, [c_void_p])
        fn("getNz", c_long, [c_void_p])
        for g in self.getters:
            fn("get" + g, _f32p, [c_void_p])
        if "DtOmegaInvQ" not in self.getters and self.has("getDtOmegaInvQ"):
            # exported by the CUDA build for every propagator, absent from the reference's 3D VTI library
            fn("getDtOmegaInvQ", _f32p, [c_void_p])
        for v in self.born:
            fn("ForwardBornInjection_" + v, None, [c_void_p] + [_f32p] * _born_args(self.physics, v))
        for v in self.images:
            extra = [c_long] if v.startswith("wavefieldsep") else []
            fn("AdjointBornAccumulation_" + v, None, [c_void_p] + [_f32p] * _image_args(self.physics, v) + extra)
        if name == "Prop2DAcoVTIDenQ_DEO2_FDTD":
            # prop2DAcoVTIDenQ_DEO2_FDTD.cc:158-176
            self.applyFirstDerivatives2D_PlusHalf = self._raw(
                name + "_applyFirstDerivatives2D_PlusHalf", None,
                [c_long, c_long, c_long, c_long, c_float, c_float, c_float, c_float, c_float, c_float,
                 _f32p, _f32p, _f32p, _f32p, c_long, c_long])

    def _raw(self, sym, restype, argtypes):
        f = getattr(self.lib, sym)
        f.restype = restype
        f.argtypes = argtypes
        return f

    def _fn(self, short, restype, argtypes):
        setattr(self, short, self._raw(self.name + "_" + short, restype, argtypes))

    def has(self, short: str) -> bool:
        return hasattr(self.lib, self.name + "_" + short)


class SourcePoint32(ctypes.Structure):
    """spacetime.cc:132-136 / src/spacetime.jl:793-797: 1-based linear index, 1-based trace index, weight."""
    _fields_ = [("iu", c_long), ("ir", c_long), ("c", c_float)]


class SpacetimeABI:
    """spacetime.cc:144-162 (injectdata_float), :184-204 (extractdata_float) and the time
    interpolation exports :228-330 (interp{forward,adjoint}_{1d,nd}_{float,double})."""

    def __init__(self, lib: ctypes.CDLL):
        self.lib = lib
        for T, ct in (("float", c_float), ("double", ctypes.c_double)):
            pp = POINTER(POINTER(ct))
            p = POINTER(ct)
            for fn, args in ((f"interpadjoint_1d_{T}", [pp, p, p, c_size_t, c_size_t, c_size_t]),
                             (f"interpforward_1d_{T}", [pp, p, p, c_size_t, c_size_t, c_size_t]),
                             (f"interpadjoint_nd_{T}", [pp, p, p, c_size_t, c_size_t, c_size_t, c_size_t, c_size_t]),
                             (f"interpforward_nd_{T}", [pp, p, p, c_size_t, c_size_t, c_size_t, c_size_t, c_size_t])):
                if hasattr(lib, fn):
                    f = getattr(lib, fn)
                    f.restype = None
                    f.argtypes = args
                    setattr(self, fn, f)
        self.injectdata_float = lib.injectdata_float
        self.injectdata_float.restype = None
        self.injectdata_float.argtypes = [_f32p, _f32p, c_size_t, c_size_t, POINTER(POINTER(SourcePoint32)),
                                          c_size_t, POINTER(c_long), c_size_t]
        self.extractdata_float = lib.extractdata_float
        self.extractdata_float.restype = None
        self.extractdata_float.argtypes = [_f32p, _f32p, POINTER(POINTER(SourcePoint32)), c_size_t,
                                           POINTER(c_long), c_size_t, c_size_t, c_size_t]
