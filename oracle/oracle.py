"""Python bindings for the checker -- TEST INFRASTRUCTURE ONLY.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module; the product
never imports it.

* `Oracle` wraps _build/liboracle_wavefd.so, the project's C restatement (wavefd_oracle.c).
* `reference_lib(name, flavour)` opens the reference's own library compiled from its sources
  by this directory's Makefile (_ref/strict: IEEE order, _ref/fast: the reference's CMake
  flags, _ref/avx2: the same with -march=x86-64-v3).
* `Oracle.*64` methods: the FP64 rerun of the restatement (wfo64_*: the same routines on double
  arrays); `Ref64` wraps _ref/strict64/libref64.so, the reference's own pass templates
  instantiated with double (ref64_harness.cc), which pins the FP64 restatement.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_float, c_long

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle_wavefd.so")
REF_DIR = os.path.join(HERE, "_ref")

_f32p = POINTER(c_float)
_f64p = POINTER(ctypes.c_double)
_i64p = POINTER(c_long)
REF64_LIB = os.path.join(REF_DIR, "strict64", "libref64.so")


class Geom(ctypes.Structure):
    _fields_ = [("ndim", c_long), ("fs", c_long), ("nx", c_long), ("ny", c_long), ("nz", c_long),
                ("dx", c_float), ("dy", c_float), ("dz", c_float), ("dt", c_float)]


def reference_lib_path(name: str, flavour: str = "strict") -> str:
    return os.path.join(REF_DIR, flavour, f"lib{name}.so")


def reference_available(flavour: str = "strict") -> bool:
    return os.path.exists(reference_lib_path("prop3DAcoIsoDenQ_DEO2_FDTD", flavour))


def reference_lib(name: str, flavour: str = "strict") -> ctypes.CDLL:
    path = reference_lib_path(name, flavour)
    if not os.path.exists(path):
        raise FileNotFoundError(f"reference library not built: {path} (run make -C oracle ref)")
    return ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"], "float32 C-contiguous array expected"
    return a.ctypes.data_as(_f32p)


def _p64(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "float64 C-contiguous array expected"
    return a.ctypes.data_as(_f64p)


class Oracle:
    """C restatement of the reference's per-step arithmetic (see wavefd_oracle.h)."""

    def __init__(self, path: str = ORACLE_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library not built: {path} (run make -C oracle)")
        self.lib = ctypes.CDLL(path)

    def geom(self, ndim, fs, nx, ny, nz, dx, dy, dz, dt):
        return Geom(ndim, int(bool(fs)), nx, ny if ndim == 3 else 1, nz, dx, dy, dz, dt)

    def setup_q(self, g, nsponge, freqQ, qMin, qInterior, q):
        self.lib.wfo_setup_q(ctypes.byref(g), c_long(nsponge), c_float(freqQ), c_float(qMin), c_float(qInterior), _p(q))

    def step_iso(self, g, v, b, q, pcur, pold, pspace):
        self.lib.wfo_step_iso(ctypes.byref(g), _p(v), _p(b), _p(q), _p(pcur), _p(pold), _p(pspace))

    def step_vti(self, g, linear, v, eps, eta, b, f, q, pcur, mcur, pold, mold, pspace, mspace):
        self.lib.wfo_step_vti(ctypes.byref(g), c_long(int(linear)), _p(v), _p(eps), _p(eta), _p(b), _p(f), _p(q),
                              _p(pcur), _p(mcur), _p(pold), _p(mold), _p(pspace), _p(mspace))

    def step_tti(self, g, v, eps, eta, b, f, q, sint, cost, sinp, cosp, pcur, mcur, pold, mold, pspace, mspace):
        self.lib.wfo_step_tti(ctypes.byref(g), _p(v), _p(eps), _p(eta), _p(b), _p(f), _p(q), _p(sint), _p(cost),
                              _p(sinp), _p(cosp), _p(pcur), _p(mcur), _p(pold), _p(mold), _p(pspace), _p(mspace))

    def scale(self, g, v, b, pspace, mspace=None):
        self.lib.wfo_scale(ctypes.byref(g), _p(v), _p(b), _p(pspace), _p(mspace))

    def dplus(self, g, a, ox, oy, oz):
        self.lib.wfo_dplus(ctypes.byref(g), _p(a), _p(ox), _p(oy), _p(oz))

    def dminus(self, g, a, ox, oy, oz):
        self.lib.wfo_dminus(ctypes.byref(g), _p(a), _p(ox), _p(oy), _p(oz))

    def born_iso(self, g, which, v, b, dv, db, p, dp, pcur):
        self.lib.wfo_born_iso(ctypes.byref(g), c_long(which), _p(v), _p(b), _p(dv), _p(db), _p(p), _p(dp), _p(pcur))

    def born_aniso_v(self, g, v, dv, dp, dm, pcur, mcur):
        self.lib.wfo_born_aniso_v(ctypes.byref(g), _p(v), _p(dv), _p(dp), _p(dm), _p(pcur), _p(mcur))

    def born_vea(self, g, tti, v, eps, eta, b, f, sint, cost, sinp, cosp, dv, de, da, p, m, dp, dm, pcur, mcur):
        self.lib.wfo_born_vea(ctypes.byref(g), c_long(int(tti)), _p(v), _p(eps), _p(eta), _p(b), _p(f), _p(sint),
                              _p(cost), _p(sinp), _p(cosp), _p(dv), _p(de), _p(da), _p(p), _p(m), _p(dp), _p(dm),
                              _p(pcur), _p(mcur))

    def image_iso(self, g, which, v, b, p, dp, pold, dv, db):
        self.lib.wfo_image_iso(ctypes.byref(g), c_long(which), _p(v), _p(b), _p(p), _p(dp), _p(pold), _p(dv), _p(db))

    def image_aniso_v(self, g, v, b, dp, dm, pold, mold, dv):
        self.lib.wfo_image_aniso_v(ctypes.byref(g), _p(v), _p(b), _p(dp), _p(dm), _p(pold), _p(mold), _p(dv))

    def image_vea(self, g, tti, v, eps, eta, b, f, sint, cost, sinp, cosp, p, m, dp, dm, pold, mold, dv, de, da):
        self.lib.wfo_image_vea(ctypes.byref(g), c_long(int(tti)), _p(v), _p(eps), _p(eta), _p(b), _p(f), _p(sint),
                               _p(cost), _p(sinp), _p(cosp), _p(p), _p(m), _p(dp), _p(dm), _p(pold), _p(mold),
                               _p(dv), _p(de), _p(da))

    def image_wavefieldsep(self, g, isfwi, v, b, dp, pold, dm, mold, dv):
        self.lib.wfo_image_wavefieldsep(ctypes.byref(g), c_long(int(isfwi)), _p(v), _p(b), _p(dp), _p(pold),
                                        _p(dm), _p(mold), _p(dv))

    def inject(self, field, data_colmajor, it, nt, iu, ir, c):
        iu = np.ascontiguousarray(iu, dtype=np.int64)
        ir = np.ascontiguousarray(ir, dtype=np.int64)
        c = np.ascontiguousarray(c, dtype=np.float32)
        self.lib.wfo_inject(_p(field), _p(data_colmajor), c_long(it), c_long(nt), iu.ctypes.data_as(_i64p),
                            ir.ctypes.data_as(_i64p), _p(c), c_long(len(c)))

    def illum(self, accum, field):
        """wfo_illum_float: field = field^2 (accum None) or accum += field^2, in place."""
        self.lib.wfo_illum_float(_p(accum), _p(field), c_long(field.size))

    def interp(self, forward, h, out, inp, nh, nout, nin, nslow):
        """Time interpolation (wfo_interpforward_* / wfo_interpadjoint_*), float32 or float64 arrays."""
        dbl = out.dtype == np.float64
        ptr = (lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) if dbl else _p
        name = ("wfo_interpforward_" if forward else "wfo_interpadjoint_") + ("double" if dbl else "float")
        getattr(self.lib, name)(ptr(np.ascontiguousarray(h)), ptr(out), ptr(inp), c_long(nh), c_long(nout),
                                c_long(nin), c_long(nslow))

    def extract(self, data_colmajor, field, it, nt, iu, ir, c):
        iu = np.ascontiguousarray(iu, dtype=np.int64)
        ir = np.ascontiguousarray(ir, dtype=np.int64)
        c = np.ascontiguousarray(c, dtype=np.float32)
        self.lib.wfo_extract(_p(data_colmajor), _p(field), c_long(it), c_long(nt), iu.ctypes.data_as(_i64p),
                             ir.ctypes.data_as(_i64p), _p(c), c_long(len(c)))

    # ---- FP64 rerun (double arrays) -------------------------------------------------------------
    def step_iso64(self, g, v, b, q, pcur, pold, pspace):
        self.lib.wfo64_step_iso(ctypes.byref(g), _p64(v), _p64(b), _p64(q), _p64(pcur), _p64(pold), _p64(pspace))

    def step_vti64(self, g, linear, v, eps, eta, b, f, q, pcur, mcur, pold, mold, pspace, mspace):
        self.lib.wfo64_step_vti(ctypes.byref(g), c_long(int(linear)), _p64(v), _p64(eps), _p64(eta), _p64(b), _p64(f),
                                _p64(q), _p64(pcur), _p64(mcur), _p64(pold), _p64(mold), _p64(pspace), _p64(mspace))

    def step_tti64(self, g, v, eps, eta, b, f, q, sint, cost, sinp, cosp, pcur, mcur, pold, mold, pspace, mspace):
        self.lib.wfo64_step_tti(ctypes.byref(g), _p64(v), _p64(eps), _p64(eta), _p64(b), _p64(f), _p64(q), _p64(sint),
                                _p64(cost), _p64(sinp), _p64(cosp), _p64(pcur), _p64(mcur), _p64(pold), _p64(mold),
                                _p64(pspace), _p64(mspace))

    def scale64(self, g, v, b, pspace, mspace=None):
        self.lib.wfo64_scale(ctypes.byref(g), _p64(v), _p64(b), _p64(pspace), _p64(mspace))

    def born_aniso_v64(self, g, v, dv, dp, dm, pcur, mcur):
        self.lib.wfo64_born_aniso_v(ctypes.byref(g), _p64(v), _p64(dv), _p64(dp), _p64(dm), _p64(pcur), _p64(mcur))

    def image_aniso_v64(self, g, v, b, dp, dm, pold, mold, dv):
        self.lib.wfo64_image_aniso_v(ctypes.byref(g), _p64(v), _p64(b), _p64(dp), _p64(dm), _p64(pold), _p64(mold),
                                     _p64(dv))

    def born_iso64(self, g, which, v, b, dv, db, p, dp, pcur):
        self.lib.wfo64_born_iso(ctypes.byref(g), c_long(which), _p64(v), _p64(b), _p64(dv), _p64(db), _p64(p),
                                _p64(dp), _p64(pcur))

    def image_iso64(self, g, which, v, b, p, dp, pold, dv, db):
        self.lib.wfo64_image_iso(ctypes.byref(g), c_long(which), _p64(v), _p64(b), _p64(p), _p64(dp), _p64(pold),
                                 _p64(dv), _p64(db))

    def inject64(self, field, data_colmajor, it, nt, iu, ir, c):
        iu = np.ascontiguousarray(iu, dtype=np.int64)
        ir = np.ascontiguousarray(ir, dtype=np.int64)
        c = np.ascontiguousarray(c, dtype=np.float64)
        self.lib.wfo64_inject(_p64(field), _p64(data_colmajor), c_long(it), c_long(nt), iu.ctypes.data_as(_i64p),
                              ir.ctypes.data_as(_i64p), _p64(c), c_long(len(c)))

    def extract64(self, data_colmajor, field, it, nt, iu, ir, c):
        iu = np.ascontiguousarray(iu, dtype=np.int64)
        ir = np.ascontiguousarray(ir, dtype=np.int64)
        c = np.ascontiguousarray(c, dtype=np.float64)
        self.lib.wfo64_extract(_p64(data_colmajor), _p64(field), c_long(it), c_long(nt), iu.ctypes.data_as(_i64p),
                               ir.ctypes.data_as(_i64p), _p64(c), c_long(len(c)))


def ref64_available() -> bool:
    return os.path.exists(REF64_LIB)


class Ref64:
    """The reference's time-step pass templates instantiated with double (ref64_harness.cc).

    `step(physics, ndim, g, a, scratch, linear)` advances the dict of float64 arrays `a` (getter
    names) by one step in place, pointer swap included. `scratch` holds the six pass-1 arrays of
    one propagator object (zero at construction and kept across its steps, as the reference's
    tmp arrays are); `new_scratch(shape)` makes them."""

    def __init__(self, path: str = REF64_LIB):
        if not os.path.exists(path):
            raise FileNotFoundError(f"FP64 reference harness not built: {path} (run make -C oracle ref)")
        self.lib = ctypes.CDLL(path, mode=ctypes.RTLD_LOCAL)

    @staticmethod
    def new_scratch(shape):
        return [np.zeros(shape, np.float64) for _ in range(6)]

    def step(self, physics, ndim, g, a, scratch, linear=False):
        t = [_p64(x) for x in scratch]
        L = self.lib
        fs, nx, ny, nz = c_long(g.fs), c_long(g.nx), c_long(g.ny), c_long(g.nz)
        dx, dy, dz, dt = c_float(g.dx), c_float(g.dy), c_float(g.dz), c_float(g.dt)
        P = lambda k: _p64(a[k])
        if physics == "iso" and ndim == 3:
            L.ref64_step_iso3d(fs, nx, ny, nz, dx, dy, dz, dt, P("V"), P("B"), P("DtOmegaInvQ"), P("PCur"), P("POld"),
                               P("PSpace"), t[0], t[1], t[2])
        elif physics == "iso":
            L.ref64_step_iso2d(fs, nx, nz, dx, dz, dt, P("V"), P("B"), P("DtOmegaInvQ"), P("PCur"), P("POld"),
                               P("PSpace"), t[0], t[1])
        elif physics == "vti" and ndim == 3:
            L.ref64_step_vti3d(fs, c_long(int(linear)), nx, ny, nz, dx, dy, dz, dt, P("V"), P("Eps"), P("Eta"), P("B"),
                               P("F"), P("DtOmegaInvQ"), P("PCur"), P("MCur"), P("POld"), P("MOld"), P("PSpace"),
                               P("MSpace"), *t)
        elif physics == "vti":
            L.ref64_step_vti2d(fs, c_long(int(linear)), nx, nz, dx, dz, dt, P("V"), P("Eps"), P("Eta"), P("B"), P("F"),
                               P("DtOmegaInvQ"), P("PCur"), P("MCur"), P("POld"), P("MOld"), P("PSpace"), P("MSpace"),
                               *t[:4])
        elif ndim == 3:
            # the reference takes the angle arrays as float (prop3DAcoTTIDenQ_DEO2_FDTD.h:811-814)
            keep = [np.ascontiguousarray(a[k], dtype=np.float32) for k in ("SinTheta", "CosTheta", "SinPhi", "CosPhi")]
            L.ref64_step_tti3d(fs, nx, ny, nz, dx, dy, dz, dt, P("V"), P("Eps"), P("Eta"), P("B"), P("F"),
                               P("DtOmegaInvQ"), *[k.ctypes.data_as(_f32p) for k in keep], P("PCur"), P("MCur"),
                               P("POld"), P("MOld"), P("PSpace"), P("MSpace"), *t)
        else:
            keep = [np.ascontiguousarray(a[k], dtype=np.float32) for k in ("SinTheta", "CosTheta")]
            L.ref64_step_tti2d(fs, nx, nz, dx, dz, dt, P("V"), P("Eps"), P("Eta"), P("B"), P("F"), P("DtOmegaInvQ"),
                               *[k.ctypes.data_as(_f32p) for k in keep], P("PCur"), P("MCur"), P("POld"), P("MOld"),
                               P("PSpace"), P("MSpace"), *t[:4])
        a["PCur"], a["POld"] = a["POld"], a["PCur"]
        if physics != "iso":
            a["MCur"], a["MOld"] = a["MOld"], a["MCur"]
