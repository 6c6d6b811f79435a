"""Shared test helpers: seeded small models and a runner that drives any library exporting the
reference's propagator ABI (the CUDA build, or the reference itself built as the checker), plus
the same sequence replayed on the C restatement."""
from __future__ import annotations

import ctypes

import numpy as np

from wavefd_b200.abi import PROPAGATORS, PropagatorABI

SMALL_SHAPES = {2: (44, 1, 38), 3: (28, 22, 24)}  # (nz, ny, nx); nz*4 a multiple of 16 (TMA rows)


def geometry(name):
    ndim, physics = PROPAGATORS[name][:2]
    return ndim, physics


def make_model(ndim, physics, shape, seed=0, dx=0.01, dt=0.001):
    """Seeded model: velocity 1.5-3 km/s with 10 m cells and 1 ms steps (Courant <= 0.3)."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    full = (nx, ny, nz) if ndim == 3 else (nx, nz)

    def smooth(lo, hi):
        a = rng.random(full)
        for ax in range(a.ndim):
            a = (a + np.roll(a, 1, ax) + np.roll(a, -1, ax)) / 3
        a = (a - a.min()) / max(a.max() - a.min(), 1e-6)
        return (lo + (hi - lo) * a).astype(np.float32)

    m = {"V": smooth(1.5, 3.0), "B": smooth(0.4, 1.0)}
    if physics in ("vti", "tti"):
        m["Eps"] = smooth(0.0, 0.3)
        m["Eta"] = smooth(0.0, 0.15)
        m["F"] = np.full(full, 0.85, np.float32)
    if physics == "tti":
        th = smooth(0.0, np.pi / 4)
        m["SinTheta"] = np.sin(th).astype(np.float32)
        m["CosTheta"] = np.cos(th).astype(np.float32)
        if ndim == 3:
            ph = smooth(0.0, 2 * np.pi)
            m["SinPhi"] = np.sin(ph).astype(np.float32)
            m["CosPhi"] = np.cos(ph).astype(np.float32)
    fields = ["PCur", "POld"] + (["MCur", "MOld"] if physics != "iso" else [])
    for f in fields:
        m[f] = (rng.standard_normal(full) * 1e-2).astype(np.float32)
    return {k: np.ascontiguousarray(v) for k, v in m.items()}


class ABIRunner:
    """Drives one propagator object through the C ABI (arrays seen through the getters)."""

    def __init__(self, lib: ctypes.CDLL, name, shape, fs=True, nsponge=6, dx=0.01, dt=0.001, nthread=4,
                 freqQ=5.0, qMin=0.1, qInterior=100.0):
        self.abi = PropagatorABI(lib, name)
        self.name = name
        self.ndim, self.physics = geometry(name)
        self.nz, self.ny, self.nx = shape
        if self.ndim == 3:
            self.p = self.abi.alloc(int(fs), nthread, self.nx, self.ny, self.nz, nsponge, dx, dx, dx, dt, 8, 8, self.nz)
        else:
            self.p = self.abi.alloc(int(fs), nthread, self.nx, self.nz, nsponge, dx, dx, dt, 8, self.nz)
        self.abi.SetupDtOmegaInvQ(self.p, freqQ, qMin, qInterior)

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz) if self.ndim == 3 else (self.nx, self.nz)

    def arr(self, getter):
        ptr = getattr(self.abi, "get" + getter)(self.p)
        return np.ctypeslib.as_array(ptr, shape=self.shape)

    def load(self, model):
        for k, v in model.items():
            self.arr(k)[...] = v

    def close(self):
        if self.p:
            self.abi.free(self.p)
            self.p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class OracleRunner:
    """The same object semantics replayed on the C restatement (pointer swap included)."""

    def __init__(self, oracle, name, shape, fs=True, nsponge=6, dx=0.01, dt=0.001, freqQ=5.0, qMin=0.1,
                 qInterior=100.0):
        self.o = oracle
        self.name = name
        self.ndim, self.physics = geometry(name)
        self.nz, self.ny, self.nx = shape
        self.g = oracle.geom(self.ndim, fs, self.nx, self.ny, self.nz, dx, dx, dx, dt)
        shp = (self.nx, self.ny, self.nz) if self.ndim == 3 else (self.nx, self.nz)
        self.a = {k: np.zeros(shp, np.float32) for k in PROPAGATORS[name][2]}
        for k in ("DtOmegaInvQ", "SinPhi", "CosPhi", "MSpace", "MCur", "MOld"):
            self.a.setdefault(k, np.zeros(shp, np.float32))
        oracle.setup_q(self.g, nsponge, freqQ, qMin, qInterior, self.a["DtOmegaInvQ"])

    def load(self, model):
        for k, v in model.items():
            self.a[k][...] = v

    def arr(self, k):
        return self.a[k]

    def step(self, linear=False):
        a, o, g = self.a, self.o, self.g
        if self.physics == "iso":
            o.step_iso(g, a["V"], a["B"], a["DtOmegaInvQ"], a["PCur"], a["POld"], a["PSpace"])
        elif self.physics == "vti":
            o.step_vti(g, linear, a["V"], a["Eps"], a["Eta"], a["B"], a["F"], a["DtOmegaInvQ"], a["PCur"],
                       a["MCur"], a["POld"], a["MOld"], a["PSpace"], a["MSpace"])
        else:
            o.step_tti(g, a["V"], a["Eps"], a["Eta"], a["B"], a["F"], a["DtOmegaInvQ"], a["SinTheta"],
                       a["CosTheta"], a["SinPhi"], a["CosPhi"], a["PCur"], a["MCur"], a["POld"], a["MOld"],
                       a["PSpace"], a["MSpace"])
        a["PCur"], a["POld"] = a["POld"], a["PCur"]
        a["MCur"], a["MOld"] = a["MOld"], a["MCur"]

    def scale(self):
        a = self.a
        self.o.scale(self.g, a["V"], a["B"], a["PSpace"], None if self.physics == "iso" else a["MSpace"])


class OracleRunner64:
    """The FP64 rerun of the restatement with the same object semantics: the FP32 model (Q from the
    FP32 profile) promoted to double, then every step in double precision."""

    def __init__(self, oracle, name, shape, fs=True, nsponge=6, dx=0.01, dt=0.001, freqQ=5.0, qMin=0.1,
                 qInterior=100.0):
        base = OracleRunner(oracle, name, shape, fs=fs, nsponge=nsponge, dx=dx, dt=dt, freqQ=freqQ, qMin=qMin,
                            qInterior=qInterior)
        self.o, self.g, self.physics, self.ndim = oracle, base.g, base.physics, base.ndim
        self.a = {k: v.astype(np.float64) for k, v in base.a.items()}

    def load(self, model):
        for k, v in model.items():
            self.a[k][...] = v

    def arr(self, k):
        return self.a[k]

    def step(self, linear=False):
        a, o, g = self.a, self.o, self.g
        if self.physics == "iso":
            o.step_iso64(g, a["V"], a["B"], a["DtOmegaInvQ"], a["PCur"], a["POld"], a["PSpace"])
        elif self.physics == "vti":
            o.step_vti64(g, linear, a["V"], a["Eps"], a["Eta"], a["B"], a["F"], a["DtOmegaInvQ"], a["PCur"],
                         a["MCur"], a["POld"], a["MOld"], a["PSpace"], a["MSpace"])
        else:
            o.step_tti64(g, a["V"], a["Eps"], a["Eta"], a["B"], a["F"], a["DtOmegaInvQ"], a["SinTheta"],
                         a["CosTheta"], a["SinPhi"], a["CosPhi"], a["PCur"], a["MCur"], a["POld"], a["MOld"],
                         a["PSpace"], a["MSpace"])
        a["PCur"], a["POld"] = a["POld"], a["PCur"]
        a["MCur"], a["MOld"] = a["MOld"], a["MCur"]


class Ref64Runner(OracleRunner64):
    """The reference's own passes instantiated with double (oracle Ref64), same object semantics."""

    def __init__(self, ref64, oracle, name, shape, **kw):
        super().__init__(oracle, name, shape, **kw)
        self.r = ref64
        self.scratch = ref64.new_scratch(self.a["V"].shape)

    def step(self, linear=False):
        self.r.step(self.physics, self.ndim, self.g, self.a, self.scratch, linear=linear)


def same(a, b):
    """Bitwise equality up to the sign of zero."""
    return np.array_equal(a, b)


def mismatch_report(a, b):
    d = np.abs(a.astype(np.float64) - b.astype(np.float64))
    idx = np.unravel_index(np.argmax(d), d.shape)
    return f"max |diff| {d.max():.3e} at {idx}: {a[idx]!r} vs {b[idx]!r}; n_diff={int((a != b).sum())}"


def rel_l2(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))
