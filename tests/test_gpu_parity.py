"""GPU parity: the CUDA library, driven through the reference's C ABI, against the C restatement
(oracle/) on the same seeded inputs.

* strict mode (IEEE order, no FMA): bitwise equality (up to the sign of zero) after several steps,
  for every propagator, free surface on and off, fused and unfused step kernels, and for Born
  injection and the imaging conditions;
* fast mode (FMA contraction, approximate division): relative L2 <= 1e-5 per field after 40 steps;
* wavefield separation (FFT rounding differs from the double-precision oracle): relative L2 <= 1e-5.
"""
import ctypes

import numpy as np
import pytest

from tests.harness import (ABIRunner, OracleRunner, SMALL_SHAPES, fptr, make_model, mismatch_report, rel_l2,
                           same)
from wavefd_b200.abi import PROPAGATORS

pytestmark = pytest.mark.gpu

NAMES = list(PROPAGATORS)
FAST_TOL = 1e-5

# odd sizes: partial tiles in z and y, and x split into several fused-kernel chunks; nz = 37 takes
# the fused kernel that stages tiles with ordinary loads, nz = 36 the TMA-staged one; nz = 100,
# ny = 53 gives tiles whose halo lies wholly inside the interior
ODD_SHAPES = {2: [(45, 1, 150)], 3: [(37, 21, 140), (36, 21, 150), (100, 53, 60)]}


@pytest.fixture(scope="module")
def lib():
    from wavefd_b200 import _lib
    return _lib.library()


def _pair(lib, oracle, name, fs, shape=None, seed=2, strict=True, fused=True):
    ndim, physics = PROPAGATORS[name][:2]
    shape = shape or SMALL_SHAPES[ndim]
    gpu = ABIRunner(lib, name, shape, fs=fs)
    lib.WFD_Prop_SetStrict(ctypes.c_void_p(gpu.p), int(strict))
    lib.WFD_Prop_SetFused(ctypes.c_void_p(gpu.p), int(fused))
    orc = OracleRunner(oracle, name, shape, fs=fs)
    model = make_model(ndim, physics, shape, seed=seed)
    gpu.load(model)
    orc.load(model)
    return gpu, orc


def _fields(name, linear=False):
    physics = PROPAGATORS[name][1]
    f = ["PCur", "POld"] + ([] if physics == "iso" else ["MCur", "MOld"])
    if not linear:
        f += ["PSpace"] + ([] if physics == "iso" else ["MSpace"])
    return f


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("fs", [True, False])
@pytest.mark.parametrize("fused", [True, False])
def test_step_strict_bitwise(lib, oracle, name, fs, fused):
    gpu, orc = _pair(lib, oracle, name, fs, fused=fused)
    for _ in range(5):
        gpu.abi.TimeStep(gpu.p)
        orc.step()
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    for k in _fields(name):
        assert same(gpu.arr(k), orc.arr(k)), f"{name} fs={fs} fused={fused} {k}: {mismatch_report(gpu.arr(k), orc.arr(k))}"
    gpu.close()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("fs", [True, False])
@pytest.mark.parametrize("which", [0, 1, 2])
def test_step_strict_bitwise_odd_sizes(lib, oracle, name, fs, which):
    ndim = PROPAGATORS[name][0]
    if which >= len(ODD_SHAPES[ndim]):
        pytest.skip("one odd shape in 2D")
    gpu, orc = _pair(lib, oracle, name, fs, shape=ODD_SHAPES[ndim][which], seed=5)
    for _ in range(3):
        gpu.abi.TimeStep(gpu.p)
        orc.step()
    for k in _fields(name):
        assert same(gpu.arr(k), orc.arr(k)), f"{name} {k}: {mismatch_report(gpu.arr(k), orc.arr(k))}"
    gpu.close()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("fs", [True, False])
def test_step_fast_close(lib, oracle, name, fs):
    gpu, orc = _pair(lib, oracle, name, fs, strict=False)
    for _ in range(40):
        gpu.abi.TimeStep(gpu.p)
        orc.step()
    for k in _fields(name):
        err = rel_l2(gpu.arr(k), orc.arr(k))
        assert err <= FAST_TOL, f"{name} {k}: rel L2 {err:.3e}"
    gpu.close()


@pytest.mark.parametrize("name", [n for n in NAMES if PROPAGATORS[n][0] == 3])
@pytest.mark.parametrize("fs", [True, False])
def test_step_fast_close_interior_tiles(lib, oracle, name, fs):
    gpu, orc = _pair(lib, oracle, name, fs, shape=ODD_SHAPES[3][2], seed=9, strict=False)
    for _ in range(30):
        gpu.abi.TimeStep(gpu.p)
        orc.step()
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    for k in _fields(name):
        err = rel_l2(gpu.arr(k), orc.arr(k))
        assert err <= FAST_TOL, f"{name} {k}: rel L2 {err:.3e}"
    gpu.close()


@pytest.mark.parametrize("name", [n for n in NAMES if PROPAGATORS[n][5]])
@pytest.mark.parametrize("strict", [True, False])
def test_step_linear(lib, oracle, name, strict):
    gpu, orc = _pair(lib, oracle, name, True, strict=strict)
    for _ in range(4):
        gpu.abi.TimeStepLinear(gpu.p)
        orc.step(linear=True)
    for k in _fields(name, linear=True):
        if strict:
            assert same(gpu.arr(k), orc.arr(k)), f"{name} {k}: {mismatch_report(gpu.arr(k), orc.arr(k))}"
        else:
            assert rel_l2(gpu.arr(k), orc.arr(k)) <= FAST_TOL
    gpu.close()


@pytest.mark.parametrize("name", NAMES)
def test_scale_and_q(lib, oracle, name):
    gpu, orc = _pair(lib, oracle, name, True)
    assert same(gpu.arr("DtOmegaInvQ"), orc.arr("DtOmegaInvQ"))
    gpu.abi.TimeStep(gpu.p)
    orc.step()
    gpu.abi.ScaleSpatialDerivatives(gpu.p)
    orc.scale()
    for k in ["PSpace"] + ([] if PROPAGATORS[name][1] == "iso" else ["MSpace"]):
        assert same(gpu.arr(k), orc.arr(k)), mismatch_report(gpu.arr(k), orc.arr(k))
    gpu.close()


def _rand(shape, seed, scale=1e-2):
    return (np.random.default_rng(seed).standard_normal(shape) * scale).astype(np.float32)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("variant", ["V", "VB", "B", "VEA"])
@pytest.mark.parametrize("fs", [True, False])
def test_born_strict_bitwise(lib, oracle, name, variant, fs):
    physics = PROPAGATORS[name][1]
    if variant not in PROPAGATORS[name][3]:
        pytest.skip("variant not defined for this physics")
    gpu, orc = _pair(lib, oracle, name, fs)
    shp = orc.arr("V").shape
    dv, db, de, da = _rand(shp, 11), _rand(shp, 12), _rand(shp, 13), _rand(shp, 14)
    P, DP, M, DM = _rand(shp, 15), _rand(shp, 16), _rand(shp, 17), _rand(shp, 18)
    fn = getattr(gpu.abi, "ForwardBornInjection_" + variant)
    a = orc.a
    tti = physics == "tti"
    if physics == "iso":
        args = {"V": (dv, DP), "VB": (dv, db, P, DP), "B": (db, P, DP)}[variant]
        fn(gpu.p, *[fptr(x) for x in args])
        oracle.born_iso(orc.g, {"V": 0, "VB": 1, "B": 2}[variant], a["V"], a["B"], dv, db, P, DP, a["PCur"])
        keys = ["PCur"]
    elif variant == "V":
        fn(gpu.p, fptr(dv), fptr(DP), fptr(DM))
        oracle.born_aniso_v(orc.g, a["V"], dv, DP, DM, a["PCur"], a["MCur"])
        keys = ["PCur", "MCur"]
    else:
        fn(gpu.p, *[fptr(x) for x in (dv, de, da, P, M, DP, DM)])
        oracle.born_vea(orc.g, tti, a["V"], a["Eps"], a["Eta"], a["B"], a["F"], a["SinTheta"] if tti else None,
                        a["CosTheta"] if tti else None, a["SinPhi"], a["CosPhi"], dv, de, da, P, M, DP, DM,
                        a["PCur"], a["MCur"])
        keys = ["PCur", "MCur"]
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    for k in keys:
        assert same(gpu.arr(k), orc.arr(k)), f"{name} {variant} {k}: {mismatch_report(gpu.arr(k), orc.arr(k))}"
    gpu.close()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("variant", ["V", "VB", "B", "VEA"])
@pytest.mark.parametrize("fs", [True, False])
def test_imaging_strict_bitwise(lib, oracle, name, variant, fs):
    physics = PROPAGATORS[name][1]
    if variant not in PROPAGATORS[name][4]:
        pytest.skip("variant not defined for this physics")
    gpu, orc = _pair(lib, oracle, name, fs)
    shp = orc.arr("V").shape
    P, DP, M, DM = _rand(shp, 25), _rand(shp, 26), _rand(shp, 27), _rand(shp, 28)
    img = {k: _rand(shp, 30 + i) for i, k in enumerate(("v", "b", "e", "a"))}
    mine = {k: v.copy() for k, v in img.items()}
    fn = getattr(gpu.abi, "AdjointBornAccumulation_" + variant)
    a = orc.a
    tti = physics == "tti"
    if physics == "iso":
        if variant == "V":
            fn(gpu.p, fptr(img["v"]), fptr(DP))
        elif variant == "VB":
            fn(gpu.p, fptr(img["v"]), fptr(img["b"]), fptr(P), fptr(DP))
        else:
            fn(gpu.p, fptr(img["b"]), fptr(P), fptr(DP))
        oracle.image_iso(orc.g, {"V": 0, "VB": 1, "B": 2}[variant], a["V"], a["B"], P, DP, a["POld"], mine["v"],
                         mine["b"])
        keys = {"V": ["v"], "VB": ["v", "b"], "B": ["b"]}[variant]
    elif variant == "V":
        fn(gpu.p, fptr(img["v"]), fptr(DP), fptr(DM))
        oracle.image_aniso_v(orc.g, a["V"], a["B"], DP, DM, a["POld"], a["MOld"], mine["v"])
        keys = ["v"]
    else:
        fn(gpu.p, *[fptr(x) for x in (img["v"], img["e"], img["a"], P, M, DP, DM)])
        oracle.image_vea(orc.g, tti, a["V"], a["Eps"], a["Eta"], a["B"], a["F"], a["SinTheta"] if tti else None,
                         a["CosTheta"] if tti else None, a["SinPhi"], a["CosPhi"], P, M, DP, DM, a["POld"],
                         a["MOld"], mine["v"], mine["e"], mine["a"])
        keys = ["v", "e", "a"]
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    for k in keys:
        assert same(img[k], mine[k]), f"{name} {variant} image {k}: {mismatch_report(img[k], mine[k])}"
    gpu.close()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("variant", ["VB", "B", "VEA"])
def test_born_imaging_fast_close(lib, oracle, name, variant):
    """The fast build (FMA contraction, approximate division) of the VB/B/VEA Born injections and
    imaging conditions, whose gradient triples and D- are formed per cell: what each call adds to
    pCur/mCur or to the images, against the checker's, relative L2 <= 1e-5."""
    physics = PROPAGATORS[name][1]
    if variant not in PROPAGATORS[name][3]:
        pytest.skip("variant not defined for this physics")
    tti = physics == "tti"
    # Born injection
    gpu, orc = _pair(lib, oracle, name, True, strict=False)
    shp = orc.arr("V").shape
    dv, db, de, da = _rand(shp, 51), _rand(shp, 52), _rand(shp, 53), _rand(shp, 54)
    P, DP, M, DM = _rand(shp, 55), _rand(shp, 56), _rand(shp, 57), _rand(shp, 58)
    keys = ["PCur"] if physics == "iso" else ["PCur", "MCur"]
    before = {k: orc.arr(k).copy() for k in keys}
    a = orc.a
    fn = getattr(gpu.abi, "ForwardBornInjection_" + variant)
    if physics == "iso":
        args = {"VB": (dv, db, P, DP), "B": (db, P, DP)}[variant]
        fn(gpu.p, *[fptr(x) for x in args])
        oracle.born_iso(orc.g, {"VB": 1, "B": 2}[variant], a["V"], a["B"], dv, db, P, DP, a["PCur"])
    else:
        fn(gpu.p, *[fptr(x) for x in (dv, de, da, P, M, DP, DM)])
        oracle.born_vea(orc.g, tti, a["V"], a["Eps"], a["Eta"], a["B"], a["F"], a["SinTheta"] if tti else None,
                        a["CosTheta"] if tti else None, a["SinPhi"], a["CosPhi"], dv, de, da, P, M, DP, DM,
                        a["PCur"], a["MCur"])
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    for k in keys:
        err = rel_l2(gpu.arr(k) - before[k], orc.arr(k) - before[k])
        assert err <= 1e-5, f"{name} Born {variant} {k}: rel L2 of the increment {err:.2e}"
    gpu.close()
    # imaging condition
    if variant not in PROPAGATORS[name][4]:
        return
    gpu, orc = _pair(lib, oracle, name, True, strict=False)
    img = {k: _rand(shp, 60 + i) for i, k in enumerate(("v", "b", "e", "a"))}
    start = {k: v.copy() for k, v in img.items()}
    mine = {k: v.copy() for k, v in img.items()}
    a = orc.a
    fn = getattr(gpu.abi, "AdjointBornAccumulation_" + variant)
    if physics == "iso":
        if variant == "VB":
            fn(gpu.p, fptr(img["v"]), fptr(img["b"]), fptr(P), fptr(DP))
        else:
            fn(gpu.p, fptr(img["b"]), fptr(P), fptr(DP))
        oracle.image_iso(orc.g, {"VB": 1, "B": 2}[variant], a["V"], a["B"], P, DP, a["POld"], mine["v"], mine["b"])
        ks = {"VB": ["v", "b"], "B": ["b"]}[variant]
    else:
        fn(gpu.p, *[fptr(x) for x in (img["v"], img["e"], img["a"], P, M, DP, DM)])
        oracle.image_vea(orc.g, tti, a["V"], a["Eps"], a["Eta"], a["B"], a["F"], a["SinTheta"] if tti else None,
                         a["CosTheta"] if tti else None, a["SinPhi"], a["CosPhi"], P, M, DP, DM, a["POld"],
                         a["MOld"], mine["v"], mine["e"], mine["a"])
        ks = ["v", "e", "a"]
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    for k in ks:
        err = rel_l2(img[k] - start[k], mine[k] - start[k])
        assert err <= 1e-5, f"{name} imaging {variant} {k}: rel L2 of the increment {err:.2e}"
    gpu.close()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("isfwi", [0, 1])
@pytest.mark.parametrize("nz", [26, 32])  # Bluestein length and power-of-two length
def test_wavefieldsep_close(lib, oracle, name, isfwi, nz):
    ndim, physics = PROPAGATORS[name][:2]
    shape = (nz,) + SMALL_SHAPES[ndim][1:]
    gpu, orc = _pair(lib, oracle, name, True, shape=shape)
    shp = orc.arr("V").shape
    DP, DM = _rand(shp, 41), _rand(shp, 42)
    img = _rand(shp, 43)
    mine = img.copy()
    a = orc.a
    if physics == "iso":
        gpu.abi.AdjointBornAccumulation_wavefieldsep(gpu.p, fptr(img), fptr(DP), isfwi)
        oracle.image_wavefieldsep(orc.g, isfwi, a["V"], a["B"], DP, a["POld"], None, None, mine)
    else:
        gpu.abi.AdjointBornAccumulation_wavefieldsep_V(gpu.p, fptr(img), fptr(DP), fptr(DM), isfwi)
        oracle.image_wavefieldsep(orc.g, isfwi, a["V"], a["B"], DP, a["POld"], DM, a["MOld"], mine)
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    err = rel_l2(img - _rand(shp, 43), mine - _rand(shp, 43))
    assert err <= 1e-5, f"rel L2 of the accumulated term {err:.3e}"
    gpu.close()


@pytest.mark.parametrize("name", ["Prop3DAcoIsoDenQ_DEO2_FDTD", "Prop3DAcoTTIDenQ_DEO2_FDTD"])
def test_host_writes_through_getters_in_a_loop(lib, oracle, name):
    """A time loop that asks for pCur before every step (as the reference's Julia loop does) stops
    moving that array back to the device after two steps; host writes into it, and into the model,
    made between steps through the getters' pointers must still reach the next step: bitwise against
    the restatement doing the same writes."""
    gpu, orc = _pair(lib, oracle, name, True)
    rng = np.random.default_rng(21)
    for it in range(8):
        gpu.arr("PCur")  # the getter, every step
        if it in (4, 6):  # host writes into the streaked array and into a model array
            d = (rng.standard_normal(gpu.arr("PCur").shape) * 1e-3).astype(np.float32)
            for r in (gpu, orc):
                a = r.arr("PCur")
                a[...] = a + d
            v = gpu.arr("V")
            v[2:5, 3:6] *= np.float32(1.01)
            w = orc.arr("V")
            w[2:5, 3:6] *= np.float32(1.01)
        gpu.abi.TimeStep(gpu.p)
        orc.step()
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    for k in _fields(name):
        assert same(gpu.arr(k), orc.arr(k)), f"{name} {k}: {mismatch_report(gpu.arr(k), orc.arr(k))}"
    gpu.close()
