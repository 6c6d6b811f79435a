"""Pin the C restatement (oracle/) to the reference itself.

The reference's C++ is compiled from its own sources with IEEE semantics (oracle/_ref/strict),
driven through its C ABI, and compared bitwise (up to the sign of zero) with the restatement
on seeded models: every propagator, free surface on and off, several steps, the linear step,
the spatial-derivative scaling, the Q/sponge profile, Born injection, the imaging conditions,
and injection/extraction. Wavefield separation uses FFTs whose rounding differs (the reference
goes through a DFT shim, the restatement through a double-precision DFT), so it is held to a
tolerance instead.
"""
import ctypes

import numpy as np
import pytest

from oracle.oracle import reference_available, reference_lib
from tests.harness import (ABIRunner, OracleRunner, SMALL_SHAPES, fptr, make_model, mismatch_report, rel_l2,
                           same)
from wavefd_b200.abi import PROPAGATORS, SourcePoint32, SpacetimeABI

pytestmark = pytest.mark.skipif(not reference_available("strict"), reason="reference not built (make -C oracle ref)")

NAMES = list(PROPAGATORS)


def _pair(oracle, name, fs, seed=1):
    ndim = PROPAGATORS[name][0]
    shape = SMALL_SHAPES[ndim]
    ref = ABIRunner(reference_lib(name.replace("Prop", "prop"), "strict"), name, shape, fs=fs)
    orc = OracleRunner(oracle, name, shape, fs=fs)
    model = make_model(ndim, PROPAGATORS[name][1], shape, seed=seed)
    # 3D VTI has no DtOmegaInvQ getter; both sides then use the profile from SetupDtOmegaInvQ
    ref.load({k: v for k, v in model.items() if ref.abi.has("get" + k)})
    orc.load({k: v for k, v in model.items() if ref.abi.has("get" + k)})
    return ref, orc


def _compare(ref, orc, keys):
    for k in keys:
        a, b = ref.arr(k), orc.arr(k)
        assert same(a, b), f"{ref.name} {k}: {mismatch_report(a, b)}"


def _fields(name):
    physics = PROPAGATORS[name][1]
    return ["PCur", "POld", "PSpace"] + ([] if physics == "iso" else ["MCur", "MOld", "MSpace"])


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("fs", [True, False])
def test_timestep_bitwise(oracle, name, fs):
    ref, orc = _pair(oracle, name, fs)
    for _ in range(3):
        ref.abi.TimeStep(ref.p)
        orc.step()
    _compare(ref, orc, _fields(name))
    ref.close()


@pytest.mark.parametrize("name", [n for n in NAMES if PROPAGATORS[n][5]])
def test_timestep_linear_bitwise(oracle, name):
    ref, orc = _pair(oracle, name, True)
    for _ in range(2):
        ref.abi.TimeStepLinear(ref.p)
        orc.step(linear=True)
    _compare(ref, orc, ["PCur", "POld", "MCur", "MOld"])
    ref.close()


@pytest.mark.parametrize("name", NAMES)
def test_scale_bitwise(oracle, name):
    ref, orc = _pair(oracle, name, True)
    ref.abi.TimeStep(ref.p)
    orc.step()
    ref.abi.ScaleSpatialDerivatives(ref.p)
    orc.scale()
    _compare(ref, orc, ["PSpace"] + ([] if PROPAGATORS[name][1] == "iso" else ["MSpace"]))
    ref.close()


@pytest.mark.parametrize("name", [n for n in NAMES if "DtOmegaInvQ" in PROPAGATORS[n][2]])
@pytest.mark.parametrize("fs", [True, False])
@pytest.mark.parametrize("q", [(5.0, 0.1, 100.0), (12.0, 0.5, 40.0), (3.0, 0.0, 0.0)])
def test_q_profile_bitwise(oracle, name, fs, q):
    ref, orc = _pair(oracle, name, fs)
    ref.arr("DtOmegaInvQ")[...] = 0
    orc.arr("DtOmegaInvQ")[...] = 0
    ref.abi.SetupDtOmegaInvQ(ref.p, *q)
    g = orc.g
    oracle.setup_q(g, 6, q[0], q[1], q[2], orc.arr("DtOmegaInvQ"))
    _compare(ref, orc, ["DtOmegaInvQ"])
    ref.close()


def _rand(shape, seed, scale=1e-2):
    return (np.random.default_rng(seed).standard_normal(shape) * scale).astype(np.float32)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("variant", ["V", "VB", "B", "VEA"])
@pytest.mark.parametrize("fs", [True, False])
def test_born_injection_bitwise(oracle, name, variant, fs):
    physics = PROPAGATORS[name][1]
    if variant not in PROPAGATORS[name][3]:
        pytest.skip("variant not defined for this physics")
    ref, orc = _pair(oracle, name, fs)
    shp = orc.arr("V").shape
    dv, db, de, da = _rand(shp, 11), _rand(shp, 12), _rand(shp, 13), _rand(shp, 14)
    P, DP, M, DM = _rand(shp, 15), _rand(shp, 16), _rand(shp, 17), _rand(shp, 18)
    fn = getattr(ref.abi, "ForwardBornInjection_" + variant)
    a = orc.a
    if physics == "iso":
        args = {"V": (dv, DP), "VB": (dv, db, P, DP), "B": (db, P, DP)}[variant]
        fn(ref.p, *[fptr(x) for x in args])
        oracle.born_iso(orc.g, {"V": 0, "VB": 1, "B": 2}[variant], a["V"], a["B"], dv, db, P, DP, a["PCur"])
        keys = ["PCur"]
    elif variant == "V":
        fn(ref.p, fptr(dv), fptr(DP), fptr(DM))
        oracle.born_aniso_v(orc.g, a["V"], dv, DP, DM, a["PCur"], a["MCur"])
        keys = ["PCur", "MCur"]
    else:
        fn(ref.p, *[fptr(x) for x in (dv, de, da, P, M, DP, DM)])
        oracle.born_vea(orc.g, physics == "tti", a["V"], a["Eps"], a["Eta"], a["B"], a["F"], a["SinTheta"] if physics == "tti" else None,
                        a["CosTheta"] if physics == "tti" else None, a["SinPhi"], a["CosPhi"], dv, de, da, P, M, DP, DM,
                        a["PCur"], a["MCur"])
        keys = ["PCur", "MCur"]
    _compare(ref, orc, keys)
    ref.close()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("variant", ["V", "VB", "B", "VEA"])
@pytest.mark.parametrize("fs", [True, False])
def test_imaging_bitwise(oracle, name, variant, fs):
    physics = PROPAGATORS[name][1]
    if variant not in PROPAGATORS[name][4]:
        pytest.skip("variant not defined for this physics")
    ref, orc = _pair(oracle, name, fs)
    shp = orc.arr("V").shape
    P, DP, M, DM = _rand(shp, 25), _rand(shp, 26), _rand(shp, 27), _rand(shp, 28)
    img = {k: _rand(shp, 30 + i) for i, k in enumerate(("v", "b", "e", "a"))}
    mine = {k: v.copy() for k, v in img.items()}
    fn = getattr(ref.abi, "AdjointBornAccumulation_" + variant)
    a = orc.a
    if physics == "iso":
        if variant == "V":
            fn(ref.p, fptr(img["v"]), fptr(DP))
        elif variant == "VB":
            fn(ref.p, fptr(img["v"]), fptr(img["b"]), fptr(P), fptr(DP))
        else:
            fn(ref.p, fptr(img["b"]), fptr(P), fptr(DP))
        oracle.image_iso(orc.g, {"V": 0, "VB": 1, "B": 2}[variant], a["V"], a["B"], P, DP, a["POld"], mine["v"], mine["b"])
        keys = {"V": ["v"], "VB": ["v", "b"], "B": ["b"]}[variant]
    elif variant == "V":
        fn(ref.p, fptr(img["v"]), fptr(DP), fptr(DM))
        oracle.image_aniso_v(orc.g, a["V"], a["B"], DP, DM, a["POld"], a["MOld"], mine["v"])
        keys = ["v"]
    else:
        fn(ref.p, *[fptr(x) for x in (img["v"], img["e"], img["a"], P, M, DP, DM)])
        oracle.image_vea(orc.g, physics == "tti", a["V"], a["Eps"], a["Eta"], a["B"], a["F"],
                         a["SinTheta"] if physics == "tti" else None, a["CosTheta"] if physics == "tti" else None,
                         a["SinPhi"], a["CosPhi"], P, M, DP, DM, a["POld"], a["MOld"], mine["v"], mine["e"], mine["a"])
        keys = ["v", "e", "a"]
    for k in keys:
        assert same(img[k], mine[k]), f"{name} {variant} image {k}: {mismatch_report(img[k], mine[k])}"
    ref.close()


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("isfwi", [0, 1])
def test_wavefieldsep_close(oracle, name, isfwi):
    physics = PROPAGATORS[name][1]
    ref, orc = _pair(oracle, name, True)
    shp = orc.arr("V").shape
    DP, DM = _rand(shp, 41), _rand(shp, 42)
    img = np.zeros(shp, np.float32)
    mine = img.copy()
    a = orc.a
    if physics == "iso":
        ref.abi.AdjointBornAccumulation_wavefieldsep(ref.p, fptr(img), fptr(DP), isfwi)
        oracle.image_wavefieldsep(orc.g, isfwi, a["V"], a["B"], DP, a["POld"], None, None, mine)
    else:
        ref.abi.AdjointBornAccumulation_wavefieldsep_V(ref.p, fptr(img), fptr(DP), fptr(DM), isfwi)
        oracle.image_wavefieldsep(orc.g, isfwi, a["V"], a["B"], DP, a["POld"], DM, a["MOld"], mine)
    assert rel_l2(mine, img) < 2e-6, rel_l2(mine, img)
    ref.close()


def _points(n, npts_grid, nr, seed):
    rng = np.random.default_rng(seed)
    iu = np.sort(rng.integers(1, npts_grid + 1, n))  # sorted by iu with repeats, as source_blocking leaves them
    ir = rng.integers(1, nr + 1, n)
    c = rng.standard_normal(n).astype(np.float32)
    return iu, ir, c


def test_inject_extract_bitwise(oracle):
    lib = reference_lib("spacetime", "strict")
    st = SpacetimeABI(lib)
    ngrid, nr, nt = 500, 7, 13
    iu, ir, c = _points(300, ngrid, nr, 3)
    rng = np.random.default_rng(4)
    data = rng.standard_normal(nr * nt).astype(np.float32)
    field = rng.standard_normal(ngrid).astype(np.float32)
    pts = (SourcePoint32 * len(c))(*[SourcePoint32(int(a), int(b), float(x)) for a, b, x in zip(iu, ir, c)])
    parts = (ctypes.POINTER(SourcePoint32) * 1)(ctypes.cast(pts, ctypes.POINTER(SourcePoint32)))
    npp = (ctypes.c_long * 1)(len(c))
    f_ref, f_or = field.copy(), field.copy()
    st.injectdata_float(fptr(f_ref), fptr(data), 5, nt, parts, 1, npp, 1)
    oracle.inject(f_or, data, 5, nt, iu, ir, c)
    assert same(f_ref, f_or), mismatch_report(f_ref, f_or)
    d_ref, d_or = data.copy(), data.copy()
    st.extractdata_float(fptr(d_ref), fptr(field), parts, 1, npp, 9, nt, 1)
    oracle.extract(d_or, field, 9, nt, iu, ir, c)
    assert same(d_ref, d_or), mismatch_report(d_ref, d_or)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nh,nd", [(1, 7), (2, 8), (4, 13), (5, 40)])
def test_time_interpolation_bitwise(oracle, dtype, nh, nd):
    """spacetime.cc:4-127 (interp{forward,adjoint}_nd) against the restatement, both directions."""
    from wavefd_b200.abi import SpacetimeABI
    from wavefd_b200.spacetime import interp, interpfilters
    st = SpacetimeABI(reference_lib("spacetime", "strict"))
    rng = np.random.default_rng(nh * 100 + nd)
    h = interpfilters(0.001, 0.001 * nh, mode=0, dtype=dtype) + rng.standard_normal((nh, 8)).astype(dtype) * 1e-3
    for nm in (nd * nh - nh + 1, nd * nh, nd * nh - 2 * nh):
        if nm < 1:
            continue
        fine = rng.standard_normal((3, nm)).astype(dtype)
        coarse = rng.standard_normal((3, nd)).astype(dtype)
        want_f = interp(st, True, h, fine, nd)
        want_a = interp(st, False, h, coarse, nm)
        got_f = np.zeros_like(want_f)
        got_a = np.zeros_like(want_a)
        oracle.interp(True, h, got_f, fine, nh, nd, nm, 3)
        oracle.interp(False, h, got_a, coarse, nh, nm, nd, 3)
        assert np.array_equal(got_f, want_f), (nh, nd, nm)
        assert np.array_equal(got_a, want_a), (nh, nd, nm)


def test_illumination_bitwise(oracle):
    """illumination.c:3-53 (srcillum_helper_float, illum_accumulate_float) against the restatement."""
    lib = reference_lib("illumination", "strict")
    f32p = ctypes.POINTER(ctypes.c_float)
    lib.srcillum_helper_float.argtypes = [f32p, ctypes.c_size_t, ctypes.c_int]
    lib.illum_accumulate_float.argtypes = [f32p, f32p, ctypes.c_size_t, ctypes.c_int]
    rng = np.random.default_rng(9)
    f = rng.standard_normal(10001).astype(np.float32)
    acc = rng.standard_normal(10001).astype(np.float32)
    a1, a2 = acc.copy(), acc.copy()
    lib.illum_accumulate_float(fptr(a1), fptr(f.copy()), f.size, 4)
    oracle.illum(a2, f.copy())
    assert np.array_equal(a1, a2)
    g1, g2 = f.copy(), f.copy()
    lib.srcillum_helper_float(fptr(g1), f.size, 4)
    oracle.illum(None, g2)
    assert np.array_equal(g1, g2)
