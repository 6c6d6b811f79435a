"""The time step with the Born-V injection, the V imaging condition or the derivative scaling fused
into it (WFD_Prop_TimeStepBorn / WFD_Prop_TimeStepImage / WFD_Prop_TimeStepScaled) against the
reference's call sequence on the same library (TimeStep or TimeStepLinear, then
ForwardBornInjection_V, AdjointBornAccumulation_V or ScaleSpatialDerivatives), and against the
checker.

Strict build: bitwise (up to the sign of zero), fields and image, after several steps, for the 3D
propagators on TMA shapes (the epilogue inside the step kernel), on a shape whose nz is not a
multiple of 4 and in 2D (the separate kernels after the step). Fast build: relative L2 <= 1e-5.
"""
import ctypes

import numpy as np
import pytest

from tests.harness import ABIRunner, OracleRunner, make_model, mismatch_report, rel_l2
from wavefd_b200.abi import PROPAGATORS

pytestmark = pytest.mark.gpu

CASES = [("Prop3DAcoIsoDenQ_DEO2_FDTD", (40, 36, 44)), ("Prop3DAcoVTIDenQ_DEO2_FDTD", (40, 36, 44)),
         ("Prop3DAcoTTIDenQ_DEO2_FDTD", (40, 36, 44)), ("Prop3DAcoTTIDenQ_DEO2_FDTD", (37, 21, 30)),
         ("Prop3DAcoIsoDenQ_DEO2_FDTD", (37, 21, 30)), ("Prop2DAcoIsoDenQ_DEO2_FDTD", (44, 1, 38)),
         ("Prop2DAcoVTIDenQ_DEO2_FDTD", (44, 1, 38))]


@pytest.fixture(scope="module")
def lib():
    from wavefd_b200 import _lib
    lib = _lib.library()
    return lib


def _dev(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _fields(physics):
    return ["PCur", "POld", "PSpace"] + ([] if physics == "iso" else ["MCur", "MOld", "MSpace"])


@pytest.mark.parametrize("name,shape", CASES)
@pytest.mark.parametrize("kind", ["born", "image", "image_linear", "scaled"])
@pytest.mark.parametrize("strict", [True, False])
def test_fused_step_epilogue(lib, oracle, name, shape, kind, strict):
    import torch
    ndim, physics = PROPAGATORS[name][:2]
    aniso = physics != "iso"
    if kind == "image_linear" and physics != "vti":
        pytest.skip("the linear step is VTI only")
    model = make_model(ndim, physics, shape, seed=4)
    runs = []
    for fused in (True, False):
        gpu = ABIRunner(lib, name, shape)
        lib.WFD_Prop_SetStrict(ctypes.c_void_p(gpu.p), int(strict))
        gpu.load(model)
        shp = gpu.arr("V").shape
        rng = np.random.default_rng(12)
        dv = torch.from_numpy((rng.standard_normal(shp) * 0.02).astype(np.float32)).cuda()
        img = torch.from_numpy((rng.standard_normal(shp) * 1e-3).astype(np.float32)).cuda()
        dps = [torch.from_numpy((rng.standard_normal(shp) * 1e-2).astype(np.float32)).cuda() for _ in range(4)]
        dms = [torch.from_numpy((rng.standard_normal(shp) * 1e-2).astype(np.float32)).cuda() for _ in range(4)]
        torch.cuda.synchronize()
        for i in range(4):
            dp, dm = dps[i], dms[i] if aniso else None
            pp = ctypes.c_void_p(gpu.p)
            if fused:
                if kind == "born":
                    rc = lib.WFD_Prop_TimeStepBorn(pp, _dev(dv), _dev(dp), _dev(dm))
                elif kind == "scaled":
                    rc = lib.WFD_Prop_TimeStepScaled(pp)
                else:
                    rc = lib.WFD_Prop_TimeStepImage(pp, _dev(img), _dev(dp), _dev(dm), int(kind == "image_linear"))
                assert rc == 0, lib.WFD_Prop_Message(pp)
                assert lib.WFD_Prop_Synchronize(pp) == 0
            else:
                if kind == "image_linear":
                    gpu.abi.TimeStepLinear(gpu.p)
                else:
                    gpu.abi.TimeStep(gpu.p)
                f = ctypes.POINTER(ctypes.c_float)
                cast = lambda t: ctypes.cast(ctypes.c_void_p(t.data_ptr()), f) if t is not None else None
                if kind == "scaled":
                    gpu.abi.ScaleSpatialDerivatives(gpu.p)
                else:
                    args = [cast(dv if kind == "born" else img), cast(dp)] + ([cast(dm)] if aniso else [])
                    getattr(gpu.abi, "ForwardBornInjection_V" if kind == "born" else "AdjointBornAccumulation_V")(
                        gpu.p, *args)
            assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
        torch.cuda.synchronize()
        out = {k: gpu.arr(k).copy() for k in _fields(physics)}
        out["img"] = img.cpu().numpy()
        runs.append(out)
        gpu.close()
    fused_out, seq_out = runs
    for k in fused_out:
        a, b = fused_out[k], seq_out[k]
        if strict:
            assert np.array_equal(a, b), f"{name} {kind} {k}: {mismatch_report(a, b)}"
        else:
            assert rel_l2(a, b) <= 1e-5, f"{name} {kind} {k}: rel L2 {rel_l2(a, b):.2e}"


@pytest.mark.parametrize("name", ["Prop3DAcoIsoDenQ_DEO2_FDTD", "Prop3DAcoTTIDenQ_DEO2_FDTD"])
def test_fused_born_step_matches_checker(lib, oracle, name):
    """Strict build against the FP32 restatement: step, then Born-V injection, three times."""
    import torch
    ndim, physics = PROPAGATORS[name][:2]
    shape = (40, 36, 44)
    model = make_model(ndim, physics, shape, seed=6)
    gpu = ABIRunner(lib, name, shape)
    lib.WFD_Prop_SetStrict(ctypes.c_void_p(gpu.p), 1)
    gpu.load(model)
    orc = OracleRunner(oracle, name, shape)
    orc.load(model)
    shp = gpu.arr("V").shape
    rng = np.random.default_rng(3)
    dv = (rng.standard_normal(shp) * 0.02).astype(np.float32)
    dv_d = torch.from_numpy(dv).cuda()
    for _ in range(3):
        dp = (rng.standard_normal(shp) * 1e-2).astype(np.float32)
        dm = (rng.standard_normal(shp) * 1e-2).astype(np.float32)
        dp_d, dm_d = torch.from_numpy(dp).cuda(), torch.from_numpy(dm).cuda()
        torch.cuda.synchronize()
        assert lib.WFD_Prop_TimeStepBorn(ctypes.c_void_p(gpu.p), _dev(dv_d), _dev(dp_d), _dev(dm_d)) == 0
        assert lib.WFD_Prop_Synchronize(ctypes.c_void_p(gpu.p)) == 0
        orc.step()
        a = orc.a
        if physics == "iso":
            oracle.born_iso(orc.g, 0, a["V"], a["B"], dv, dv, dp, dp, a["PCur"])
        else:
            oracle.born_aniso_v(orc.g, a["V"], dv, dp, dm, a["PCur"], a["MCur"])
    for k in _fields(physics):
        assert np.array_equal(gpu.arr(k), orc.arr(k)), f"{k}: {mismatch_report(gpu.arr(k), orc.arr(k))}"
    gpu.close()
