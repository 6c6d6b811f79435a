"""The FP64 rerun (CPU, no GPU needed).

* The restatement instantiated in double (wfo64_*) against the reference's own pass templates
  instantiated in double (oracle/ref64_harness.cc, built from the reference's headers): bitwise for
  every propagator whose passes are written in the template type throughout. The 3D VTI pass 1
  declares its interior temporaries `float` (prop3DAcoVTIDenQ_DEO2_FDTD.h:902-949), so the
  reference's own double instantiation rounds them through FP32 there; it is compared at relative
  L2 <= 1e-5 instead, and the FP64 rerun used elsewhere is the restatement's.
* The FP32 restatement (pinned to the reference) against the FP64 rerun: relative L2 <= 1e-5 after
  20 steps, a sanity check of both (the GPU long-run tests report the errors on the workloads).
"""
import numpy as np
import pytest

from oracle.oracle import Ref64, ref64_available
from tests.harness import OracleRunner, OracleRunner64, Ref64Runner, SMALL_SHAPES, make_model, rel_l2
from wavefd_b200.abi import PROPAGATORS

NAMES = list(PROPAGATORS)


def _fields(physics):
    return ["PCur", "POld", "PSpace"] + ([] if physics == "iso" else ["MCur", "MOld", "MSpace"])


@pytest.mark.skipif(not ref64_available(), reason="FP64 reference harness not built (make -C oracle ref)")
@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("fs", [True, False])
def test_fp64_restatement_matches_reference_fp64(oracle, name, fs):
    ndim, physics = PROPAGATORS[name][:2]
    shape = SMALL_SHAPES[ndim]
    ref = Ref64Runner(Ref64(), oracle, name, shape, fs=fs)
    res = OracleRunner64(oracle, name, shape, fs=fs)
    model = make_model(ndim, physics, shape, seed=7)
    ref.load(model)
    res.load(model)
    for _ in range(8):
        ref.step()
        res.step()
    for k in _fields(physics):
        a, b = res.arr(k), ref.arr(k)
        if name == "Prop3DAcoVTIDenQ_DEO2_FDTD":
            assert rel_l2(a, b) <= 1e-5, f"{name} fs={fs} {k}: rel L2 {rel_l2(a, b):.2e}"
        else:
            assert np.array_equal(a, b), f"{name} fs={fs} {k}: max |diff| {np.abs(a - b).max():.3e}"


@pytest.mark.skipif(not ref64_available(), reason="FP64 reference harness not built (make -C oracle ref)")
def test_fp64_vti_linear_step(oracle):
    name = "Prop3DAcoVTIDenQ_DEO2_FDTD"
    shape = SMALL_SHAPES[3]
    ref = Ref64Runner(Ref64(), oracle, name, shape)
    res = OracleRunner64(oracle, name, shape)
    model = make_model(3, "vti", shape, seed=8)
    ref.load(model)
    res.load(model)
    for _ in range(6):
        ref.step(linear=True)
        res.step(linear=True)
    for k in ("PCur", "POld", "MCur", "MOld"):
        assert rel_l2(res.arr(k), ref.arr(k)) <= 1e-5


@pytest.mark.parametrize("name", NAMES)
def test_fp32_restatement_close_to_fp64(oracle, name):
    ndim, physics = PROPAGATORS[name][:2]
    shape = SMALL_SHAPES[ndim]
    f32 = OracleRunner(oracle, name, shape)
    f64 = OracleRunner64(oracle, name, shape)
    model = make_model(ndim, physics, shape, seed=9)
    f32.load(model)
    f64.load(model)
    for _ in range(20):
        f32.step()
        f64.step()
    for k in _fields(physics):
        err = rel_l2(f32.arr(k), f64.arr(k))
        assert err <= 1e-5, f"{name} {k}: FP32 vs FP64 rel L2 {err:.2e}"
