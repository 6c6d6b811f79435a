"""Failure detection on the GPU, without a GPU fault.

* A wait that runs out: the tile-load waits of the TMA step kernels are bounded (2 s). With the
  limit shortened to 1 ns (WFD_Debug_SetPipelineWait) a wait gives up while its copy is still in
  flight; the kernel records the timeout in its device status word, lets every copy it issued land
  (the drain waits keep their own limit) and leaves, and the object reports WFD_ERR_TIMEOUT. The
  context stays usable: with the limit restored a new object steps bitwise like the checker.
* An allocation that fails (WAVEFD_B200_FAIL_ALLOC, in a child process): the constructor returns
  NULL with WFD_ERR_ALLOC, and the next object of the same process works.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from tests.harness import ABIRunner, OracleRunner, make_model, mismatch_report

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WFD_ERR_TIMEOUT = 5


@pytest.fixture(scope="module")
def lib():
    from wavefd_b200 import _lib
    return _lib.library()


@pytest.mark.parametrize("name,physics", [("Prop3DAcoIsoDenQ_DEO2_FDTD", "iso"), ("Prop3DAcoVTIDenQ_DEO2_FDTD", "vti"),
                                          ("Prop3DAcoTTIDenQ_DEO2_FDTD", "tti")])
def test_wait_that_runs_out_reports_timeout(lib, oracle, name, physics):
    shape = (64, 48, 96)  # nz % 4 == 0: the TMA-staged step kernel
    gpu = ABIRunner(lib, name, shape)
    gpu.load(make_model(3, physics, shape, seed=1))
    lib.WFD_Debug_SetPipelineWait.restype = ctypes.c_int
    lib.WFD_Debug_SetPipelineWait.argtypes = [ctypes.c_ulonglong]
    try:
        assert lib.WFD_Debug_SetPipelineWait(1) == 0
        gpu.abi.TimeStep(gpu.p)
        status = lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p))
    finally:
        assert lib.WFD_Debug_SetPipelineWait(0) == 0
    gpu.close()
    assert status == WFD_ERR_TIMEOUT, f"status {status}"
    # the context is intact: a new object steps like the checker
    gpu = ABIRunner(lib, name, shape)
    lib.WFD_Prop_SetStrict(ctypes.c_void_p(gpu.p), 1)
    orc = OracleRunner(oracle, name, shape)
    model = make_model(3, physics, shape, seed=2)
    gpu.load(model)
    orc.load(model)
    for _ in range(3):
        gpu.abi.TimeStep(gpu.p)
        orc.step()
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    for k in ("PCur", "POld", "PSpace"):
        assert np.array_equal(gpu.arr(k), orc.arr(k)), f"{k}: {mismatch_report(gpu.arr(k), orc.arr(k))}"
    gpu.close()


PROBE = r"""
import ctypes, sys
sys.path.insert(0, {root!r})
from wavefd_b200 import _lib
from wavefd_b200.abi import PropagatorABI
lib = _lib.library()
abi = PropagatorABI(lib, "Prop3DAcoIsoDenQ_DEO2_FDTD")
p = abi.alloc(1, 1, 40, 36, 44, 4, 10.0, 10.0, 10.0, 0.001, 8, 8, 44)
print("first", "NULL" if not p else "OBJECT", lib.WFD_LastError(), lib.WFD_LastErrorMessage().decode())
q = abi.alloc(1, 1, 40, 36, 44, 4, 10.0, 10.0, 10.0, 0.001, 8, 8, 44)
abi.SetupDtOmegaInvQ(q, 5.0, 0.1, 100.0)
abi.TimeStep(q)
print("second", "NULL" if not q else "OBJECT", lib.WFD_Prop_Status(ctypes.c_void_p(q)))
abi.free(q)
"""


def test_injected_allocation_failure_then_recovery():
    env = dict(os.environ, WAVEFD_B200_FAIL_ALLOC="3")
    r = subprocess.run([sys.executable, "-c", PROBE.format(root=ROOT)], capture_output=True, text=True, env=env,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    first = [l for l in lines if l.startswith("first")][0]
    second = [l for l in lines if l.startswith("second")][0]
    assert first.startswith("first NULL 2 ") and "injected" in first, first
    assert second == "second OBJECT 0", second
