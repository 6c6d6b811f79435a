"""Failure detection on the host (no GPU needed): the allocation fault injector.

WAVEFD_B200_FAIL_ALLOC=N makes the Nth allocation of the process fail without calling CUDA. The
object constructor then returns NULL with WFD_ERR_ALLOC and a message that names the injected
failure, and nothing it had allocated is left behind. Each case runs in its own process (the
count is process-wide)."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import ctypes, sys
sys.path.insert(0, {root!r})
from wavefd_b200 import _lib
from wavefd_b200.abi import PropagatorABI
lib = _lib.library()
abi = PropagatorABI(lib, "Prop3DAcoIsoDenQ_DEO2_FDTD")
p = abi.alloc(1, 1, 16, 16, 16, 4, 10.0, 10.0, 10.0, 0.001, 8, 8, 16)
print("NULL" if not p else "OBJECT", lib.WFD_LastError(), lib.WFD_LastErrorMessage().decode())
"""


def _probe(env_value):
    env = dict(os.environ)
    env.pop("WAVEFD_B200_FAIL_ALLOC", None)
    if env_value is not None:
        env["WAVEFD_B200_FAIL_ALLOC"] = env_value
    env["CUDA_VISIBLE_DEVICES"] = ""  # host-side paths only: no device is used by this test
    r = subprocess.run([sys.executable, "-c", PROBE.format(root=ROOT)], capture_output=True, text=True, env=env,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    return r.stdout.strip().splitlines()[-1]


def test_injected_allocation_failure_is_reported():
    out = _probe("1")
    assert out.startswith("NULL 2 "), out  # WFD_ERR_ALLOC
    assert "injected" in out and "WAVEFD_B200_FAIL_ALLOC" in out, out


def test_without_injection_no_injected_note():
    out = _probe(None)
    # no device here: the real allocation fails, and the message does not claim an injection
    assert "injected" not in out, out
