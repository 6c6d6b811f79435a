"""Batched shots on the GPU: a ShotBatch of uneven Iso/VTI/TTI objects against the same objects
stepped one by one through the C ABI (with injection and extraction through the device point
tables). Strict build: bitwise; fast build: relative L2 <= 1e-5. The batch's CUDA graph, every plan
and the autotuner (which must restore what its trial launches overwrite) give the same results.
Ginsu crop / scatter-add against numpy (bitwise)."""
import ctypes

import numpy as np
import pytest

from tests.harness import ABIRunner, make_model, mismatch_report, rel_l2, same
from wavefd_b200.spacetime import SOURCEPOINT32

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-5
# (name, (nz, ny, nx)): uneven windows, several x-chunks for small chunk targets, partial tiles
SHOTS = [
    ("Prop3DAcoIsoDenQ_DEO2_FDTD", (36, 21, 50)),
    ("Prop3DAcoVTIDenQ_DEO2_FDTD", (40, 30, 37)),
    ("Prop3DAcoIsoDenQ_DEO2_FDTD", (28, 22, 24)),
    ("Prop3DAcoTTIDenQ_DEO2_FDTD", (32, 20, 33)),
    ("Prop3DAcoVTIDenQ_DEO2_FDTD", (44, 26, 61)),
]
NT = 12


@pytest.fixture(scope="module")
def lib():
    from wavefd_b200 import _lib
    return _lib.library()


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _acq(shape, seed):
    """A few source points near the centre (one wavelet trace) and a surface receiver line with one
    off-grid receiver spread over two cells."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    cell = lambda x, y, z: (x * ny + y) * nz + z + 1
    src = np.zeros(4, SOURCEPOINT32)
    for i, (dx, dy, dz) in enumerate([(0, 0, 0), (1, 0, 0), (0, 1, 1), (0, 0, 1)]):
        src[i] = (cell(nx // 2 + dx, ny // 2 + dy, nz // 2 + dz), 1, rng.uniform(0.2, 1.0))
    xs = np.arange(5, nx - 5, 3)
    rec = np.zeros(len(xs) + 2, SOURCEPOINT32)
    for i, x in enumerate(xs):
        rec[i] = (cell(x, ny // 2, 2), i + 1, 1.0)
    rec[len(xs)] = (cell(6, 6, 3), len(xs) + 1, 0.25)
    rec[len(xs) + 1] = (cell(6, 7, 3), len(xs) + 1, 0.75)
    return src, rec, len(xs) + 1


class Shot:
    def __init__(self, lib, torch, name, shape, seed, strict):
        self.runner = ABIRunner(lib, name, shape, fs=True)
        self.p = self.runner.p
        lib.WFD_Prop_SetStrict(ctypes.c_void_p(self.p), int(strict))
        ndim, physics = 3, self.runner.physics
        self.runner.load(make_model(ndim, physics, shape, seed=seed))
        self.src, self.rec, self.nrec = _acq(shape, seed)
        rng = np.random.default_rng(100 + seed)
        self.wavelet = torch.from_numpy(rng.standard_normal(NT).astype(np.float32)).cuda()
        self.traces = torch.zeros(self.nrec * NT, device="cuda")
        self.physics = physics

    def fields(self):
        f = ["PCur", "POld", "PSpace"] + ([] if self.physics == "iso" else ["MCur", "MOld", "MSpace"])
        return {k: self.runner.arr(k).copy() for k in f}


def _make(lib, torch, strict, seed0=0):
    shots = [Shot(lib, torch, n, s, seed0 + i, strict) for i, (n, s) in enumerate(SHOTS)]
    torch.cuda.synchronize()
    return shots


def _step_alone(lib, shots, nsteps, it0=1):
    from wavefd_b200.abi import SourcePoint32
    tabs = []
    for s in shots:
        ts = lib.WFD_Points_Create(s.src.ctypes.data_as(ctypes.POINTER(SourcePoint32)), len(s.src), 0)
        tr = lib.WFD_Points_Create(s.rec.ctypes.data_as(ctypes.POINTER(SourcePoint32)), len(s.rec), 1)
        tabs.append((ts, tr))
    for k in range(nsteps):
        it = it0 + k
        for s, (ts, tr) in zip(shots, tabs):
            s.runner.abi.TimeStep(s.p)
            stream = ctypes.c_void_p(lib.WFD_Prop_Stream(ctypes.c_void_p(s.p)))
            pc = ctypes.c_void_p(ctypes.cast(s.runner.abi.getPCur(s.p), ctypes.c_void_p).value)
            if it <= NT:
                assert lib.WFD_Inject(ts, pc, ctypes.c_void_p(s.wavelet.data_ptr()), it, NT, stream) == 0
                assert lib.WFD_Extract(tr, ctypes.c_void_p(s.traces.data_ptr()), pc, it, NT, stream) == 0
            assert lib.WFD_Prop_Synchronize(ctypes.c_void_p(s.p)) == 0
    for ts, tr in tabs:
        lib.WFD_Points_Free(ts)
        lib.WFD_Points_Free(tr)


def _batch(shots, plan=None):
    from wavefd_b200.batch import ShotBatch
    b = ShotBatch([s.runner for s in shots])
    for i, s in enumerate(shots):
        b.set_acquisition(i, s.src, s.wavelet, s.rec, s.traces, NT)
    if plan is not None:
        b.plan(*plan)
    return b


def _compare(a_shots, b_shots, strict, what):
    for i, (a, b) in enumerate(zip(a_shots, b_shots)):
        fa, fb = a.fields(), b.fields()
        fa["traces"] = a.traces.cpu().numpy()
        fb["traces"] = b.traces.cpu().numpy()
        for k in fa:
            if strict:
                assert same(fa[k], fb[k]), f"{what} shot {i} {k}: {mismatch_report(fa[k], fb[k])}"
            else:
                assert rel_l2(fa[k], fb[k]) <= FAST_TOL, f"{what} shot {i} {k}: rel L2 {rel_l2(fa[k], fb[k]):.2e}"


def _close(shots):
    for s in shots:
        s.runner.close()


@pytest.mark.parametrize("strict", [True, False])
def test_batch_matches_objects_stepped_alone(lib, torch, strict):
    ref = _make(lib, torch, strict)
    _step_alone(lib, ref, 7)
    shots = _make(lib, torch, strict)
    b = _batch(shots, plan=(16, 0, True))
    b.run(7, it0=1, graph=True)  # three graph replays and one single step
    b.synchronize()
    info = b.info()
    assert info["classes"]["iso"]["shots"] == 2 and info["classes"]["vti"]["shots"] == 2
    assert info["classes"]["tti"]["shots"] == 1
    _compare(ref, shots, strict, "batch vs alone")
    b.free()
    _close(ref)
    _close(shots)


def test_batch_graph_and_plans_agree(lib, torch):
    base = _make(lib, torch, True)
    b0 = _batch(base, plan=(0, 0, True))
    b0.run(5, graph=False)
    b0.synchronize()
    for plan in [(16, 1, False), (24, 0, False), (48, 1, True)]:
        shots = _make(lib, torch, True)
        b = _batch(shots, plan=plan)
        # split runs: the parity bookkeeping across calls (odd then even counts)
        b.run(3, it0=1, graph=True)
        b.run(2, it0=4, graph=True)
        b.synchronize()
        _compare(base, shots, True, f"plan {plan}")
        b.free()
        _close(shots)
    b0.free()
    _close(base)


def test_batch_tuner_restores_state(lib, torch):
    ref = _make(lib, torch, True)
    bref = _batch(ref, plan=(32, 0, True))
    bref.run(4)
    bref.synchronize()
    shots = _make(lib, torch, True)
    b = _batch(shots)
    b.run(1)
    b.tune(reps=1)
    info = b.info()
    assert info["tuned"]
    b.run(3, it0=2)
    b.synchronize()
    _compare(ref, shots, True, "tuned")
    b.free()
    bref.free()
    _close(ref)
    _close(shots)


def test_ginsu_crop_and_accumulate(torch):
    from wavefd_b200.batch import ginsu_accumulate, ginsu_crop
    rng = np.random.default_rng(3)
    S = (30, 25, 40)  # (nx, ny, nz) of the survey
    survey = rng.standard_normal(S).astype(np.float32)
    d_survey = torch.from_numpy(survey).cuda()
    for origin, shape in [((3, 4, 0), (10, 12, 40)), ((-4, 20, 8), (12, 9, 36))]:
        d_shot = torch.empty(shape, device="cuda")
        ginsu_crop(d_survey, S, origin, d_shot, shape)
        xs = np.clip(origin[0] + np.arange(shape[0]), 0, S[0] - 1)
        ys = np.clip(origin[1] + np.arange(shape[1]), 0, S[1] - 1)
        zs = np.clip(origin[2] + np.arange(shape[2]), 0, S[2] - 1)
        want = survey[np.ix_(xs, ys, zs)]
        torch.cuda.synchronize()
        assert np.array_equal(d_shot.cpu().numpy(), want)
        img = rng.standard_normal(shape).astype(np.float32)
        acc = rng.standard_normal(S).astype(np.float32)
        d_acc = torch.from_numpy(acc).cuda()
        ginsu_accumulate(d_acc, S, origin, torch.from_numpy(img).cuda(), shape)
        torch.cuda.synchronize()
        for x in range(shape[0]):
            for y in range(shape[1]):
                sx, sy = origin[0] + x, origin[1] + y
                if not (0 <= sx < S[0] and 0 <= sy < S[1]):
                    continue
                for z in range(shape[2]):
                    sz = origin[2] + z
                    if 0 <= sz < S[2]:
                        acc[sx, sy, sz] = np.float32(acc[sx, sy, sz] + img[x, y, z])
        assert np.array_equal(d_acc.cpu().numpy(), acc)
