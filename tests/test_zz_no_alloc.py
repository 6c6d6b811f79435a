"""The allocation-free entry point (WFD_AdjointBornAccumulation_wavefieldsep_NoAlloc), for callers
that cannot call cudaMalloc, against the regular wavefield-separation entry point.

It is called through the C ABI on device arrays and must give the regular entry point's result
within the wavefield-separation tolerance of the other GPU tests (relative L2 1e-5), on two calls
in a row (the second call reuses the library's fixed scratch array left by the first). This file
is collected last so that a run stopping at the first failure has run everything else first.
"""
import ctypes

import numpy as np
import pytest

from tests.harness import ABIRunner, SMALL_SHAPES, fptr, make_model, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def lib():
    from wavefd_b200 import _lib
    lib = _lib.library()
    f = lib.WFD_AdjointBornAccumulation_wavefieldsep_NoAlloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_long] * 4 + [ctypes.c_void_p] * 7 + [ctypes.c_void_p]
    return lib


def _dev(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("name", ["Prop3DAcoIsoDenQ_DEO2_FDTD", "Prop3DAcoTTIDenQ_DEO2_FDTD",
                                  "Prop2DAcoVTIDenQ_DEO2_FDTD"])
@pytest.mark.parametrize("nz", [26, 32])  # Bluestein length and power-of-two length
@pytest.mark.parametrize("isfwi", [0, 1])
def test_no_alloc_matches_regular_entry_point(lib, name, nz, isfwi):
    import torch
    from wavefd_b200.abi import PROPAGATORS
    ndim, physics = PROPAGATORS[name][:2]
    shape = (nz,) + SMALL_SHAPES[ndim][1:]
    gpu = ABIRunner(lib, name, shape, fs=True)
    gpu.load(make_model(ndim, physics, shape, seed=7))
    shp = gpu.arr("V").shape
    rng = np.random.default_rng(11)
    DP = (rng.standard_normal(shp) * 1e-2).astype(np.float32)
    DM = (rng.standard_normal(shp) * 1e-2).astype(np.float32)
    img0 = (rng.standard_normal(shp) * 1e-3).astype(np.float32)
    aniso = physics != "iso"

    # regular entry point, twice, host arrays
    ref = img0.copy()
    for _ in range(2):
        if aniso:
            gpu.abi.AdjointBornAccumulation_wavefieldsep_V(gpu.p, fptr(ref), fptr(DP), fptr(DM), isfwi)
        else:
            gpu.abi.AdjointBornAccumulation_wavefieldsep(gpu.p, fptr(ref), fptr(DP), isfwi)
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0

    # allocation-free entry point, twice, device arrays; model and adjoint fields straight from
    # the object's managed arrays
    d_dp = torch.from_numpy(DP).cuda()
    d_dm = torch.from_numpy(DM).cuda()
    d_img = torch.from_numpy(img0).cuda()
    torch.cuda.synchronize()
    ptr = lambda g: ctypes.c_void_p(ctypes.cast(getattr(gpu.abi, "get" + g)(gpu.p), ctypes.c_void_p).value)
    nx, ny = shp[0], (shp[1] if ndim == 3 else 1)
    for _ in range(2):
        rc = lib.WFD_AdjointBornAccumulation_wavefieldsep_NoAlloc(
            nx, ny, nz, isfwi, ptr("V"), ptr("B"), _dev(d_dp), ptr("POld"),
            _dev(d_dm) if aniso else None, ptr("MOld") if aniso else None, _dev(d_img), None)
        assert rc == 0, lib.WFD_LastErrorMessage()
    torch.cuda.synchronize()
    got = d_img.cpu().numpy()
    err = rel_l2(got - img0, ref - img0)
    assert err <= TOL, f"{name} nz={nz} isfwi={isfwi}: rel L2 of the accumulated term {err:.3e}"
    gpu.close()


@pytest.mark.parametrize("nz", [2047, 2048])  # the largest Bluestein length (fills the scratch) and the limit
def test_no_alloc_at_the_size_limit(lib, nz):
    """nz = 2047: n = 4094, Bluestein length 8192, 20478 of the scratch's 20480 entries; nz = 2048:
    the largest accepted (power of two). Isotropic 2D, against the regular entry point."""
    import torch
    name = "Prop2DAcoIsoDenQ_DEO2_FDTD"
    shape = (nz, 1, 12)
    gpu = ABIRunner(lib, name, shape, fs=True)
    gpu.load(make_model(2, "iso", shape, seed=3))
    shp = gpu.arr("V").shape
    rng = np.random.default_rng(5)
    DP = (rng.standard_normal(shp) * 1e-2).astype(np.float32)
    img0 = (rng.standard_normal(shp) * 1e-3).astype(np.float32)
    ref = img0.copy()
    for _ in range(2):
        gpu.abi.AdjointBornAccumulation_wavefieldsep(gpu.p, fptr(ref), fptr(DP), 0)
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0
    d_dp = torch.from_numpy(DP).cuda()
    d_img = torch.from_numpy(img0).cuda()
    ptr = lambda g: ctypes.c_void_p(ctypes.cast(getattr(gpu.abi, "get" + g)(gpu.p), ctypes.c_void_p).value)
    for i in range(2):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        rc = lib.WFD_AdjointBornAccumulation_wavefieldsep_NoAlloc(shp[0], 1, nz, 0, ptr("V"), ptr("B"), _dev(d_dp),
                                                                  ptr("POld"), None, None, _dev(d_img), None)
        assert rc == 0, lib.WFD_LastErrorMessage()
        torch.cuda.synchronize()
        if i == 1:  # the first call on a device may load the library's module; the second allocates nothing
            assert torch.cuda.mem_get_info()[0] == free0, "device memory in use changed across a call"
    err = rel_l2(d_img.cpu().numpy() - img0, ref - img0)
    assert err <= TOL, f"nz={nz}: rel L2 of the accumulated term {err:.3e}"
    gpu.close()


def test_no_alloc_rejects_oversize_and_host_arrays(lib):
    import torch
    d = torch.zeros(16, device="cuda")
    p = _dev(d)
    assert lib.WFD_AdjointBornAccumulation_wavefieldsep_NoAlloc(1, 1, 2049, 0, p, p, p, p, None, None, p, None) != 0
    h = np.zeros(64, np.float32)
    hp = ctypes.c_void_p(h.ctypes.data)
    assert lib.WFD_AdjointBornAccumulation_wavefieldsep_NoAlloc(2, 1, 32, 0, hp, hp, hp, hp, None, None, hp, None) != 0
