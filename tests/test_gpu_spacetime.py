"""Injection/extraction on the GPU against the oracle (bitwise): the drop-in libspacetime
entry points with host and managed arrays, and the device-resident point tables."""
import ctypes

import numpy as np
import pytest

from tests.harness import fptr, mismatch_report, same
from wavefd_b200.abi import SourcePoint32, SpacetimeABI

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from wavefd_b200 import _lib
    return _lib.library()


def _points(n, ngrid, nr, seed, sort_by="iu"):
    rng = np.random.default_rng(seed)
    iu = rng.integers(1, ngrid + 1, n)
    ir = rng.integers(1, nr + 1, n)
    c = rng.standard_normal(n).astype(np.float32)
    order = np.argsort(iu if sort_by == "iu" else ir, kind="stable")
    return iu[order], ir[order], c[order]


def _partitions(key, iu, ir, c, nparts):
    """Split into contiguous partitions the way source_blocking does (equal keys kept together)."""
    n = len(c)
    bounds = [0]
    step = max(1, n // nparts)
    while bounds[-1] < n:
        b = min(n, bounds[-1] + step)
        while b < n and key[b] == key[b - 1]:
            b += 1
        bounds.append(b)
    parts = []
    keep = []
    for a, b in zip(bounds[:-1], bounds[1:]):
        arr = (SourcePoint32 * (b - a))(*[SourcePoint32(int(iu[i]), int(ir[i]), float(c[i])) for i in range(a, b)])
        keep.append(arr)
        parts.append(ctypes.cast(arr, ctypes.POINTER(SourcePoint32)))
    pp = (ctypes.POINTER(SourcePoint32) * len(parts))(*parts)
    npp = (ctypes.c_long * len(parts))(*[b - a for a, b in zip(bounds[:-1], bounds[1:])])
    return pp, npp, len(parts), keep


@pytest.mark.parametrize("nparts,npts,nr", [(1, 3000, 9), (4, 3000, 9), (3, 30000, 20000)])
def test_dropin_inject_extract_host_arrays(lib, oracle, nparts, npts, nr):
    """30000 points: the host loops over the points (comparison with the cached table, gather and
    scatter of the host arrays) run on the caller's threads."""
    st = SpacetimeABI(lib)
    ngrid, nt = 40000, 17
    iu, ir, c = _points(npts, ngrid, nr, 7)
    pp, npp, npart, keep = _partitions(iu, iu, ir, c, nparts)
    rng = np.random.default_rng(8)
    data = rng.standard_normal(nr * nt).astype(np.float32)
    field = rng.standard_normal(ngrid).astype(np.float32)
    f_gpu, f_or = field.copy(), field.copy()
    st.injectdata_float(fptr(f_gpu), fptr(data), 4, nt, pp, npart, npp, 4)
    oracle.inject(f_or, data, 4, nt, iu, ir, c)
    assert same(f_gpu, f_or), mismatch_report(f_gpu, f_or)
    iu2, ir2, c2 = _points(npts, ngrid, nr, 9, sort_by="ir")
    pp2, npp2, npart2, keep2 = _partitions(ir2, iu2, ir2, c2, nparts)
    d_gpu, d_or = data.copy(), data.copy()
    st.extractdata_float(fptr(d_gpu), fptr(field), pp2, npart2, npp2, 11, nt, 4)
    oracle.extract(d_or, field, 11, nt, iu2, ir2, c2)
    assert same(d_gpu, d_or), mismatch_report(d_gpu, d_or)
    # the same partitions again (the cached table), then changed contents behind the same pointers
    st.extractdata_float(fptr(d_gpu), fptr(field), pp2, npart2, npp2, 12, nt, 4)
    oracle.extract(d_or, field, 12, nt, iu2, ir2, c2)
    assert same(d_gpu, d_or), mismatch_report(d_gpu, d_or)
    first = keep2[-1]
    first[len(first) - 1].c = first[len(first) - 1].c * 0.5
    c2 = c2.copy()
    c2[-1] = np.float32(c2[-1] * np.float32(0.5))
    st.extractdata_float(fptr(d_gpu), fptr(field), pp2, npart2, npp2, 13, nt, 4)
    oracle.extract(d_or, field, 13, nt, iu2, ir2, c2)
    assert same(d_gpu, d_or), mismatch_report(d_gpu, d_or)


def test_dropin_inject_into_managed_field(lib, oracle):
    from wavefd_b200.props import PCur, Prop3DAcoIsoDenQ_DEO2_FDTD, free
    prop = Prop3DAcoIsoDenQ_DEO2_FDTD(nz=24, ny=20, nx=22, dz=10, dy=10, dx=10, dt=0.001)
    pcur = PCur(prop)
    rng = np.random.default_rng(3)
    pcur[...] = rng.standard_normal(pcur.shape).astype(np.float32)
    flat = pcur.reshape(-1)
    ref = flat.copy()
    st = SpacetimeABI(lib)
    iu, ir, c = _points(500, flat.size, 3, 4)
    pp, npp, npart, keep = _partitions(iu, iu, ir, c, 2)
    nt = 6
    data = rng.standard_normal(3 * nt).astype(np.float32)
    st.injectdata_float(flat.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), fptr(data), 2, nt, pp, npart, npp, 2)
    oracle.inject(ref, data, 2, nt, iu, ir, c)
    assert same(flat, ref), mismatch_report(flat, ref)
    free(prop)


def test_device_tables_inject_extract(lib, oracle):
    import torch
    ngrid, nr, nt = 5000, 11, 13
    iu, ir, c = _points(4000, ngrid, nr, 21)
    pts = (SourcePoint32 * len(c))(*[SourcePoint32(int(a), int(b), float(x)) for a, b, x in zip(iu, ir, c)])
    tin = lib.WFD_Points_Create(pts, len(c), 0)
    tout = lib.WFD_Points_Create(pts, len(c), 1)
    assert tin and tout
    rng = np.random.default_rng(22)
    data = rng.standard_normal(nr * nt).astype(np.float32)
    field = rng.standard_normal(ngrid).astype(np.float32)
    fd = torch.from_numpy(field).cuda()
    dd = torch.from_numpy(data).cuda()
    s = torch.cuda.current_stream().cuda_stream
    assert lib.WFD_Inject(tin, ctypes.c_void_p(fd.data_ptr()), ctypes.c_void_p(dd.data_ptr()), 5, nt, ctypes.c_void_p(s)) == 0
    assert lib.WFD_Extract(tout, ctypes.c_void_p(dd.data_ptr()), ctypes.c_void_p(fd.data_ptr()), 6, nt, ctypes.c_void_p(s)) == 0
    torch.cuda.synchronize()
    f_or, d_or = field.copy(), data.copy()
    oracle.inject(f_or, data, 5, nt, iu, ir, c)
    o2 = np.argsort(ir, kind="stable")
    oracle.extract(d_or, f_or, 6, nt, iu[o2], ir[o2], c[o2])
    assert same(fd.cpu().numpy(), f_or)
    assert same(dd.cpu().numpy(), d_or)
    lib.WFD_Points_Free(tin)
    lib.WFD_Points_Free(tout)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("nh,nd", [(1, 7), (4, 13), (8, 250)])
def test_time_interpolation_dropin_bitwise(lib, oracle, dtype, nh, nd):
    """interp{forward,adjoint}_nd_{float,double} (spacetime.cc:228-330) on the GPU, host arrays, against
    the restatement (pinned to the compiled reference)."""
    from wavefd_b200.spacetime import interp, interpfilters
    st = SpacetimeABI(lib)
    rng = np.random.default_rng(nh + nd)
    h = interpfilters(0.0005, 0.0005 * nh, dtype=dtype)
    nm = nd * nh - nh // 2
    fine = rng.standard_normal((5, nm)).astype(dtype)
    coarse = rng.standard_normal((5, nd)).astype(dtype)
    got_f = interp(st, True, h, fine, nd)
    got_a = interp(st, False, h, coarse, nm)
    want_f, want_a = np.zeros_like(got_f), np.zeros_like(got_a)
    oracle.interp(True, h, want_f, fine, nh, nd, nm, 5)
    oracle.interp(False, h, want_a, coarse, nh, nm, nd, 5)
    assert np.array_equal(got_f, want_f)
    assert np.array_equal(got_a, want_a)


def test_time_interpolation_device_and_streamed_extraction(lib, oracle):
    """WFD_Interp on device arrays, and WFD_ExtractInterp (extraction streamed into the forward
    interpolation) against extraction into a fine buffer followed by interpforward: bitwise."""
    import torch
    from wavefd_b200.spacetime import interpfilters
    nh, nd = 4, 60
    nm = nd * nh
    h = interpfilters(0.0005, 0.002)
    dh = torch.from_numpy(h).cuda()
    rng = np.random.default_rng(3)
    # device interpolation, both directions
    fine = rng.standard_normal((7, nm)).astype(np.float32)
    coarse = rng.standard_normal((7, nd)).astype(np.float32)
    out_f = torch.zeros((7, nd), device="cuda")
    out_a = torch.zeros((7, nm), device="cuda")
    assert lib.WFD_Interp(1, ctypes.c_void_p(dh.data_ptr()), ctypes.c_void_p(out_f.data_ptr()),
                          ctypes.c_void_p(torch.from_numpy(fine).cuda().data_ptr()), nh, nm, nd, 7, None) == 0
    assert lib.WFD_Interp(0, ctypes.c_void_p(dh.data_ptr()), ctypes.c_void_p(out_a.data_ptr()),
                          ctypes.c_void_p(torch.from_numpy(coarse).cuda().data_ptr()), nh, nm, nd, 7, None) == 0
    torch.cuda.synchronize()
    want_f, want_a = np.zeros((7, nd), np.float32), np.zeros((7, nm), np.float32)
    oracle.interp(True, h, want_f, fine, nh, nd, nm, 7)
    oracle.interp(False, h, want_a, coarse, nh, nm, nd, 7)
    assert np.array_equal(out_f.cpu().numpy(), want_f)
    assert np.array_equal(out_a.cpu().numpy(), want_a)
    # streamed extraction: 9 receivers (one spread over 3 points) on a 2000-cell field over nm steps
    ngrid, nrec = 2000, 9
    iu = np.concatenate([rng.integers(1, ngrid + 1, nrec), rng.integers(1, ngrid + 1, 2)])
    ir = np.concatenate([np.arange(1, nrec + 1), [4, 4]])
    c = rng.standard_normal(len(iu)).astype(np.float32)
    order = np.argsort(ir, kind="stable")
    iu, ir, c = iu[order], ir[order], c[order]
    pts = (SourcePoint32 * len(c))(*[SourcePoint32(int(a), int(b), float(w)) for a, b, w in zip(iu, ir, c)])
    tab = lib.WFD_Points_Create(ctypes.cast(pts, ctypes.POINTER(SourcePoint32)), len(c), 1)
    dcoarse = torch.zeros((nrec, nd), device="cuda")
    fine_traces = np.zeros((nrec, nm), np.float32)
    for it in range(1, nm + 1):
        field = rng.standard_normal(ngrid).astype(np.float32)
        dfield = torch.from_numpy(field).cuda()
        assert lib.WFD_ExtractInterp(tab, ctypes.c_void_p(dcoarse.data_ptr()), ctypes.c_void_p(dfield.data_ptr()),
                                     ctypes.c_void_p(dh.data_ptr()), nh, it, nm, nd, None) == 0
        oracle.extract(fine_traces.reshape(-1), field, it, nm, iu, ir, c)
        torch.cuda.synchronize()
    lib.WFD_Points_Free(tab)
    want = np.zeros((nrec, nd), np.float32)
    oracle.interp(True, h, want, fine_traces, nh, nd, nm, nrec)
    got = dcoarse.cpu().numpy()
    assert np.array_equal(got, want), mismatch_report(got, want)


def test_illumination_bitwise(lib, oracle):
    """srcillum_helper_float / illum_accumulate_float (illumination.c:3-53) on host and device arrays, and
    the WFD_IllumAccumulate add-on, against the restatement."""
    import torch
    f32p = ctypes.POINTER(ctypes.c_float)
    lib.srcillum_helper_float.argtypes = [f32p, ctypes.c_size_t, ctypes.c_int]
    lib.illum_accumulate_float.argtypes = [f32p, f32p, ctypes.c_size_t, ctypes.c_int]
    rng = np.random.default_rng(10)
    f = rng.standard_normal(100003).astype(np.float32)
    acc = rng.standard_normal(100003).astype(np.float32)
    want = acc.copy()
    oracle.illum(want, f.copy())
    a = acc.copy()
    lib.illum_accumulate_float(fptr(a), fptr(f.copy()), f.size, 4)  # host arrays
    assert np.array_equal(a, want)
    da, dfield = torch.from_numpy(acc.copy()).cuda(), torch.from_numpy(f).cuda()
    assert lib.WFD_IllumAccumulate(ctypes.c_void_p(da.data_ptr()), ctypes.c_void_p(dfield.data_ptr()), f.size,
                                   None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(da.cpu().numpy(), want)
    g, gw = f.copy(), f.copy()
    lib.srcillum_helper_float(fptr(g), f.size, 4)
    oracle.illum(None, gw)
    assert np.array_equal(g, gw)


@pytest.mark.parametrize("name,shape", [("Prop2DAcoIsoDenQ_DEO2_FDTD", (44, 1, 38)),
                                        ("Prop2DAcoVTIDenQ_DEO2_FDTD", (44, 1, 38)),
                                        ("Prop2DAcoTTIDenQ_DEO2_FDTD", (44, 1, 38)),
                                        ("Prop3DAcoTTIDenQ_DEO2_FDTD", (28, 22, 24))])
@pytest.mark.parametrize("use_graph", [1, 0])
def test_prop_run_matches_stepping(lib, name, shape, use_graph):
    """WFD_Prop_Run (a pair of steps with injection and extraction replayed from a CUDA graph, the time
    index on the device) against TimeStep + WFD_Inject + WFD_Extract per step: bitwise, pointer state
    included, over an odd number of steps."""
    import torch
    from tests.harness import ABIRunner, make_model
    from wavefd_b200.abi import PROPAGATORS
    ndim, physics = PROPAGATORS[name][:2]
    nz, ny, nx = shape
    nt, nsteps = 30, 11
    runs = []
    for mode in ("run", "steps"):
        g = ABIRunner(lib, name, shape, fs=True)
        lib.WFD_Prop_SetStrict(ctypes.c_void_p(g.p), 1)
        g.load(make_model(ndim, physics, shape, seed=4))
        ncell = nz * ny * nx
        src = (SourcePoint32 * 2)(SourcePoint32(ncell // 2 + 1, 1, 0.75), SourcePoint32(ncell // 2 + 3, 1, 0.25))
        rec = (SourcePoint32 * 3)(*[SourcePoint32(3 + i * nz * 5, i + 1, 1.0) for i in range(3)])
        ts = lib.WFD_Points_Create(ctypes.cast(src, ctypes.POINTER(SourcePoint32)), 2, 0)
        tr = lib.WFD_Points_Create(ctypes.cast(rec, ctypes.POINTER(SourcePoint32)), 3, 1)
        wav = torch.from_numpy(np.random.default_rng(1).standard_normal(nt).astype(np.float32)).cuda()
        trc = torch.zeros(3 * nt, device="cuda")
        torch.cuda.synchronize()
        g.abi.TimeStep(g.p)  # one ordinary step first (an odd pointer parity)
        stream = ctypes.c_void_p(lib.WFD_Prop_Stream(ctypes.c_void_p(g.p)))
        if mode == "run":
            assert lib.WFD_Prop_Run(ctypes.c_void_p(g.p), nsteps, 2, ts, ctypes.c_void_p(wav.data_ptr()), tr,
                                    ctypes.c_void_p(trc.data_ptr()), nt, use_graph) == 0
        else:
            for it in range(2, 2 + nsteps):
                assert lib.WFD_Prop_TimeStepAsync(ctypes.c_void_p(g.p), 1, 0) == 0
                pc = ctypes.c_void_p(ctypes.cast(g.abi.getPCur(g.p), ctypes.c_void_p).value)
                assert lib.WFD_Inject(ts, pc, ctypes.c_void_p(wav.data_ptr()), it, nt, stream) == 0
                assert lib.WFD_Extract(tr, ctypes.c_void_p(trc.data_ptr()), pc, it, nt, stream) == 0
        assert lib.WFD_Prop_Synchronize(ctypes.c_void_p(g.p)) == 0
        f = ["PCur", "POld", "PSpace"] + ([] if physics == "iso" else ["MCur", "MOld"])
        runs.append(({k: g.arr(k).copy() for k in f}, trc.cpu().numpy()))
        lib.WFD_Points_Free(ts)
        lib.WFD_Points_Free(tr)
        g.close()
    (fa, ta), (fb, tb) = runs
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), (k, mismatch_report(fa[k], fb[k]))
    assert np.array_equal(ta, tb)


@pytest.mark.parametrize("nrec", [0, 600])
def test_prop_run_index_advance(lib, nrec):
    """The time index of WFD_Prop_Run advances once per step whether the extraction launch has no
    receivers (one block, index advance only) or several blocks of them (the last block to finish
    advances it): the run equals TimeStep + WFD_Inject (+ WFD_Extract) per step, bitwise."""
    import torch
    from tests.harness import ABIRunner, make_model
    name, shape = "Prop2DAcoIsoDenQ_DEO2_FDTD", (44, 1, 38)
    nz, ny, nx = shape
    nt, nsteps = 40, 13
    runs = []
    for mode in ("run", "steps"):
        g = ABIRunner(lib, name, shape, fs=True)
        lib.WFD_Prop_SetStrict(ctypes.c_void_p(g.p), 1)
        g.load(make_model(2, "iso", shape, seed=6))
        ncell = nz * ny * nx
        src = (SourcePoint32 * 1)(SourcePoint32(ncell // 2 + 5, 1, 1.0))
        ts = lib.WFD_Points_Create(ctypes.cast(src, ctypes.POINTER(SourcePoint32)), 1, 0)
        tr = None
        if nrec:
            rec = (SourcePoint32 * nrec)(*[SourcePoint32((7 * i) % ncell + 1, i + 1, 1.0) for i in range(nrec)])
            tr = lib.WFD_Points_Create(ctypes.cast(rec, ctypes.POINTER(SourcePoint32)), nrec, 1)
        wav = torch.from_numpy(np.random.default_rng(2).standard_normal(nt).astype(np.float32)).cuda()
        trc = torch.zeros(max(nrec, 1) * nt, device="cuda")
        torch.cuda.synchronize()
        stream = ctypes.c_void_p(lib.WFD_Prop_Stream(ctypes.c_void_p(g.p)))
        if mode == "run":
            assert lib.WFD_Prop_Run(ctypes.c_void_p(g.p), nsteps, 1, ts, ctypes.c_void_p(wav.data_ptr()), tr,
                                    ctypes.c_void_p(trc.data_ptr()) if nrec else None, nt, 1) == 0
        else:
            for it in range(1, 1 + nsteps):
                assert lib.WFD_Prop_TimeStepAsync(ctypes.c_void_p(g.p), 1, 0) == 0
                pc = ctypes.c_void_p(ctypes.cast(g.abi.getPCur(g.p), ctypes.c_void_p).value)
                assert lib.WFD_Inject(ts, pc, ctypes.c_void_p(wav.data_ptr()), it, nt, stream) == 0
                if nrec:
                    assert lib.WFD_Extract(tr, ctypes.c_void_p(trc.data_ptr()), pc, it, nt, stream) == 0
        assert lib.WFD_Prop_Synchronize(ctypes.c_void_p(g.p)) == 0
        runs.append(({k: g.arr(k).copy() for k in ("PCur", "POld", "PSpace")}, trc.cpu().numpy()))
        lib.WFD_Points_Free(ts)
        if tr:
            lib.WFD_Points_Free(tr)
        g.close()
    (fa, ta), (fb, tb) = runs
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), (k, mismatch_report(fa[k], fb[k]))
    assert np.array_equal(ta, tb)
    if nrec:
        assert np.count_nonzero(ta.reshape(nrec, nt)[:, :nsteps]) > 0


@pytest.mark.parametrize("name,shape", [("Prop3DAcoIsoDenQ_DEO2_FDTD", (36, 21, 30)),
                                        ("Prop3DAcoIsoDenQ_DEO2_FDTD", (37, 21, 30)),
                                        ("Prop3DAcoVTIDenQ_DEO2_FDTD", (28, 22, 24)),
                                        ("Prop3DAcoVTIDenQ_DEO2_FDTD", (30, 22, 24)),
                                        ("Prop3DAcoTTIDenQ_DEO2_FDTD", (28, 22, 24)),
                                        ("Prop2DAcoIsoDenQ_DEO2_FDTD", (44, 1, 38))])
def test_illumination_fused_into_step(lib, name, shape):
    """WFD_Prop_SetIllumination: every step adds pCur^2 (the field it reads) to the sum, inside the 3D
    Iso, VTI and TTI step kernels (nz % 4 == 0) or as a separate pass otherwise (nz % 4 != 0, 2D);
    bitwise against float32 numpy."""
    import torch
    from tests.harness import ABIRunner, make_model
    from wavefd_b200.abi import PROPAGATORS
    ndim, physics = PROPAGATORS[name][:2]
    g = ABIRunner(lib, name, shape, fs=True)
    g.load(make_model(ndim, physics, shape, seed=6))
    n = int(np.prod(shape))
    acc = torch.zeros(n, device="cuda")
    torch.cuda.synchronize()
    assert lib.WFD_Prop_SetIllumination(ctypes.c_void_p(g.p), ctypes.c_void_p(acc.data_ptr())) == 0
    want = np.zeros(n, np.float32)
    for _ in range(4):
        pc = g.arr("PCur").reshape(-1).copy()
        want = want + pc * pc  # float32: one rounding per operation
        g.abi.TimeStep(g.p)
    assert lib.WFD_Prop_Status(ctypes.c_void_p(g.p)) == 0
    torch.cuda.synchronize()
    assert np.array_equal(acc.cpu().numpy(), want)
    assert lib.WFD_Prop_SetIllumination(ctypes.c_void_p(g.p), None) == 0
    g.close()


@pytest.mark.parametrize("spread", ["local", "far"])
@pytest.mark.parametrize("shape", [(200, 1, 90), (1000, 1, 400)])
@pytest.mark.parametrize("name", ["Prop2DAcoIsoDenQ_DEO2_FDTD", "Prop2DAcoVTIDenQ_DEO2_FDTD",
                                  "Prop2DAcoTTIDenQ_DEO2_FDTD"])
def test_prop_run_2d_tiles(lib, spread, shape, name):
    """The 2D whole-loop launch on a grid of many tiles in both directions (16 x 64 cells each),
    receiver groups of two points one row apart or 40 rows apart (more than two tiles), sources in one
    tile, on a tile corner, on the free-surface rows and outside the interior (cells the step does
    not write), against TimeStep + WFD_Inject + WFD_Extract per step, bitwise (strict build). At
    200 x 90 (24 tiles) every tile stays in one CTA for the whole loop; at 1000 x 400 (400 tiles,
    more than the CTAs that fit at once) the CTAs take turns over the tiles (2D Iso; the 2D VTI and TTI
    loop always shares the tiles out over the CTAs)."""
    import torch
    from tests.harness import ABIRunner, make_model
    from wavefd_b200.abi import PROPAGATORS
    physics = PROPAGATORS[name][1]
    nz, ny, nx = shape
    nt, nsteps = 40, 17
    gap = nz * (1 if spread == "local" else 40)  # the second point of a group: 1 or 40 rows further in x
    pts = []
    for i in range(12):
        k = (5 + 6 * i) * nz + 7 + 13 * i
        pts.append(SourcePoint32(k + 1, i + 1, 0.6))
        pts.append(SourcePoint32(min(k + gap, nz * nx - 1) + 1, i + 1, 0.4))
    runs = []
    for mode in ("run", "steps"):
        g = ABIRunner(lib, name, shape, fs=True)
        lib.WFD_Prop_SetStrict(ctypes.c_void_p(g.p), 1)
        g.load(make_model(2, physics, shape, seed=8))
        h = nx // 2
        spts = [SourcePoint32(h * nz + 3, 1, 1.0),             # free-surface row kz 2
                SourcePoint32(h * nz + 6, 2, 0.5),             # the same tile
                SourcePoint32(h * nz + 6, 1, 0.25),            # the same cell, a second contribution
                SourcePoint32(1 * nz + 10, 2, 0.75),           # row x 1: outside the interior
                SourcePoint32((h + 1) * nz + nz - 1, 1, 0.6),  # kz nz-2: outside the interior
                SourcePoint32(80 * nz + 64 + 1, 2, 0.3)]       # the tile corner (x 80, z 64)
        src = (SourcePoint32 * len(spts))(*spts)
        ts = lib.WFD_Points_Create(ctypes.cast(src, ctypes.POINTER(SourcePoint32)), len(spts), 0)
        rec = (SourcePoint32 * len(pts))(*pts)
        tr = lib.WFD_Points_Create(ctypes.cast(rec, ctypes.POINTER(SourcePoint32)), len(pts), 1)
        wav = torch.from_numpy(np.random.default_rng(3).standard_normal(2 * nt).astype(np.float32)).cuda()
        trc = torch.zeros(12 * nt, device="cuda")
        torch.cuda.synchronize()
        stream = ctypes.c_void_p(lib.WFD_Prop_Stream(ctypes.c_void_p(g.p)))
        if mode == "run":
            assert lib.WFD_Prop_Run(ctypes.c_void_p(g.p), nsteps, 1, ts, ctypes.c_void_p(wav.data_ptr()), tr,
                                    ctypes.c_void_p(trc.data_ptr()), nt, 1) == 0
            assert lib.WFD_Prop_RunLaunches(ctypes.c_void_p(g.p)) == 1
        else:
            for it in range(1, 1 + nsteps):
                assert lib.WFD_Prop_TimeStepAsync(ctypes.c_void_p(g.p), 1, 0) == 0
                pc = ctypes.c_void_p(ctypes.cast(g.abi.getPCur(g.p), ctypes.c_void_p).value)
                assert lib.WFD_Inject(ts, pc, ctypes.c_void_p(wav.data_ptr()), it, nt, stream) == 0
                assert lib.WFD_Extract(tr, ctypes.c_void_p(trc.data_ptr()), pc, it, nt, stream) == 0
        assert lib.WFD_Prop_Synchronize(ctypes.c_void_p(g.p)) == 0
        assert lib.WFD_Prop_Status(ctypes.c_void_p(g.p)) == 0
        keys = ("PCur", "POld", "PSpace") + (() if physics == "iso" else ("MCur", "MOld", "MSpace"))
        runs.append(({k: g.arr(k).copy() for k in keys}, trc.cpu().numpy()))
        lib.WFD_Points_Free(ts)
        lib.WFD_Points_Free(tr)
        g.close()
    (fa, ta), (fb, tb) = runs
    for k in fa:
        assert np.array_equal(fa[k], fb[k]), (k, mismatch_report(fa[k], fb[k]))
    assert np.array_equal(ta, tb)
    assert np.count_nonzero(ta) > 0
