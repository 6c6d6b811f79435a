"""Parity over whole records: the CUDA library through the reference's C ABI and its call sequence
(TimeStep, injectdata_float, extractdata_float with host partitions), against the FP32
restatement, with every result's error against the FP64 rerun stated.

* 2D AcoIsoDenQ, the reference's CPU-runnable workload whole: 501 x 501, 10 m, dt 1 ms,
  nt 2000, 60-cell sponge, constant Q 100, 15 Hz causal Ricker at the centre of the top row,
  receivers on every surface cell.
* 3D AcoIsoDenQ, AcoVTIDenQ and AcoTTIDenQ on 96^3 (the 3D workloads' model generator: layered
  plus smooth random velocity, Gardner density, block Q with the sponge ramp, layered anisotropy,
  smooth random tilt and azimuth), 10 m, dt 0.5 ms, 1000 steps, 20-cell sponge, 12 Hz causal
  Ricker near the surface centre, 16 x 16 surface receivers.

Strict build: bitwise equal to the FP32 restatement (up to the sign of zero) after the whole
record, wavefields and traces, hence within any tolerance of the reference.

Fast build (FMA contraction, approximate division and square root): over a whole record the
reference's own FP32 result drifts from the FP64 rerun by rounding alone (relative L2 about 1e-5
on the 2D record, 1-2e-4 on the 3D ones after 1000 steps), and any FP32 evaluation that rounds
differently drifts by the same amount, so a fixed 1e-5 bound against the FP32 result cannot hold
there. The fast build is held to relative L2 <= max(1e-5, 2 x the FP32 restatement's own error
against FP64), field by field: it is no further from the reference than the reference is from exact
arithmetic. (Over 40 steps the fast build is held to 1e-5 in test_gpu_parity.py.)

Each result's relative L2 against the FP64 rerun is printed (and appended as JSON lines to the
file named by WFD_PARITY_REPORT, when set).
"""
import ctypes
import json
import os

import numpy as np
import pytest

from tests.harness import ABIRunner, OracleRunner, OracleRunner64, fptr, rel_l2
from wavefd_b200.abi import SpacetimeABI
from wavefd_b200.spacetime import _partition_args, causal_ricker, receiver_blocking, source_blocking

pytestmark = pytest.mark.gpu

FAST_TOL = 1e-5

CASES = {
    "iso2d_501": dict(name="Prop2DAcoIsoDenQ_DEO2_FDTD", physics="iso", ndim=2, nx=501, ny=1, nz=501, d=10.0,
                      dt=0.001, nt=2000, nsponge=60, fpeak=15.0, q_model=False),
    "iso3d_96": dict(name="Prop3DAcoIsoDenQ_DEO2_FDTD", physics="iso", ndim=3, nx=96, ny=96, nz=96, d=10.0,
                     dt=0.0005, nt=1000, nsponge=20, fpeak=12.0, q_model=True),
    "vti3d_96": dict(name="Prop3DAcoVTIDenQ_DEO2_FDTD", physics="vti", ndim=3, nx=96, ny=96, nz=96, d=10.0,
                     dt=0.0005, nt=1000, nsponge=20, fpeak=12.0, q_model=True),
    "tti3d_96": dict(name="Prop3DAcoTTIDenQ_DEO2_FDTD", physics="tti", ndim=3, nx=96, ny=96, nz=96, d=10.0,
                     dt=0.0005, nt=1000, nsponge=20, fpeak=12.0, q_model=True),
}


@pytest.fixture(scope="module")
def lib():
    from wavefd_b200 import _lib
    return _lib.library()


def _model(c):
    from wavefd_b200 import synthetic
    shp = (c["nx"], c["ny"], c["nz"])
    m = synthetic.earth_model(shp, c["physics"], seed=1, d=c["d"], dt=c["dt"], nsponge=c["nsponge"],
                              q_blocks=c["q_model"], device="cpu")
    out = {}
    for k, t in m.items():
        if k == "DtOmegaInvQ" and not c["q_model"]:
            continue  # constant Q: the object's own sponge profile (SetupDtOmegaInvQ)
        a = t.numpy()
        out[k] = np.ascontiguousarray(a.reshape(c["nx"], c["nz"]) if c["ndim"] == 2 else a)
    return out


def _acquisition(c):
    from wavefd_b200 import synthetic
    if c["ndim"] == 2:
        return synthetic.surface_acquisition_2d((c["nx"], c["nz"]), c["d"])
    shp = (c["nx"], c["ny"], c["nz"])
    return synthetic.center_source(shp, c["d"]), synthetic.surface_receivers(shp, 16, 16, c["nsponge"])


def _fields(physics):
    return ["PCur", "POld", "PSpace"] + ([] if physics == "iso" else ["MCur", "MOld", "MSpace"])


_ORACLE = {}


def _oracle_run(oracle, key):
    """FP32 restatement and FP64 rerun over the whole record (cached per case)."""
    if key in _ORACLE:
        return _ORACLE[key]
    c = CASES[key]
    shape = (c["nz"], c["ny"], c["nx"])
    model = _model(c)
    src, rec = _acquisition(c)
    nt = c["nt"]
    wav = causal_ricker(c["dt"] * np.arange(nt), f=c["fpeak"]).astype(np.float32)
    kw = dict(fs=True, nsponge=c["nsponge"], dx=c["d"], dt=c["dt"])
    r32 = OracleRunner(oracle, c["name"], shape, **kw)
    r64 = OracleRunner64(oracle, c["name"], shape, **kw)
    r32.load(model)
    r64.load(model)
    tr32 = np.zeros(len(rec) * nt, np.float32)
    tr64 = np.zeros(len(rec) * nt, np.float64)
    wav64 = wav.astype(np.float64)
    for it in range(1, nt + 1):
        r32.step()
        r64.step()
        oracle.inject(r32.arr("PCur"), wav, it, nt, src["iu"], src["ir"], src["c"])
        oracle.extract(tr32, r32.arr("PCur"), it, nt, rec["iu"], rec["ir"], rec["c"])
        oracle.inject64(r64.arr("PCur"), wav64, it, nt, src["iu"], src["ir"], src["c"])
        oracle.extract64(tr64, r64.arr("PCur"), it, nt, rec["iu"], rec["ir"], rec["c"])
    res = ({k: r32.arr(k).copy() for k in _fields(c["physics"])}, tr32,
           {k: r64.arr(k).copy() for k in _fields(c["physics"])}, tr64, model, src, rec, wav)
    _ORACLE[key] = res
    return res


def _gpu_run(lib, key, strict, model, src, rec, wav):
    c = CASES[key]
    shape = (c["nz"], c["ny"], c["nx"])
    gpu = ABIRunner(lib, c["name"], shape, fs=True, nsponge=c["nsponge"], dx=c["d"], dt=c["dt"])
    lib.WFD_Prop_SetStrict(ctypes.c_void_p(gpu.p), int(strict))
    gpu.load(model)
    st = SpacetimeABI(lib)
    sp, sc = _partition_args(sb := source_blocking(src, 4))
    rp, rc = _partition_args(rb := receiver_blocking(rec, 4))
    nt = c["nt"]
    traces = np.zeros(len(rec) * nt, np.float32)
    getp = getattr(gpu.abi, "getPCur")
    for it in range(1, nt + 1):
        gpu.abi.TimeStep(gpu.p)
        pc = getp(gpu.p)
        st.injectdata_float(pc, fptr(wav), it, nt, sp, len(sb), sc, 4)
        st.extractdata_float(fptr(traces), pc, rp, len(rb), rc, it, nt, 4)
    assert lib.WFD_Prop_Status(ctypes.c_void_p(gpu.p)) == 0, lib.WFD_Prop_Message(ctypes.c_void_p(gpu.p))
    out = {k: gpu.arr(k).copy() for k in _fields(c["physics"])}
    gpu.close()
    return out, traces


def _report(rec):
    line = json.dumps(rec)
    print(line)
    path = os.environ.get("WFD_PARITY_REPORT")
    if path:
        with open(path, "a") as f:
            f.write(line + "\n")


@pytest.mark.parametrize("key", list(CASES))
@pytest.mark.parametrize("strict", [True, False])
def test_whole_record_parity(lib, oracle, key, strict):
    f32, tr32, f64, tr64, model, src, rec, wav = _oracle_run(oracle, key)
    g, trg = _gpu_run(lib, key, strict, model, src, rec, wav)
    assert np.isfinite(tr32).all() and np.abs(tr32).max() > 0, "the record carries no signal"
    errs = {}
    for k in f32:
        e_or = rel_l2(g[k], f32[k])
        errs[k] = {"vs_fp32_restatement": e_or, "gpu_vs_fp64": rel_l2(g[k], f64[k]),
                   "fp32_restatement_vs_fp64": rel_l2(f32[k], f64[k])}
        if strict:
            assert np.array_equal(g[k], f32[k]), f"{key} strict {k}: rel L2 {e_or:.3e}"
        else:
            bound = max(FAST_TOL, 2 * errs[k]["fp32_restatement_vs_fp64"])
            assert e_or <= bound, f"{key} fast {k}: rel L2 {e_or:.3e} > {bound:.3e}"
    e_tr = rel_l2(trg, tr32)
    errs["traces"] = {"vs_fp32_restatement": e_tr, "gpu_vs_fp64": rel_l2(trg, tr64),
                      "fp32_restatement_vs_fp64": rel_l2(tr32, tr64)}
    if strict:
        assert np.array_equal(trg, tr32), f"{key} strict traces: rel L2 {e_tr:.3e}"
    else:
        bound = max(FAST_TOL, 2 * errs["traces"]["fp32_restatement_vs_fp64"])
        assert e_tr <= bound, f"{key} fast traces: rel L2 {e_tr:.3e} > {bound:.3e}"
    c = CASES[key]
    _report({"case": key, "build": "strict" if strict else "fast", "grid": [c["nx"], c["ny"], c["nz"]],
             "nt": c["nt"], "errors": errs})


@pytest.mark.parametrize("strict", [True, False])
def test_whole_record_prop_run_2d(lib, oracle, strict):
    """Config 0 whole through the whole-loop launch (WFD_Prop_Run: 2000 steps, injection and
    extraction inside one cooperative kernel with neighbour-only synchronisation between tiles)
    against the FP32 restatement: bitwise in the strict build, within the fast bound otherwise."""
    import torch
    from wavefd_b200.abi import SourcePoint32
    key = "iso2d_501"
    f32, tr32, f64, tr64, model, src, rec, wav = _oracle_run(oracle, key)
    c = CASES[key]
    shape = (c["nz"], c["ny"], c["nx"])
    gpu = ABIRunner(lib, c["name"], shape, fs=True, nsponge=c["nsponge"], dx=c["d"], dt=c["dt"])
    lib.WFD_Prop_SetStrict(ctypes.c_void_p(gpu.p), int(strict))
    gpu.load(model)
    nt = c["nt"]
    ts = lib.WFD_Points_Create(src.ctypes.data_as(ctypes.POINTER(SourcePoint32)), len(src), 0)
    tr = lib.WFD_Points_Create(rec.ctypes.data_as(ctypes.POINTER(SourcePoint32)), len(rec), 1)
    d_wav = torch.from_numpy(np.ascontiguousarray(wav, np.float32)).cuda()
    d_tr = torch.zeros(len(rec) * nt, device="cuda")
    torch.cuda.synchronize()
    assert lib.WFD_Prop_Run(ctypes.c_void_p(gpu.p), nt, 1, ts, ctypes.c_void_p(d_wav.data_ptr()), tr,
                            ctypes.c_void_p(d_tr.data_ptr()), nt, 1) == 0
    assert lib.WFD_Prop_Synchronize(ctypes.c_void_p(gpu.p)) == 0
    assert lib.WFD_Prop_RunLaunches(ctypes.c_void_p(gpu.p)) == 1
    g = {k: gpu.arr(k).copy() for k in _fields(c["physics"])}
    trg = d_tr.cpu().numpy()
    lib.WFD_Points_Free(ts)
    lib.WFD_Points_Free(tr)
    gpu.close()
    for k in f32:
        if strict:
            assert np.array_equal(g[k], f32[k]), f"{k}: rel L2 {rel_l2(g[k], f32[k]):.3e}"
        else:
            assert rel_l2(g[k], f32[k]) <= max(FAST_TOL, 2 * rel_l2(f32[k], f64[k]))
    if strict:
        assert np.array_equal(trg, tr32)
    else:
        assert rel_l2(trg, tr32) <= max(FAST_TOL, 2 * rel_l2(tr32, tr64))
