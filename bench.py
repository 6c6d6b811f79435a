#!/usr/bin/env python
"""Headline benchmark: Mcells/s and % of the HBM roofline of the 3D visco-acoustic time step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload iso512|tti400]

A "step" is one time step of the single-shot forward workload: the propagator step, the injection
of the source sample and the extraction of the receiver samples of that time index. Default
workload: 3D AcoIsoDenQ forward, 512^3 cells, 10 m, dt 0.5 ms, 40-cell sponge, 12 Hz Ricker source
at the centre, 256 x 256 surface receivers (synthetic, seeded). Inputs are resident in HBM and far
larger than L2 (537 MB per field). Under torchrun each rank runs its own shot (weak scaling, no
collective on the data path); value = all ranks' cells x steps / the slowest rank's time.

--impl reference times the reference's own C++/OpenMP implementation (compiled from its sources into
oracle/_ref) on the host cores for the same workload and prints the same JSON line.
"""
from __future__ import annotations

import os

# The reference's benchmark binds its OpenMP threads (benchmark/README.md: OMP_PROC_BIND=close); set
# before any library that starts an OpenMP runtime is loaded in this process.
os.environ.setdefault("OMP_PROC_BIND", "close")
os.environ.setdefault("OMP_PLACES", "cores")

import argparse
import ctypes
import json
import math
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "iso512": dict(physics="iso", name="Prop3DAcoIsoDenQ_DEO2_FDTD", shape=(512, 512, 512), d=10.0, dt=0.0005,
                   nt=1000, nsponge=40, fpeak=12.0, nrec=(256, 256), bytes_per_cell=28,
                   label="3D AcoIsoDenQ single-shot forward, 512^3 (134M cells), 10 m, dt 0.5 ms, nt 1000, "
                         "40-cell sponge, 12 Hz Ricker, 256x256 surface receivers"),
    # the reference's own CPU-runnable case: 2D, small enough to sit in L2 (latency-bound on a GPU)
    "iso2d": dict(physics="iso", name="Prop2DAcoIsoDenQ_DEO2_FDTD", shape=(501, 1, 501), d=10.0, dt=0.001,
                  nt=2000, nsponge=60, fpeak=15.0, nrec=(501, 1), bytes_per_cell=28, ndim=2,
                  label="2D AcoIsoDenQ forward, 501 x 501, 10 m, dt 1 ms, nt 2000, 60-cell sponge, constant Q "
                        "100, 15 Hz Ricker at the centre of the top row, receivers on every surface cell"),
    # profiling-size case of the same kernel (fields still larger than L2: 67 MB each)
    # the fused 2D VTI and TTI steps on the same grid (the time loop as a CUDA graph of two steps)
    "vti2d": dict(physics="vti", name="Prop2DAcoVTIDenQ_DEO2_FDTD", shape=(501, 1, 501), d=10.0, dt=0.0005,
                  nt=2000, nsponge=60, fpeak=15.0, nrec=(501, 1), bytes_per_cell=56, ndim=2,
                  label="2D AcoVTIDenQ forward, 501 x 501, 10 m, dt 0.5 ms, nt 2000, 60-cell sponge, "
                        "receivers on every surface cell"),
    "tti2d": dict(physics="tti", name="Prop2DAcoTTIDenQ_DEO2_FDTD", shape=(501, 1, 501), d=10.0, dt=0.0005,
                  nt=2000, nsponge=60, fpeak=15.0, nrec=(501, 1), bytes_per_cell=64, ndim=2,
                  label="2D AcoTTIDenQ forward, 501 x 501, 10 m, dt 0.5 ms, nt 2000, 60-cell sponge, "
                        "receivers on every surface cell"),
    "iso256": dict(physics="iso", name="Prop3DAcoIsoDenQ_DEO2_FDTD", shape=(256, 256, 256), d=10.0, dt=0.0005,
                   nt=1000, nsponge=40, fpeak=12.0, nrec=(128, 128), bytes_per_cell=28,
                   label="3D AcoIsoDenQ forward, 256^3 (16.8M cells), profiling size"),
    "tti400": dict(physics="tti", name="Prop3DAcoTTIDenQ_DEO2_FDTD", shape=(400, 400, 400), d=10.0, dt=0.0005,
                   nt=2000, nsponge=40, fpeak=12.0, nrec=(256, 256), bytes_per_cell=72,
                   label="3D AcoTTIDenQ forward, 400^3 (64M cells), 10 m, dt 0.5 ms, nt 2000, 40-cell sponge, "
                         "12 Hz Ricker, 256x256 surface receivers"),
    "vti400": dict(physics="vti", name="Prop3DAcoVTIDenQ_DEO2_FDTD", shape=(400, 400, 400), d=10.0, dt=0.0005,
                   nt=2000, nsponge=40, fpeak=12.0, nrec=(256, 256), bytes_per_cell=56,
                   label="3D AcoVTIDenQ forward, 400^3 (64M cells), 10 m, dt 0.5 ms, nt 2000, 40-cell sponge, "
                         "12 Hz Ricker, 256x256 surface receivers"),
    # profiling-size case of the VTI kernel (fields still larger than L2: 67 MB each)
    "vti256": dict(physics="vti", name="Prop3DAcoVTIDenQ_DEO2_FDTD", shape=(256, 256, 256), d=10.0, dt=0.0005,
                   nt=2000, nsponge=40, fpeak=12.0, nrec=(128, 128), bytes_per_cell=56,
                   label="3D AcoVTIDenQ forward, 256^3 (16.8M cells), profiling size"),
    # profiling-size case of the TTI kernel (fields still larger than L2: 67 MB each)
    "tti256": dict(physics="tti", name="Prop3DAcoTTIDenQ_DEO2_FDTD", shape=(256, 256, 256), d=10.0, dt=0.0005,
                   nt=2000, nsponge=40, fpeak=12.0, nrec=(128, 128), bytes_per_cell=72,
                   label="3D AcoTTIDenQ forward, 256^3 (16.8M cells), profiling size"),
    # batched shots: 64 ginsu windows of a 1024 x 1024 x 400 survey, apertures U{160..320} per axis,
    # depth 400, Iso/VTI 50/50 by seed, one persistent launch per physics class, CUDA-graph time loop
    "batch64": dict(physics="mixed", name="batch", survey=(1024, 1024, 400), nshots=64, aperture=(160, 320),
                    d=10.0, dt=0.0005, nt=1500, nsponge=40, fpeak=12.0, nrec=(32, 32),
                    label="batched 3D AcoIso/VTI DenQ forward: 64 ginsu windows (160-320)^2 x 400 of a "
                          "1024x1024x400 survey, Iso/VTI 50/50, nt 1500, one persistent launch per physics "
                          "class, CUDA-graph time loop, autotuned plan"),
    # the learned codec alone: encode and decode of one 512x512x400 field
    "codec512": dict(physics="none", name="codec", shape=(512, 512, 400),
                     label="learned wavefield codec: encode + decode of one 512x512x400 FP32 field"),
    # Born imaging of one TTI shot with learned compression of the saved forward fields against plain
    # FP32 storage in pinned host memory; a sample of the time loop, scaled to the full record
    "born512": dict(physics="tti", name="born", shape=(512, 512, 400), d=10.0, dt=0.0005, nt=3000, every=4,
                    nsponge=40, fpeak=12.0, nrec=(64, 64),
                    label="3D TTI DenQ Born imaging of one shot of the 16-shot job's shape, 512x512x400, nt 3000, "
                          "snapshots every 4 steps: learned BF16 autoencoder compression vs plain FP32 storage "
                          "(pinned host memory; checkpointed recomputation on the device; disk)"),
}
METRIC = "Mcells/s & %HBM roofline, 3D Iso/TTI step; Born image s/shot learned vs plain"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs, burst copy)"
    return 6650.0, "fallback 6.65 TB/s"


def profiled_traffic(kernel_key):
    """Per-launch DRAM bytes from the committed ncu summary, if one exists for this kernel."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        j = json.load(f)
    return j.get(kernel_key)


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = f"/tmp/wfd_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.dev)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        # nvidia-smi takes a moment to start: wait (at most 5 s) for its first sample, so that the
        # samples cover the load that follows
        t0 = time.perf_counter()
        while self.proc and time.perf_counter() - t0 < 5.0:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.02)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for n, v in zip(names, r[5:9]):
                if "Active" in v and "Not" not in v:
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------------------------------------
def _dist_env():
    """(world, rank, local rank, torch.distributed or None); the process group is created once."""
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        if not dist.is_initialized():
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return world, rank, local, dist


def run_ours(args, W):
    """One single-shot workload on this rank's GPU; returns the JSON line (dict) on rank 0."""
    import torch

    from wavefd_b200 import _lib, props, synthetic

    world, rank, local, dist = _dist_env()
    lib = _lib.library()
    nx, ny, nz = W["shape"]
    ncells = nx * ny * nz
    cls = getattr(props, W["name"])
    prop = cls(nz=nz, ny=ny, nx=nx, nsponge=W["nsponge"], dz=W["d"], dy=W["d"], dx=W["d"], dt=W["dt"],
               freesurface=True, freqQ=5.0, qMin=0.1, qInterior=100.0)
    model = synthetic.earth_model((nx, ny, nz), W["physics"], seed=1 + rank, d=W["d"], dt=W["dt"],
                                  nsponge=W["nsponge"], device="cuda")
    # write the model into the object's managed arrays on the device (no host round trip)
    for k, t in model.items():
        if W.get("ndim", 3) == 2 and k in ("SinPhi", "CosPhi"):
            continue  # (2D TTI has no azimuth)
        dst = _managed_tensor(prop, k, (nx, ny, nz))
        dst.copy_(t)
    del model
    torch.cuda.synchronize()
    prop.prefetch()
    stream = torch.cuda.ExternalStream(prop.stream())
    sptr = ctypes.c_void_p(prop.stream())
    # acquisition
    if W.get("ndim", 3) == 2:
        src, rec = synthetic.surface_acquisition_2d((nx, nz), W["d"])
    else:
        src = synthetic.center_source((nx, ny, nz), W["d"])
        rec = synthetic.surface_receivers((nx, ny, nz), W["nrec"][0], W["nrec"][1], W["nsponge"])
    from wavefd_b200.abi import SourcePoint32
    tsrc = lib.WFD_Points_Create(src.ctypes.data_as(ctypes.POINTER(SourcePoint32)), len(src), 0)
    trec = lib.WFD_Points_Create(rec.ctypes.data_as(ctypes.POINTER(SourcePoint32)), len(rec), 1)
    nt = W["nt"]
    from wavefd_b200.spacetime import causal_ricker
    wav = torch.from_numpy(causal_ricker(W["dt"] * np.arange(nt), f=W["fpeak"])).cuda()
    nrec = len(rec)
    traces = torch.zeros(nrec * nt, device="cuda")
    getp = getattr(prop.abi, "getPCur")

    def step(it):
        _lib.check(lib.WFD_Prop_TimeStepAsync(prop.p, 1, 0), "step", prop.p)
        pc = ctypes.c_void_p(ctypes.cast(getp(prop.p), ctypes.c_void_p).value)
        _lib.check(lib.WFD_Inject(tsrc, pc, ctypes.c_void_p(wav.data_ptr()), it, nt, sptr), "inject")
        _lib.check(lib.WFD_Extract(trec, ctypes.c_void_p(traces.data_ptr()), pc, it, nt, sptr), "extract")

    K, Wu = args.steps, args.warmup
    if W.get("ndim", 3) == 2:
        # a small grid is bound by launch latency: the whole time loop runs through WFD_Prop_Run
        return run_graph_2d(args, W, lib, prop, stream, tsrc, trec, wav, traces, nt, ncells, rank, world, dist)
    it = 0
    for _ in range(Wu):
        it = it % nt + 1
        step(it)
    prop.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # -- device-timed region: K full steps, plus per-step events around the step kernel(s) -------------
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    with ClockSampler(local) as clk:
        # untimed load of about a second first, so that the clock samples (every 200 ms) cover the GPU
        # under load; the samples end with the timed region
        t_load = time.perf_counter()
        nload = 0
        while time.perf_counter() - t_load < 1.0:
            it = it % nt + 1
            step(it)
            nload += 1
            if nload % 50 == 0:
                prop.synchronize()
        ev0.record(stream)
        for i in range(K):
            it = it % nt + 1
            kev[i][0].record(stream)
            _lib.check(lib.WFD_Prop_TimeStepAsync(prop.p, 1, 0), "step", prop.p)
            kev[i][1].record(stream)
            pc = ctypes.c_void_p(ctypes.cast(getp(prop.p), ctypes.c_void_p).value)
            _lib.check(lib.WFD_Inject(tsrc, pc, ctypes.c_void_p(wav.data_ptr()), it, nt, sptr), "inject")
            _lib.check(lib.WFD_Extract(trec, ctypes.c_void_p(traces.data_ptr()), pc, it, nt, sptr), "extract")
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    kms = [a.elapsed_time(b) for a, b in kev]
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_per_step = ms / K
    value = world * ncells * K / (ms / 1e3) / 1e6
    # -- end-to-end through the public API with host buffers: per step the source sample goes up
    #    from pinned memory and the receiver samples of that step come back to pinned memory -------
    h_wav = torch.from_numpy(causal_ricker(W["dt"] * np.arange(nt), f=W["fpeak"])).pin_memory()
    h_rec = torch.empty(nrec, pin_memory=True)
    d_sample = torch.zeros(1, device="cuda")
    d_rec = torch.zeros(nrec, device="cuda")
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    with torch.cuda.stream(stream):
        for i in range(K):
            it = it % nt + 1
            d_sample.copy_(h_wav[it - 1:it], non_blocking=True)
            _lib.check(lib.WFD_Prop_TimeStepAsync(prop.p, 1, 0), "step", prop.p)
            pc = ctypes.c_void_p(ctypes.cast(getp(prop.p), ctypes.c_void_p).value)
            _lib.check(lib.WFD_Inject(tsrc, pc, ctypes.c_void_p(d_sample.data_ptr()), 1, 1, sptr), "inject")
            d_rec.zero_()
            _lib.check(lib.WFD_Extract(trec, ctypes.c_void_p(d_rec.data_ptr()), pc, 1, 1, sptr), "extract")
            h_rec.copy_(d_rec, non_blocking=True)
            stream.synchronize()
    t_e2e = time.perf_counter() - t0
    if dist:
        t = torch.tensor([t_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    e2e = world * ncells * K / t_e2e / 1e6
    dropin = _dropin_loop(args, W, lib, prop, src, rec, nt, ncells, world, dist)
    # -- roofline of the step kernel(s) --------------------------------------------------------------
    kern_ms = statistics.mean(kms)
    alg_bytes = W["bytes_per_cell"] * ncells
    achieved = alg_bytes / (kern_ms / 1e3) / 1e9
    peak, peak_src = peaks()
    epilogues = _epilogue_legs(lib, prop, W, K, stream, ncells, peak)
    traffic = profiled_traffic(W["name"])
    launches_per_step = lib.WFD_Prop_StepKernels(prop.p)
    clocks = clk.summary()
    clocks["window"] = f"{nload} untimed steps (about 1 s) then the {K} timed steps"
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mcells/s", "n_gpus": world, "steps": K, "warmup": Wu,
        "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded layered+random earth model, Gardner density, block Q)",
        "config": {"workload": W["label"], "grid": list(W["shape"]), "time_steps_per_shot": nt,
                   "l2": (f"inputs larger than L2 ({ncells * 4 / 1e6:.0f} MB per field, 126 MB L2)"
                          if ncells * 4 > 126e6 else
                          f"L2-resident by nature ({ncells * 4 / 1e6:.1f} MB per field), not flushed"),
                   "parallelism": f"shots x{world}"},
        # end to end through the reference-facing C ABI: the reference's own per-step calls with host
        # arrays (the drop-in a Julia caller of the reference makes)
        "e2e": dropin,
        # the same through this library's add-on calls: asynchronous step, device point tables, one
        # source sample up from pinned memory and the step's receiver samples back per step
        "e2e_addon": {"value": round(e2e, 1), "unit": "Mcells/s", "h2d_bytes_per_step": 4,
                      "d2h_bytes_per_step": 4 * nrec,
                      "calls": "WFD_Prop_TimeStepAsync + WFD_Inject + WFD_Extract, pinned host buffers"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": traffic,
                     "kernel": "step kernel(s) of " + W["name"], "algorithmic_bytes_per_cell": W["bytes_per_cell"],
                     "kernel_ms": round(kern_ms, 4), "peak_source": peak_src},
        "gpu_launches": K * (launches_per_step + 2),
        "clocks": clocks,
    }
    if epilogues:
        out["fused_epilogues"] = epilogues
    # tensors used on the object's stream go before the stream does
    del traces, wav, d_sample, d_rec, h_rec, h_wav
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    lib.WFD_Points_Free(tsrc)
    lib.WFD_Points_Free(trec)
    props.free(prop)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(W)
    if dist:
        dist.barrier()
    return out if rank == 0 else None


def _epilogue_legs(lib, prop, W, K, stream, ncells, peak):
    """The 3D step with the Born-V injection (WFD_Prop_TimeStepBorn) and with the V imaging condition
    (WFD_Prop_TimeStepImage) fused into it: K launches of each, timed with CUDA events on the
    object's stream. Algorithmic bytes: the step's plus the add-on's, Born-V reading dV and DP (and
    DM), the imaging condition reading DP (and DM) and reading and writing the image."""
    import torch

    from wavefd_b200 import _lib
    if W.get("ndim", 3) != 3:
        return None
    aniso = W["physics"] != "iso"
    gen = torch.Generator(device="cuda")
    gen.manual_seed(3)

    def rnd(scale):
        return torch.randn(tuple(W["shape"]), device="cuda", generator=gen) * scale

    dv, dp = rnd(0.02), rnd(1e-2)
    dm = rnd(1e-2) if aniso else None
    img = torch.zeros(tuple(W["shape"]), device="cuda")
    torch.cuda.synchronize()

    def vp(t):
        return ctypes.c_void_p(t.data_ptr()) if t is not None else None

    out = {}
    for kind in ("born", "image"):
        def launch():
            if kind == "born":
                rc = lib.WFD_Prop_TimeStepBorn(prop.p, vp(dv), vp(dp), vp(dm))
            else:
                rc = lib.WFD_Prop_TimeStepImage(prop.p, vp(img), vp(dp), vp(dm), 0)
            _lib.check(rc, kind, prop.p)

        for _ in range(3):
            launch()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            launch()
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / K
        extra = (12 if aniso else 8) if kind == "born" else (16 if aniso else 12)
        bpc = W["bytes_per_cell"] + extra
        ach = bpc * ncells / (ms / 1e3) / 1e9
        out[kind] = {"entry": "WFD_Prop_TimeStepBorn" if kind == "born" else "WFD_Prop_TimeStepImage",
                     "kernel_ms": round(ms, 4), "mcells_s": round(ncells / (ms / 1e3) / 1e6, 1),
                     "algorithmic_bytes_per_cell": bpc, "achieved_gbs": round(ach, 1),
                     "frac": round(ach / peak, 4)}
    del dv, dp, dm, img
    torch.cuda.synchronize()
    return out


def _dropin_loop(args, W, lib, prop, src, rec, nt, ncells, world, dist):
    """The reference's own call sequence (src/spacetime.jl:1157-1199 around propagateforward!):
    TimeStep, injectdata_float and extractdata_float with host partitions (source_blocking /
    receiver_blocking), a host wavelet and a host trace array, timed end to end on the host clock."""
    import torch

    from wavefd_b200.abi import SpacetimeABI
    from wavefd_b200.spacetime import _partition_args, causal_ricker, receiver_blocking, source_blocking
    st = SpacetimeABI(lib)
    sb, rb = source_blocking(src, 8), receiver_blocking(rec, 8)
    sp, sc = _partition_args(sb)
    rp, rc = _partition_args(rb)
    wav = causal_ricker(W["dt"] * np.arange(nt), f=W["fpeak"]).astype(np.float32)
    traces = np.zeros(len(rec) * nt, np.float32)
    fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    step = getattr(prop.abi, "TimeStep")
    getp = getattr(prop.abi, "getPCur")
    it = 0

    def one():
        nonlocal it
        it = it % nt + 1
        step(prop.p)
        pc = getp(prop.p)
        st.injectdata_float(pc, fp(wav), it, nt, sp, len(sb), sc, 8)
        st.extractdata_float(fp(traces), pc, rp, len(rb), rc, it, nt, 8)

    for _ in range(3):
        one()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    K = args.steps
    t0 = time.perf_counter()
    for _ in range(K):
        one()
    t = time.perf_counter() - t0
    if dist:
        tt = torch.tensor([t], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = float(tt.item())
    return {"value": round(world * ncells * K / t / 1e6, 1), "unit": "Mcells/s", "steps": K,
            "calls": "TimeStep + injectdata_float + extractdata_float (host wavelet, host traces, host partitions), "
                     "synchronous as in the reference",
            # injection reads the step's wavelet sample of every source point; extraction reads and writes
            # back the step's sample of every receiver trace
            "h2d_bytes_per_step": 4 * (len(src) + len(rec)), "d2h_bytes_per_step": 4 * len(rec)}


def run_codec(args, W):
    """Encode and decode throughput of the learned codec (HBM roofline: the kernels read the field
    once and write the code, or read the code and write the field)."""
    import torch

    from wavefd_b200.codec import WavefieldCodec

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    shape = W["shape"]
    n = int(np.prod(shape))
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0)
    f = torch.randn(shape, generator=gen, device="cuda")
    for _ in range(2):  # smooth it a little (wavefield-like blocks)
        f = (f + f.roll(1, 0) + f.roll(1, 1) + f.roll(1, 2)) * 0.25
    codec = WavefieldCodec(seed=1)
    code = codec.empty_code(shape)
    out = torch.empty(shape, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # larger than L2
    cb = codec.code_bytes(shape)
    peak, peak_src = peaks()
    bytes_e = 4 * n + cb  # read the field, write the code (the raw-block copy reads 1 % again)
    bytes_d = 4 * n + cb
    K = args.steps

    def time_engine(name):
        codec.engine = name
        for _ in range(max(3, args.warmup)):
            codec.encode(f, shape, code)
            codec.decode(code, shape, out)
        torch.cuda.synchronize()
        te, td = [], []
        for _ in range(K):
            flush.zero_()
            e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
            e0.record()
            codec.encode(f, shape, code)
            e1.record()
            flush.zero_()
            e2.record()
            codec.decode(code, shape, out)
            e3.record()
            e3.synchronize()
            te.append(e0.elapsed_time(e1))
            td.append(e2.elapsed_time(e3))
        codec.status()
        rel = float(torch.linalg.norm(out - f) / torch.linalg.norm(f))
        ms_e, ms_d = statistics.median(te), statistics.median(td)
        ach_e, ach_d = bytes_e / (ms_e / 1e3) / 1e9, bytes_d / (ms_d / 1e3) / 1e9
        return {"encode": {"ms": round(ms_e, 4), "GB_s": round(ach_e, 1), "frac": round(ach_e / peak, 4)},
                "decode": {"ms": round(ms_d, 4), "GB_s": round(ach_d, 1), "frac": round(ach_d / peak, 4)},
                "field_rel_l2": rel}

    with ClockSampler(0) as clk:
        legacy = time_engine("mma.sync")
        umma = time_engine("tcgen05")
        mixed = time_engine("mixed")
    head = mixed  # the default engine: encode on mma.sync, decode on tcgen05
    ms_e, ms_d = head["encode"]["ms"], head["decode"]["ms"]
    ach_e = head["encode"]["GB_s"]
    out_j = {
        "metric": "learned codec throughput (encode + decode of one field)", "value": round(n / ((ms_e + ms_d) / 1e3) / 1e6, 1),
        "unit": "Mcells/s", "n_gpus": 1, "steps": K, "warmup": args.warmup, "ms_per_step": round(ms_e + ms_d, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 weights, fp32 accumulation",
        "data": "synthetic smoothed random field", "config": {"workload": W["label"], "grid": list(shape),
                                                              "l2": "L2 flushed (256 MB write) before each launch"},
        "code_bytes": cb, "compression_ratio_bytes": round(4 * n / cb, 2),
        "encode": head["encode"], "decode": head["decode"], "field_rel_l2": head["field_rel_l2"],
        "engines": {"tcgen05": umma, "mma.sync": legacy, "mixed (default)": mixed}, "grids": codec.grids(),
        "roofline": {"bound": "hbm", "achieved": round(ach_e, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(ach_e / peak, 4), "traffic": None,
                     "kernel": "k_encode (mma.sync, the default engine's encoder; + raw-block selection)",
                     "peak_source": peak_src},
        "e2e": {"value": round(n / ((ms_e + ms_d) / 1e3) / 1e6, 1), "unit": "Mcells/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
    }
    print(json.dumps(out_j), flush=True)


def _host_mem_gb():
    try:
        return os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES") / 1e9
    except (ValueError, OSError):
        return float("nan")


def run_born(args, W):
    """Seconds per Born-imaged shot with the learned codec and with plain storage, on a sample of the
    time loop (args.steps steps forward and adjoint) scaled to the full record length."""
    import torch

    from wavefd_b200 import _lib, imaging
    from wavefd_b200.codec import WavefieldCodec, train_on_propagated

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    _lib.library()
    every = W["every"]
    ns = max(every, (args.steps // every) * every)  # learned store: this many steps (3000 = the whole record)
    ns_plain = min(ns, 200)  # plain pinned-host store: a sample (a whole shot's 629 GB exceeds host memory)
    codec = WavefieldCodec(seed=1)
    t0 = time.perf_counter()
    hist, nblocks = train_on_propagated(codec)
    t_train = time.perf_counter() - t0
    shot = imaging.make_shot("tti", W["shape"], seed=4, d=W["d"], dt=W["dt"], nsponge=W["nsponge"], fpeak=W["fpeak"],
                             nt=ns, nrec=W["nrec"])
    data = imaging.born_data(shot)
    # warm-up (first launches, tensor maps, allocator)
    warm = dict(shot, nt=min(ns, 2 * every))
    imaging.born_image(warm, data, imaging.DeviceStore(W["shape"], 2, 2), every=every, nt=2 * every)
    with ClockSampler(0) as clk:
        plain = imaging.HostStore(W["shape"], ns_plain // every, 2)
        img_plain, t_plain_sample = imaging.born_image(shot, data, plain, every=every, nt=ns_plain)
        del plain
        learned = imaging.CodecStore(codec, W["shape"], ns // every, 2)
        img_codec, t_codec = imaging.born_image(shot, data, learned, every=every)
    t_plain = t_plain_sample * ns / ns_plain  # the plain store's cost per step is the same at every step
    # plain storage in a snapshot file on local disk (O_DIRECT), the fallback when 629 GB per shot fit
    # in neither device nor host memory: a shorter sample (at most 64 steps) so that it stays within
    # the box's disk and a couple of minutes
    disk = None
    nsnap = ns // every
    disk_steps = min(ns, 64)
    disk_bytes = (disk_steps // every) * 2 * int(np.prod(W["shape"])) * 4
    tmpdir = os.environ.get("WFD_SNAP_DIR", tempfile.gettempdir())
    st = os.statvfs(tmpdir)
    if st.f_bavail * st.f_frsize > 1.5 * disk_bytes:
        dstore = imaging.DiskStore(W["shape"], disk_steps // every, 2,
                                   os.path.join(tmpdir, f"wfd_born_{os.getpid()}.snap"), direct=True)
        _, t_disk = imaging.born_image(shot, data, dstore, every=every, nt=disk_steps)
        dstore.close()
        disk = {"s_per_shot": round(t_disk * W["nt"] / disk_steps, 3), "sample_steps": disk_steps,
                "bytes_written": disk_bytes, "speedup_learned_vs_disk": round(t_disk / disk_steps / (t_codec / ns), 3),
                "where": f"{tmpdir} (O_DIRECT where the file system allows)"}
    else:
        disk = {"unavailable": f"less than {1.5 * disk_bytes / 1e9:.0f} GB free in {tmpdir}"}
    # plain FP32 snapshots held on the device by recomputation: checkpoints of the full state every
    # 200 steps, each segment's snapshots recomputed before the adjoint run crosses it (one forward
    # pass more); timed over the whole record. Then the image error at this shape over the whole
    # record: the same checkpointed run with the learned store filled in its forward pass, both images
    # through one adjoint wavefield (exact snapshots against decoded ones)
    import torch
    del learned
    torch.cuda.empty_cache()
    seg = 200
    img_ck, t_ck, _ = imaging.born_image_checkpointed(shot, data, every=every, seg=seg)
    del img_ck
    torch.cuda.empty_cache()
    img_e, _, img_l = imaging.born_image_checkpointed(shot, data, every=every, seg=seg,
                                                      learned=imaging.CodecStore(codec, W["shape"], ns // every, 2))
    ae, al = img_e.double(), img_l.double()
    img_norm = float(torch.linalg.norm(ae))
    rel_full = float(torch.linalg.norm(al - ae) / torch.linalg.norm(ae).clamp_min(1e-30))
    del img_e, img_l, ae, al
    torch.cuda.empty_cache()
    # image error over a whole record (the sample's first steps image nothing yet): 128^3, 1000 steps
    small = imaging.make_shot("tti", (128, 128, 128), seed=4, d=W["d"], dt=W["dt"], nsponge=20, fpeak=W["fpeak"],
                              nt=1000, nrec=(32, 32))
    sdata = imaging.born_data(small)
    img_exact, _ = imaging.born_image(small, sdata, imaging.DeviceStore(small["shape"], 250, 2), every=every)
    img_small, _ = imaging.born_image(small, sdata, imaging.CodecStore(codec, small["shape"], 250, 2), every=every)
    a, b = img_small.cpu().numpy().astype(np.float64), img_exact.cpu().numpy().astype(np.float64)
    rel = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
    scale = W["nt"] / ns  # 1 when the whole record was run
    ncells = int(np.prod(W["shape"]))
    out = {
        "metric": "Born image s/shot, learned compression vs plain storage (3D TTI DenQ)",
        "value": round(t_codec * scale, 3), "unit": "s/shot", "n_gpus": 1, "steps": ns, "warmup": 2 * every,
        "ms_per_step": round(t_codec / ns * 1e3, 4), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (codec: bf16 weights, fp32 accumulation)",
        "data": "synthetic (seeded TTI earth model, sparse +-2% reflectors on 20 horizons)",
        "config": {"workload": W["label"], "grid": list(W["shape"]), "time_steps_per_shot": W["nt"],
                   "learned_steps": ns, "plain_host_steps": ns_plain, "snapshot_every": every,
                   "scaling_note": (f"learned: forward + adjoint of {ns} steps timed end to end"
                                    + (f", times {W['nt']}/{ns}" if ns != W["nt"] else " (the whole record)")
                                    + f"; plain pinned-host: {ns_plain} steps, times {W['nt']}/{ns_plain}")},
        "plain_s_per_shot": round(t_plain * scale, 3),
        "speedup_learned_vs_plain": round(t_plain / t_codec, 3),
        "plain_disk": disk,
        "plain_host_note": (f"pinned-host plain storage timed on a {ns_plain}-step sample; a whole shot needs "
                            f"{2 * ncells * 4 * (W['nt'] // every) / 1e9:.0f} GB of pinned host memory "
                            f"(this host: {_host_mem_gb():.0f} GB), so beyond the sample it is the disk store"),
        "image_rel_l2_learned_vs_plain": rel,
        "image_check": "TTI 128^3, nt 1000, snapshots every 4 steps, learned vs exact FP32 storage",
        "image_rel_l2_at_bench_shape": rel_full,
        "image_l2_norm_at_bench_shape": img_norm,
        "image_check_at_bench_shape": (f"TTI {'x'.join(map(str, W['shape']))}, the bench shot's {ns}-step record, "
                                       f"learned snapshots vs exact FP32 snapshots recomputed from checkpoints every "
                                       f"{seg} steps, both imaged through one adjoint wavefield"),
        "plain_checkpointed": {"s_per_shot": round(t_ck * scale, 3), "steps": ns,
                               "speedup_learned_vs_checkpointed": round(t_ck / t_codec, 3),
                               "how": (f"exact FP32 snapshots on the device by recomputation: full-state checkpoints "
                                       f"every {seg} steps, each segment recomputed before the adjoint run crosses "
                                       f"it (one forward pass more; {seg // every} snapshots resident)")},
        "snapshot_bytes": {"plain": 2 * ncells * 4, "learned": 2 * codec.code_bytes(W["shape"])},
        "codec_training": {"seconds": round(t_train, 2), "blocks": nblocks, "steps": len(hist),
                           "final_loss": float(np.mean(hist[-50:]))},
        "e2e": {"value": round(t_codec * scale, 3), "unit": "s/shot", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "clocks": clk.summary(),
    }
    print(json.dumps(out), flush=True)


def batch_layout(W):
    """The shot windows of the batched workload: (physics, (nx, ny, nz), (x0, y0)) per shot, seeded."""
    rng = np.random.default_rng(3)
    snx, sny, snz = W["survey"]
    lo, hi = W["aperture"]
    shots = []
    for _ in range(W["nshots"]):
        nx, ny = (int(v) for v in rng.integers(lo, hi + 1, 2))
        phys = "iso" if rng.random() < 0.5 else "vti"
        x0 = int(rng.integers(0, snx - nx + 1))
        y0 = int(rng.integers(0, sny - ny + 1))
        shots.append((phys, (nx, ny, snz), (x0, y0)))
    return shots


def run_batch(args, W):
    import torch

    from wavefd_b200 import _lib, props, synthetic
    from wavefd_b200.batch import ShotBatch, ginsu_crop
    from wavefd_b200.spacetime import causal_ricker

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    _lib.library()
    nt = W["nt"]
    layout = batch_layout(W)
    survey = synthetic.earth_model(W["survey"], "vti", seed=3 + rank, d=W["d"], dt=W["dt"], nsponge=W["nsponge"],
                                   q_blocks=False, device="cuda")
    shots, srcs, recs, wavs, trcs = [], [], [], [], []
    wav = torch.from_numpy(causal_ricker(W["dt"] * np.arange(nt), f=W["fpeak"]).astype(np.float32))
    for phys, (nx, ny, nz), (x0, y0) in layout:
        cls = props.Prop3DAcoIsoDenQ_DEO2_FDTD if phys == "iso" else props.Prop3DAcoVTIDenQ_DEO2_FDTD
        p = cls(nz=nz, ny=ny, nx=nx, nsponge=W["nsponge"], dz=W["d"], dy=W["d"], dx=W["d"], dt=W["dt"],
                freesurface=True, freqQ=5.0, qMin=0.1, qInterior=100.0)
        names = ["V", "B"] + (["Eps", "Eta", "F"] if phys == "vti" else [])
        for k in names:
            dst = _managed_tensor(p, k, (nx, ny, nz))
            ginsu_crop(survey[k], W["survey"], (x0, y0, 0), dst, (nx, ny, nz))
        shots.append(p)
        srcs.append(synthetic.center_source((nx, ny, nz), W["d"]))
        recs.append(synthetic.surface_receivers((nx, ny, nz), W["nrec"][0], W["nrec"][1], W["nsponge"]))
        wavs.append(wav.cuda())
        trcs.append(torch.zeros(len(recs[-1]) * nt, device="cuda"))
    del survey
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    for p in shots:
        p.prefetch()
    batch = ShotBatch(shots)
    for i in range(len(shots)):
        batch.set_acquisition(i, srcs[i], wavs[i], recs[i], trcs[i], nt)
    torch.cuda.synchronize()
    t_tune = time.perf_counter()
    batch.tune(reps=2)
    t_tune = time.perf_counter() - t_tune
    info = batch.info()
    stream = torch.cuda.ExternalStream(batch.stream())
    cells = sum(nx * ny * nz for _, (nx, ny, nz), _ in layout)
    alg = sum(nx * ny * nz * (28 if ph == "iso" else 56) for ph, (nx, ny, nz), _ in layout)
    K, Wu = args.steps, args.warmup
    if K % 2:
        K += 1  # whole graph replays
    batch.run(Wu, it0=1)
    batch.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        batch.run(K, it0=Wu + 1, graph=True)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    batch.synchronize()
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = world * cells * K / (ms / 1e3) / 1e6
    # end to end: every step pair, the pair's source samples go up from pinned host memory into the
    # shots' wavelets and the pair's receiver samples come back to pinned host memory
    h_wav = wav.clone().pin_memory()
    h_rec = [torch.empty((len(r), 2), pin_memory=True) for r in recs]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    it = Wu + K + 1
    t0 = time.perf_counter()
    h2d = d2h = 0
    with torch.cuda.stream(stream):
        for _ in range(K // 2):
            for i in range(len(shots)):
                wavs[i][it - 1:it + 1].copy_(h_wav[it - 1:it + 1], non_blocking=True)
                h2d += 8
            batch.run(2, it0=it, graph=True)
            for i in range(len(shots)):
                nr = len(recs[i])
                h_rec[i].copy_(trcs[i].view(nr, nt)[:, it - 1:it + 1], non_blocking=True)
                d2h += 8 * nr
            it += 2
            stream.synchronize()
    t_e2e = time.perf_counter() - t0
    if dist:
        t = torch.tensor([t_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    e2e = world * cells * K / t_e2e / 1e6
    peak, peak_src = peaks()
    achieved = alg / (ms / K / 1e3) / 1e9
    niso = sum(1 for ph, _, _ in layout if ph == "iso")
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mcells/s", "n_gpus": world, "steps": K, "warmup": Wu,
        "ms_per_step": round(ms / K, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded layered+random survey model, Gardner density, ginsu windows)",
        "config": {"workload": W["label"], "survey": list(W["survey"]), "shots": len(layout), "iso_shots": niso,
                   "vti_shots": len(layout) - niso, "cells_per_step": cells, "time_steps_per_shot": nt,
                   "l2": "inputs larger than L2 (about 50 GB of shot arrays)", "parallelism": f"shots x{world}",
                   "plan": info, "tune_s": round(t_tune, 2)},
        "e2e": {"value": round(e2e, 1), "unit": "Mcells/s", "h2d_bytes_per_step": h2d // K,
                "d2h_bytes_per_step": d2h // K},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "kernel": "batched step launches (Iso and VTI classes) + injection/extraction, per step",
                     "algorithmic_bytes_per_cell": "28 Iso, 56 VTI", "kernel_ms": round(ms / K, 4),
                     "peak_source": peak_src},
        "gpu_launches": K * info["kernels_per_step"],
        "clocks": clk.summary(),
    }
    # tensors used on the batch's stream (device and pinned host memory) go before the stream does
    del wavs, trcs, h_wav, h_rec
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    batch.free()
    for p in shots:
        props.free(p)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline_batch(W, layout)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_graph_2d(args, W, lib, prop, stream, tsrc, trec, wav, traces, nt, ncells, rank, world, dist):
    """2D workload: K steps (source injection and receiver extraction included) replayed from a CUDA
    graph of two steps; end to end in chunks of 100 steps, each chunk's source samples uploaded from
    pinned host memory before it and its receiver samples read back after it."""
    import torch

    from wavefd_b200 import _lib, props
    from wavefd_b200.spacetime import causal_ricker
    K, Wu = args.steps, args.warmup
    nrec = traces.numel() // nt
    pp = ctypes.c_void_p(prop.p)
    wp, tp = ctypes.c_void_p(wav.data_ptr()), ctypes.c_void_p(traces.data_ptr())
    _lib.check(lib.WFD_Prop_Run(pp, Wu, 1, tsrc, wp, trec, tp, nt, 1), "run", prop.p)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        ev0.record(stream)
        _lib.check(lib.WFD_Prop_Run(pp, K, Wu + 1, tsrc, wp, trec, tp, nt, 1), "run", prop.p)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    timed_launches = int(lib.WFD_Prop_RunLaunches(prop.p))
    value = ncells * K / (ms / 1e3) / 1e6
    # end to end: chunks of C steps, wavelet chunk up, traces chunk down (pinned host memory)
    C = 100
    h_wav = torch.from_numpy(causal_ricker(W["dt"] * np.arange(nt), f=W["fpeak"]).astype(np.float32)).pin_memory()
    h_trc = torch.empty((nrec, C), pin_memory=True)
    d_wav = torch.zeros(C, device="cuda")
    d_trc = torch.zeros(nrec * C, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    done = 0
    with torch.cuda.stream(stream):
        while done < K:
            c = min(C, K - done)
            d_wav[:c].copy_(h_wav[(done % nt):(done % nt) + c] if (done % nt) + c <= nt else h_wav[:c], non_blocking=True)
            d_trc.zero_()
            _lib.check(lib.WFD_Prop_Run(pp, c, 1, tsrc, ctypes.c_void_p(d_wav.data_ptr()), trec,
                                        ctypes.c_void_p(d_trc.data_ptr()), C, 1), "run", prop.p)
            h_trc[:, :c].copy_(d_trc.view(nrec, C)[:, :c], non_blocking=True)
            stream.synchronize()
            done += c
    t_e2e = time.perf_counter() - t0
    peak, peak_src = peaks()
    achieved = W["bytes_per_cell"] * ncells / (ms / K / 1e3) / 1e9
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "Mcells/s", "n_gpus": world, "steps": K, "warmup": Wu,
        "ms_per_step": round(ms / K, 5), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded layered+random earth model, Gardner density, block Q)",
        "config": {"workload": W["label"], "grid": list(W["shape"]), "time_steps_per_shot": nt,
                   "l2": f"L2-resident by nature ({ncells * 4 / 1e6:.1f} MB per field), not flushed",
                   "parallelism": f"shots x{world}",
                   "time_loop": "WFD_Prop_Run: the whole loop in one cooperative launch (grid-wide barrier "
                                "between steps)" if timed_launches == 1 else "WFD_Prop_Run: CUDA graph of two steps"},
        "e2e": {"value": round(ncells * K / t_e2e / 1e6, 1), "unit": "Mcells/s", "h2d_bytes_per_step": 4,
                "d2h_bytes_per_step": 4 * nrec},
        "roofline": {"bound": "latency (L2-resident)", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "traffic": None,
                     "kernel": "whole step (kernels of " + W["name"] + " + injection + extraction)",
                     "algorithmic_bytes_per_cell": W["bytes_per_cell"], "kernel_ms": round(ms / K, 5),
                     "peak_source": peak_src},
        # kernels of the timed WFD_Prop_Run: one cooperative launch for the whole loop (2D Iso), else
        # per step the step kernel(s), the injection unless the step kernel applied it, the extraction
        "gpu_launches": timed_launches,
        "clocks": clk.summary(),
    }
    del traces, wav, d_wav, d_trc, h_trc, h_wav
    torch.cuda.synchronize()
    lib.WFD_Points_Free(tsrc)
    lib.WFD_Points_Free(trec)
    props.free(prop)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(W)
    return out if rank == 0 else None


def _managed_tensor(prop, getter, shape):
    import torch
    ptr = ctypes.cast(getattr(prop.abi, "get" + getter)(prop.p), ctypes.c_void_p).value

    class _CAI:
        __cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (ptr, False), "version": 3,
                                    "strides": None}
    return torch.as_tensor(_CAI(), device="cuda")


# ---------------------------------------------------------------------------------------------------
def _ref_flavour():
    from oracle.oracle import reference_lib_path
    for fl in ("avx2", "fast"):
        if os.path.exists(reference_lib_path("prop3DAcoIsoDenQ_DEO2_FDTD", fl)):
            if fl == "avx2":
                flags = open("/proc/cpuinfo").read()
                if " avx2" not in flags or " fma" not in flags:
                    continue
            return fl
    return None


def _count_physical_cores():
    """Physical cores among the CPUs this process may run on: the distinct hyperthread-sibling sets of
    those CPUs (sysfs topology), else the CPU count."""
    cpus = sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else list(range(os.cpu_count() or 1))
    sets = set()
    for c in cpus:
        try:
            with open(f"/sys/devices/system/cpu/cpu{c}/topology/thread_siblings_list") as f:
                sets.add(f.read().strip())
        except OSError:
            return max(1, len(cpus))
    return max(1, len(sets))


# counted before any OpenMP runtime binds this process's main thread to one core (OMP_PROC_BIND
# narrows the affinity that a later count would see)
_PHYS_CORES = _count_physical_cores()


def _physical_cores():
    return _PHYS_CORES


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _ref_object(W, lib_name, fl, th, shape, nby, nbx):
    from oracle.oracle import reference_lib
    from wavefd_b200.abi import PropagatorABI
    lib = reference_lib(lib_name, fl)
    abi = PropagatorABI(lib, W["name"])
    nx, ny, nz = shape
    if W.get("ndim", 3) == 2:
        p = abi.alloc(1, th, nx, nz, W["nsponge"], W["d"], W["d"], W["dt"], nbx, nz)
    else:
        p = abi.alloc(1, th, nx, ny, nz, W["nsponge"], W["d"], W["d"], W["d"], W["dt"], nbx, nby, nz)
    abi.SetupDtOmegaInvQ(p, 5.0, 0.1, 100.0)
    arr = lambda g: np.ctypeslib.as_array(getattr(abi, "get" + g)(p), shape=shape)
    arr("V")[...] = np.linspace(1500, 4500, nz, dtype=np.float32)[None, None, :]
    arr("B")[...] = 0.5
    if W["physics"] != "iso":
        arr("Eps")[...] = 0.1
        arr("Eta")[...] = 0.05
        arr("F")[...] = 0.85
    if W["physics"] == "tti":
        angles = (("SinTheta", 0.3), ("CosTheta", 0.954)) + (() if W.get("ndim", 3) == 2 else
                                                               (("SinPhi", 0.5), ("CosPhi", 0.866)))
        for g, v in angles:
            arr(g)[...] = v
    rng = np.random.default_rng(0)
    arr("PCur")[:, :, :64] = rng.standard_normal((nx, ny, min(64, nz))).astype(np.float32)[:, :, :64] * 1e-3
    return abi, p, arr


_TILE_CACHE = {}


def _cpu_tile(W, fl, th):
    """The reference's tile knobs for this grid on these cores: nbz = nz, and (nby, nbx) chosen like
    its tilesize() (src/prop3DAcoIsoDenQ_DEO2_FDTD.jl:159-185, which times every pair of 4:2:64) on
    the pairs {4, 8, 16, 32, 64}^2, each timed over 3 steps (median, after one) on a 32-plane slab of
    the grid. Returns (nby, nbx, note)."""
    key = (W["name"], tuple(W["shape"]), fl, th)
    if key in _TILE_CACHE:
        return _TILE_CACHE[key]
    nx, ny, nz = W["shape"]
    if W.get("ndim", 3) == 2:
        cands = [(1, b) for b in (4, 8, 16, 32, 64)]
    else:
        cands = [(by, bx) for by in (4, 8, 16, 32, 64) for bx in (4, 8, 16, 32, 64)]
    slab = (min(nx, 32), ny, nz)
    best, rates = None, {}
    for by, bx in cands:
        abi, p, _ = _ref_object(W, W["name"].replace("Prop", "prop"), fl, th, slab, by, bx)
        abi.TimeStep(p)
        ts = []
        for _ in range(3):
            t1 = time.perf_counter()
            abi.TimeStep(p)
            ts.append(time.perf_counter() - t1)
        abi.free(p)
        rates[(by, bx)] = slab[0] * slab[1] * slab[2] / statistics.median(ts) / 1e6
        if best is None or rates[(by, bx)] > rates[best]:
            best = (by, bx)
    note = (f"tiles nbz=nz, (nby, nbx) = {best} chosen from {{4,8,16,32,64}}^2 on a {slab[0]}-plane slab "
            f"({rates[best]:.0f} Mcells/s there; (8, 8) gave {rates.get((8, 8), float('nan')):.0f})")
    _TILE_CACHE[key] = (best[0], best[1], note)
    return _TILE_CACHE[key]


def _cpu_run(W, nsteps_max, seconds, warmup=1, with_acq=True):
    """Reference propagator on the host cores (oracle/_ref): returns (Mcells/s, steps, threads, flavour,
    step times, note). One OpenMP thread per physical core, bound close to cores (set at the top of
    this file), tiles from _cpu_tile."""
    fl = _ref_flavour()
    if fl is None:
        return None
    from oracle.oracle import reference_lib
    from wavefd_b200.abi import SpacetimeABI
    name = W["name"]
    nx, ny, nz = W["shape"]
    th = _physical_cores()
    two = W.get("ndim", 3) == 2
    nby, nbx, tile_note = _cpu_tile(W, fl, th)
    shp = (nx, ny, nz)
    abi, p, arr = _ref_object(W, name.replace("Prop", "prop"), fl, th, shp, nby, nbx)
    st = None
    if with_acq:
        from wavefd_b200 import synthetic
        st = SpacetimeABI(reference_lib("spacetime", fl))
        if two:
            src, rec = synthetic.surface_acquisition_2d((nx, nz), W["d"])
        else:
            src = synthetic.center_source(shp, W["d"])
            rec = synthetic.surface_receivers(shp, W["nrec"][0], W["nrec"][1], W["nsponge"])
        from wavefd_b200.spacetime import receiver_blocking, source_blocking, _partition_args
        sb, rb = source_blocking(src, th), receiver_blocking(rec, th)
        sp, sc = _partition_args(sb)
        rp, rc = _partition_args(rb)
        nt = W["nt"]
        from wavefd_b200.spacetime import causal_ricker
        wav = causal_ricker(W["dt"] * np.arange(nt), f=W["fpeak"])
        traces = np.zeros(len(rec) * nt, np.float32)
        fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    it = 0

    def one():
        nonlocal it
        it = it % W["nt"] + 1
        abi.TimeStep(p)
        if st is not None:
            pc = abi.getPCur(p)
            st.injectdata_float(pc, fp(wav), it, nt, sp, len(sb), sc, th)
            st.extractdata_float(fp(traces), pc, rp, len(rb), rc, it, nt, th)

    for _ in range(warmup):
        one()
    n, t0 = 0, time.perf_counter()
    times = []
    while n < nsteps_max and (time.perf_counter() - t0) < seconds:
        t1 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t1)
        n += 1
    abi.free(p)
    return nx * ny * nz / statistics.median(times) / 1e6, n, th, fl, times, tile_note


def cpu_baseline(W):
    r = _cpu_run(W, nsteps_max=50, seconds=15.0)
    if r is None:
        return {"value": None, "unit": "Mcells/s", "cores": None, "kind": "reference",
                "sample": "reference library not built"}
    v, n, th, fl, _, tile_note = r
    return {"value": round(v, 1), "unit": "Mcells/s", "cores": th, "kind": "reference", "cpu": _cpu_model(),
            "sample": f"{W['name']} TimeStep + injectdata_float + extractdata_float on the full "
                      f"{'x'.join(map(str, W['shape']))} grid, median of {n} steps after 1 warm-up, "
                      f"{th} OpenMP threads (one per physical core, OMP_PROC_BIND={os.environ.get('OMP_PROC_BIND')}, "
                      f"OMP_PLACES={os.environ.get('OMP_PLACES')}), {tile_note}, reference built with "
                      f"-O3 -ffast-math ({fl})"}


def _batch_sample_ws(W, layout):
    """Reference sample shots of the batched workload: one Iso and one VTI window of the mean size."""
    ws = {}
    n = len(layout)
    mx = int(round(sum(s[1][0] for s in layout) / n)) // 4 * 4
    my = int(round(sum(s[1][1] for s in layout) / n)) // 4 * 4
    for ph, name in (("iso", "Prop3DAcoIsoDenQ_DEO2_FDTD"), ("vti", "Prop3DAcoVTIDenQ_DEO2_FDTD")):
        ws[ph] = dict(W, physics=ph, name=name, shape=(mx, my, W["survey"][2]))
    return ws


def _batch_cpu_rate(W, layout, steps, warmup, seconds):
    """Mcells/s of the whole batch on the host cores: each physics timed on a mean-size sample shot,
    the batch's cells per step divided by the time the two rates give."""
    ws = _batch_sample_ws(W, layout)
    rates, notes, th, fl = {}, [], None, None
    for ph, w in ws.items():
        r = _cpu_run(w, nsteps_max=steps, seconds=seconds, warmup=warmup)
        if r is None:
            return None
        rates[ph], n, th, fl, _, tile_note = r
        notes.append(f"{ph} {'x'.join(map(str, w['shape']))}: {rates[ph]:.1f} Mcells/s over {n} steps, {tile_note}")
    t = sum(nx * ny * nz / rates[ph] for ph, (nx, ny, nz), _ in layout)
    cells = sum(nx * ny * nz for _, (nx, ny, nz), _ in layout)
    return cells / t, th, fl, "; ".join(notes)


def cpu_baseline_batch(W, layout):
    r = _batch_cpu_rate(W, layout, steps=10, warmup=1, seconds=10.0)
    if r is None:
        return {"value": None, "unit": "Mcells/s", "cores": None, "kind": "reference",
                "sample": "reference library not built"}
    v, th, fl, notes = r
    return {"value": round(v, 1), "unit": "Mcells/s", "cores": th, "kind": "reference", "cpu": _cpu_model(),
            "sample": f"reference TimeStep + injectdata_float + extractdata_float on one mean-size Iso and one "
                      f"VTI window ({notes}), median step times, combined over the batch's 64 windows; "
                      f"{th} OpenMP threads (one per physical core, bound close to cores), -O3 -ffast-math ({fl})"}


def _unavailable(why):
    return {"impl": "reference", "unavailable": why}


def run_reference(args, W):
    """The reference's own C++/OpenMP implementation (oracle/_ref, compiled from its sources) on this
    host's cores, same workload, metric and unit; returns the JSON line (rank 0 only)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return None
    if _ref_flavour() is None:
        return _unavailable("reference library not built (make -C oracle ref)")
    if W["name"] == "codec":
        return _unavailable("the reference compresses with CvxCompress, a Julia package absent from the "
                            "reference tree and from this image")
    if W["name"] == "born":
        return _unavailable("the reference's Born imaging stores its snapshots through CvxCompress "
                            "(src/compressedio.jl), a Julia package absent here")
    if W["name"] == "batch":
        layout = batch_layout(W)
        v, th, fl, notes = _batch_cpu_rate(W, layout, steps=args.steps, warmup=args.warmup, seconds=60.0)
        cells = sum(nx * ny * nz for _, (nx, ny, nz), _ in layout)
        return {
            "metric": METRIC, "value": round(v, 1), "unit": "Mcells/s", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(cells / v / 1e3, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": W["label"], "parallelism": f"OpenMP x{th}"},
            "cpu_baseline": {"value": round(v, 1), "unit": "Mcells/s", "cores": th, "kind": "reference",
                             "cpu": _cpu_model(), "sample": notes},
            "e2e": {"value": round(v, 1), "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
    r = _cpu_run(W, nsteps_max=args.steps, seconds=1e9, warmup=args.warmup)
    v, n, th, fl, times, tile_note = r
    ms = statistics.mean(times) * 1e3
    return {
        "metric": METRIC, "value": round(v, 1), "unit": "Mcells/s", "n_gpus": 0, "steps": n, "warmup": args.warmup,
        "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic", "impl": "reference",
        "config": {"workload": W["label"], "grid": list(W["shape"]), "parallelism": f"OpenMP x{th}"},
        "cpu_baseline": {"value": round(v, 1), "unit": "Mcells/s", "cores": th, "kind": "reference",
                         "cpu": _cpu_model(),
                         "sample": f"{n} full-grid steps (TimeStep + inject + extract), median; {th} OpenMP threads "
                                   f"(one per physical core, bound close to cores); {tile_note}; -O3 -ffast-math "
                                   f"({fl})"},
        "e2e": {"value": round(v, 1), "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


# Secondary workloads timed in the same run as the headline one (same JSON line, key "legs"): the
# 3D TTI step is the north-star kernel, timed on the 3D TTI workload's 400^3 grid.
LEGS = {"iso512": ["tti400"]}


def _relaunch_distributed(args):
    """--gpus N without a launcher: run this script as N ranks (one per GPU) under torchrun."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="iso512", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-legs", action="store_true", help="time the headline workload only")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return _relaunch_distributed(args)
    if world != args.gpus and args.impl == "ours":
        raise SystemExit(f"--gpus {args.gpus} but this launch has {world} ranks")
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    W = WORKLOADS[args.workload]
    legs = [] if args.no_legs else LEGS.get(args.workload, [])
    if args.impl == "reference":
        out = run_reference(args, W)
        if out is not None and "unavailable" not in out and legs:
            out["legs"] = {k: run_reference(args, WORKLOADS[k]) for k in legs}
    elif W["name"] == "batch":
        run_batch(args, W)
        return 0
    elif W["name"] == "born":
        run_born(args, W)
        return 0
    elif W["name"] == "codec":
        run_codec(args, W)
        return 0
    else:
        out = run_ours(args, W)
        leg_out = {k: run_ours(args, WORKLOADS[k]) for k in legs}
        if out is not None and legs:
            out["legs"] = leg_out
            out["gpu_launches"] += sum(v.get("gpu_launches", 0) for v in leg_out.values())
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
