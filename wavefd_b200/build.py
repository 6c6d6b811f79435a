"""Build the CUDA library in-tree: wavefd_b200/lib/libwavefd_b200.so (sm_100a).

Kernel sources are compiled twice, once with IEEE order of operations (-fmad=false; namespace
wfd_strict, the bitwise-parity build) and once for speed (FMA contraction; namespace wfd_fast).
The library exports the reference's C ABI by name; `lib/` also gets one symlink per reference
library name (libprop3DAcoIsoDenQ_DEO2_FDTD.so, ..., libspacetime.so) so that a loader that asks
for the reference's libraries by name finds this one.

    python -m wavefd_b200.build [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
BUILD = os.path.join(HERE, "_build")
LIBNAME = "libwavefd_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I", os.path.join(ROOT, "include"),
          "--expt-relaxed-constexpr"]
STRICT = ["-DWFD_STRICT=1", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]
FAST = ["-DWFD_STRICT=0", "-fmad=true", "-prec-div=false", "-prec-sqrt=false", "-ftz=true"]
HOST = ["-Xcompiler", "-fopenmp"]  # host loops of the drop-in calls use the caller's thread count

KERNEL_SOURCES = ["wfd_generic.cu", "wfd_fused.cu", "wfd_fused_iso3d.cu", "wfd_fused_iso3d_tma.cu",
                  "wfd_fused_aniso3d_tma.cu", "wfd_fused_vti3d_tma.cu", "wfd_fused_iso2d.cu", "wfd_fused_aniso2d.cu",
                  "wfd_wavefieldsep.cu"]
HOST_SOURCES = ["wfd_prop.cu", "wfd_bornimage.cu", "wfd_capi.cu", "wfd_addon.cu", "wfd_spacetime.cu",
                "wfd_tma_host.cu", "wfd_noalloc.cu", "wfd_batch.cu", "wfd_codec.cu", "wfd_interp.cu", "wfd_illum.cu", "wfd_snapio.cu"]

REFERENCE_NAMES = ["prop2DAcoIsoDenQ_DEO2_FDTD", "prop2DAcoVTIDenQ_DEO2_FDTD", "prop2DAcoTTIDenQ_DEO2_FDTD",
                   "prop3DAcoIsoDenQ_DEO2_FDTD", "prop3DAcoVTIDenQ_DEO2_FDTD", "prop3DAcoTTIDenQ_DEO2_FDTD",
                   "spacetime", "illumination"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "wavefd_b200.h")]
    return max(os.path.getmtime(f) for f in files)


def _compile(args):
    src, obj, flags = args
    cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    out = os.path.join(LIBDIR, LIBNAME)
    if not force and os.path.exists(out) and os.path.getmtime(out) >= _deps():
        _links()
        return out
    jobs = []
    for f in KERNEL_SOURCES:
        stem = os.path.splitext(f)[0]
        jobs.append((os.path.join(CSRC, f), os.path.join(BUILD, stem + "_strict.o"), STRICT))
        jobs.append((os.path.join(CSRC, f), os.path.join(BUILD, stem + "_fast.o"), FAST))
    for f in HOST_SOURCES:
        stem = os.path.splitext(f)[0]
        jobs.append((os.path.join(CSRC, f), os.path.join(BUILD, stem + ".o"), HOST))
    with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(_compile, jobs))
    tmp = out + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "shared", "-Xcompiler", "-fopenmp", "-o", tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, out)
    _links()
    if verbose:
        print(out)
    return out


def _links():
    for name in REFERENCE_NAMES:
        link = os.path.join(LIBDIR, f"lib{name}.so")
        if os.path.islink(link) or os.path.exists(link):
            continue
        os.symlink(LIBNAME, link)


def ptxas_report(source: str = "wfd_fused_iso3d.cu", strict: bool = False) -> str:
    """-Xptxas -v register/shared-memory report of one kernel source (for tuning notes)."""
    cmd = [nvcc()] + ARCH + COMMON + (STRICT if strict else FAST) + ["-Xptxas", "-v", "-c",
                                                                      os.path.join(CSRC, source), "-o", os.devnull]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return r.stderr


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", default=None, help="print -Xptxas -v for one source instead of building")
    a = ap.parse_args()
    if a.ptxas:
        print(ptxas_report(a.ptxas))
        sys.exit(0)
    print(build(force=a.force, verbose=True))
