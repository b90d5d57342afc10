"""Build recipe for librgf.so (sm_100a) -- run ``python -m rgf_b200.build``.

The shared library is built in-tree (``rgf_b200/librgf.so``) with nvcc,
statically linked against the CUDA runtime so it loads without touching
torch's bundled runtime.  ``librgf_peak.so`` (the FP64 peak microbenchmark
bench.py uses as its roofline denominator) is built beside it.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "librgf.so"
PEAK_OUT = PKG / "librgf_peak.so"
SOURCES = ["channels.cu", "sweep.cu", "persist.cu", "rgf_api.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def build(verbose: bool = False, force: bool = False) -> Path:
    srcs = [CSRC / s for s in SOURCES]
    deps = srcs + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "rgf.h"]
    if OUT.exists() and not force:
        newest = max(p.stat().st_mtime for p in deps)
        if OUT.stat().st_mtime >= newest:
            build_peak(verbose, force)
            return OUT
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    objs = []
    for src in srcs:
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(PKG.parent / "include"), "-c", "-o", str(obj), str(src)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *objs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    build_peak(verbose, force)
    return OUT


def build_peak(verbose: bool = False, force: bool = False) -> Path:
    src = CSRC / "peak.cu"
    if PEAK_OUT.exists() and not force and PEAK_OUT.stat().st_mtime >= src.stat().st_mtime:
        return PEAK_OUT
    tmp = PEAK_OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, *FLAGS, "-shared", "-cudart", "static", "-o", str(tmp), str(src)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, PEAK_OUT)
    return PEAK_OUT


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
