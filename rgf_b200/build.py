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
SELFTEST_SRC = PKG.parent / "tests" / "cuda" / "selftest.cu"
SELFTEST_OUT = PKG.parent / "tests" / "cuda" / "libselftest.so"
MEXSTUB_DIR = PKG.parent / "tests" / "mexstub"
MEXSTUB_OUT = MEXSTUB_DIR / "libmexstub.so"
MEX_GATEWAY = PKG.parent / "matlab" / "rgf_mex.c"
SOURCES = ["channels.cu", "sweep.cu", "persist.cu", "mixed.cu", "rgf_api.cu"]
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
            build_selftest(verbose, force)
            build_mexstub(verbose, force)
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
    build_selftest(verbose, force)
    build_mexstub(verbose, force)
    return OUT


def build_peak(verbose: bool = False, force: bool = False) -> Path:
    src = CSRC / "peak.cu"
    if PEAK_OUT.exists() and not force and PEAK_OUT.stat().st_mtime >= max(src.stat().st_mtime,
                                                                            (CSRC / "tc32.cuh").stat().st_mtime):
        return PEAK_OUT
    tmp = PEAK_OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(PKG.parent / "include"), "-shared", "-cudart", "static", "-o", str(tmp),
           str(src)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, PEAK_OUT)
    return PEAK_OUT


def build_selftest(verbose: bool = False, force: bool = False) -> Path:
    """Unit-test kernels for device functions without a C-ABI entry (tests only)."""
    if not SELFTEST_SRC.exists():
        return SELFTEST_OUT
    deps = [SELFTEST_SRC, CSRC / "recip.cuh", CSRC / "rgf_internal.cuh", CSRC / "tc32.cuh"]
    if SELFTEST_OUT.exists() and not force and SELFTEST_OUT.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return SELFTEST_OUT
    tmp = SELFTEST_OUT.with_suffix(".so.tmp")
    cmd = [nvcc(), *ARCH, *FLAGS, "-I", str(PKG.parent / "include"), "-shared", "-cudart", "static", "-o", str(tmp),
           str(SELFTEST_SRC)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, SELFTEST_OUT)
    return SELFTEST_OUT


def build_mexstub(verbose: bool = False, force: bool = False) -> Path:
    """The MEX gateway (matlab/rgf_mex.c) compiled against the test harness's
    stand-in for MATLAB's MEX API (tests/mexstub), linked to librgf.so: lets
    the tests drive mexFunction without MATLAB."""
    src = MEXSTUB_DIR / "mexstub.c"
    if not src.exists():
        return MEXSTUB_OUT
    deps = [src, MEXSTUB_DIR / "mex.h", MEX_GATEWAY, PKG.parent / "include" / "rgf.h", OUT]
    if MEXSTUB_OUT.exists() and not force and MEXSTUB_OUT.stat().st_mtime >= max(p.stat().st_mtime for p in deps):
        return MEXSTUB_OUT
    tmp = MEXSTUB_OUT.with_suffix(".so.tmp")
    cmd = [os.environ.get("CC", "gcc"), "-std=gnu11", "-O2", "-Wall", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I", str(MEXSTUB_DIR), "-I", str(PKG.parent / "include"), str(src), str(MEX_GATEWAY),
           "-L", str(PKG), "-lrgf", "-Wl,-rpath,$ORIGIN/../../rgf_b200", "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, MEXSTUB_OUT)
    return MEXSTUB_OUT


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
