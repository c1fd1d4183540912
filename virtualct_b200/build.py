"""Build libvct.so (and the drop-in executables) for sm_100a with nvcc.

Usage: python -m virtualct_b200.build [--force]

Outputs, all in-tree so they travel with the repository snapshot:
  virtualct_b200/lib/libvct.so         C-ABI library (include/vct.h)
  virtualct_b200/lib/libvct_bounds.so  the same library with index checks in the
                                       kernels (-DVCT_BOUNDS=1): a failed check
                                       skips its access and is counted
                                       (vct_bounds_violations); for tests
  virtualct_b200/bin/vct_mbfpa         drop-in for Release_MBFPA_CPU_human/mvct.exe
  virtualct_b200/bin/vct_fbp           drop-in for Release_FBP_CPU/mvct.exe
  virtualct_b200/bin/vct_bhc           drop-in for the beam-hardening correction
  virtualct_b200/lib/libvct_peaks.so   bench.py's roofline denominators (L2 read,
                                       FP64 and FP32 FMA probes); not part of
                                       the product library
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INC = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
BINDIR = os.path.join(PKG, "bin")
LIB = os.path.join(LIBDIR, "libvct.so")
LIB_BOUNDS = os.path.join(LIBDIR, "libvct_bounds.so")
LIB_PEAKS = os.path.join(LIBDIR, "libvct_peaks.so")
PEAKS_SRC = os.path.join(CSRC, "probe", "vct_peaks.cu")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INC, "-I", CSRC]

# Per-translation-unit flags.  The walk (vct_walk.cuh, in the forward and the
# adjoint) must not fuse a*b+c: the reference (x86-64, -O2, no FMA) rounds
# every product and sum separately, and the walk's segment boundaries depend
# on those roundings.
CU_SOURCES = {
    "vct_forward.cu": ["--fmad=false"],
    "vct_fbp.cu": [],
    "vct_fbp_noalloc.cu": [],
    "vct_adjoint.cu": ["--fmad=false"],
    "vct_descent.cu": [],
    "vct_lengthproj.cu": ["--fmad=false"],
    "vct_ir.cu": ["--fmad=false"],
    "vct_measured.cu": ["--fmad=false"],
}
CPP_SOURCES = ["vct_host.cpp", "vct_io.cpp", "vct_batch.cpp"]
APPS = {"vct_mbfpa": "vct_mbfpa_main.cpp", "vct_fbp": "vct_fbp_main.cpp", "vct_bhc": "vct_bhc_main.cpp"}
HEADERS = ["vct_internal.h", "vct_philox.h", "vct_walk.cuh", "vct_fastmath.cuh", "vct_ctx.h"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")


def _library(lib: str, objdir: str, defines: list[str], force: bool, verbose: bool, hdrs: list[str]) -> str:
    """Compile every translation unit (in parallel) and link `lib`."""
    os.makedirs(objdir, exist_ok=True)
    jobs, objs = [], []
    for src, extra in list(CU_SOURCES.items()) + [(c, None) for c in CPP_SOURCES]:
        s = os.path.join(CSRC, src)
        o = os.path.join(objdir, src + ".o")
        objs.append(o)
        if force or not _newer(o, [s] + hdrs + [__file__]):
            arch = ARCH if extra is not None else []
            jobs.append([nvcc(), *arch, *NVCC_COMMON, *defines, *(extra or []), "-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4) or 1) as pool:
        for cmd in jobs:
            if verbose:
                print(" ".join(cmd))
        list(pool.map(_run, jobs))
    if force or not _newer(lib, objs):
        _run([nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", lib, "-cudart", "static"])
    return lib


def build(force: bool = False, verbose: bool = False, bounds: bool = True) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BINDIR, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INC, h) for h in ("vct.h", "vct_io.h")]
    _library(LIB, BUILD, [], force, verbose, hdrs)
    if bounds:
        _library(LIB_BOUNDS, os.path.join(BUILD, "bounds"), ["-DVCT_BOUNDS=1"], force, verbose, hdrs)
    if force or not _newer(LIB_PEAKS, [PEAKS_SRC, __file__]):
        _run([nvcc(), *ARCH, "-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", PEAKS_SRC,
              "-o", LIB_PEAKS, "-cudart", "static"])
    for app, src in APPS.items():
        s = os.path.join(CSRC, src)
        exe = os.path.join(BINDIR, app)
        if force or not _newer(exe, [s, LIB] + hdrs):
            _run([nvcc(), *NVCC_COMMON, s, "-o", exe, "-L", LIBDIR, "-lvct", "-Xlinker", "-rpath=$ORIGIN/../lib"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
