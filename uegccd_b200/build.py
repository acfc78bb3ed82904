"""Builds the sm_100a CUDA library of the package in-tree (nvcc, no GPU needed).

    python -m uegccd_b200.build        # -> uegccd_b200/libuegccd.so

The library holds the C ABI of include/uegccd.h, the FP64 and mixed-precision
kernels and the host-side momentum-block planner.  It is compiled for sm_100a
only; there is no other code path.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libuegccd.so")
ZCODE = os.path.join(PKG, "uegccd_zcode")
OBJDIR = os.path.join(PKG, "_build")

SOURCES = ["capi.cu", "kernels_fp64.cu", "kernels_tc.cu", "plan.cpp", "heg_host.cpp", "zcode.cpp", "mp2_static.cu",
           "diis_api.cu", "heg_device.cu", "two_channel.cu"]
# bench.py's FP64 tensor-core peak measurement: a library of its own beside bench.py
BENCH_PEAK_SRC = os.path.join(ROOT, "bench_peak.cu")
BENCH_PEAK_LIB = os.path.join(ROOT, "bench_peak.so")
HEADERS = ["kernels.h", "plan.h", "uegccd_internal.h", "listdir.h", "heg_device.h", "two_channel.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    nvcc = _nvcc()
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", f) for f in ("uegccd.h", "uegccd_host.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJDIR, src + ".o")
        objs.append(o)
        if not _stale(o, [s] + hdrs):
            continue
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-c", s, "-o", o]
        if ptxas_verbose and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    if os.path.exists(BENCH_PEAK_SRC) and _stale(BENCH_PEAK_LIB, [BENCH_PEAK_SRC]):
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-shared", BENCH_PEAK_SRC, "-o", BENCH_PEAK_LIB, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    main = os.path.join(CSRC, "zcode_main.cpp")
    if _stale(ZCODE, [LIB, main] + hdrs):
        # the drop-in executable for the reference's ZCode program, linked to the library beside it
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), main, "-o", ZCODE, "-L", PKG,
               "-luegccd", "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_verbose="-v" in sys.argv)
    print(LIB)
