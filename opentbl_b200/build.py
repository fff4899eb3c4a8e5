"""Builds the in-tree extension opentbl_b200/libotbl.so for sm_100a.

One nvcc invocation compiles the CUDA kernels (csrc/kernels.cu), the C ABI
(csrc/otbl_capi.cu) and the host-side coefficient setup (csrc/coef.cpp) into
a shared library with the CUDA runtime linked statically, so the library has
no dependency on torch and can be bound from C, Fortran (iso_c_binding) or
Python (ctypes).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libotbl.so")
DRIVER = os.path.join(HERE, "otbl_driver")
SOURCES = ["kernels.cu", "k_xlines.cu", "k_ylines.cu", "k_ydense.cu", "k_stats.cu", "otbl_capi.cu",
           "otbl_graph.cu", "coef.cpp"]
HEADERS = ["otbl_internal.cuh", "fft.cuh", "devcommon.cuh", "tma.cuh", "zline.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_compiler() -> list[str]:
    # the default gcc on PATH may lack its runtime spec files; prefer the
    # system compiler when present
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def stale() -> bool:
    if not os.path.exists(LIB) or not os.path.exists(DRIVER):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS + ["otbl_driver.c"]]
    deps += [os.path.join(HERE, "..", "include", h) for h in ("otbl.h", "otbl_layout.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return LIB
    cmd = [nvcc(), *host_compiler(), *ARCH, "-O3", "-lineinfo", "-std=c++17",
           "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
           "--expt-relaxed-constexpr",
           "-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libotbl.so")
    if verbose:
        sys.stderr.write(r.stderr)
    build_driver()
    return LIB


def build_driver() -> str:
    """The C program csrc/otbl_driver.c, linked against libotbl.so alone
    (it finds the library next to itself at run time)."""
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else (shutil.which("gcc") or "cc")
    cmd = [cc, "-O2", "-std=c11", "-Wall", "-o", DRIVER, os.path.join(CSRC, "otbl_driver.c"),
           "-L" + HERE, "-lotbl", "-Wl,-rpath,$ORIGIN", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("gcc failed building otbl_driver")
    return DRIVER


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
