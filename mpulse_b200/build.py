"""Builds the CUDA library libmpulse_b200.so in-tree for sm_100a.

    python -m mpulse_b200.build          # or: mpulse_b200.build.build()

Every .cu file under csrc/ is compiled with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked into one shared
library next to this file.  Objects go to csrc/_build/ and are rebuilt only
when a source or header is newer.

``build(checked=True)`` makes libmpulse_b200_checked.so from the same sources
with -DMPB_CHECKED=1 (objects in csrc/_build_checked/): the step kernels test
every state index against its array's size and report skipped accesses
(MP_ERR_BOUNDS) instead of touching memory outside an array.  Select it with
MPULSE_B200_LIB.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(CSRC, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "libmpulse_b200.so")
LIB_CHECKED = os.path.join(HERE, "libmpulse_b200_checked.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# cuFFT: the once-per-block spectral precompute of gauss_inject
CUDA_LIB = "/usr/local/cuda/lib64"
LINK_LIBS = ["-L" + CUDA_LIB, "-lcufft", "-Xlinker", "-rpath=" + CUDA_LIB]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I" + INCLUDE, "-I" + CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, checked: bool = False) -> str:
    bdir, lib = (BUILD + "_checked", LIB_CHECKED) if checked else (BUILD, LIB)
    flags = NVCC_FLAGS + (["-DMPB_CHECKED=1"] if checked else [])
    os.makedirs(bdir, exist_ok=True)
    headers = (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) +
               glob.glob(os.path.join(INCLUDE, "*.h")))
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(bdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if _newer(obj, [src, *headers, __file__]):
            cmd = [nvcc(), *ARCH, *flags, "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if _newer(lib, objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", lib, *objs, "-lcudart", *LINK_LIBS]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


def ptxas_report() -> str:
    """Register / spill / shared-memory report of the step kernels."""
    out = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        r = subprocess.run([nvcc(), *ARCH, *NVCC_FLAGS, "-Xptxas", "-v", "-c", src, "-o", os.devnull],
                           capture_output=True, text=True)
        out.append(r.stderr)
    return "\n".join(out)


if __name__ == "__main__":
    if "--ptxas" in sys.argv:
        print(ptxas_report())
    else:
        print(build(verbose=True, checked="--checked" in sys.argv))
