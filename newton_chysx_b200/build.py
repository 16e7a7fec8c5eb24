"""Builds ``libvbd_b200.so`` in-tree with nvcc for sm_100a (``python -m newton_chysx_b200.build``)."""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
SOURCES = ["vbd_b200.cu", "vbd_noalloc.cu"]
HEADERS = ["vbd_math.cuh", "vbd_elements.cuh", "vbd_kernels.cuh", "vbd_ell.cuh", "vbd_dual.cuh", "vbd_adjoint.cuh"]
OUT = os.path.join(HERE, "libvbd_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "vbd_b200.h"),
                                                                 __file__]  # fmt: skip
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        return OUT
    tmp = OUT + ".tmp"
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
           "-Wno-deprecated-declarations", "-I", os.path.join(ROOT, "include"), "-o", tmp,
           *[os.path.join(CSRC, s) for s in SOURCES]]  # fmt: skip
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
