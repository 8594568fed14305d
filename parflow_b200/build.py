"""Builds libpfgpu.so (the CUDA library behind include/pfgpu.h) in-tree for
sm_100a with nvcc.  ``python -m parflow_b200.build`` or ``build()``."""

from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libpfgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def deps():
    return sources() + sorted(glob.glob(os.path.join(HERE, "csrc", "*.h*"))) + \
        sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
        [os.path.join(ROOT, "include", "pfgpu.h")]


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(d) <= t for d in deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                    "-I" + os.path.join(ROOT, "include"), "--expt-relaxed-constexpr"]
    if verbose:
        flags += ["-Xptxas", "-v"]
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [nvcc()] + flags + ["-c", src, "-o", obj]
        subprocess.check_call(cmd)
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
