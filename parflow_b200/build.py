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
# the device-side Newton control restates host arithmetic: no contracted
# multiply-adds there
NO_FMAD_SOURCES = {"nk_control.cu"}
NO_FMAD = ["-fmad=false"]


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
    headers = [d for d in deps() if not d.endswith(".cu")]
    newest_header = max(os.path.getmtime(h) for h in headers)
    jobs, objs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if (force or not os.path.exists(obj) or os.path.getmtime(obj) < os.path.getmtime(src)
                or os.path.getmtime(obj) < newest_header):
            extra = NO_FMAD if os.path.basename(src) in NO_FMAD_SOURCES else []
            jobs.append([nvcc()] + flags + extra + ["-c", src, "-o", obj])
    # one nvcc per translation unit, in parallel
    from concurrent.futures import ThreadPoolExecutor

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for rc, cmd in zip(ex.map(lambda c: subprocess.call(c), jobs), jobs):
            if rc != 0:
                raise subprocess.CalledProcessError(rc, cmd)
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
