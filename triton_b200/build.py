"""Builds the library in-tree: triton_b200/lib/libtriton_b200.so (sm_100a).

``python -m triton_b200.build`` or ``triton_b200.build.build()``.  The
object of each .cu file is rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
HOST = os.path.join(HERE, "host")
LIBDIR = os.path.join(HERE, "lib")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(LIBDIR, "libtriton_b200.so")
EXE = os.path.join(LIBDIR, "triton_b200")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false keeps every product and sum separately rounded, as the
# reference's CPU build computes them; double division and sqrt are IEEE.
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--fmad=false", "-Xcompiler", "-fPIC",
                  "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
# The FP32 precision form is held to a tolerance against FP64, not to bit
# parity; its approximate divisions are explicit intrinsics in the source.  No
# compiler licence to contract products or approximate divisions: where a
# compiler uses it depends on what a function was inlined into, and a member of
# a batch must compute exactly what the same domain computes alone.
PER_FILE = {"tri_step_f32.cu": ["--fmad=false", "-ftz=true"]}


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False):
    nvcc = _nvcc()
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _newer(obj, [src] + headers):
            flags = [f for f in NVFLAGS if not (f.startswith("--fmad") and os.path.basename(src) in PER_FILE)]
            cmd = [nvcc] + flags + PER_FILE.get(os.path.basename(src), []) + ["-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    if _newer(LIB, objs):
        cmd = [nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    host_srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    if host_srcs:
        hdrs = glob.glob(os.path.join(HOST, "*.h")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
        if _newer(EXE, host_srcs + hdrs + [LIB]):
            cmd = ["g++", "-std=c++20", "-O2", "-pthread", "-I" + os.path.join(ROOT, "include"), "-I" + HOST] + \
                host_srcs + \
                ["-o", EXE, "-L" + LIBDIR, "-ltriton_b200", "-Wl,-rpath,$ORIGIN"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(LIB)
