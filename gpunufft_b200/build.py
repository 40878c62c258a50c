"""Build the native library ``libgpunufft_b200.so`` in-tree for sm_100a.

Usage: ``python -m gpunufft_b200.build`` (or ``build()`` from Python).
Sources live in ``gpunufft_b200/csrc``; objects go to ``gpunufft_b200/_build``.
Only files whose sources (or headers) changed are recompiled.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libgpunufft_b200.so")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler",
          "-fPIC,-ffp-contract=off,-fvisibility=hidden",
          "-I" + os.path.join(HERE, "..", "include")]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) +
                  glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return (glob.glob(os.path.join(CSRC, "*.cuh")) +
            glob.glob(os.path.join(CSRC, "*.hpp")) +
            glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def _obj(src):
    base = os.path.basename(src)
    return os.path.join(BUILD, base + ".o")


def _stale(src, obj, hdr_mtime):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or hdr_mtime > t


def _compile(src):
    obj = _obj(src)
    cmd = [NVCC] + ARCH + COMMON + ["-c", src, "-o", obj]
    if src.endswith(".cu"):
        cmd[1:1] = ["-Xptxas", "-warn-spills"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n"
                           f"{r.stderr}")
    return obj, r.stderr


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr = max([os.path.getmtime(h) for h in _headers()] + [0.0])
    srcs = _sources()
    todo = [s for s in srcs if _stale(s, _obj(s), hdr)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for obj, err in ex.map(_compile, todo):
                if verbose and err.strip():
                    print(err, file=sys.stderr)
    objs = [_obj(s) for s in srcs]
    if todo or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcufft", "-lcudart", "-lpthread",
            "-Xlinker", "-rpath", "-Xlinker",
            os.path.join(CUDA_HOME, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n"
                               f"{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
