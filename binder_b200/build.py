"""Build the sm_100a shared library ``binder_b200/lib/libbinder_b200.so`` in place with nvcc.

Usage: ``python -m binder_b200.build`` (or ``build()`` from Python).  Objects go to
``binder_b200/_build``; the library is rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libbinder_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", os.path.join(ROOT, "include")]
# per-file extra flags: the FP64 Jacobian/topology kernels must not contract a*b+c into FMA so
# the determinants match the reference's CPU evaluation bit for bit
EXTRA = {"topology.cu": ["-fmad=false"]}
SOURCES = ["layout.cu", "transform.cu", "umma_transform.cu", "mstep2d.cu", "estep.cu",
           "topology.cu", "resample.cu", "engine.cu", "multires.cu", "preprocess.cu", "initnet.cu", "capi.cu"]


def _newest(paths):
    return max(os.path.getmtime(p) for p in paths)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "binder_b200.h"))
    hdr_time = _newest(headers)
    src_time = max(hdr_time, _newest([os.path.join(CSRC, s) for s in SOURCES]))
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= src_time:
        return LIB  # up to date (objects may be absent where only the library was shipped)
    objs, cmds = [], []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time):
            cmds.append([NVCC, *ARCH, *COMMON, *EXTRA.get(src, []), "-c", s, "-o", o])
    # the translation units compile independently: one nvcc per host core at most
    from concurrent.futures import ThreadPoolExecutor

    def compile_one(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(compile_one, c) for c in cmds]:
            f.result()
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
