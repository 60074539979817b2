"""
Build the native libraries in-tree:

* ``cms_cuda/libcms_b200.so`` -- the CUDA library (sm_100a) with the C ABI
  declared in ``include/cms_b200.h``;
* ``cms_cuda/libcms_synth.so`` -- the seeded synthetic-complex generator
  (host C, OpenMP).

FP64 geometry must round like NumPy, so everything is compiled with
``-fmad=false`` (no contraction of a*b+c); kernels that want FMA (the FP32
nearest-dot filter) call ``__fmaf_rn`` explicitly.

Usage: ``python cms-cuda_b200/build.py [--force]``
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
PKG = os.path.join(HERE, "cms_cuda")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")

CUDA_SOURCES = ["k_scan.cu", "k_surface.cu", "k_dots.cu", "k_readout.cu", "k_adjoint.cu", "k_refine.cu", "capi.cu", "k_noalloc.cu"]
HEADERS = ["cms_math.cuh", "cms_internal.cuh", "cms_kernels.cuh", "cms_readout.cuh", "cms_circle.cuh", "cms_dual.cuh"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
              "--expt-relaxed-constexpr", "-I", INCLUDE]

LIB = os.path.join(PKG, "libcms_b200.so")
SYNTH = os.path.join(PKG, "libcms_synth.so")
BUILD_DIR = os.path.join(HERE, "_build")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(p) > t for p in deps)


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_cuda(force=False, verbose_ptxas=False):
    os.makedirs(BUILD_DIR, exist_ok=True)
    deps = [os.path.join(CSRC, f) for f in CUDA_SOURCES + HEADERS] + [os.path.join(INCLUDE, "cms_b200.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    objs = []
    hdrs = [os.path.join(CSRC, f) for f in HEADERS] + [os.path.join(INCLUDE, "cms_b200.h")]
    for src in CUDA_SOURCES:
        obj = os.path.join(BUILD_DIR, src.replace(".cu", ".o"))
        s = os.path.join(CSRC, src)
        if force or _stale(obj, [s] + hdrs):
            extra = ["-Xptxas", "-v"] if verbose_ptxas else []
            _run([NVCC] + ARCH + NVCC_FLAGS + extra + ["-c", s, "-o", obj])
        objs.append(obj)
    _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs)
    return LIB


def build_synth(force=False):
    src = os.path.join(CSRC, "synth.c")
    if not force and not _stale(SYNTH, [src]):
        return SYNTH
    _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-std=gnu11", "-o", SYNTH, src, "-lm"])
    return SYNTH


def build(force=False):
    build_synth(force)
    build_cuda(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
