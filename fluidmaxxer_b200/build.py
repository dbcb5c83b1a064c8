"""In-tree build of the native libraries.

* ``fluidmaxxer_b200/libfm.so``       -- the CUDA library behind ``include/fm.h``
  (sm_100a only).
* ``fluidmaxxer_b200/libfm_synth.so`` -- host-only synthetic geometry generators.

Usage: ``python -m fluidmaxxer_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# --fmad=false: no multiply-add contraction, so every FP32 expression rounds as the
# reference kernels' source spells it and the FP32 path reproduces their results
# bit for bit (division stays IEEE round-to-nearest, -prec-div=true by default).
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
              "--fmad=false"]

LIBFM = os.path.join(PKG, "libfm.so")
LIBSYNTH = os.path.join(PKG, "libfm_synth.so")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose=False):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(cmd))
    return r.stdout


def build_libfm(force=False, verbose=False):
    srcs = [os.path.join(CSRC, "fm_abi.cu"), os.path.join(CSRC, "fm_static.cu"), os.path.join(CSRC, "fm_vti.cpp")]
    deps = srcs + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(ROOT, "include", "fm.h"), __file__]
    if force or _stale(LIBFM, deps):
        extra = ["-Xptxas", "-v"] if verbose else []
        _run([NVCC, *ARCH, *NVCC_FLAGS, *extra, "-o", LIBFM, *srcs], verbose)
    return LIBFM


def build_synth(force=False):
    src = os.path.join(CSRC, "synth.c")
    if force or _stale(LIBSYNTH, [src, __file__]):
        _run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-o", LIBSYNTH, src, "-lm"])
    return LIBSYNTH


def build(force=False, verbose=False):
    build_synth(force)
    build_libfm(force, verbose)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print("built", LIBFM, LIBSYNTH)
