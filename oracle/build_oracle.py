"""Build recipe for the oracle libraries (test infrastructure only).

* ``oracle/libfmoracle_{f64,f32}.so`` -- the plain-C restatement
  ``oracle/fm_oracle.c``; always built.
* ``oracle/_ref/ref_cuda_bench_{f64,f32}`` -- the reference's own CUDA kernels for
  sm_100a with a timing driver (``oracle/ref_cuda_bench.cu``); built on request
  (``python oracle/build_oracle.py --cuda``), for the reference-CUDA baseline.
* ``oracle/_ref/libfmref_vti.so`` -- the reference's header-only readVTI behind
  a C wrapper (``oracle/ref_vti.cpp``), the checker of the VTI reader.
* ``oracle/_ref/libfmref_{f64,f32}.so`` -- the reference's own kernel bodies
  compiled for the host.  Built only where the reference tree is present (the
  container that holds it); elsewhere the prebuilt file is used.  Each kernel
  file is streamed, cut before its class glue (which uses ``<<<>>>`` launches),
  from where it lies into ``g++`` through ``oracle/shim/fm_ref_shim.h``; no
  reference source is copied anywhere.  The objects are linked with
  ``oracle/ref_driver.cpp``.

Both are compiled with ``-ffp-contract=off`` so that the restatement and the
reference kernels agree bit for bit.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference checkout: FM_REFERENCE_ROOT, else a `reference` folder beside
# this repository's own folder
REF_ROOT = os.environ.get("FM_REFERENCE_ROOT", os.path.normpath(os.path.join(HERE, "..", "..", "reference")))
REF_OUT = os.path.join(HERE, "_ref")
CUDA_INC = "/usr/local/cuda/include"

# (file under the reference's src/, last line of its kernel part; 0 = whole file)
REF_KERNEL_FILES = [
    ("src/collision/BGKCollision.cu", 177),
    ("src/collision/PorousBGKCollision.cu", 155),
    ("src/collision/ADBGKCollision.cu", 128),
    ("src/core/Macros.cu", 61),
    ("src/boundary/ns/PressureDirichlet.cu", 96),
    ("src/boundary/ns/VelocityDirichletNEQ.cu", 96),
    ("src/boundary/ns/VelocityDirichlet.cu", 84),
    ("src/boundary/ns/BounceBack.cu", 31),
    ("src/boundary/ad/ADDirichlet.cu", 30),
    ("src/boundary/ad/ADNeumannOutlet.cu", 31),
    ("src/boundary/ad/ADDirichletTanhPulse.cu", 31),
    ("src/reaction/LinearLDF.cu", 48),
    ("src/reaction/LangmuirLDF.cu", 41),
    ("src/core/D3Q19Constants.cu", 0),
    ("src/core/D3Q7Constants.cu", 0),
]

CFLAGS = ["-O3", "-march=x86-64-v3", "-fPIC", "-fopenmp", "-ffp-contract=off"]
# the descriptors' constexpr tables are C++17 inline variables; g++ would emit them as
# process-wide unique symbols, making the f32 and f64 builds share one copy.
REF_CXXFLAGS = ["-fno-gnu-unique"]


def _run(cmd, stdin_bytes=None):
    r = subprocess.run(cmd, input=stdin_bytes, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        sys.stderr.write(r.stdout.decode(errors="replace"))
        raise RuntimeError("oracle build step failed: " + " ".join(cmd[:4]) + " ...")


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_restatement(force=False):
    src = os.path.join(HERE, "fm_oracle.c")
    hdr = os.path.join(HERE, "fm_oracle.h")
    for tag, real in (("f64", "double"), ("f32", "float")):
        out = os.path.join(HERE, f"libfmoracle_{tag}.so")
        if not force and _newer(out, [src, hdr, __file__]):
            continue
        _run(["gcc", "-std=c11", *CFLAGS, "-shared", f"-DFMO_REAL={real}", "-o", out, src, "-lm"])


def reference_present():
    return os.path.isfile(os.path.join(REF_ROOT, "src/collision/BGKCollision.cu"))


def build_reference(force=False):
    """Compile the reference kernels for the host; returns False if absent."""
    if not reference_present():
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    shim = os.path.join(HERE, "shim", "fm_ref_shim.h")
    drv = os.path.join(HERE, "ref_driver.cpp")
    deps = [shim, drv, os.path.join(HERE, "fm_oracle.h"), os.path.join(HERE, "shim/core/Types.hpp"), __file__]
    for tag, real in (("f64", "double"), ("f32", "float")):
        lib = os.path.join(REF_OUT, f"libfmref_{tag}.so")
        if not force and _newer(lib, deps):
            continue
        objs = []
        common = ["g++", "-x", "c++", "-std=c++17", *CFLAGS, *REF_CXXFLAGS, f"-DFM_REF_REAL={real}",
                  "-include", shim, "-I", os.path.join(HERE, "shim"),
                  "-I", os.path.join(REF_ROOT, "include"), "-I", CUDA_INC]
        for rel, last in REF_KERNEL_FILES:
            with open(os.path.join(REF_ROOT, rel), "rb") as fh:
                text = fh.read()
            if last:
                text = b"".join(text.splitlines(keepends=True)[:last])
            obj = os.path.join(REF_OUT, f"{tag}_{os.path.basename(rel)[:-3]}.o")
            _run(common + ["-c", "-", "-o", obj], stdin_bytes=text)
            objs.append(obj)
        drv_obj = os.path.join(REF_OUT, f"{tag}_ref_driver.o")
        _run(["g++", "-std=c++17", *CFLAGS, f"-DFM_REF_REAL={real}", "-I", HERE,
              "-I", CUDA_INC, "-c", drv, "-o", drv_obj])
        _run(["g++", "-shared", "-fopenmp", "-Wl,-Bsymbolic", "-o", lib, drv_obj, *objs])
        for o in objs + [drv_obj]:
            os.remove(o)
    return True


def build_reference_vti(force=False):
    """The reference's header-only readVTI behind a C wrapper (oracle/ref_vti.cpp)."""
    if not reference_present():
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    src = os.path.join(HERE, "ref_vti.cpp")
    lib = os.path.join(REF_OUT, "libfmref_vti.so")
    if force or not _newer(lib, [src, __file__]):
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-I", os.path.join(REF_ROOT, "include"),
              "-o", lib, src])
    return True


REF_CUDA_SOURCES = [
    "src/core/CudaHelpers.cu", "src/core/D3Q19Constants.cu", "src/core/D3Q7Constants.cu", "src/core/Macros.cu",
    "src/collision/BGKCollision.cu", "src/collision/PorousBGKCollision.cu", "src/collision/ADBGKCollision.cu",
    "src/boundary/ad/ADDirichlet.cu", "src/boundary/ad/ADDirichletTanhPulse.cu", "src/boundary/ad/ADNeumannOutlet.cu",
    "src/boundary/ns/BounceBack.cu", "src/boundary/ns/PressureDirichlet.cu", "src/boundary/ns/VelocityDirichlet.cu",
    "src/boundary/ns/VelocityDirichletNEQ.cu", "src/reaction/LinearLDF.cu", "src/reaction/LangmuirLDF.cu",
]


def build_reference_cuda(force=False):
    """The reference's own CUDA implementation for sm_100a: all 16 kernel files
    (the two its CMakeLists.txt omits included), its own flags (--use_fast_math,
    separable compilation), linked with oracle/ref_cuda_bench.cu into
    oracle/_ref/ref_cuda_bench_{f64,f32}.  Measurement only."""
    if not reference_present():
        return False
    os.makedirs(REF_OUT, exist_ok=True)
    drv = os.path.join(HERE, "ref_cuda_bench.cu")
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    for tag, real in (("f64", "double"), ("f32", "float")):
        exe = os.path.join(REF_OUT, f"ref_cuda_bench_{tag}")
        if not force and _newer(exe, [drv, __file__]):
            continue
        inc = ["-I", os.path.join(HERE, "shim"), f"-DFM_REF_REAL={real}"] if tag == "f32" else []
        srcs = [os.path.join(REF_ROOT, r) for r in REF_CUDA_SOURCES]
        _run([nvcc, "-std=c++17", "-O3", "--use_fast_math", "-rdc=true", "-gencode", "arch=compute_100a,code=sm_100a",
              *inc, "-I", os.path.join(REF_ROOT, "include"), "-o", exe, drv, *srcs])
    return True


def build(force=False):
    build_restatement(force)
    have = build_reference(force)
    build_reference_vti(force)
    return have


if __name__ == "__main__":
    have_ref = build(force="--force" in sys.argv)
    if "--cuda" in sys.argv:
        build_reference_cuda(force="--force" in sys.argv)
    print("restatement built;", "reference kernels built" if have_ref else "reference tree absent")
