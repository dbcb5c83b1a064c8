"""Seeded synthetic geometries (host-only; wraps ``csrc/synth.c``).

The reference takes its geometry from a VTI file it does not ship; these
generators stand in for it with seeded solid masks.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libfm_synth.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `python -m fluidmaxxer_b200.build`")
        lib = C.CDLL(path)
        lib.fm_synth_uniform.argtypes = [C.c_uint64, C.c_long, C.c_void_p]
        lib.fm_synth_bernoulli.argtypes = [C.c_int] * 3 + [C.c_double, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_void_p]
        lib.fm_synth_sphere_pack.argtypes = [C.c_int] * 3 + [C.c_double, C.c_double, C.c_int, C.c_int,
                                                              C.c_uint64, C.c_long, C.c_void_p, C.c_void_p]
        lib.fm_synth_sphere_pack.restype = C.c_long
        lib.fm_synth_smooth_noise.argtypes = [C.c_int] * 3 + [C.c_double, C.c_uint64, C.c_void_p]
        lib.fm_synth_smooth_noise.restype = C.c_int
        _LIB = lib
    return _LIB


def uniform(seed: int, n: int) -> np.ndarray:
    out = np.empty(int(n), dtype=np.float64)
    _lib().fm_synth_uniform(seed, int(n), out.ctypes.data)
    return out


def bernoulli(nx, ny, nz, p, seed, fluid_lo=0, fluid_hi=0, walls=False) -> np.ndarray:
    m = np.empty(nx * ny * nz, dtype=np.uint8)
    _lib().fm_synth_bernoulli(nx, ny, nz, float(p), seed, fluid_lo, fluid_hi, int(walls), m.ctypes.data)
    return m


def sphere_pack(nx, ny, nz, radius, target_porosity, buffer, seed, walls=False, max_failures=20000):
    """Random sequential addition of non-overlapping spheres; returns
    ``(mask, n_spheres, achieved_slab_porosity)``."""
    m = np.empty(nx * ny * nz, dtype=np.uint8)
    por = C.c_double(0.0)
    ns = _lib().fm_synth_sphere_pack(nx, ny, nz, float(radius), float(target_porosity), buffer,
                                     int(walls), seed, int(max_failures), m.ctypes.data, C.byref(por))
    if ns < 0:
        raise MemoryError("sphere pack allocation failed")
    return m, int(ns), float(por.value)


def smooth_noise(nx, ny, nz, sigma, seed) -> np.ndarray:
    out = np.empty(nx * ny * nz, dtype=np.float64)
    if _lib().fm_synth_smooth_noise(nx, ny, nz, float(sigma), seed, out.ctypes.data):
        raise MemoryError("smooth_noise allocation failed")
    return out
