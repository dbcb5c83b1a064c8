"""ctypes declarations of every entry point in ``include/fm.h``.

Loading fails loudly when ``libfm.so`` is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBFM_PATH = os.path.join(_HERE, "libfm.so")

FM_OK = 0
FM_ERR_ARG, FM_ERR_STATE, FM_ERR_CUDA, FM_ERR_UNSUPPORTED, FM_ERR_NOMEM, FM_ERR_DEVICE = -1, -2, -3, -4, -5, -6
FM_F32, FM_F16_SHIFTED, FM_BF16_SHIFTED, FM_F64, FM_F16_FIXED_AD = 0, 1, 2, 3, 4
FM_COLL_BGK, FM_COLL_POROUS = 0, 1
FM_ISO_NONE, FM_ISO_LINEAR, FM_ISO_LANGMUIR = 0, 1, 2
FM_FIELD_RHO, FM_FIELD_UX, FM_FIELD_UY, FM_FIELD_UZ, FM_FIELD_C, FM_FIELD_Q = range(6)


class FmParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("rho0", C.c_double), ("tau", C.c_double), ("tau_ad", C.c_double),
        ("phi0", C.c_double), ("min_concentration", C.c_double),
        ("periodic_x", C.c_int), ("periodic_y", C.c_int), ("periodic_z", C.c_int),
    ]


_vp, _u8p, _dp, _fp, _sz, _i, _d, _f = C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_double, C.c_float

# name -> (restype, argtypes); kept in the order of include/fm.h
SIGNATURES = {
    "fm_last_error": (C.c_char_p, []),
    "fm_abi_version": (_i, []),
    "fm_lattice_create": (_i, [C.POINTER(FmParams), _i, _vp, C.POINTER(_vp)]),
    "fm_lattice_destroy": (_i, [_vp]),
    "fm_set_obstacle_mask": (_i, [_vp, _u8p, _sz]),
    "fm_set_obstacle_bits": (_i, [_vp, _vp, _sz]),
    "fm_set_porosity_from_mask": (_i, [_vp, _u8p, _sz, _d, _d]),
    "fm_set_porosity": (_i, [_vp, _dp, _sz]),
    "fm_set_tau_field": (_i, [_vp, _dp, _sz]),
    "fm_build_tau_field": (_i, [_i, _i, _i, _d, _d, _u8p, _sz, _d, _d, _dp]),
    "fm_set_collision": (_i, [_vp, _i]),
    "fm_set_coupling": (_i, [_vp, _i]),
    "fm_set_isotherm_linear": (_i, [_vp, _u8p, _sz, _d, _d]),
    "fm_set_isotherm_langmuir": (_i, [_vp, _u8p, _sz, _d, _d, _d]),
    "fm_clear_isotherm": (_i, [_vp]),
    "fm_add_ns_velocity_eq": (_i, [_vp, _u8p, _sz, _d, _d, _d]),
    "fm_add_ns_velocity_neq": (_i, [_vp, _u8p, _sz, _d, _d, _d]),
    "fm_add_ns_pressure": (_i, [_vp, _u8p, _sz, _d]),
    "fm_add_ns_bounceback": (_i, [_vp, _u8p, _sz]),
    "fm_add_ad_dirichlet": (_i, [_vp, _u8p, _sz, _d]),
    "fm_add_ad_tanh_pulse": (_i, [_vp, _u8p, _sz, _d, _d, _i, _i, _d]),
    "fm_add_ad_neumann": (_i, [_vp, _u8p, _sz]),
    "fm_init_equilibrium": (_i, [_vp]),
    "fm_step": (_i, [_vp, _i]),
    "fm_synchronize": (_i, [_vp]),
    "fm_step_count": (C.c_longlong, [_vp]),
    "fm_get_field": (_i, [_vp, _i, _dp, _sz]),
    "fm_get_field_f32": (_i, [_vp, _i, _fp, _sz]),
    "fm_get_fields": (_i, [_vp, C.POINTER(C.c_void_p), C.c_size_t]),
    "fm_get_fields_f32": (_i, [_vp, C.POINTER(C.c_void_p), C.c_size_t]),
    "fm_set_outlet_probe": (_i, [_vp, _u8p, _sz, _i]),
    "fm_get_breakthrough": (_i, [_vp, _dp, _i, C.POINTER(_i)]),
    "fm_reduce": (_i, [_vp, _dp]),
    "fm_get_state": (_i, [_vp, _dp, _dp, _dp, _dp]),
    "fm_set_state": (_i, [_vp, _dp, _dp, _dp, _dp]),
    "fm_launch_henry_ldf_source_d3q7": (_i, [_i, _vp, _vp, _vp, _vp, _f, _f, _f, _vp]),
    "fm_launch_langmuir_ldf_source_d3q7": (_i, [_i, _vp, _vp, _vp, _vp, _f, _f, _f, _f, _vp]),
    "fm_batch_create": (_i, [C.POINTER(_vp), _i, _vp, C.POINTER(_vp)]),
    "fm_batch_destroy": (_i, [_vp]),
    "fm_batch_step": (_i, [_vp, _i]),
    "fm_batch_synchronize": (_i, [_vp]),
    "fm_batch_cells": (C.c_longlong, [_vp]),
    "fm_batch_set_config": (_i, [_vp, _i, _i, _i]),
    "fm_batch_set_mode": (_i, [_vp, _i, _i, _i, _i]),
    "fm_batch_autotune": (_i, [_vp, _i, C.POINTER(_i), C.POINTER(_i), C.POINTER(_i), C.POINTER(_i),
                               C.POINTER(C.c_double)]),
    "fm_outlet_stats": (_i, [_vp, _dp]),
    "fm_pack_zplane": (_i, [_vp, _i, _vp]),
    "fm_unpack_zplane": (_i, [_vp, _i, _vp]),
    "fm_pack_zhalo": (_i, [_vp, _i, _i, _vp]),
    "fm_unpack_zhalo": (_i, [_vp, _i, _i, _vp]),
    "fm_step_planes": (_i, [_vp, _i, _i]),
    "fm_step_finish": (_i, [_vp]),
    "fm_reduce_zrange": (_i, [_vp, _i, _i, _dp]),
    "fm_vti_info": (_i, [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                         C.POINTER(C.c_longlong)]),
    "fm_vti_read": (_i, [C.c_char_p, C.c_double, _vp, _dp, C.c_size_t]),
    "fm_vti_write": (_i, [C.c_char_p, _i, _i, _i, _dp, _i, C.c_char_p, _i]),
    "fm_adjoint_breakthrough": (_i, [_vp, _i, _dp, _i, _i, _i, _dp, _dp, _dp]),
    "fm_adjoint_release": (_i, [_vp]),
    "fm_adjoint_stats": (_i, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "fm_reduce_static": (_i, [_vp, _vp, _vp, C.c_longlong, C.c_longlong, _dp, _vp]),
    "fm_profile_enable": (_i, [_vp, _i]),
    "fm_profile_read": (_i, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]),
    "fm_bench_pull_copy": (_i, [_vp, _i, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fm_set_monitor": (_i, [_vp, _i]),
    "fm_get_monitor": (_i, [_vp, _dp, _i, C.POINTER(_i)]),
    "fm_trim_memory": (_i, [C.c_size_t]),
    "fm_set_pair_layout": (_i, [_vp, _i]),
    "fm_storage_layout": (_i, [_vp]),
    "fm_set_pair_kernel": (_i, [_vp, _i]),
    "fm_step_kernel": (_i, [_vp]),
    "fm_step_status": (_i, [_vp, C.POINTER(_i)]),
    "fm_set_prefetch_distance": (_i, [_vp, _i]),
    "fm_launches_per_step": (_i, [_vp]),
    "fm_debug_layout": (_i, [_vp, C.POINTER(C.c_longlong), C.POINTER(_i)]),
    "fm_debug_set_status": (_i, [_vp, _i]),
}

_LIB = None


class FmError(RuntimeError):
    """Raised for a nonzero fm_status; carries the code and fm_last_error()."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBFM_PATH):
            raise ImportError(f"{LIBFM_PATH} is missing: the CUDA path has no fallback; "
                              "run `python -m fluidmaxxer_b200.build`")
        L = C.CDLL(LIBFM_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc):
    if rc != FM_OK:
        raise FmError(rc, lib().fm_last_error().decode(errors="replace"))
    return rc
