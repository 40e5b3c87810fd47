"""Loader for ``libbinder_b200.so`` (the sm_100a engine behind the C ABI in include/binder_b200.h).

There is no fallback: if the library is missing or cannot be loaded, importing the package's
compute entry points raises ImportError.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libbinder_b200.so")

STATUS_NAMES = {1: "invalid argument", 2: "CUDA error", 3: "unsupported", 4: "not ready",
                5: "device fault"}

# every entry point declared in include/binder_b200.h
EXPORTS = [
    "binder_last_error", "binder_backend", "binder_has_topology_correction",
    "binder_registration_create", "binder_registration_destroy",
    "binder_registration_set_mi_likelihood", "binder_registration_set_nonlinear_transformation",
    "binder_registration_set_mi_likelihood_filter",
    "binder_registration_set_ssd_likelihood_filter", "binder_registration_get_ssd_filter_parameters",
    "binder_registration_em", "binder_registration_sampler", "binder_registration_sampler_chains",
    "binder_registration_get_final_locations", "binder_registration_get_dream_locations",
    "binder_registration_set_dream_locations", "binder_registration_add_displacement",
    "binder_registration_get_likelihood_parameters", "binder_registration_get_shape", "binder_registration_get_iteration_stats",
    "binder_registration_get_state", "binder_registration_last_elapsed_ms",
    "binder_registration_set_stream", "binder_registration_set_chain",
    "binder_registration_reset", "binder_registration_correct_topology",
    "binder_kernel_launch_count", "binder_registration_get_stream",
    "binder_registration_profile_stage", "binder_registration_set_precision",
    "binder_registration_set_histogram_precision",
    "binder_transform_set_precision",
    "binder_transform_create", "binder_transform_destroy",
    "binder_transform_smooth_deformation", "binder_transform_sample_deformation_field",
    "binder_transform_get_shape", "binder_jacobian_determinant_3d", "binder_topology_correct_3d",
    "binder_topology_correct_2d",
    "binder_jacobian_determinant_3d_noalloc", "binder_jacobian_noalloc_max_voxels",
    "binder_jacobian_determinant_2d", "binder_transform_up_sample", "binder_resize_linear",
    "binder_resample_matrix", "binder_pyramid_create", "binder_pyramid_destroy",
    "binder_pyramid_level", "binder_pinned_alloc", "binder_pinned_free",
    "binder_bin_signal_robust", "binder_bin_signal", "binder_center_of_mass", "binder_warp_image",
    "binder_registration_set_ssd_likelihood", "binder_registration_get_ssd_parameters",
    "binder_initnet_create", "binder_initnet_destroy", "binder_initnet_parameter_count",
    "binder_initnet_get_parameters", "binder_initnet_set_parameters", "binder_initnet_predict",
    "binder_initnet_train_step", "binder_initnet_gradients",
    "binder_batch_create", "binder_batch_destroy", "binder_batch_em", "binder_gemm_bf16",
    "binder_registration_set_estep_grid",
]


class BinderError(RuntimeError):
    """A non-zero status from the C ABI (the reference raises std::runtime_error here)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"binder_b200 {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_f32 = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_f64 = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_P = C.c_void_p
_i, _d, _u32, _u64 = C.c_int, C.c_double, C.c_uint32, C.c_uint64


def _declare(lib):
    lib.binder_last_error.restype = C.c_char_p
    lib.binder_backend.restype = C.c_char_p
    lib.binder_has_topology_correction.restype = _i
    lib.binder_kernel_launch_count.restype = C.c_longlong
    lib.binder_jacobian_noalloc_max_voxels.restype = C.c_longlong
    sig = {
        "binder_registration_create": [C.POINTER(_P), _f32, _i, _f32, _P] + [_i] * 7 + [_d],
        "binder_registration_destroy": [_P],
        "binder_registration_set_mi_likelihood": [_P, _d, _f32, _i, _i, _i, _i32, _i32],
        "binder_registration_set_mi_likelihood_filter": [_P, _d, _f32, _i, _i32, _i32, _i, _i, _i],
        "binder_registration_set_ssd_likelihood_filter": [_P, _f64, _i, _f64, _f64, _f64, _i, _d,
                                                          _d, _i, _i],
        "binder_registration_get_ssd_filter_parameters": [_P, _f64, _f64],
        "binder_registration_set_nonlinear_transformation": [_P] + [_d] * 9 + [_f32],
        "binder_registration_em": [_P, _i, _d, _i, _i, C.POINTER(_i)],
        "binder_registration_sampler": [_P, _u64, _i, _i, _i, _i, _i, _i, _i, _f64, _f64],
        "binder_registration_sampler_chains": [_P, _u64] + [_i] * 8 + [_P] * 4,
        "binder_registration_get_final_locations": [_P, _f32],
        "binder_registration_get_dream_locations": [_P, _f32],
        "binder_registration_set_dream_locations": [_P, _f32],
        "binder_registration_add_displacement": [_P, _P, _i, _i, _i],
        "binder_registration_get_likelihood_parameters": [_P, _f32],
        "binder_registration_get_shape": [_P, _i32],
        "binder_registration_get_iteration_stats": [_P, _f64, _i, C.POINTER(_i)],
        "binder_registration_get_state": [_P, _f64, C.POINTER(_d), C.POINTER(C.c_ulonglong),
                                          C.POINTER(C.c_uint)],
        "binder_registration_last_elapsed_ms": [_P, C.POINTER(_d)],
        "binder_registration_set_stream": [_P, _P],
        "binder_registration_set_chain": [_P, _u32],
        "binder_registration_reset": [_P],
        "binder_registration_set_precision": [_P, _i],
        "binder_registration_set_histogram_precision": [_P, _i],
        "binder_transform_set_precision": [_P, _i],
        "binder_registration_get_stream": [_P, C.POINTER(_P)],
        "binder_registration_profile_stage": [_P, _i, _i, C.POINTER(_d)],
        "binder_registration_correct_topology": [_P, _d, _d, _i, _i, _f64, _P],
        "binder_transform_create": [C.POINTER(_P)] + [_d] * 9 + [_f32, _i, _i, _i, _i, _d, _d],
        "binder_transform_destroy": [_P],
        "binder_transform_smooth_deformation": [_P, _f32, _f32, C.POINTER(_d)],
        "binder_transform_sample_deformation_field": [_P, _f32, _i, _f32],
        "binder_transform_get_shape": [_P, _i32],
        "binder_jacobian_determinant_3d": [_f64, _i, _i, _i, _d, _d, _d, _f64],
        "binder_jacobian_determinant_2d": [_f64, _i, _i, _d, _d, _f64],
        "binder_transform_up_sample": [_f64, _i, _i, _i, _i, _i, _i, _i, _f64],
        "binder_resize_linear": [_f64, _i, _i, _i, _i, _i, _i, _i, _d, _f64],
        "binder_resample_matrix": [_i, _i, _i, _f64],
        "binder_pyramid_create": [C.POINTER(_P), _i32, _i32, _P, _i, _i, _i, _i, _i, _i, _f64,
                                  _f64, _d, _i, _i, _i, _i],
        "binder_pyramid_destroy": [_P],
        "binder_pinned_alloc": [C.c_size_t, C.POINTER(_P)],
        "binder_pinned_free": [_P, C.c_size_t],
        "binder_bin_signal_robust": [_P, _i, C.c_longlong, _i, _d, _d, _P, _P],
        "binder_bin_signal": [_P, _i, C.c_longlong, _i, _P],
        "binder_registration_set_ssd_likelihood": [_P, _i, _i, _d, _i, _d, _d, _i32, _i32, _d,
                                                   _d],
        "binder_registration_get_ssd_parameters": [_P, _f64],
        "binder_center_of_mass": [_i32, _i, _i, _i, _f64],
        "binder_warp_image": [_f64, _i, _i, _i, _f64, C.c_longlong, _i, _f64],
        "binder_pyramid_level": [_P, _i, _P, _i, _d, _P, _i, _i, _P, _P],
        "binder_jacobian_determinant_3d_noalloc": [_f64, _i, _i, _i, _d, _d, _d, _f64,
                                                   C.POINTER(_d), C.POINTER(C.c_longlong)],
        "binder_topology_correct_3d": [_f64, _d, _d, _i, _i, _i, _f64, _i, _i, _i, _f64, _P],
        "binder_topology_correct_2d": [_f64, _d, _d, _i, _i, _i, _f64, _i, _i, _f64, _P],
        "binder_initnet_create": [C.POINTER(_P), _i, _i, _i, _u64],
        "binder_initnet_destroy": [_P],
        "binder_initnet_parameter_count": [_P, C.POINTER(C.c_longlong)],
        "binder_initnet_get_parameters": [_P, _P],
        "binder_initnet_set_parameters": [_P, _P],
        "binder_initnet_predict": [_P, _P, _P],
        "binder_initnet_train_step": [_P, _P, _P, _d, C.POINTER(_d), _P],
        "binder_initnet_gradients": [_P, _P, _P, C.POINTER(_d), _P],
        "binder_batch_create": [_P, _i, C.POINTER(_P)],
        "binder_gemm_bf16": [_P, _P, _P, _i, _i, _i],
        "binder_batch_destroy": [_P],
        "binder_batch_em": [_P, _i, _d, _i, _i32, C.POINTER(_d)],
        "binder_registration_set_estep_grid": [_P, _i],
    }
    for name, args in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _i
    return lib


_LIB = None


def lib():
    """The loaded C library (ImportError when it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m binder_b200.build` "
                "(the package has no CPU fallback)")
        _LIB = _declare(C.CDLL(LIB_PATH))
    return _LIB


def check(status: int) -> None:
    if status != 0:
        raise BinderError(status, lib().binder_last_error().decode(errors="replace"))
