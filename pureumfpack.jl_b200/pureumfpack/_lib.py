"""ctypes binding of libmfgpu.so (declarations in include/mfgpu.h).

The library is required: there is no CPU fallback for the numeric phase, so
importing a GPU entry point without the built library raises.
"""

from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libmfgpu.so")

i64 = ctypes.c_int64
i32 = ctypes.c_int32
f64 = ctypes.c_double
vp = ctypes.c_void_p
i64p = ctypes.POINTER(ctypes.c_int64)
f64p = ctypes.POINTER(ctypes.c_double)
f32p = ctypes.POINTER(ctypes.c_float)
cp = ctypes.c_char_p

# (name, restype, argtypes) for every symbol of include/mfgpu.h
SIGNATURES = [
    ("mfgpu_row_scaling", ctypes.c_int, [i64, i64p, i64p, f64p, i32, f64p]),
    ("mfgpu_row_scaling_f32", ctypes.c_int, [i64, i64p, i64p, f32p, i32, f32p]),
    ("mfgpu_row_scaling_c64", ctypes.c_int, [i64, i64p, i64p, f64p, i32, f64p]),
    ("mfgpu_amd_order", ctypes.c_int, [i64, i64p, i64p, f64, i64p]),
    ("mfgpu_colamd_order", ctypes.c_int, [i64, i64, i64p, i64p, f64, i64p]),
    ("mfgpu_symbolic_create", ctypes.c_int, [i64, i64p, i64p, i64p, ctypes.POINTER(vp)]),
    ("mfgpu_symbolic_create_batch", ctypes.c_int, [i64, i64p, ctypes.POINTER(vp), ctypes.POINTER(vp), i32,
                                                   ctypes.POINTER(vp)]),
    ("mfgpu_symbolic_destroy", None, [vp]),
    ("mfgpu_symbolic_relax", ctypes.c_int, [vp]),
    ("mfgpu_symbolic_sizes", ctypes.c_int, [vp, i64p]),
    ("mfgpu_symbolic_get", ctypes.c_int, [vp, i64p, i64p, i64p, i64p, i64p, i64p, i64p, i64p]),
    ("mfgpu_symbolic_predicted_fill", i64, [vp]),
    ("mfgpu_factor_colptrs", ctypes.c_int, [vp, i64p, i64p]),
    ("mfgpu_host_last_error", cp, []),
    ("mfgpu_create", ctypes.c_int, [vp, ctypes.POINTER(vp)]),
    ("mfgpu_destroy", None, [vp]),
    ("mfgpu_last_error", cp, [vp]),
    ("mfgpu_set_stream", ctypes.c_int, [vp, vp]),
    ("mfgpu_set_precision", ctypes.c_int, [vp, i32]),
    ("mfgpu_set_growth_limit", ctypes.c_int, [vp, f64]),
    ("mfgpu_set_wait_limit", ctypes.c_int, [vp, f64]),
    ("mfgpu_test_stall", ctypes.c_int, [vp, ctypes.c_int32]),
    ("mfgpu_analyze", ctypes.c_int, [vp, i64, i64p, i64p, i64p, i64p, i64, i64p, i64p, i64p]),
    ("mfgpu_analyze_symbolic", ctypes.c_int, [vp, i64, i64p, i64p, vp]),
    ("mfgpu_factor", ctypes.c_int, [vp, f64p, f64p, i32]),
    ("mfgpu_factor_device", ctypes.c_int, [vp, vp, vp, i32]),
    ("mfgpu_factor_scaled", ctypes.c_int, [vp, f64p, i32, i32]),
    ("mfgpu_get_row_scaling", ctypes.c_int, [vp, f64p]),
    ("mfgpu_factor_sizes", ctypes.c_int, [vp, i64p]),
    ("mfgpu_get_factors", ctypes.c_int, [vp, i64p, i64p, f64p, i64p, i64p, f64p, i64p, i64p, i64p]),
    ("mfgpu_factor_f32", ctypes.c_int, [vp, f32p, f32p, i32]),
    ("mfgpu_get_factors_f32", ctypes.c_int, [vp, i64p, i64p, f32p, i64p, i64p, f32p, i64p, i64p, i64p]),
    ("mfgpu_solve_f32", ctypes.c_int, [vp, i64, f32p, f32p, i32]),
    ("mfgpu_factor_c64", ctypes.c_int, [vp, f64p, f64p, i32]),
    ("mfgpu_get_factors_c64", ctypes.c_int, [vp, i64p, i64p, f64p, i64p, i64p, f64p, i64p, i64p, i64p]),
    ("mfgpu_solve_c64", ctypes.c_int, [vp, i64, f64p, f64p, i32]),
    ("mfgpu_solve", ctypes.c_int, [vp, i64, f64p, i64, f64p, i64, i32]),
    ("mfgpu_factor_solve", ctypes.c_int, [vp, f64p, f64p, i32, i64, f64p, i64, f64p, i64, i32]),
    ("mfgpu_solve_device", ctypes.c_int, [vp, i64, vp, i64, vp, i64, i32]),
    ("mfgpu_backward_error_device", ctypes.c_int, [vp, i64, vp, i64, vp, i64, f64p]),
    ("mfgpu_backward_error_noalloc", ctypes.c_int, [vp, i64, vp, i64, vp, i64, f64p]),
    ("mfgpu_stats_json", ctypes.c_int, [vp, ctypes.c_char_p, i64]),
    ("mfgpu_set_profiling", ctypes.c_int, [vp, i32]),
    ("mfgpu_launch_records", ctypes.c_int, [vp, ctypes.c_char_p, i64]),
    ("mfgpu_batch_analyze", ctypes.c_int, [vp, i64, i64p, ctypes.POINTER(vp), ctypes.POINTER(vp), i32]),
    ("mfgpu_batch_layout", ctypes.c_int, [vp, i64p, i64p, i64p]),
    ("mfgpu_batch_factor", ctypes.c_int, [vp, ctypes.POINTER(vp), i32, i32, i64p]),
    ("mfgpu_batch_solve", ctypes.c_int, [vp, i64, ctypes.POINTER(vp), ctypes.POINTER(vp), i32]),
    ("mfgpu_batch_factor_sizes", ctypes.c_int, [vp, i64, i64p]),
    ("mfgpu_batch_get_factors", ctypes.c_int, [vp, i64, i64p, i64p, f64p, i64p, i64p, f64p, i64p, i64p, i64p]),
    ("mfgpu_gplu_create", ctypes.c_int, [i32, ctypes.POINTER(vp)]),
    ("mfgpu_gplu_destroy", None, [vp]),
    ("mfgpu_gplu_last_error", cp, [vp]),
    ("mfgpu_gplu_set_initial_capacity", ctypes.c_int, [vp, i64]),
    ("mfgpu_gplu_factor", ctypes.c_int, [vp, i64, i64p, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                         ctypes.POINTER(vp), ctypes.POINTER(vp), f64, i32, i32, i64p]),
    ("mfgpu_gplu_sizes", ctypes.c_int, [vp, i64, i64p]),
    ("mfgpu_gplu_get_factors", ctypes.c_int, [vp, i64, i64p, i64p, f64p, i64p, i64p, f64p, i64p, i64p, i64p]),
    ("mfgpu_gplu_solve", ctypes.c_int, [vp, i64, ctypes.POINTER(vp), ctypes.POINTER(vp), i32]),
    ("mfgpu_gplu_timings", ctypes.c_int, [vp, f64p]),
    ("mfgpu_gplu_factor_f32", ctypes.c_int, [vp, i64, i64p, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                             ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp), f64, i32,
                                             i32, i64p]),
    ("mfgpu_gplu_get_factors_f32", ctypes.c_int, [vp, i64, i64p, i64p, f32p, i64p, i64p, f32p, i64p, i64p, i64p]),
    ("mfgpu_gplu_solve_f32", ctypes.c_int, [vp, i64, ctypes.POINTER(vp), ctypes.POINTER(vp), i32]),
    ("mfgpu_gplu_factor_c64", ctypes.c_int, [vp, i64, i64p, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                             ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp), f64, i32,
                                             i32, i64p]),
    ("mfgpu_gplu_get_factors_c64", ctypes.c_int, [vp, i64, i64p, i64p, f64p, i64p, i64p, f64p, i64p, i64p, i64p]),
    ("mfgpu_gplu_solve_c64", ctypes.c_int, [vp, i64, ctypes.POINTER(vp), ctypes.POINTER(vp), i32]),
    ("mfgpu_tune_features", ctypes.c_int, [vp, i64, i64p, f32p, i64]),
    ("mfgpu_tune_set_choice", ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int8), i64]),
    ("mfgpu_mlp_create", ctypes.c_int, [i32, i32, i32, ctypes.c_uint64, ctypes.POINTER(vp)]),
    ("mfgpu_mlp_destroy", None, [vp]),
    ("mfgpu_mlp_last_error", cp, [vp]),
    ("mfgpu_mlp_nparams", i32, [vp]),
    ("mfgpu_mlp_get_params", ctypes.c_int, [vp, f32p]),
    ("mfgpu_mlp_set_params", ctypes.c_int, [vp, f32p]),
    ("mfgpu_mlp_predict", ctypes.c_int, [vp, f32p, i64, f32p]),
    ("mfgpu_mlp_loss_grad", ctypes.c_int, [vp, f32p, f32p, i64, f32p, f32p]),
    ("mfgpu_mlp_train", ctypes.c_int, [vp, f32p, f32p, i64, i32, ctypes.c_float, f32p]),
]

_lib = None


class LibraryMissing(RuntimeError):
    pass


def lib():
    """Load libmfgpu.so (built by pureumfpack.jl_b200/build.py)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LibraryMissing(
                f"{LIB_PATH} is not built; run `python pureumfpack.jl_b200/build.py` "
                "(there is no CPU fallback for the numeric factorization)"
            )
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class MfOptions(ctypes.Structure):
    _fields_ = [("device", i32), ("precision", i32), ("flags", i32), ("reserved", i32)]


def ptr_array(arrays):
    """ctypes array of the data pointers of contiguous numpy arrays."""
    return (vp * len(arrays))(*[a.ctypes.data for a in arrays])


def ptr(a, ty=i64p):
    """ctypes pointer to a contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(ty)
