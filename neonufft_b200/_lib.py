"""ctypes binding of libneonufft_b200.so (the C ABI declared in include/neonufft_gpu.h).

Loading fails loudly: there is no CPU fallback. The library is looked up next to this file
(in-tree build, see build.py) unless NEONUFFT_B200_LIB points elsewhere.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(os.environ.get("NEONUFFT_B200_LIB", Path(__file__).resolve().parent / "libneonufft_b200.so"))

# NeonufftError (include/neonufft/errors.h)
SUCCESS, GENERIC_ERROR, MEMORY_ALLOC_ERROR, UNKNOWN_ERROR, INTERNAL_ERROR, INPUT_ERROR, \
    GPU_ERROR, NOT_IMPLEMENTED_ERROR = range(8)

NNB_FLOAT, NNB_DOUBLE = 0, 1
NNB_BATCH_SERIAL, NNB_BATCH_STREAMS, NNB_BATCH_GRAPH = 0, 1, 2
NNB_BATCH_FUSED, NNB_BATCH_FUSED_GRAPH = 3, 4
STAGES = ("bin", "spread", "fft", "deconv", "interp", "phase")


class NnbOptions(C.Structure):
    _fields_ = [
        ("tol", C.c_double), ("upsampfac", C.c_double), ("recenter_threshold", C.c_double),
        ("num_threads", C.c_int), ("sort_input", C.c_int), ("sort_output", C.c_int),
        ("kernel_approximation", C.c_int), ("order", C.c_int), ("kernel_type", C.c_int),
        ("tile", C.c_int * 3), ("spread_method", C.c_int), ("n_spread", C.c_int),
        ("reserved", C.c_int * 7),
    ]


AllocFn = C.CFUNCTYPE(C.c_void_p, C.c_void_p, C.c_size_t)
FreeFn = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p)


class NnbAllocator(C.Structure):
    _fields_ = [("allocate", AllocFn), ("deallocate", FreeFn), ("ctx", C.c_void_p)]


class NnbPlanInfo(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("precision", C.c_int), ("n_spread", C.c_int), ("spread_method", C.c_int),
        ("es_beta", C.c_double), ("grid", C.c_int64 * 3), ("spread_grid", C.c_int64 * 3),
        ("tile", C.c_int * 3), ("num_in", C.c_int64), ("num_out", C.c_int64),
        ("batch_size", C.c_int64), ("device_bytes", C.c_uint64),
        ("input_offset", C.c_double * 3), ("output_offset", C.c_double * 3),
        ("gamma", C.c_double * 3), ("h", C.c_double * 3),
    ]


# Every exported entry point and its signature: (name, restype, argtypes).
_P = C.c_void_p
_E = C.c_int
_I64 = C.c_int64
_PP = C.POINTER(C.c_void_p)
_PI64 = C.POINTER(C.c_int64)
_PD = C.POINTER(C.c_double)
SIGNATURES = [
    ("nnb_options_default", None, [C.POINTER(NnbOptions)]),
    ("nnb_plan_create", _E, [C.POINTER(_P), C.c_int, C.c_int, C.POINTER(NnbOptions), C.c_int, _I64, _PP, _PI64, _P, C.POINTER(NnbAllocator)]),
    ("nnb_plan_set_points", _E, [_P, _I64, _PP]),
    ("nnb_plan_transform_type_1", _E, [_P, _P, _P, _PI64]),
    ("nnb_plan_transform_type_2", _E, [_P, _P, _PI64, _P]),
    ("nnb_plan_transform_type_1_many", _E, [_P, _I64, _P, _I64, _P, _I64, _PI64]),
    ("nnb_plan_destroy", _E, [_P]),
    ("nnb_plan_t3_grid_memory_size", _E, [C.c_int, C.c_int, C.POINTER(NnbOptions), _PD, _PD, _PD, _PD, C.POINTER(C.c_uint64)]),
    ("nnb_plan_t3_create", _E, [C.POINTER(_P), C.c_int, C.c_int, C.POINTER(NnbOptions), C.c_int, _I64, _PP, _I64, _PP, _P, _I64, C.POINTER(NnbAllocator)]),
    ("nnb_plan_t3_create_bounds", _E, [C.POINTER(_P), C.c_int, C.c_int, C.POINTER(NnbOptions), C.c_int, _PD, _PD, _PD, _PD, _P, _I64, C.POINTER(NnbAllocator)]),
    ("nnb_plan_t3_set_input_points", _E, [_P, _I64, _PP]),
    ("nnb_plan_t3_set_output_points", _E, [_P, _I64, _PP]),
    ("nnb_plan_t3_add_input", _E, [_P, _P, _I64]),
    ("nnb_plan_t3_transform", _E, [_P, _P, _I64]),
    ("nnb_plan_t3_reset", _E, [_P]),
    ("nnb_plan_t3_destroy", _E, [_P]),
    ("nnb_last_error_message", C.c_char_p, []),
    ("nnb_device_alloc", _E, [C.POINTER(_P), C.c_size_t]),
    ("nnb_device_free", _E, [_P]),
    ("nnb_plan_info", _E, [_P, C.POINTER(NnbPlanInfo)]),
    ("nnb_plan_t3_info", _E, [_P, C.POINTER(NnbPlanInfo)]),
    ("nnb_plan_enable_timing", _E, [_P, C.c_int]),
    ("nnb_plan_stage_times", _E, [_P, _PD, _PI64, C.c_int]),
    ("nnb_plan_t3_enable_timing", _E, [_P, C.c_int]),
    ("nnb_plan_t3_stage_times", _E, [_P, _PD, _PI64, C.c_int]),
    ("nnb_direct_type1_f64", _E, [C.c_int, C.c_int, _I64, _PP, _P, _I64, _P, _P, _P]),
    ("nnb_direct_type1_f64_noalloc", _E, [C.c_int, C.c_int, _I64, _PP, _P, _I64, _P, _P, _P]),
    ("nnb_direct_type2_f64", _E, [C.c_int, C.c_int, _PI64, _P, _PP, _I64, _P, _P, _P]),
    ("nnb_direct_type3_f64", _E, [C.c_int, C.c_int, _I64, _PP, _P, _PP, _I64, _P, _P, _P]),
    ("nnb_es_kernel_params", _E, [C.c_double, C.c_double, C.c_int, C.POINTER(C.c_int), _PD, _PD]),
    ("nnb_plan_t3_geometry", _E, [C.c_int, C.c_int, C.POINTER(NnbOptions), _PD, _PD, _PD, _PD, _PI64, _PI64, _PD, _PD, _PD, _PD]),
    ("nnb_deconv_factors", _E, [C.c_double, C.c_double, C.c_int, _I64, _PD]),
    ("nnb_batch_create", _E, [C.POINTER(_P), C.c_int, C.POINTER(NnbOptions), C.c_int, _P, C.POINTER(NnbAllocator)]),
    ("nnb_batch_add", _E, [_P, C.c_int, C.c_int, C.c_int, _I64, _PP, _PI64, _P, _P, _PI64, C.POINTER(NnbOptions), _PI64]),
    ("nnb_batch_execute", _E, [_P, C.c_int]),
    ("nnb_batch_size", _E, [_P, _PI64]),
    ("nnb_batch_info", _E, [_P, _I64, C.POINTER(NnbPlanInfo)]),
    ("nnb_batch_destroy", _E, [_P]),
    ("nnb_mlp_param_count", _E, [C.c_int, C.POINTER(C.c_int), _PI64]),
    ("nnb_mlp_forward", _E, [C.c_int, C.POINTER(C.c_int), _P, _P, _I64, _P, _P]),
    ("nnb_mlp_backward", _E, [C.c_int, C.POINTER(C.c_int), _P, _P, _P, _P, _I64, _P, _P]),
    ("nnb_mlp_mse", _E, [_P, _P, _I64, _P, _P, _P]),
    ("nnb_mlp_adam", _E, [_I64, _P, _P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_float, _I64, _P]),
    ("nnb_version", C.c_char_p, []),
    ("nnb_kernel_launches", C.c_int64, []),
    ("nnb_is_checked_build", C.c_int, []),
    ("nnb_check_device_status", _E, []),
]

_lib = None


def load() -> C.CDLL:
    """Loads the engine library once; raises RuntimeError if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"neonufft_b200: {LIB_PATH} not found; build it with `python -m neonufft_b200.build` "
            "(the engine has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, res, args in SIGNATURES:
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def ptr_array(ptrs) -> C.Array:
    arr = (C.c_void_p * max(1, len(ptrs)))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr


def i64_array(vals) -> C.Array:
    arr = (C.c_int64 * max(1, len(vals)))()
    for i, v in enumerate(vals):
        arr[i] = int(v)
    return arr


def f64_array(vals) -> C.Array:
    arr = (C.c_double * max(1, len(vals)))()
    for i, v in enumerate(vals):
        arr[i] = float(v)
    return arr
