"""ctypes binding of ``libfastpls_b200.so`` (the C ABI in include/fastpls_b200.h).

There is no CPU fallback: importing works without a GPU, but every compute
call goes through the CUDA library, and a missing library raises at load.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfastpls_b200.so")

_vp, _i, _d, _sz = C.c_void_p, C.c_int, C.c_double, C.c_size_t
_ull = C.c_ulonglong
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_cp = C.c_char_p

# name -> (restype, argtypes); mirrors include/fastpls_b200.h
SIGNATURES = {
    "fastpls_cuda_gemm": (_i, [_vp, _vp, _i, _i, _i, _i, _vp, _cp, _sz]),
    "fastpls_resident_simpls_cv_classification": (
        _i, [_vp, _vp, _vp, _i, _i, _i, _i, _vp, _i, _i, _i, _i, _i, _ull, _i,
             _i, _vp, _vp, _vp, _vp, _cp, _sz]),
    "fastpls_resident_simpls_cv_regression": (
        _i, [_vp, _vp, _vp, _i, _i, _i, _i, _vp, _i, _i, _i, _i, _i, _ull, _i,
             _vp, _vp, _vp, _vp, _vp, _vp, _cp, _sz]),
    "fastpls_resident_plssvd_cv_classification": (
        _i, [_vp, _vp, _vp, _i, _i, _i, _i, _vp, _i, _i, _i, _i, _i, _ull, _i,
             _i, _vp, _vp, _vp, _vp, _cp, _sz]),
    "fastpls_resident_plssvd_cv_regression": (
        _i, [_vp, _vp, _vp, _i, _i, _i, _i, _vp, _i, _i, _i, _i, _i, _ull, _i,
             _vp, _vp, _vp, _vp, _vp, _vp, _cp, _sz]),
    "fastpls_resident_simpls_create": (
        _vp, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _ull, _cp, _sz]),
    "fastpls_resident_plssvd_create": (
        _vp, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _ull, _cp, _sz]),
    "fastpls_resident_opls_create": (
        _vp, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _ull, _i, _cp,
              _sz]),
    "fastpls_resident_kernelpls_create": (
        _vp, [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _i, _ull, _i, _d,
              _i, _d, _cp, _sz]),
    "fastpls_resident_predict_path": (_i, [_vp, _vp, _i, _vp, _i, _i, _vp, _cp, _sz]),
    "fastpls_resident_simpls_destroy": (None, [_vp]),
    "fastpls_resident_export": (_i, [_vp, _i, _vp, _sz, _cp, _sz]),
    "fastpls_resident_classify_path": (_i, [_vp, _vp, _i, _vp, _i, _i, _i, _vp, _cp, _sz]),
    "fastpls_resident_classify_response_path": (
        _i, [_vp, _vp, _i, _vp, _i, _i, _i, _vp, _vp, _cp, _sz]),
    "fastpls_resident_response_sums": (_i, [_vp, _vp, _vp, _vp, _i, _i, _vp, _cp, _sz]),
    "fastpls_resident_project": (_i, [_vp, _vp, _i, _i, _vp, _cp, _sz]),
    "fastpls_resident_controls": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _cp, _sz]),
    "fastpls_resident_compact": (_i, [_vp, _i, _cp, _sz]),
    "fastpls_b200_device_count": (_i, []),
    "fastpls_b200_launch_count": (_ull, []),
    "fastpls_b200_set_stream": (None, [_vp]),
    "fastpls_b200_server_create": (_vp, [_sz, _i, _cp, _sz]),
    "fastpls_b200_server_destroy": (None, [_vp]),
    "fastpls_b200_server_submit_fit": (
        _i, [_vp, _i, _vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _d, _i, _d,
             C.POINTER(C.c_ulonglong), _cp, _sz]),
    "fastpls_b200_server_submit_predict": (
        _i, [_vp, _ull, _vp, _i, _i, _i, _vp, _i, _i, C.POINTER(C.c_ulonglong), _cp, _sz]),
    "fastpls_b200_server_wait": (_i, [_vp, _ull, _d, _vp, _sz, _dp, _dp, _cp, _sz]),
    "fastpls_b200_server_release": (_i, [_vp, _ull, _cp, _sz]),
    "fastpls_b200_server_stats": (_i, [_vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t),
                                       C.POINTER(C.c_size_t)]),
    "fastpls_b200_server_batch_stats": (_i, [_vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "fastpls_b200_server_set_borrow": (_i, [_vp, _i]),
    "fastpls_b200_fastcor": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _i, _i, _vp, _cp, _sz]),
    "fastpls_b200_fastsvd": (_i, [_vp, _i, _i, _i, _i, _i, _i, _ull, _vp, _vp, _vp, _cp, _sz]),
    "fastpls_b200_simpls_cv_permutation_classification": (
        _i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, _i, _i, _vp, _vp, _cp, _sz]),
    "fastpls_b200_simpls_cv_permutation_classification_head": (
        _i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, _i, _i, _i, _vp, _vp, _cp, _sz]),
    "fastpls_b200_resident_vip": (_i, [_vp, _vp, _sz, _cp, _sz]),
    "fastpls_b200_model_import": (_vp, [_i, _i, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp,
                                        _vp, _vp, _cp, _sz]),
    "fastpls_b200_fastsvd_audited": (_i, [_vp, _i, _i, _i, _i, _i, _i, _ull, _vp, _vp, _vp, _vp,
                                          _cp, _sz]),
    "fastpls_b200_crossprod_noalloc": (
        _i, [_vp, _i, _i, _i, C.c_long, _vp, C.c_long, _i, _vp, C.c_long, _vp, _cp, _sz]),
    "fastpls_b200_fp64_peak": (_i, [_dp, _cp, _sz]),
    "fastpls_b200_profile_gemm": (None, [_i]),
    "fastpls_b200_profile_gemm_read": (None, [_dp, _dp, C.POINTER(C.c_ulonglong)]),
    "fastpls_b200_set_product_digits": (None, [_i]),
    "fastpls_b200_product_digits": (_i, []),
    "fastpls_b200_set_batch_lanes": (None, [_i]),
    "fastpls_b200_batch_lanes": (_i, []),
    "fastpls_b200_set_argmax_guard": (None, [_d]),
    "fastpls_b200_argmax_guard": (_d, []),
    "fastpls_b200_guard_refits": (_i, []),
    "fastpls_b200_last_fit_times": (None, [_dp, _dp]),
    "fastpls_b200_set_persistent": (None, [_i]),
    "fastpls_b200_int8_wait_test": (None, [_i, C.c_longlong]),
    "fastpls_b200_persistent_wait_test": (None, [_i, C.c_longlong]),
    "fastpls_b200_persistent": (_i, []),
    "fastpls_b200_set_autotune": (None, [_i]),
    "fastpls_b200_autotune": (_i, []),
    "fastpls_b200_batched_stats": (None, [C.POINTER(C.c_int)] * 6),
    "fastpls_b200_release_workspace": (None, []),
    "fastpls_b200_profile_int8": (None, [_i]),
    "fastpls_b200_profile_int8_read": (None, [_dp, _dp, C.POINTER(C.c_ulonglong)]),
    "fastpls_b200_int8_crossprod": (
        _i, [_vp, _i, _vp, _i, _i, _i, _i, _i, _i, _i, _i, _vp, _i, _cp, _sz]),
    "fastpls_b200_simpls_cv_permutation": (
        _i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, _i, _i, _i, _vp, _vp,
             _vp, _vp, _vp, _cp, _sz]),
    "fastpls_b200_simpls_cv_permutation_device": (
        _i, [_vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _vp, _i, _i, _i, _vp, _vp,
             _vp, _vp, _vp, _cp, _sz]),
}

_lib = None


def load() -> C.CDLL:
    """Load the library once; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m fastpls_b200.build`"
                " (the fitting path has no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class FastplsError(RuntimeError):
    """Error reported by the CUDA library through its error buffer."""


def error_buffer(size: int = 1024):
    return C.create_string_buffer(size), C.c_size_t(size)


def check(rc: int, err) -> None:
    if rc != 0:
        raise FastplsError(err.value.decode(errors="replace"))
