"""ctypes binding of libmojoblas_gpu.so (the C ABI declared in include/mojoblas_gpu.h).

The library is loaded from this package directory.  There is no fallback: if
the shared object is missing, importing raises and names the build command.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmojoblas_gpu.so"
TUNING_PATH = Path(__file__).resolve().parent / "tuning_b200.json"

MBG_OK = 0
MBG_ERR_CUDA = -1
MBG_ERR_ALLOC = -2
MBG_ERR_UNSUPPORTED = -3
MBG_ERR_NO_DEVICE = -4
MBG_ERR_TIMEOUT = -5
MBG_ERR_INVALID_MODE = -6
MBG_ERR_SCRATCH_LIMIT = -7

MODE_PLAIN = 0
MODE_BF16X3 = 1
MODE_BF16X6 = 2
MODE_OZAKI = 3

i64 = C.c_int64
_ch = C.c_char
_vp = C.c_void_p
_f, _d, _i = C.c_float, C.c_double, C.c_int

# name -> argtypes (restype int unless listed in _RESTYPES)
SIGNATURES = {
    "mbg_sgemm": [_ch, _ch, i64, i64, i64, _f, _vp, i64, _vp, i64, _f, _vp, i64],
    "mbg_dgemm": [_ch, _ch, i64, i64, i64, _d, _vp, i64, _vp, i64, _d, _vp, i64],
    "mbg_sgemm_ex": [_i, _ch, _ch, i64, i64, i64, _f, _vp, i64, _vp, i64, _f, _vp, i64],
    "mbg_dgemm_ex": [_i, _i, _ch, _ch, i64, i64, i64, _d, _vp, i64, _vp, i64, _d, _vp, i64],
    "mbg_ssyrk": [_ch, _ch, i64, i64, _f, _vp, i64, _f, _vp, i64],
    "mbg_dsyrk": [_ch, _ch, i64, i64, _d, _vp, i64, _d, _vp, i64],
    "mbg_ssyrk_ex": [_i, _ch, _ch, i64, i64, _f, _vp, i64, _f, _vp, i64],
    "mbg_dsyrk_ex": [_i, _i, _ch, _ch, i64, i64, _d, _vp, i64, _d, _vp, i64],
    "mbg_strsm": [_ch, _ch, _ch, _ch, i64, i64, _f, _vp, i64, _vp, i64],
    "mbg_dtrsm": [_ch, _ch, _ch, _ch, i64, i64, _d, _vp, i64, _vp, i64],
    "mbg_strsm_ex": [_i, _i, _ch, _ch, _ch, _ch, i64, i64, _f, _vp, i64, _vp, i64],
    "mbg_dtrsm_ex": [_i, _i, _i, _ch, _ch, _ch, _ch, i64, i64, _d, _vp, i64, _vp, i64],
    "mbg_sgemv": [_ch, i64, i64, _f, _vp, i64, _vp, i64, _f, _vp, i64],
    "mbg_dgemv": [_ch, i64, i64, _d, _vp, i64, _vp, i64, _d, _vp, i64],
    "mbg_strsv": [_ch, _ch, _ch, i64, _vp, i64, _vp, i64],
    "mbg_dtrsv": [_ch, _ch, _ch, i64, _vp, i64, _vp, i64],
    "mbg_ssymm": [_ch, _ch, i64, i64, _f, _vp, i64, _vp, i64, _f, _vp, i64],
    "mbg_dsymm": [_ch, _ch, i64, i64, _d, _vp, i64, _vp, i64, _d, _vp, i64],
    "mbg_ssymm_ex": [_i, _ch, _ch, i64, i64, _f, _vp, i64, _vp, i64, _f, _vp, i64],
    "mbg_dsymm_ex": [_i, _i, _ch, _ch, i64, i64, _d, _vp, i64, _vp, i64, _d, _vp, i64],
    "mbg_ssyr2k": [_ch, _ch, i64, i64, _f, _vp, i64, _vp, i64, _f, _vp, i64],
    "mbg_dsyr2k": [_ch, _ch, i64, i64, _d, _vp, i64, _vp, i64, _d, _vp, i64],
    "mbg_ssyr2k_ex": [_i, _ch, _ch, i64, i64, _f, _vp, i64, _vp, i64, _f, _vp, i64],
    "mbg_dsyr2k_ex": [_i, _i, _ch, _ch, i64, i64, _d, _vp, i64, _vp, i64, _d, _vp, i64],
    "mbg_strmm": [_ch, _ch, _ch, _ch, i64, i64, _f, _vp, i64, _vp, i64],
    "mbg_dtrmm": [_ch, _ch, _ch, _ch, i64, i64, _d, _vp, i64, _vp, i64],
    "mbg_strmm_ex": [_i, _ch, _ch, _ch, _ch, i64, i64, _f, _vp, i64, _vp, i64],
    "mbg_dtrmm_ex": [_i, _i, _ch, _ch, _ch, _ch, i64, i64, _d, _vp, i64, _vp, i64],
    "mbg_sgemm_adjoint": [_i, _ch, _ch, i64, i64, i64, _f, _vp, i64, _vp, i64, _vp, i64, _vp, i64, _vp, i64],
    "mbg_dgemm_adjoint": [_i, _i, _ch, _ch, i64, i64, i64, _d, _vp, i64, _vp, i64, _vp, i64, _vp, i64, _vp, i64],
    "mbg_strsm_adjoint": [_i, _ch, _ch, _ch, _ch, i64, i64, _f, _vp, i64, _vp, i64, _vp, i64, _vp, i64, _vp, i64],
    "mbg_dtrsm_adjoint": [_i, _i, _ch, _ch, _ch, _ch, i64, i64, _d, _vp, i64, _vp, i64, _vp, i64, _vp, i64, _vp,
                          i64],
    "mbg_sgemm_ex_noalloc": [_i, _ch, _ch, i64, i64, i64, _f, _vp, i64, _vp, i64, _f, _vp, i64],
    "mbg_cgemm": [_ch, _ch, i64, i64, i64, _vp, _vp, i64, _vp, i64, _vp, _vp, i64],
    "mbg_zgemm": [_ch, _ch, i64, i64, i64, _vp, _vp, i64, _vp, i64, _vp, _vp, i64],
    "mbg_cgemm_ex": [_i, _ch, _ch, i64, i64, i64, _vp, _vp, i64, _vp, i64, _vp, _vp, i64],
    "mbg_zgemm_ex": [_i, _i, _ch, _ch, i64, i64, i64, _vp, _vp, i64, _vp, i64, _vp, _vp, i64],
    "mbg_set_stream": [_vp],
    "mbg_set_thread_stream": [_i, _vp],
    "mbg_get_stream": [],
    "mbg_set_sync": [_i],
    "mbg_synchronize": [],
    "mbg_status_string": [_i],
    "mbg_last_error": [],
    "mbg_version": [],
    "mbg_release_workspace": [],
    "mbg_prof_enable": [_i],
    "mbg_prof_reset": [],
    "mbg_prof_query": [C.c_char_p, C.POINTER(_d), C.POINTER(i64)],
    "mbg_launch_count": [],
    "mbg_debug_fail_alloc": [_i],
    "mbg_debug_wait_probe": [i64],
    "mbg_debug_set_noalloc_error": [_i],
    "mbg_probe_peaks": [C.POINTER(_d)] * 4,
    "mbg_set_tuning": [C.c_char_p, i64],
    "mbg_get_tuning": [C.c_char_p],
    "mbg_load_tuning": [C.c_char_p],
    "mbg_sgemm_grouped_plan": [_i, _i, _vp, C.POINTER(_vp)],
    "mbg_strsm_grouped_plan": [_i, _i, _vp, C.POINTER(_vp)],
    "mbg_plan_execute": [_vp],
    "mbg_plan_destroy": [_vp],
    "mbg_sgemm_grouped": [_i, _i, _vp],
    "mbg_strsm_grouped": [_i, _i, _vp],
}
_RESTYPES = {
    "mbg_get_stream": _vp,
    "mbg_status_string": C.c_char_p,
    "mbg_last_error": C.c_char_p,
    "mbg_launch_count": i64,
    "mbg_get_tuning": i64,
}

class SgemmProblem(C.Structure):
    """mbg_sgemm_problem (include/mojoblas_gpu.h)."""
    _fields_ = [("trans_a", C.c_char), ("trans_b", C.c_char), ("m", i64), ("n", i64), ("k", i64),
                ("alpha", C.c_float), ("beta", C.c_float), ("a", C.c_void_p), ("lda", i64),
                ("b", C.c_void_p), ("ldb", i64), ("c", C.c_void_p), ("ldc", i64)]


class StrsmProblem(C.Structure):
    """mbg_strsm_problem (include/mojoblas_gpu.h)."""
    _fields_ = [("side", C.c_char), ("uplo", C.c_char), ("trans_a", C.c_char), ("diag", C.c_char),
                ("m", i64), ("n", i64), ("alpha", C.c_float), ("a", C.c_void_p), ("lda", i64),
                ("b", C.c_void_p), ("ldb", i64)]


_lib = None


def load() -> C.CDLL:
    """Load the CUDA library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH.name} is missing: build it with `python -m mojoblas_b200.build` "
                "(nvcc, sm_100a); there is no CPU fallback")
        lib = C.CDLL(str(LIB_PATH))
        for name, argtypes in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPES.get(name, _i)
        _lib = lib
        if TUNING_PATH.exists():  # the autotuner's table for B200 (mojoblas_b200/autotune.py)
            lib.mbg_load_tuning(str(TUNING_PATH).encode())
    return _lib


def last_error() -> str:
    return (load().mbg_last_error() or b"").decode()


def status_string(st: int) -> str:
    return (load().mbg_status_string(int(st)) or b"").decode()
