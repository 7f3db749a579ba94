"""Python mirror of mojoBLAS's level-2 gemv and trsv on the CUDA library.

Same routine names, argument order and meaning as the reference
(src/level2/gemv.mojo:23, src/level2/trsv.mojo:20): column-major A with a
leading dimension, strided vectors (incx, incy; negative increments follow
Netlib's convention), results written in place into `y` (gemv) or `x` (trsv).
As in the reference, gemv's `trans` must be "N", "T" or "C" in upper case.
Buffers may be numpy arrays (the library stages them), torch tensors or raw
integer addresses with an explicit dtype.  An invalid argument prints
"<routine>: Info <n>" and returns n; a CUDA-side failure raises MbgError.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L
from .level3 import _ch, _dtype_of, _ptr, _report


def gemv(trans, m, n, alpha, a, lda, x, incx, beta, y, incy, *, dtype=None) -> int:
    """y := alpha*op(A)*x + beta*y (mojoBLAS gemv, gemv.mojo:23-212)."""
    dt = _dtype_of(y, dtype)
    lib = L.load()
    args = (_ch(trans), m, n, float(alpha), _ptr(a), lda, _ptr(x), incx, float(beta), _ptr(y), incy)
    if dt == np.float32:
        st = lib.mbg_sgemv(*args)
    elif dt == np.float64:
        st = lib.mbg_dgemv(*args)
    else:
        raise TypeError(f"unsupported dtype {dt}")
    return _report("gemv", st)


def trsv(uplo, trans, diag, n, a, lda, x, incx, *, dtype=None) -> int:
    """op(A) x = b, the solution overwrites x (mojoBLAS trsv, trsv.mojo:20-214)."""
    dt = _dtype_of(x, dtype)
    lib = L.load()
    args = (_ch(uplo), _ch(trans), _ch(diag), n, _ptr(a), lda, _ptr(x), incx)
    if dt == np.float32:
        st = lib.mbg_strsv(*args)
    elif dt == np.float64:
        st = lib.mbg_dtrsv(*args)
    else:
        raise TypeError(f"unsupported dtype {dt}")
    return _report("trsv", st)
