"""Python mirror of mojoBLAS's level-3 routines on the CUDA library.

Same routine names, argument order and meaning as the reference
(src/level3/gemm.mojo:56, syrk.mojo:20, trsm.mojo:20, symm.mojo:20, syr2k.mojo:20,
trmm.mojo:20; docs/reference.md:264-325): column-major storage with leading
dimensions, Netlib transpose / uplo / side / diag characters, results written in
place into `c` (gemm, syrk, symm, syr2k) or `b` (trsm, trmm).
The dtype is taken from the buffers (float32 or float64), as the reference
takes it from its `dtype` parameter; gemm also takes complex64 / complex128
buffers (cgemm / zgemm, with trans 'C' the conjugate transpose).

Buffers may be numpy arrays (host memory; the library stages the copies),
torch tensors (host or CUDA) or raw integer addresses with an explicit dtype.
An invalid argument behaves like the reference: "<routine>: Info <n>" is
printed and n is returned.  A CUDA-side failure raises MbgError.

Keyword extensions (not in the reference): `mode` (PLAIN, BF16X3, BF16X6 for
float32; PLAIN, OZAKI for float64), `slices` (Ozaki int8 slices, 2..8; s slices
keep 8s - 2 bits, and the default 7 meets plain FP64's error) and
`refine` (trsm iterative-refinement steps).
"""
from __future__ import annotations

import numpy as np

from . import _lib as L

PLAIN, BF16X3, BF16X6, OZAKI = L.MODE_PLAIN, L.MODE_BF16X3, L.MODE_BF16X6, L.MODE_OZAKI


class MbgError(RuntimeError):
    def __init__(self, routine: str, status: int):
        self.status = status
        super().__init__(f"{routine}: {L.status_string(status)} ({status}): {L.last_error()}")


def _dtype_of(x, dtype=None):
    if dtype is not None:
        return np.dtype(dtype)
    if isinstance(x, np.ndarray):
        return x.dtype
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return {torch.float32: np.dtype(np.float32), torch.float64: np.dtype(np.float64),
                    torch.complex64: np.dtype(np.complex64), torch.complex128: np.dtype(np.complex128)}[x.dtype]
    except ImportError:
        pass
    raise TypeError("pass dtype= for raw pointers")


def _ptr(x) -> int:
    if x is None:
        return 0
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        if not (x.flags.f_contiguous or x.flags.c_contiguous and x.ndim == 1):
            raise ValueError("numpy buffers must be contiguous column-major storage")
        return x.ctypes.data
    return int(x.data_ptr())  # torch.Tensor


def _ch(t: str) -> bytes:
    return t.encode()[:1] if isinstance(t, str) else bytes(t)[:1]


def _report(routine: str, st: int) -> int:
    if st > 0:
        print(f"{routine}: Info", st)  # the reference prints and returns (gemm.mojo:211-213)
        return st
    if st < 0:
        raise MbgError(routine, st)
    return 0


def gemm(trans_a, trans_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, *, mode=PLAIN,
         slices=7, dtype=None) -> int:
    """C := alpha*op(A)*op(B) + beta*C (mojoBLAS gemm, gemm.mojo:56-124)."""
    dt = _dtype_of(c, dtype)
    lib = L.load()
    if dt == np.float32:
        args = (_ch(trans_a), _ch(trans_b), m, n, k, float(alpha), _ptr(a), lda, _ptr(b), ldb,
                float(beta), _ptr(c), ldc)
        st = lib.mbg_sgemm(*args) if mode == PLAIN else lib.mbg_sgemm_ex(mode, *args)
    elif dt == np.float64:
        args = (_ch(trans_a), _ch(trans_b), m, n, k, float(alpha), _ptr(a), lda, _ptr(b), ldb,
                float(beta), _ptr(c), ldc)
        st = lib.mbg_dgemm(*args) if mode == PLAIN else lib.mbg_dgemm_ex(mode, slices, *args)
    elif dt in (np.complex64, np.complex128):
        # complex (an extension: complex dtypes are on the reference's roadmap, README.md:152);
        # trans 'C' is the conjugate transpose; alpha and beta are complex scalars
        rt = np.float32 if dt == np.complex64 else np.float64
        al = np.array([complex(alpha).real, complex(alpha).imag], rt)
        be = np.array([complex(beta).real, complex(beta).imag], rt)
        args = (_ch(trans_a), _ch(trans_b), m, n, k, al.ctypes.data, _ptr(a), lda, _ptr(b), ldb,
                be.ctypes.data, _ptr(c), ldc)
        if dt == np.complex64:
            st = lib.mbg_cgemm(*args) if mode == PLAIN else lib.mbg_cgemm_ex(mode, *args)
        else:
            st = lib.mbg_zgemm(*args) if mode == PLAIN else lib.mbg_zgemm_ex(mode, slices, *args)
    else:
        raise TypeError(f"unsupported dtype {dt}")
    return _report("gemm", st)


def syrk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc, *, mode=PLAIN, slices=7, dtype=None) -> int:
    """C := alpha*A*A^T + beta*C or alpha*A^T*A + beta*C on one triangle (syrk.mojo:20-200)."""
    dt = _dtype_of(c, dtype)
    lib = L.load()
    args = (_ch(uplo), _ch(trans), n, k, float(alpha), _ptr(a), lda, float(beta), _ptr(c), ldc)
    if dt == np.float32:
        st = lib.mbg_ssyrk(*args) if mode == PLAIN else lib.mbg_ssyrk_ex(mode, *args)
    elif dt == np.float64:
        st = lib.mbg_dsyrk(*args) if mode == PLAIN else lib.mbg_dsyrk_ex(mode, slices, *args)
    else:
        raise TypeError(f"unsupported dtype {dt}")
    return _report("syrk", st)


def trsm(side, uplo, trans_a, diag, m, n, alpha, a, lda, b, ldb, *, mode=PLAIN, slices=7,
         refine=0, dtype=None) -> int:
    """op(A) X = alpha B or X op(A) = alpha B, X overwrites B (trsm.mojo:20-275)."""
    dt = _dtype_of(b, dtype)
    lib = L.load()
    args = (_ch(side), _ch(uplo), _ch(trans_a), _ch(diag), m, n, float(alpha), _ptr(a), lda,
            _ptr(b), ldb)
    if dt == np.float32:
        st = lib.mbg_strsm(*args) if (mode == PLAIN and refine == 0) else \
            lib.mbg_strsm_ex(mode, refine, *args)
    elif dt == np.float64:
        st = lib.mbg_dtrsm(*args) if (mode == PLAIN and refine == 0) else \
            lib.mbg_dtrsm_ex(mode, slices, refine, *args)
    else:
        raise TypeError(f"unsupported dtype {dt}")
    return _report("trsm", st)


def symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, *, mode=PLAIN, slices=7,
         dtype=None) -> int:
    """C := alpha*A*B + beta*C or alpha*B*A + beta*C, A symmetric (symm.mojo:20-241)."""
    dt = _dtype_of(c, dtype)
    lib = L.load()
    args = (_ch(side), _ch(uplo), m, n, float(alpha), _ptr(a), lda, _ptr(b), ldb, float(beta), _ptr(c), ldc)
    if dt == np.float32:
        st = lib.mbg_ssymm(*args) if mode == PLAIN else lib.mbg_ssymm_ex(mode, *args)
    elif dt == np.float64:
        st = lib.mbg_dsymm(*args) if mode == PLAIN else lib.mbg_dsymm_ex(mode, slices, *args)
    else:
        raise TypeError(f"unsupported dtype {dt}")
    return _report("symm", st)


def syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc, *, mode=PLAIN, slices=7,
          dtype=None) -> int:
    """C := alpha*(A*B^T + B*A^T) + beta*C or alpha*(A^T*B + B^T*A) + beta*C on one
    triangle (syr2k.mojo:20-190)."""
    dt = _dtype_of(c, dtype)
    lib = L.load()
    args = (_ch(uplo), _ch(trans), n, k, float(alpha), _ptr(a), lda, _ptr(b), ldb, float(beta), _ptr(c), ldc)
    if dt == np.float32:
        st = lib.mbg_ssyr2k(*args) if mode == PLAIN else lib.mbg_ssyr2k_ex(mode, *args)
    elif dt == np.float64:
        st = lib.mbg_dsyr2k(*args) if mode == PLAIN else lib.mbg_dsyr2k_ex(mode, slices, *args)
    else:
        raise TypeError(f"unsupported dtype {dt}")
    return _report("syr2k", st)


def trmm(side, uplo, trans_a, diag, m, n, alpha, a, lda, b, ldb, *, mode=PLAIN, slices=7,
         dtype=None) -> int:
    """B := alpha*op(A)*B or alpha*B*op(A), A triangular, B overwritten (trmm.mojo:20-305)."""
    dt = _dtype_of(b, dtype)
    lib = L.load()
    args = (_ch(side), _ch(uplo), _ch(trans_a), _ch(diag), m, n, float(alpha), _ptr(a), lda, _ptr(b), ldb)
    if dt == np.float32:
        st = lib.mbg_strmm(*args) if mode == PLAIN else lib.mbg_strmm_ex(mode, *args)
    elif dt == np.float64:
        st = lib.mbg_dtrmm(*args) if mode == PLAIN else lib.mbg_dtrmm_ex(mode, slices, *args)
    else:
        raise TypeError(f"unsupported dtype {dt}")
    return _report("trmm", st)


def set_stream(stream) -> None:
    """Use a cudaStream_t (int address or torch.cuda.Stream) for later calls."""
    h = stream if isinstance(stream, int) else (0 if stream is None else stream.cuda_stream)
    L.load().mbg_set_stream(h)


def set_sync(on: bool) -> None:
    L.load().mbg_set_sync(1 if on else 0)


def synchronize() -> None:
    st = L.load().mbg_synchronize()
    if st:
        raise MbgError("synchronize", st)
