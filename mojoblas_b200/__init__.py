"""mojoblas_b200 — B200 (sm_100a) level-3 BLAS behind mojoBLAS's routine signatures.

The product is the C-ABI shared library libmojoblas_gpu.so (include/mojoblas_gpu.h);
this package holds its sources (csrc/), its build recipe (build.py), a ctypes
binding (_lib.py) and a Python mirror of the reference routines (level3.py,
level2.py).
"""
from ._lib import LIB_PATH, load  # noqa: F401
from .level3 import (BF16X3, BF16X6, OZAKI, PLAIN, MbgError, gemm, set_stream,  # noqa: F401
                     set_sync, symm, synchronize, syr2k, syrk, trmm, trsm)
from .level2 import gemv, trsv  # noqa: F401

__all__ = ["gemm", "syrk", "trsm", "symm", "syr2k", "trmm", "gemv", "trsv", "set_stream", "set_sync", "synchronize", "MbgError",
           "PLAIN", "BF16X3", "BF16X6", "OZAKI", "load", "LIB_PATH"]
