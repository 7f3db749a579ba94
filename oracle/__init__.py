"""ORACLE — test infrastructure only.

Python access to the CPU restatement of mojoBLAS's level-3 routines and of
gemv / trsv (ref_level3.cpp, ref_level2.cpp, built into liboracle_level3.so by
the Makefile beside it) plus
float64 / extended-precision reference products.  Only tests, the smoke check
and bench.py's CPU-baseline legs import this package; the CUDA library never
does.

Matrices are numpy arrays holding column-major storage: a matrix with leading
dimension ld and n columns is a 1-D buffer (or a Fortran-ordered 2-D array)
whose element (i, j) sits at flat index i + j*ld.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_level3.so"
BUG_COMPAT = 1  # reproduce the reference's quirks (v7 alpha, right/trans trsm, symm zero skip)

_lib = None


def build() -> Path:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        i64, f32p, f64p = C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_double)
        ch = C.c_char
        sig = {
            "orc_sgemm": [ch, ch, i64, i64, i64, C.c_float, f32p, i64, f32p, i64, C.c_float, f32p, i64, C.c_int],
            "orc_dgemm": [ch, ch, i64, i64, i64, C.c_double, f64p, i64, f64p, i64, C.c_double, f64p, i64, C.c_int],
            "orc_sgemm_naive": [ch, ch, i64, i64, i64, C.c_float, f32p, i64, f32p, i64, C.c_float, f32p, i64],
            "orc_dgemm_naive": [ch, ch, i64, i64, i64, C.c_double, f64p, i64, f64p, i64, C.c_double, f64p, i64],
            "orc_sgemm_v11": [i64, i64, i64, C.c_float, f32p, i64, f32p, i64, C.c_float, f32p, i64],
            "orc_dgemm_v3": [i64, i64, i64, C.c_double, f64p, i64, f64p, i64, C.c_double, f64p, i64],
            "orc_dgemm_v7": [i64, i64, i64, C.c_double, f64p, i64, f64p, i64, C.c_double, f64p, i64, C.c_int],
            "orc_ssyrk": [ch, ch, i64, i64, C.c_float, f32p, i64, C.c_float, f32p, i64],
            "orc_dsyrk": [ch, ch, i64, i64, C.c_double, f64p, i64, C.c_double, f64p, i64],
            "orc_strsm": [ch, ch, ch, ch, i64, i64, C.c_float, f32p, i64, f32p, i64, C.c_int],
            "orc_dtrsm": [ch, ch, ch, ch, i64, i64, C.c_double, f64p, i64, f64p, i64, C.c_int],
            "orc_ssymm": [ch, ch, i64, i64, C.c_float, f32p, i64, f32p, i64, C.c_float, f32p, i64, C.c_int],
            "orc_dsymm": [ch, ch, i64, i64, C.c_double, f64p, i64, f64p, i64, C.c_double, f64p, i64, C.c_int],
            "orc_ssyr2k": [ch, ch, i64, i64, C.c_float, f32p, i64, f32p, i64, C.c_float, f32p, i64],
            "orc_dsyr2k": [ch, ch, i64, i64, C.c_double, f64p, i64, f64p, i64, C.c_double, f64p, i64],
            "orc_strmm": [ch, ch, ch, ch, i64, i64, C.c_float, f32p, i64, f32p, i64],
            "orc_sgemv": [ch, i64, i64, C.c_float, f32p, i64, f32p, i64, C.c_float, f32p, i64],
            "orc_dgemv": [ch, i64, i64, C.c_double, f64p, i64, f64p, i64, C.c_double, f64p, i64],
            "orc_strsv": [ch, ch, ch, i64, f32p, i64, f32p, i64],
            "orc_dtrsv": [ch, ch, ch, i64, f64p, i64, f64p, i64],
            "orc_dtrmm": [ch, ch, ch, ch, i64, i64, C.c_double, f64p, i64, f64p, i64],
        }
        for name, argtypes in sig.items():
            fn = getattr(_lib, name)
            fn.argtypes = argtypes
            fn.restype = C.c_int
        _lib.orc_dgemm_dot2_rows.argtypes = [ch, ch, i64, i64, f64p, i64, f64p, i64, C.POINTER(C.c_int64), i64,
                                             f64p]
        _lib.orc_dgemm_dot2_rows.restype = C.c_int
        _lib.orc_fma.argtypes = [i64, f64p, f64p, f64p, f64p]
        _lib.orc_fma.restype = C.c_int
        _lib.orc_set_threads.argtypes = [C.c_int]
        _lib.orc_max_threads.restype = C.c_int
        _lib.orc_naive_threads.restype = C.c_int
    return _lib


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def max_threads() -> int:
    return lib().orc_max_threads()


def naive_threads() -> int:
    """Threads that ran the column loop of the last gemm_naive call (1 below the
    reference's parallel threshold of 64 columns, gemm.mojo:255)."""
    return lib().orc_naive_threads()


def _p(x: np.ndarray, dt):
    assert x.dtype == dt and (x.flags.f_contiguous or x.ndim == 1), "column-major buffer expected"
    return x.ctypes.data_as(C.POINTER(C.c_float if dt == np.float32 else C.c_double))


def _c(t) -> bytes:
    return t.encode() if isinstance(t, str) else t


def _dt(x):
    return np.float32 if x.dtype == np.float32 else np.float64


def gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, flags=0) -> int:
    """The reference's gemm dispatch (gemm.mojo:56-124), in place on c."""
    dt = _dt(c)
    fn = lib().orc_sgemm if dt == np.float32 else lib().orc_dgemm
    return fn(_c(ta), _c(tb), m, n, k, alpha, _p(a, dt), lda, _p(b, dt), ldb, beta, _p(c, dt), ldc, flags)


def gemm_naive(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> int:
    dt = _dt(c)
    fn = lib().orc_sgemm_naive if dt == np.float32 else lib().orc_dgemm_naive
    return fn(_c(ta), _c(tb), m, n, k, alpha, _p(a, dt), lda, _p(b, dt), ldb, beta, _p(c, dt), ldc)


def sgemm_v11(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> int:
    f = np.float32
    return lib().orc_sgemm_v11(m, n, k, alpha, _p(a, f), lda, _p(b, f), ldb, beta, _p(c, f), ldc)


def dgemm_v7(m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, flags=0) -> int:
    f = np.float64
    return lib().orc_dgemm_v7(m, n, k, alpha, _p(a, f), lda, _p(b, f), ldb, beta, _p(c, f), ldc, flags)


def syrk(uplo, trans, n, k, alpha, a, lda, beta, c, ldc) -> int:
    dt = _dt(c)
    fn = lib().orc_ssyrk if dt == np.float32 else lib().orc_dsyrk
    return fn(_c(uplo), _c(trans), n, k, alpha, _p(a, dt), lda, beta, _p(c, dt), ldc)


def trsm(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb, flags=0) -> int:
    dt = _dt(b)
    fn = lib().orc_strsm if dt == np.float32 else lib().orc_dtrsm
    return fn(_c(side), _c(uplo), _c(ta), _c(diag), m, n, alpha, _p(a, dt), lda, _p(b, dt), ldb, flags)


def symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc, flags=0) -> int:
    """The reference's symm (symm.mojo:20-241), in place on c."""
    dt = _dt(c)
    fn = lib().orc_ssymm if dt == np.float32 else lib().orc_dsymm
    return fn(_c(side), _c(uplo), m, n, alpha, _p(a, dt), lda, _p(b, dt), ldb, beta, _p(c, dt), ldc, flags)


def syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> int:
    """The reference's syr2k (syr2k.mojo:20-190), in place on c."""
    dt = _dt(c)
    fn = lib().orc_ssyr2k if dt == np.float32 else lib().orc_dsyr2k
    return fn(_c(uplo), _c(trans), n, k, alpha, _p(a, dt), lda, _p(b, dt), ldb, beta, _p(c, dt), ldc)


def trmm(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb) -> int:
    """The reference's trmm (trmm.mojo:20-305), in place on b."""
    dt = _dt(b)
    fn = lib().orc_strmm if dt == np.float32 else lib().orc_dtrmm
    return fn(_c(side), _c(uplo), _c(ta), _c(diag), m, n, alpha, _p(a, dt), lda, _p(b, dt), ldb)


def gemv(trans, m, n, alpha, a, lda, x, incx, beta, y, incy) -> int:
    """The reference's gemv (src/level2/gemv.mojo:23-212), in place on y."""
    dt = _dt(y)
    fn = lib().orc_sgemv if dt == np.float32 else lib().orc_dgemv
    return fn(_c(trans), m, n, alpha, _p(a, dt), lda, _p(x, dt), incx, beta, _p(y, dt), incy)


def trsv(uplo, trans, diag, n, a, lda, x, incx) -> int:
    """The reference's trsv (src/level2/trsv.mojo:20-214), in place on x."""
    dt = _dt(x)
    fn = lib().orc_strsv if dt == np.float32 else lib().orc_dtrsv
    return fn(_c(uplo), _c(trans), _c(diag), n, _p(a, dt), lda, _p(x, dt), incx)


def vec(buf: np.ndarray, n: int, inc: int) -> np.ndarray:
    """The n-vector stored in buf with increment inc (inc < 0: element 0 at (1 - n) * inc)."""
    start = 0 if inc > 0 else (1 - n) * inc
    return buf[start + np.arange(n) * inc]


def gemv_f64(trans, m, n, alpha, a, lda, x, incx, beta, y, incy) -> np.ndarray:
    """float64 y := alpha op(A) x + beta y as a dense vector (y untouched)."""
    A = view(a, m, n, lda).astype(np.float64)
    notrans = _c(trans) in (b"N", b"n")
    lenx, leny = (n, m) if notrans else (m, n)
    out = float(alpha) * ((A if notrans else A.T) @ vec(x, lenx, incx).astype(np.float64))
    if beta != 0:
        out = out + float(beta) * vec(y, leny, incy).astype(np.float64)
    return out


def trsv_f64(uplo, trans, diag, n, a, lda, x, incx) -> np.ndarray:
    """float64 solution of op(A) z = x as a dense vector (x untouched)."""
    import scipy.linalg as sl
    A = op(tri(view(a, n, n, lda).astype(np.float64), uplo, diag), trans)
    lower = (_c(uplo) in (b"L", b"l")) == (_c(trans) in (b"N", b"n"))
    return sl.solve_triangular(A, vec(x, n, incx).astype(np.float64), lower=lower)


# ---------------------------------------------------------------------------
# float64 references (Netlib semantics, independent of the reference's code)
# ---------------------------------------------------------------------------

def view(buf: np.ndarray, rows: int, cols: int, ld: int) -> np.ndarray:
    """The rows x cols column-major matrix stored in buf with leading dimension ld."""
    flat = buf.reshape(-1, order="F")
    if rows > 0 and cols > 0:
        assert rows <= ld and (cols - 1) * ld + rows <= flat.size, "matrix exceeds its buffer"
    return np.lib.stride_tricks.as_strided(flat, shape=(rows, cols),
                                           strides=(flat.itemsize, flat.itemsize * ld))


def op(x: np.ndarray, t) -> np.ndarray:
    return x if _c(t) in (b"N", b"n") else x.T


def gemm_f64(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> np.ndarray:
    """float64 C = alpha*op(A)op(B) + beta*C as an m x n array (c untouched)."""
    A = op(view(a, *( (m, k) if _c(ta) in (b"N", b"n") else (k, m)), lda), ta).astype(np.float64)
    B = op(view(b, *( (k, n) if _c(tb) in (b"N", b"n") else (n, k)), ldb), tb).astype(np.float64)
    out = float(alpha) * (A @ B)
    if beta != 0:
        out = out + float(beta) * view(c, m, n, ldc).astype(np.float64)
    return out


def tri(x: np.ndarray, uplo, diag) -> np.ndarray:
    t = np.tril(x) if _c(uplo) in (b"L", b"l") else np.triu(x)
    if _c(diag) in (b"U", b"u"):
        t = t.copy()
        np.fill_diagonal(t, 1.0)
    return t


def trsm_f64(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb) -> np.ndarray:
    """float64 Netlib trsm result X (m x n); b untouched."""
    import scipy.linalg as sl
    na = m if _c(side) in (b"L", b"l") else n
    A = tri(view(a, na, na, lda).astype(np.float64), uplo, diag)
    opA = op(A, ta)
    B = float(alpha) * view(b, m, n, ldb).astype(np.float64)
    lower = bool(np.allclose(opA, np.tril(opA)))
    if _c(side) in (b"L", b"l"):
        return sl.solve_triangular(opA, B, lower=lower)
    # X opA = B  <=>  opA^T X^T = B^T
    return sl.solve_triangular(opA.T, B.T, lower=not lower).T


def sym(x: np.ndarray, uplo) -> np.ndarray:
    """The symmetric matrix whose `uplo` triangle is stored in x (the other triangle ignored)."""
    t = np.tril(x) if _c(uplo) in (b"L", b"l") else np.triu(x)
    return t + t.T - np.diag(np.diag(x))


def symm_f64(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc) -> np.ndarray:
    """float64 Netlib symm result (m x n); c untouched."""
    na = m if _c(side) in (b"L", b"l") else n
    A = sym(view(a, na, na, lda).astype(np.float64), uplo)
    B = view(b, m, n, ldb).astype(np.float64)
    out = float(alpha) * (A @ B if _c(side) in (b"L", b"l") else B @ A)
    if beta != 0:
        out = out + float(beta) * view(c, m, n, ldc).astype(np.float64)
    return out


def syr2k_f64(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc) -> np.ndarray:
    """float64 Netlib syr2k result as a full n x n array; only its `uplo` triangle is defined."""
    shape = (n, k) if _c(trans) in (b"N", b"n") else (k, n)
    A = view(a, *shape, lda).astype(np.float64)
    B = view(b, *shape, ldb).astype(np.float64)
    if _c(trans) not in (b"N", b"n"):
        A, B = A.T, B.T
    out = float(alpha) * (A @ B.T + B @ A.T)
    if beta != 0:
        out = out + float(beta) * view(c, n, n, ldc).astype(np.float64)
    return out


def trmm_f64(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb) -> np.ndarray:
    """float64 Netlib trmm result (m x n); b untouched."""
    na = m if _c(side) in (b"L", b"l") else n
    opA = op(tri(view(a, na, na, lda).astype(np.float64), uplo, diag), ta)
    B = view(b, m, n, ldb).astype(np.float64)
    return float(alpha) * (opA @ B if _c(side) in (b"L", b"l") else B @ opA)


def gemm_rows_dot2(ta, tb, n, k, a, lda, b, ldb, rows) -> np.ndarray:
    """Rows `rows` of op(A) op(B) (float64 inputs, shape (len(rows), n)), every element a
    compensated dot product (dot2.cpp): as accurate as a twice-working-precision sum,
    so a float64 GEMM's own rounding error shows against it."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    out = np.empty((len(rows), n), dtype=np.float64, order="F")
    lib().orc_dgemm_dot2_rows(_c(ta), _c(tb), n, k, _p(a, np.float64), lda, _p(b, np.float64), ldb,
                              rows.ctypes.data_as(C.POINTER(C.c_int64)), len(rows), _p(out, np.float64))
    return out


def ozaki_max_k(slices: int) -> int:
    """The longest k one Ozaki launch keeps exact in int32: s pairs of digits of magnitude
    at most 128 per k step, rounded down to the 32-byte k slab."""
    return ((2 ** 31 - 1) // (int(slices) * 128 * 128)) // 32 * 32


def ozaki_gemm_emulated(ta, tb, m, n, k, alpha, a, lda, b, ldb, slices, beta=0.0, c=None, ldc=None) -> np.ndarray:
    """The library's Ozaki dgemm restated step by step on the CPU, as the checker for
    bit-for-bit comparisons with the GPU result.  For each k chunk of at most
    ozaki_max_k(s) columns (one GPU launch each):

    1. e = frexp exponent of the largest magnitude of each row of op(A) and each
       column of op(B) within the chunk (0 for an all-zero one): every value is below 2^e;
    2. G = trunc(x 2^(8s - 2 - e)) (exact: x keeps its 53-bit significand);
    3. G's signed base-256 digits, most significant first, from the bytes of
       G + 0x80...80 (s bytes, modulo 2^64), each XOR 0x80 read as int8;
    4. for each diagonal d = p + q < s the exact integer product
       D_d = sum_{p+q=d} A_p B_q (int32 on the GPU, exact within the chunk);
    5. acc = sum of D_d 2^(-8d-12) in fp64 from d = s-1 down to 0 (each product is
       exact, so this is the kernel's fused multiply-add order), v = alpha (acc 2^(e_row + e_col)).
    The first chunk writes v (beta = 0) or C + v (beta = 1, the GPU's L2 reduction); each
    later chunk adds its v with one rounding.  beta must be 0 or 1 (c and ldc given for 1),
    and the scalings must neither overflow nor underflow.  Returns C (m x n, float64)."""
    assert beta in (0.0, 1.0)
    A = op(view(np.asarray(a, np.float64), *((m, k) if _c(ta) in (b"N", b"n") else (k, m)), lda), ta)
    Bm = op(view(np.asarray(b, np.float64), *((k, n) if _c(tb) in (b"N", b"n") else (n, k)), ldb), tb)
    s = int(slices)
    nbits = 8 * s - 2

    def exponents(x, axis):
        mx = np.max(np.abs(x), axis=axis) if x.size else np.zeros(x.shape[1 - axis])
        e = np.frexp(mx)[1].astype(np.int64)
        return np.where(mx > 0, e, 0)

    def digits(x, e):
        G = np.trunc(np.ldexp(x, (nbits - e).astype(np.int32))).astype(np.int64)
        bias = np.uint64(0x8080808080808080 >> (64 - 8 * s))
        H = G.astype(np.uint64) + bias  # modulo 2^64
        out = []
        for p in range(s):
            byte = ((H >> np.uint64(8 * (s - 1 - p))) & np.uint64(255)) ^ np.uint64(0x80)
            out.append(byte.astype(np.uint8).view(np.int8).astype(np.float64))
        return out

    out = np.array(view(np.asarray(c, np.float64), m, n, ldc), dtype=np.float64) if beta == 1.0 else None
    kc = min(k, ozaki_max_k(s))
    for k0 in range(0, k, kc):
        Ak, Bk = A[:, k0:k0 + kc], Bm[k0:k0 + kc, :]
        er, ec = exponents(Ak, 1), exponents(Bk, 0)
        # digit products in float64: every partial sum is an integer below k 128^2 s < 2^53, so the
        # BLAS product is exact in any summation order (and equals the GPU's int32 sums)
        dA, dB = digits(Ak, er[:, None]), digits(Bk, ec[None, :])
        acc = np.zeros((m, n))
        for d in range(s - 1, -1, -1):
            D = sum(dA[p] @ dB[d - p] for p in range(d + 1))
            acc = acc + D * 2.0 ** (-8 * d - 12)
        v = alpha * np.ldexp(acc, (er[:, None] + ec[None, :]).astype(np.int32))
        out = v if out is None else out + v
    return out


def ozaki_syrk_emulated(uplo, trans, n, k, alpha, a, lda, slices) -> np.ndarray:
    """The library's Ozaki dsyrk (beta = 0) restated: one set of planes and exponents
    serves op(A) and op(A)^T, so the stored triangle is the Ozaki product of
    op(A) op(A)^T as ozaki_gemm_emulated forms it; the other triangle is NaN (not
    written).  Returns n x n float64."""
    t = "N" if _c(trans) in (b"N", b"n") else "T"
    full = ozaki_gemm_emulated(t, "T" if t == "N" else "N", n, n, k, alpha, a, lda, a, lda, slices)
    keep = np.tril(np.ones((n, n), bool)) if _c(uplo) in (b"L", b"l") else np.triu(np.ones((n, n), bool))
    return np.where(keep, full, np.nan)


def fma(x, y, z) -> np.ndarray:
    """x y + z element-wise with one rounding (broadcast, float64)."""
    x, y, z = np.broadcast_arrays(*(np.asarray(v, np.float64) for v in (x, y, z)))
    shape = x.shape
    x, y, z = (np.ascontiguousarray(v).reshape(-1) for v in (x, y, z))
    out = np.empty(x.size)
    lib().orc_fma(x.size, _p(x, np.float64), _p(y, np.float64), _p(z, np.float64), _p(out, np.float64))
    return out.reshape(shape)


def ozaki_trmm_emulated(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb, slices) -> np.ndarray:
    """The library's Ozaki dtrmm (in place, triangle order within one exact chunk) restated:
    the strict triangle of op(A) goes through the Ozaki product (its exponents from the
    kept entries only), and the diagonal term is added with one fused multiply-add,
        B := fma(d, B_old, alpha (strict(op(A)) B))   (side 'L', d per row),
        B := fma(d, B_old, alpha (B strict(op(A))))   (side 'R', d per column),
    with d = alpha A(i, i) (alpha for a unit diagonal).  Returns m x n float64."""
    left = _c(side) in (b"L", b"l")
    trans = _c(ta) not in (b"N", b"n")
    lower = (_c(uplo) in (b"L", b"l")) != trans  # op(A) lower triangular
    na = m if left else n
    assert na <= ozaki_max_k(slices)
    Av = view(np.asarray(a, np.float64), na, na, lda)
    opA = Av.T if trans else Av
    strict = np.asfortranarray(np.tril(opA, -1) if lower else np.triu(opA, 1))
    d = np.full(na, float(alpha)) if _c(diag) in (b"U", b"u") else alpha * np.diagonal(Av)
    B = np.asfortranarray(view(np.asarray(b, np.float64), m, n, ldb))
    if left:
        v = ozaki_gemm_emulated("N", "N", m, n, m, alpha, strict, na, B, m, slices)
        return fma(d[:, None], B, v)
    v = ozaki_gemm_emulated("N", "N", m, n, n, alpha, B, m, strict, na, slices)
    return fma(d[None, :], B, v)


def trsm_lower_longdouble(L: np.ndarray, B: np.ndarray) -> np.ndarray:
    """X with L X = B for a lower-triangular L, by forward substitution in x86 extended
    precision (numpy longdouble, 64-bit significand: unit roundoff 2^-64, 2048 times
    below float64's), as a checker for float64 solves whose own error is near 1e-16."""
    n = L.shape[0]
    Ll = np.asarray(L, dtype=np.longdouble)
    X = np.array(B, dtype=np.longdouble, copy=True)
    for i in range(n):
        X[i] = X[i] / Ll[i, i]
        if i + 1 < n:
            X[i + 1:] -= np.outer(Ll[i + 1:, i], X[i])
    return X


def max_rel_err(x: np.ndarray, ref: np.ndarray) -> float:
    """max|x - ref| / max|ref| (normwise, the error metric quoted with every result)."""
    den = float(np.max(np.abs(ref)))
    return float(np.max(np.abs(x.astype(np.float64) - ref))) / (den if den > 0 else 1.0)


def elementwise_err(x: np.ndarray, ref: np.ndarray, bound: np.ndarray) -> float:
    """max_ij |x - ref| / bound_ij, with bound = |alpha| |op(A)| |op(B)| (+|beta||C|)."""
    bound = np.where(bound > 0, bound, 1.0)
    return float(np.max(np.abs(x.astype(np.float64) - ref) / bound))
