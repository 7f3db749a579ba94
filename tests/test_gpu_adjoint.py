"""Adjoint kernels (gemm and trsm) checked three ways:

1. central finite differences in float64 along 64 seeded random directions:
   for f = <G, C(A, B)> (gemm) or f = <G, X(A, B)> (trsm), the directional
   derivative (f(+h d) - f(-h d)) / 2h must match <dA, dA_dir> + <dB, dB_dir>
   from the kernels within 1e-4 * (|dA||dA_dir| + |dB||dB_dir|) (float32 kernels);
2. the closed-form float64 gradients (numpy / scipy);
3. gradients composed from the reference's own routines (the oracle's
   restatements of mojoBLAS trsm / gemm): dB = trsm(op(A)^T, G), dA = -tri(W X^T).
"""
import numpy as np
import pytest
import scipy.linalg as sl

from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu

N_DIRS = 64


def rel(x, ref):
    return float(np.max(np.abs(np.asarray(x, np.float64) - ref)) / max(np.max(np.abs(ref)), 1e-300))


def opm(x, t):
    return x if t == "N" else x.T


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()


@pytest.mark.parametrize("mode", [L.MODE_PLAIN, L.MODE_BF16X6], ids=["plain", "bf16x6"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_gemm_adjoint(mode, ta, tb):
    lib = L.load()
    rng = np.random.default_rng(31)
    m, n, k, alpha = 96, 80, 72, 1.5
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)).astype(np.float32))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)).astype(np.float32))
    G = np.asfortranarray(rng.standard_normal((m, n)).astype(np.float32))
    dA = np.zeros_like(A, order="F")
    dB = np.zeros_like(B, order="F")
    st = lib.mbg_sgemm_adjoint(mode, ta.encode(), tb.encode(), m, n, k, alpha, A.ctypes.data, A.shape[0],
                               B.ctypes.data, B.shape[0], G.ctypes.data, m, dA.ctypes.data, A.shape[0],
                               dB.ctypes.data, B.shape[0])
    assert st == 0, L.last_error()
    A64, B64, G64 = A.astype(np.float64), B.astype(np.float64), G.astype(np.float64)
    dopA = alpha * G64 @ opm(B64, tb).T
    dopB = alpha * opm(A64, ta).T @ G64
    assert rel(dA, opm(dopA, ta)) < 2e-5
    assert rel(dB, opm(dopB, tb)) < 2e-5

    def f(a, b):
        return float(np.sum(G64 * (alpha * opm(a, ta) @ opm(b, tb))))
    h = 1e-3
    for _ in range(N_DIRS):
        ea, eb = rng.standard_normal(A.shape), rng.standard_normal(B.shape)
        fd = (f(A64 + h * ea, B64 + h * eb) - f(A64 - h * ea, B64 - h * eb)) / (2 * h)
        ad = float(np.sum(dA * ea) + np.sum(dB * eb))
        scale = np.linalg.norm(dA) * np.linalg.norm(ea) + np.linalg.norm(dB) * np.linalg.norm(eb)
        assert abs(fd - ad) <= 1e-4 * scale


@pytest.mark.parametrize("mode", [L.MODE_BF16X3, L.MODE_BF16X6], ids=["bf16x3", "bf16x6"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("m,n,k", [(300, 260, 130), (130, 390, 520), (3072, 2048, 1000)])
def test_gemm_adjoint_split_ragged(mode, ta, tb, m, n, k):
    """Split modes compute dA and dB in one launch: several tiles per product, reductions of
    different lengths (n for dA, m for dB), and leading dimensions above the row counts.  At
    3072 x 2048 x 1000 the two products' 160 wide tiles end in stream-K ranges (tiles shared
    by two ranges get two partial sums): a second call gives the same bits."""
    lib = L.load()
    rng = np.random.default_rng(m + 7 * n + 13 * k)
    pad = 5

    def padded(rows, cols, data=None):
        buf = np.zeros((rows + pad, cols), dtype=np.float32, order="F")
        if data is not None:
            buf[:rows] = data
        return buf

    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    A = padded(ar, ac, rng.uniform(-1, 1, (ar, ac)))
    B = padded(br, bc, rng.uniform(-1, 1, (br, bc)))
    G = padded(m, n, rng.standard_normal((m, n)))
    dA = padded(ar, ac)
    dB = padded(br, bc)
    dA[ar:] = dB[br:] = 7.0  # rows past the matrices stay untouched
    alpha = -0.75
    st = lib.mbg_sgemm_adjoint(mode, ta.encode(), tb.encode(), m, n, k, alpha, A.ctypes.data, ar + pad,
                               B.ctypes.data, br + pad, G.ctypes.data, m + pad, dA.ctypes.data, ar + pad,
                               dB.ctypes.data, br + pad)
    assert st == 0, L.last_error()
    dA2, dB2 = padded(ar, ac), padded(br, bc)
    st = lib.mbg_sgemm_adjoint(mode, ta.encode(), tb.encode(), m, n, k, alpha, A.ctypes.data, ar + pad,
                               B.ctypes.data, br + pad, G.ctypes.data, m + pad, dA2.ctypes.data, ar + pad,
                               dB2.ctypes.data, br + pad)
    assert st == 0, L.last_error()
    np.testing.assert_array_equal(dA2[:ar], dA[:ar])
    np.testing.assert_array_equal(dB2[:br], dB[:br])
    A64, B64, G64 = (x.astype(np.float64) for x in (A[:ar], B[:br], G[:m]))
    dopA = alpha * G64 @ opm(B64, tb).T
    dopB = alpha * opm(A64, ta).T @ G64
    tol = 2e-5 if mode == L.MODE_BF16X6 else 2e-4
    assert rel(dA[:ar], opm(dopA, ta)) < tol
    assert rel(dB[:br], opm(dopB, tb)) < tol
    assert np.all(dA[ar:] == 7.0) and np.all(dB[br:] == 7.0)


def _tri(rng, n, uplo, unit):
    a = rng.standard_normal((n, n)) / np.sqrt(n)
    a[np.arange(n), np.arange(n)] = n + np.abs(rng.standard_normal(n))
    if unit:
        a /= n
    return np.tril(a) if uplo == "L" else np.triu(a)


@pytest.mark.parametrize("mode", [L.MODE_PLAIN, L.MODE_BF16X6], ids=["plain", "bf16x6"])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
def test_trsm_adjoint(oracle, mode, side, uplo, ta, diag):
    lib = L.load()
    rng = np.random.default_rng(32)
    m, n, alpha = 96, 40, 0.75
    na = m if side == "L" else n
    A64 = _tri(rng, na, uplo, diag == "U")
    A = np.asfortranarray(A64.astype(np.float32))
    Bm = np.asfortranarray(rng.standard_normal((m, n)).astype(np.float32))
    G = np.asfortranarray(rng.standard_normal((m, n)).astype(np.float32))
    Aeff = A.astype(np.float64).copy()
    if diag == "U":
        np.fill_diagonal(Aeff, 1.0)
    opA = opm(Aeff, ta)
    low = (uplo == "L") != (ta == "T")

    def solve(a_eff, b):
        oa = opm(a_eff, ta)
        if side == "L":
            return alpha * sl.solve_triangular(oa, b, lower=low)
        return alpha * sl.solve_triangular(oa.T, b.T, lower=not low).T

    X = solve(Aeff, Bm.astype(np.float64))
    Xf = np.asfortranarray(X.astype(np.float32))
    dB = np.zeros((m, n), np.float32, order="F")
    dA = np.zeros((na, na), np.float32, order="F")
    st = lib.mbg_strsm_adjoint(mode, side.encode(), uplo.encode(), ta.encode(), diag.encode(), m, n, alpha,
                               A.ctypes.data, na, Xf.ctypes.data, m, G.ctypes.data, m, dB.ctypes.data, m,
                               dA.ctypes.data, na)
    assert st == 0, L.last_error()
    G64 = G.astype(np.float64)
    # closed form
    if side == "L":
        W = sl.solve_triangular(opA.T, G64, lower=not low)
        dopA = -W @ X.T
    else:
        W = sl.solve_triangular(opA, G64.T, lower=low).T
        dopA = -X.T @ W
    dA_ref = opm(dopA, ta)
    mask = np.tril(np.ones((na, na), bool)) if uplo == "L" else np.triu(np.ones((na, na), bool))
    if diag == "U":
        np.fill_diagonal(mask, False)
    dA_ref = np.where(mask, dA_ref, 0.0)
    assert rel(dB, alpha * W) < 2e-5
    assert rel(np.where(mask, dA, 0.0), dA_ref) < 5e-5
    if diag == "U":
        assert np.all(np.diag(dA) == 0.0)
    # gradients composed from the reference routines (oracle restatements)
    db_orc = G.copy(order="F")
    flip = "T" if ta == "N" else "N"
    oracle.trsm(side, uplo, flip, diag, m, n, alpha, A, na, db_orc, m)
    assert rel(dB, db_orc.astype(np.float64)) < 5e-5
    c_orc = np.zeros((na, na), np.float32, order="F")
    first, second = (db_orc, Xf) if (side == "L") == (ta == "N") else (Xf, db_orc)
    if side == "L":  # -(1/alpha) (first second^T)
        oracle.gemm("N", "T", na, na, n, -1.0 / alpha, first, m, second, m, 0.0, c_orc, na)
    else:            # -(1/alpha) (first^T second)
        oracle.gemm("T", "N", na, na, m, -1.0 / alpha, first, m, second, m, 0.0, c_orc, na)
    assert rel(np.where(mask, dA, 0.0), np.where(mask, c_orc, 0.0).astype(np.float64)) < 5e-5
    # finite differences along random directions on the stored triangle and B
    h = 1e-4

    def f(a_eff, b):
        return float(np.sum(G64 * solve(a_eff, b)))
    B64 = Bm.astype(np.float64)
    for _ in range(N_DIRS):
        ea = np.where(mask, rng.standard_normal((na, na)), 0.0)
        eb = rng.standard_normal((m, n))
        fd = (f(Aeff + h * ea, B64 + h * eb) - f(Aeff - h * ea, B64 - h * eb)) / (2 * h)
        ad = float(np.sum(dA * ea) + np.sum(dB * eb))
        scale = np.linalg.norm(dA * mask) * np.linalg.norm(ea) + np.linalg.norm(dB) * np.linalg.norm(eb)
        assert abs(fd - ad) <= 1e-4 * scale


def test_adjoint_info_codes():
    lib = L.load()
    z = np.zeros(64, np.float32)
    p = z.ctypes.data
    assert lib.mbg_sgemm_adjoint(0, b"X", b"N", 2, 2, 2, 1.0, p, 2, p, 2, p, 2, p, 2, p, 2) == 1
    assert lib.mbg_sgemm_adjoint(0, b"N", b"N", 2, 2, 2, 1.0, p, 2, p, 2, p, 1, p, 2, p, 2) == 12
    assert lib.mbg_strsm_adjoint(0, b"L", b"L", b"N", b"N", 2, 2, 1.0, p, 2, p, 1, p, 2, p, 2, p, 2) == 11
    assert lib.mbg_strsm_adjoint(0, b"L", b"L", b"N", b"N", 3, 2, 1.0, p, 3, p, 3, p, 3, p, 3, p, 2) == 17


# ---- double-precision adjoints: plain FP64 and 8-slice Ozaki -------------------------
@pytest.mark.parametrize("mode", [L.MODE_PLAIN, L.MODE_OZAKI], ids=["plain", "ozaki"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T")])
def test_dgemm_adjoint_closed_form(mode, ta, tb):
    """dA = alpha op^-1(G op(B)^T), dB = alpha op^-1(op(A)^T G) in float64, within the plain FP64
    (4e-16 sqrt(k)) or 8-slice Ozaki (2^-56 * 16 + that) tolerance of the float64 products."""
    lib = L.load()
    rng = np.random.default_rng(41)
    m, n, k, alpha = 300, 200, 260, 1.5
    A = np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)))
    B = np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)))
    G = np.asfortranarray(rng.standard_normal((m, n)))
    dA = np.zeros_like(A, order="F")
    dB = np.zeros_like(B, order="F")
    st = lib.mbg_dgemm_adjoint(mode, 8, ta.encode(), tb.encode(), m, n, k, alpha, A.ctypes.data, A.shape[0],
                               B.ctypes.data, B.shape[0], G.ctypes.data, m, dA.ctypes.data, A.shape[0],
                               dB.ctypes.data, B.shape[0])
    assert st == 0, L.last_error()
    dopA = alpha * G @ opm(B, tb).T
    dopB = alpha * opm(A, ta).T @ G
    tol = 4e-16 * np.sqrt(max(m, n, k)) * 4 + (16 * 2.0 ** -56 if mode == L.MODE_OZAKI else 0.0)
    assert rel(dA, opm(dopA, ta)) < tol
    assert rel(dB, opm(dopB, tb)) < tol


@pytest.mark.parametrize("mode", [L.MODE_PLAIN, L.MODE_OZAKI], ids=["plain", "ozaki"])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("ta", ["N", "T"])
def test_dtrsm_adjoint_closed_form(mode, side, uplo, ta):
    """dB = alpha op(A)^-T G and the stored triangle of dA = -tri(W X^T) (left) or -tri(X^T W)
    (right) in float64; the Ozaki mode computes the triangle-only product with int8 slices."""
    lib = L.load()
    rng = np.random.default_rng(42)
    m, n, alpha = 260, 150, 0.75
    na = m if side == "L" else n
    A = np.asfortranarray(_tri(rng, na, uplo, False))
    Bm = rng.standard_normal((m, n))
    G = np.asfortranarray(rng.standard_normal((m, n)))
    opA = opm(A, ta)
    low = (uplo == "L") != (ta == "T")
    if side == "L":
        X = alpha * sl.solve_triangular(opA, Bm, lower=low)
        W = sl.solve_triangular(opA.T, G, lower=not low)
        dopA = -W @ X.T
    else:
        X = alpha * sl.solve_triangular(opA.T, Bm.T, lower=not low).T
        W = sl.solve_triangular(opA, G.T, lower=low).T
        dopA = -X.T @ W
    Xf = np.asfortranarray(X)
    dB = np.zeros((m, n), order="F")
    dA = np.full((na, na), 7.0, order="F")  # the other triangle must survive
    st = lib.mbg_dtrsm_adjoint(mode, 8, side.encode(), uplo.encode(), ta.encode(), b"N", m, n, alpha,
                               A.ctypes.data, na, Xf.ctypes.data, m, G.ctypes.data, m, dB.ctypes.data, m,
                               dA.ctypes.data, na)
    assert st == 0, L.last_error()
    mask = np.tril(np.ones((na, na), bool)) if uplo == "L" else np.triu(np.ones((na, na), bool))
    dA_ref = opm(dopA, ta)
    tol = 4e-16 * np.sqrt(na) * 16 + (16 * 2.0 ** -56 if mode == L.MODE_OZAKI else 0.0)
    assert rel(dB, alpha * W) < tol
    assert rel(np.where(mask, dA, 0.0), np.where(mask, dA_ref, 0.0)) < tol
    assert np.all(dA[~mask] == 7.0)
