"""Pins the oracle's restatement of the Ozaki scheme (oracle.ozaki_gemm_emulated),
which the GPU tests compare with the library bit for bit, against independent
references on the CPU:

* every transpose pair agrees with a float64 product to float64 accuracy at 7
  slices, and an all-zero row gives exact zeros;
* against compensated (Dot2) products, the error falls by about 2^-8 per added
  slice and stays within the truncation bound: each operand keeps 8s - 2 bits
  of its row's (column's) scale, so |error| <= 2 k 2^-(8s-2) max|A| max|B|
  per element, relative to max|C|;
* k beyond one exact int32 chunk (each chunk with its own exponents, added to C
  one at a time) and beta = 1 stay at float64 rounding;
* the dsyrk restatement (one set of planes: an exactly symmetric product) and the
  in-place dtrmm restatement (strict triangle through the slices, the diagonal
  term by one fused multiply-add, oracle.fma) agree with float64, and never read
  the triangle's other half.
"""
import numpy as np
import pytest


def case(rng, ta, tb, m, n, k):
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ra + 1, ca)))
    b = np.asfortranarray(rng.uniform(-1, 1, (rb + 2, cb)))
    return a, ra + 1, b, rb + 2


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_transposes_and_zero_row(oracle, ta, tb):
    rng = np.random.default_rng(61)
    m, n, k = 37, 29, 55
    a, lda, b, ldb = case(rng, ta, tb, m, n, k)
    if ta == "N":
        a[3, :] = 0.0
    else:
        a[:, 3] = 0.0
    ref = oracle.gemm_f64(ta, tb, m, n, k, 1.25, a, lda, b, ldb, 0.0, np.zeros((m, n), order="F"), m)
    got = oracle.ozaki_gemm_emulated(ta, tb, m, n, k, 1.25, a, lda, b, ldb, 7)
    assert oracle.max_rel_err(got, ref) < 4e-15
    assert np.all(got[3] == 0.0)


def test_error_per_slice(oracle):
    rng = np.random.default_rng(62)
    m, n, k = 96, 80, 300
    a, lda, b, ldb = case(rng, "N", "N", m, n, k)
    ref = oracle.gemm_rows_dot2("N", "N", n, k, a, lda, b, ldb, np.arange(m))
    errs = []
    for s in range(2, 9):
        got = oracle.ozaki_gemm_emulated("N", "N", m, n, k, 1.0, a, lda, b, ldb, s)
        err = oracle.max_rel_err(got, ref)
        bound = 2 * k * 2.0 ** -(8 * s - 2) / np.max(np.abs(ref))  # max|A|, max|B| <= 1
        assert err <= bound + 4 * 2.0 ** -53, (s, err, bound)
        errs.append(err)
    for s in range(2, 7):  # about 2^-8 per slice until the fp64 epilogue's own rounding is reached
        assert errs[s - 1] < errs[s - 2] / 64, errs
    assert errs[-2] < 2 * 2.0 ** -53 and errs[-1] < 2 * 2.0 ** -53  # 7 and 8 slices: at fp64 rounding


def test_chunked_k_and_beta_one(oracle):
    """k over two chunk boundaries (8 slices: chunks of ozaki_max_k(8) = 16352), each chunk with its
    own exponents, added to C one chunk at a time; beta = 1 adds to C's values."""
    assert oracle.ozaki_max_k(8) == 16352 and oracle.ozaki_max_k(7) == 18720
    rng = np.random.default_rng(63)
    m, n, k = 16, 12, 2 * 16352 + 100
    a = np.asfortranarray(rng.uniform(-1, 1, (k, m)))  # op(A) = A^T, k-contiguous
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    a[20000:, :] *= 2.0 ** 12  # k from 20000 on (part of the second chunk, all of the third) at another scale
    c = np.asfortranarray(rng.uniform(-1, 1, (m + 1, n)))
    ref = oracle.gemm_rows_dot2("T", "N", n, k, a, k, b, k, np.arange(m))
    got0 = oracle.ozaki_gemm_emulated("T", "N", m, n, k, 1.0, a, k, b, k, 8)
    assert oracle.max_rel_err(got0, ref) < 4 * 2.0 ** -53
    got1 = oracle.ozaki_gemm_emulated("T", "N", m, n, k, 1.0, a, k, b, k, 8, beta=1.0, c=c, ldc=m + 1)
    assert oracle.max_rel_err(got1, ref + c[:m]) < 4 * 2.0 ** -53


@pytest.mark.parametrize("uplo,trans", [("L", "N"), ("U", "T")])
def test_syrk_restatement(oracle, uplo, trans):
    """The dsyrk restatement: the stored triangle of alpha op(A) op(A)^T at float64 accuracy, the
    other triangle left unwritten (NaN), symmetric entries bit-identical (one set of planes)."""
    rng = np.random.default_rng(64)
    n, k = 45, 70
    a = np.asfortranarray(rng.uniform(-1, 1, ((n if trans == "N" else k) + 1, k if trans == "N" else n)))
    lda = a.shape[0]
    got = oracle.ozaki_syrk_emulated(uplo, trans, n, k, 0.5, a, lda, 7)
    A = oracle.op(oracle.view(a, *((n, k) if trans == "N" else (k, n)), lda), trans)
    ref = 0.5 * A @ A.T
    keep = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    assert np.all(np.isnan(got[~keep]))
    assert np.max(np.abs(got[keep] - ref[keep])) / np.max(np.abs(ref)) < 4e-15
    full = oracle.ozaki_gemm_emulated("N" if trans == "N" else "T", "T" if trans == "N" else "N", n, n, k, 0.5,
                                      a, lda, a, lda, 7)
    assert np.array_equal(full, full.T)  # the same planes on both sides: an exactly symmetric product


def test_fma_rounds_once(oracle):
    x = 1.0 + 2.0 ** -30
    p = x * x  # 1 + 2^-29 + 2^-60 rounds to 1 + 2^-29
    assert oracle.fma(x, x, -p) == 2.0 ** -60
    assert np.array_equal(oracle.fma(np.array([2.0, 3.0]), 0.5, 1.0), np.array([2.0, 2.5]))


@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
def test_trmm_restatement(oracle, side, uplo, ta, diag):
    """The dtrmm restatement against float64, for every side / uplo / trans / diag; the
    triangle's other half and (for a unit diagonal) the diagonal are never read (NaN)."""
    rng = np.random.default_rng(65)
    m, n = 40, 33
    na = m if side == "L" else n
    a = rng.standard_normal((na + 1, na)) / np.sqrt(na)
    a[np.arange(na), np.arange(na)] = na + np.abs(rng.standard_normal(na))  # a dominant diagonal
    other = np.triu(np.ones((na, na), bool), 1) if uplo == "L" else np.tril(np.ones((na, na), bool), -1)
    if diag == "U":
        other |= np.eye(na, dtype=bool)
    a_nan = a.copy()
    a_nan[:na][other] = np.nan
    a, a_nan = np.asfortranarray(a), np.asfortranarray(a_nan)
    b = np.asfortranarray(rng.uniform(-1, 1, (m + 2, n)))
    ref = oracle.trmm_f64(side, uplo, ta, diag, m, n, 1.5, a, na + 1, b, m + 2)
    got = oracle.ozaki_trmm_emulated(side, uplo, ta, diag, m, n, 1.5, a_nan, na + 1, b, m + 2, 7)
    assert np.all(np.isfinite(got))
    # the float64 reference rounds too (about sqrt(na) units of 2^-53): the float64 tolerance of the parity tests
    assert oracle.max_rel_err(got, ref) < 4e-16 * np.sqrt(max(na, 16))
