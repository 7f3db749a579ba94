"""The GPU's Ozaki dgemm equals the oracle's step-by-step restatement of the same
scheme (oracle.ozaki_gemm_emulated) bit for bit: the int32 slice products are
exact and the epilogue's fp64 operations are restated in the kernel's order, so
no tolerance is needed.  Covers one-pass (s <= 4) and two-pass (s > 4) slice
counts, every transpose pair, ragged tiles, a zero row (exponent 0), rows scaled
by 2^[-20, 20], alpha != 1 and beta = 0 (C is not read: it starts as NaN); then, on
both the single-CTA and the CTA-pair kernels, k over several int32-exact chunks
with beta = 1, the dsyrk (one set of planes for both operands) and the in-place
dtrmm (strict triangle through the slices, diagonal term by one FMA)."""
import numpy as np
import pytest

import mojoblas_b200 as mb
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()
    mb.load()


@pytest.mark.parametrize("s", [2, 4, 5, 7, 8])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("m,n,k,scaled", [(96, 80, 300, False), (130, 257, 1000, True)])
def test_ozaki_bit_exact(oracle, s, ta, tb, m, n, k, scaled):
    rng = np.random.default_rng(m + n + k + s)
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ra + 1, ca)))
    b = np.asfortranarray(rng.uniform(-1, 1, (rb + 2, cb)))
    if scaled:  # rows of op(A) and the k rows of op(B) by 2^u, u in [-20, 20]
        su, sv = 2.0 ** rng.integers(-20, 21, m), 2.0 ** rng.integers(-20, 21, k)
        if ta == "N":
            a[:m, :] *= su[:, None]
        else:
            a[:, :m] *= su[None, :]
        if tb == "N":
            b[:k, :] *= sv[:, None]
        else:
            b[:, :k] *= sv[None, :]
    if ta == "N":  # one all-zero row of op(A)
        a[3, :] = 0.0
    else:
        a[:, 3] = 0.0
    c = np.full((m, n), np.nan, order="F")
    assert mb.gemm(ta, tb, m, n, k, 1.25, a, ra + 1, b, rb + 2, 0.0, c, m, mode=mb.OZAKI, slices=s) == 0
    want = oracle.ozaki_gemm_emulated(ta, tb, m, n, k, 1.25, a, ra + 1, b, rb + 2, s)
    assert np.array_equal(c, want), (np.max(np.abs(c - want)), np.sum(c != want))


@pytest.fixture(params=[0, 1], ids=["one-cta", "cta-pair"])
def ozaki_kernel(request):
    """Runs the test with the single-CTA Ozaki kernel, then with the CTA-pair kernel."""
    from mojoblas_b200 import _lib as L
    lib = L.load()
    default = lib.mbg_get_tuning(b"ozaki_cta_pair")
    assert lib.mbg_set_tuning(b"ozaki_cta_pair", request.param) == 0
    yield request.param
    lib.mbg_set_tuning(b"ozaki_cta_pair", default)


def test_ozaki_bit_exact_chunked_k_beta_one(oracle, ozaki_kernel):
    """k over two chunk boundaries of the int32-exact range (8 slices: chunks of 16352),
    each chunk with its own exponents and launch, added to C with beta = 1 (one L2
    reduction per element and chunk), part of k at another scale."""
    rng = np.random.default_rng(71)
    m, n, k = 40, 24, 2 * 16352 + 100
    a = np.asfortranarray(rng.uniform(-1, 1, (k, m)))
    b = np.asfortranarray(rng.uniform(-1, 1, (k, n)))
    a[20000:, :] *= 2.0 ** 12
    c0 = np.asfortranarray(rng.uniform(-1, 1, (m + 1, n)))
    c = c0.copy(order="F")
    assert mb.gemm("T", "N", m, n, k, 1.0, a, k, b, k, 1.0, c, m + 1, mode=mb.OZAKI, slices=8) == 0
    want = oracle.ozaki_gemm_emulated("T", "N", m, n, k, 1.0, a, k, b, k, 8, beta=1.0, c=c0, ldc=m + 1)
    assert np.array_equal(c[:m], want), (np.max(np.abs(c[:m] - want)), np.sum(c[:m] != want))
    np.testing.assert_array_equal(c[m:], c0[m:])


@pytest.mark.parametrize("uplo,trans", [("L", "N"), ("U", "T")])
def test_ozaki_syrk_bit_exact(oracle, ozaki_kernel, uplo, trans):
    """dsyrk: one set of planes for op(A) and op(A)^T; the stored triangle equals the
    restatement bit for bit, the other triangle is left as it was."""
    rng = np.random.default_rng(72)
    n, k = 300, 260
    a = np.asfortranarray(rng.uniform(-1, 1, ((n if trans == "N" else k) + 1, k if trans == "N" else n)))
    lda = a.shape[0]
    c0 = np.asfortranarray(rng.uniform(-1, 1, (n, n)))
    c = c0.copy(order="F")
    assert mb.syrk(uplo, trans, n, k, 0.5, a, lda, 0.0, c, n, mode=mb.OZAKI, slices=7) == 0
    want = oracle.ozaki_syrk_emulated(uplo, trans, n, k, 0.5, a, lda, 7)
    keep = ~np.isnan(want)
    assert np.array_equal(c[keep], want[keep])
    np.testing.assert_array_equal(c[~keep], c0[~keep])


@pytest.mark.parametrize("side,uplo,ta,diag", [("L", "L", "N", "N"), ("L", "U", "T", "U"), ("R", "L", "T", "N"),
                                               ("R", "U", "N", "U")])
def test_ozaki_trmm_bit_exact(oracle, ozaki_kernel, side, uplo, ta, diag):
    """In-place dtrmm: the strict triangle through the slices (exponents of the kept
    entries only), the diagonal term by one fused multiply-add in the epilogue."""
    rng = np.random.default_rng(73)
    m, n = 260, 200
    na = m if side == "L" else n
    a = rng.standard_normal((na + 1, na)) / np.sqrt(na)
    a[np.arange(na), np.arange(na)] = na + np.abs(rng.standard_normal(na))
    a = np.asfortranarray(a)
    b0 = np.asfortranarray(rng.uniform(-1, 1, (m + 2, n)))
    b = b0.copy(order="F")
    assert mb.trmm(side, uplo, ta, diag, m, n, 1.5, a, na + 1, b, m + 2, mode=mb.OZAKI, slices=7) == 0
    want = oracle.ozaki_trmm_emulated(side, uplo, ta, diag, m, n, 1.5, a, na + 1, b0, m + 2, 7)
    assert np.array_equal(b[:m], want), (np.max(np.abs(b[:m] - want)), np.sum(b[:m] != want))
    np.testing.assert_array_equal(b[m:], b0[m:])


def test_fused_and_separate_slicing_agree(oracle):
    """K-contiguous operands (op(A) = A^T, op(B) = B) are sliced in one pass by default;
    the separate exponent and slicing kernels give the same planes, so the same product."""
    from mojoblas_b200 import _lib as L
    lib = L.load()
    rng = np.random.default_rng(74)
    m, n, k = 200, 150, 777
    a = np.asfortranarray(rng.uniform(-1, 1, (k + 1, m)))
    b = np.asfortranarray(rng.uniform(-1, 1, (k + 3, n)))
    a[:, 5] = 0.0  # an all-zero row of op(A)
    out = []
    default = lib.mbg_get_tuning(b"ozaki_fused_slicing")
    try:
        for fused in (1, 0):
            assert lib.mbg_set_tuning(b"ozaki_fused_slicing", fused) == 0
            c = np.full((m, n), np.nan, order="F")
            assert mb.gemm("T", "N", m, n, k, 1.0, a, k + 1, b, k + 3, 0.0, c, m, mode=mb.OZAKI, slices=7) == 0
            out.append(c)
    finally:
        lib.mbg_set_tuning(b"ozaki_fused_slicing", default)
    assert np.array_equal(out[0], out[1])
    assert np.array_equal(out[0], oracle.ozaki_gemm_emulated("T", "N", m, n, k, 1.0, a, k + 1, b, k + 3, 7))
