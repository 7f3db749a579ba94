"""The Ozaki products on CTA pairs (tcgen05 cta_group::2, 256 x 128 tiles shared
by two SMs) against the single-CTA kernel (128 x 128 tiles) and against the
oracle's step-by-step restatement of the scheme.

Both kernels form the same exact int32 diagonal sums and run the same fp64
epilogue per element, so their results must be identical bit for bit, for
every epilogue form: beta = 0, general beta (C read first), beta = 1 (one L2
reduction per element: the trsm updates), the triangle-masked dsyrk, and the
in-place dtrmm (banded reduction, diagonal term by one fused multiply-add).
Tile counts cover an odd number of 128-row tiles (the last pair's second CTA
holds only padding rows), and the persistent form (each cluster looping over
several tiles) is checked against one cluster per tile, including a launch with
more tiles than clusters (3000 x 1500: 144 pair tiles).
"""
import numpy as np
import pytest

import mojoblas_b200 as mb
from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu, tri_system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    need_gpu()
    mb.load()
    lib = L.load()
    default = lib.mbg_get_tuning(b"ozaki_cta_pair")
    yield lib
    lib.mbg_set_tuning(b"ozaki_cta_pair", default)


def both(lib, call):
    """(pair kernel result, single-CTA kernel result) of call(); the pair kernel run both
    with one cluster per tile and persistent (one cluster per two SMs), which must agree."""
    default = lib.mbg_get_tuning(b"ozaki_cta_pair")
    out = []
    try:
        for pair in (1, 2, 0):
            assert lib.mbg_set_tuning(b"ozaki_cta_pair", pair) == 0
            out.append(call())
    finally:
        lib.mbg_set_tuning(b"ozaki_cta_pair", default)
    assert np.array_equal(out[0], out[1]), "persistent pair kernel differs from one cluster per tile"
    return out[0], out[2]


@pytest.mark.parametrize("s", [3, 7])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T")])
@pytest.mark.parametrize("m,n,k,beta", [(300, 200, 700, 0.0), (129, 385, 96, 0.5), (600, 130, 512, 1.0),
                                        (3000, 1500, 300, 0.5)])
def test_pair_equals_single_cta_gemm(lib, s, ta, tb, m, n, k, beta):
    rng = np.random.default_rng(m * 7 + n + k + s)
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ra, ca)))
    b = np.asfortranarray(rng.uniform(-1, 1, (rb, cb)))
    c0 = np.asfortranarray(rng.uniform(-1, 1, (m + 3, n)))

    def call():
        c = c0.copy(order="F")
        assert mb.gemm(ta, tb, m, n, k, -0.75, a, ra, b, rb, beta, c, m + 3, mode=mb.OZAKI, slices=s) == 0
        return c
    got, want = both(lib, call)
    assert np.array_equal(got, want), (float(np.max(np.abs(got - want))), int(np.sum(got != want)))
    np.testing.assert_array_equal(got[m:], c0[m:])


@pytest.mark.parametrize("m,n,k,ta,tb", [(300, 200, 700, "N", "N"), (385, 129, 1000, "T", "N")])
def test_pair_bit_exact_with_restatement(lib, oracle, m, n, k, ta, tb):
    rng = np.random.default_rng(31)
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ra, ca)))
    b = np.asfortranarray(rng.uniform(-1, 1, (rb, cb)))
    c = np.full((m, n), np.nan, order="F")
    default = lib.mbg_get_tuning(b"ozaki_cta_pair")
    try:
        assert lib.mbg_set_tuning(b"ozaki_cta_pair", 1) == 0
        assert mb.gemm(ta, tb, m, n, k, 1.25, a, ra, b, rb, 0.0, c, m, mode=mb.OZAKI, slices=7) == 0
    finally:
        lib.mbg_set_tuning(b"ozaki_cta_pair", default)
    want = oracle.ozaki_gemm_emulated(ta, tb, m, n, k, 1.25, a, ra, b, rb, 7)
    assert np.array_equal(c, want), (float(np.max(np.abs(c - want))), int(np.sum(c != want)))


@pytest.mark.parametrize("uplo,trans", [("L", "N"), ("U", "T")])
def test_pair_equals_single_cta_syrk(lib, uplo, trans):
    rng = np.random.default_rng(32)
    n, k = 333, 260
    a = np.asfortranarray(rng.uniform(-1, 1, (n, k) if trans == "N" else (k, n)))
    lda = a.shape[0]
    c0 = np.asfortranarray(rng.uniform(-1, 1, (n, n)))

    def call():
        c = c0.copy(order="F")
        assert mb.syrk(uplo, trans, n, k, 1.0, a, lda, 0.5, c, n, mode=mb.OZAKI, slices=7) == 0
        return c
    got, want = both(lib, call)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("side,uplo,ta", [("L", "L", "N"), ("L", "U", "T"), ("R", "L", "N")])
def test_pair_equals_single_cta_trmm_trsm(lib, side, uplo, ta):
    rng = np.random.default_rng(33)
    m, n = 700, 300
    a, b, lda, ldb = tri_system(rng, side, m, n, np.float64)

    def call_trmm():
        x = b.copy(order="F")
        assert mb.trmm(side, uplo, ta, "N", m, n, 0.5, a, lda, x, ldb, mode=mb.OZAKI, slices=7) == 0
        return x

    def call_trsm():
        x = b.copy(order="F")
        assert mb.trsm(side, uplo, ta, "N", m, n, 0.5, a, lda, x, ldb, mode=mb.OZAKI, slices=7) == 0
        return x
    for call in (call_trmm, call_trsm):
        got, want = both(lib, call)
        assert np.array_equal(got, want), call.__name__
