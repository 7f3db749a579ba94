"""Parity of the tensor-core precision forms with the float64 oracle and the
reference's algorithms.

Tolerances (max relative error, normwise max|X - X64| / max|X64|):
    BF16X3 (2-term bf16 split, 3 products):  TOL_X3 = 1.5e-5 (split residual ~2^-17)
    BF16X6 (3-term bf16 split, 6 products):  TOL32(k) = 1e-6 * sqrt(max(k, 16)),
                                             the plain float32 tolerance
    OZAKI s slices (8s - 2 bits kept):       TOL_OZ(s, k) = 16 * 2^(-(8 s - 2)) + TOL64(k),
                                             TOL64(k) = 4e-16 * sqrt(max(k, 16));
                                             rows scaled by 2^[-20, 20]: 64 * 2^(-7 s) + TOL64(k)
Each result is also compared with the oracle's restatement of the reference
routine on the same inputs (within the sum of both tolerances).
"""
import numpy as np
import pytest

import mojoblas_b200 as mb
from tests.gpu_util import need_gpu, rand, tri_system

pytestmark = pytest.mark.gpu

TOL_X3 = 1.5e-5


def tol32(k):
    return 1e-6 * np.sqrt(max(k, 16))


def tol64(k):
    return 4e-16 * np.sqrt(max(k, 16))


def tol_oz(s, k):
    return 16 * 2.0 ** (-(8 * s - 2)) + tol64(k)


def tol_mode(mode, k, slices=8):
    if mode == mb.BF16X3:
        return TOL_X3
    if mode == mb.BF16X6:
        return tol32(k)
    if mode == mb.OZAKI:
        return tol_oz(slices, k)
    raise ValueError(mode)


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()
    mb.load()


def _gemm(oracle, dt, mode, ta, tb, m, n, k, alpha, beta, pad=(0, 0, 0), slices=8, seed=0, scaled=False):
    rng = np.random.default_rng(seed)
    lda = (m if ta in "Nn" else k) + pad[0]
    ldb = (k if tb in "Nn" else n) + pad[1]
    ldc = m + pad[2]
    a = rand(rng, (lda, k if ta in "Nn" else m), dt)
    b = rand(rng, (ldb, n if tb in "Nn" else k), dt)
    if scaled:  # rows of op(A) scaled by 2^u, rows of op(B) (the k dimension) by 2^v, u, v in [-20, 20]
        su = np.exp2(rng.integers(-20, 21, size=m)).astype(dt)
        sv = np.exp2(rng.integers(-20, 21, size=k)).astype(dt)
        oa = oracle.op(oracle.view(a, *((m, k) if ta in "Nn" else (k, m)), lda), ta)
        oa *= su[:, None]
        ob = oracle.op(oracle.view(b, *((k, n) if tb in "Nn" else (n, k)), ldb), tb)
        ob *= sv[:, None]
    c = rand(rng, (ldc, n), dt)
    ref = oracle.gemm_f64(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    c_orc = c.copy(order="F")
    assert oracle.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c_orc, ldc) == 0
    c_gpu = c.copy(order="F")
    assert mb.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c_gpu, ldc, mode=mode, slices=slices) == 0
    return oracle.view(c_gpu, m, n, ldc), oracle.view(c_orc, m, n, ldc), ref, c, c_gpu


# ---- split-precision sgemm ---------------------------------------------------------
@pytest.mark.parametrize("mode", [mb.BF16X3, mb.BF16X6], ids=["bf16x3", "bf16x6"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("m,n,k,alpha,beta,pad", [
    (512, 512, 512, 1.5, 0.5, (0, 0, 0)),     # configuration-1 shape and scalars
    (129, 300, 257, -0.75, 0.0, (3, 1, 5)),   # ragged tiles, padded leading dims
    (1, 1, 1, 2.0, 1.0, (0, 0, 0)),
    (300, 17, 3000, 1.0, -2.0, (1, 0, 2)),
])
def test_split_sgemm_parity(oracle, mode, ta, tb, m, n, k, alpha, beta, pad):
    g, o, ref, c0, c_gpu = _gemm(oracle, np.float32, mode, ta, tb, m, n, k, alpha, beta, pad)
    t = tol_mode(mode, k)
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, o.astype(np.float64)) < t + tol32(k)
    np.testing.assert_array_equal(c_gpu[m:], c0[m:])


@pytest.mark.parametrize("mode", [mb.BF16X3, mb.BF16X6], ids=["bf16x3", "bf16x6"])
@pytest.mark.parametrize("ta,tb", [("N", "T"), ("T", "N")])
@pytest.mark.parametrize("m,n,k,beta", [
    (1000, 1500, 777, 0.0),    # 48 wide tiles: 128 x 128 tiles
    (1300, 1100, 1500, 0.5),   # 55 wide tiles, beta != 0
    (2560, 2048, 700, 0.0),    # 160 wide tiles on 148 SMs: persistent, stream-K ranges
    (2700, 2000, 1000, 0.0),   # ragged stream-K tiles (last rows and columns partial)
])
def test_split_sgemm_tile_schedules(oracle, mode, ta, tb, m, n, k, beta):
    """Mid-size products: 128 x 128 tiles where the wide ones would fill at most half of the
    SMs; with more wide tiles than SMs and beta = 0, a persistent launch whose last tiles are
    divided into equal k-slab ranges, the tiles two ranges share zeroed and both partial sums
    added.  A tile gets at most two partial sums, so a second call gives the same bits."""
    rng = np.random.default_rng(m + n + k)
    lda = (m if ta == "N" else k) + 3
    ldb = (k if tb == "N" else n) + 2
    ldc = m + 5
    a = rand(rng, (lda, k if ta == "N" else m), np.float32)
    b = rand(rng, (ldb, n if tb == "N" else k), np.float32)
    c = rand(rng, (ldc, n), np.float32)
    alpha = -1.25
    ref = oracle.gemm_f64(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    outs = []
    for _ in range(2):
        c_gpu = c.copy(order="F")
        assert mb.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c_gpu, ldc, mode=mode) == 0
        outs.append(c_gpu)
    assert oracle.max_rel_err(oracle.view(outs[0], m, n, ldc), ref) < tol_mode(mode, k)
    np.testing.assert_array_equal(outs[0][m:], c[m:])
    np.testing.assert_array_equal(outs[1], outs[0])


@pytest.mark.parametrize("mode", [mb.BF16X3, mb.BF16X6], ids=["bf16x3", "bf16x6"])
def test_split_sgemm_scaled_rows(oracle, mode):
    """Rows scaled by 2^[-20, 20]: bf16 keeps fp32's exponent range, so the split is unaffected."""
    g, _, ref, _, _ = _gemm(oracle, np.float32, mode, "N", "T", 384, 320, 1024, 1.0, 0.0, scaled=True)
    assert oracle.max_rel_err(g, ref) < tol_mode(mode, 1024)


def test_split_beats_plain_error_at_long_k(oracle):
    """BF16x6 promotes the tensor-core accumulator to fp32 registers every 128 k,
    so its error stays at or below the plain FP32 kernel's as k grows."""
    k = 8192
    g6, _, ref, _, _ = _gemm(oracle, np.float32, mb.BF16X6, "N", "T", 256, 256, k, 1.0, 0.0, seed=3)
    gp, _, ref2, _, _ = _gemm(oracle, np.float32, mb.PLAIN, "N", "T", 256, 256, k, 1.0, 0.0, seed=3)
    assert oracle.max_rel_err(g6, ref) <= oracle.max_rel_err(gp, ref2)


@pytest.mark.parametrize("mode", [mb.BF16X3, mb.BF16X6], ids=["bf16x3", "bf16x6"])
def test_split_sgemm_alpha0_k0_beta0_nan(oracle, mode):
    rng = np.random.default_rng(11)
    m, n = 70, 90
    a, b = rand(rng, (m, 8), np.float32), rand(rng, (8, n), np.float32)
    for alpha, k, beta in ((0.0, 8, 2.0), (1.0, 0, -1.0), (0.0, 8, 0.0)):
        c = rand(rng, (m, n), np.float32)
        c_o, c_g = c.copy(order="F"), c.copy(order="F")
        oracle.gemm("N", "N", m, n, k, alpha, a, m, b, 8, beta, c_o, m)
        mb.gemm("N", "N", m, n, k, alpha, a, m, b, 8, beta, c_g, m, mode=mode)
        np.testing.assert_array_equal(c_g, c_o)
    # beta == 0 never reads C (NaN in C must not leak)
    c = np.full((m, n), np.nan, np.float32, order="F")
    mb.gemm("N", "N", m, n, 8, 1.0, a, m, b, 8, 0.0, c, m, mode=mode)
    assert np.all(np.isfinite(c))


# ---- Ozaki dsyrk (triangle-only int8 product, one set of slices for both operands) ----
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_ozaki_dsyrk_parity(oracle, uplo, trans):
    rng = np.random.default_rng(13)
    n, k, alpha, beta = 600, 333, 1.25, 0.5
    lda = (n if trans == "N" else k) + 2
    a = rand(rng, (lda, k if trans == "N" else n), np.float64)
    c = rand(rng, (n + 1, n), np.float64)
    c_o, c_g = c.copy(order="F"), c.copy(order="F")
    assert oracle.syrk(uplo, trans, n, k, alpha, a, lda, beta, c_o, n + 1) == 0
    assert mb.syrk(uplo, trans, n, k, alpha, a, lda, beta, c_g, n + 1, mode=mb.OZAKI, slices=8) == 0
    A = oracle.op(oracle.view(a, *((n, k) if trans == "N" else (k, n)), lda), trans)
    ref = alpha * A @ A.T + beta * oracle.view(c, n, n, n + 1)
    mask = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    g, o = oracle.view(c_g, n, n, n + 1), oracle.view(c_o, n, n, n + 1)
    den = np.max(np.abs(ref[mask]))
    assert np.max(np.abs(g[mask] - ref[mask])) / den < tol_oz(8, k)
    assert np.max(np.abs(g[mask] - o[mask])) / den < tol_oz(8, k) + tol64(k)
    np.testing.assert_array_equal(g[~mask], oracle.view(c, n, n, n + 1)[~mask])
    np.testing.assert_array_equal(c_g[n:], c[n:])


# ---- split-precision syrk (triangular tile schedule) ---------------------------------
@pytest.mark.parametrize("mode", [mb.BF16X3, mb.BF16X6], ids=["bf16x3", "bf16x6"])
@pytest.mark.parametrize("uplo", ["L", "U"])
@pytest.mark.parametrize("trans", ["N", "T"])
def test_split_syrk_parity(oracle, mode, uplo, trans):
    rng = np.random.default_rng(12)
    n, k, alpha, beta = 600, 333, 1.25, 0.5
    lda = (n if trans == "N" else k) + 2
    a = rand(rng, (lda, k if trans == "N" else n), np.float32)
    c = rand(rng, (n + 1, n), np.float32)
    c_o, c_g = c.copy(order="F"), c.copy(order="F")
    assert oracle.syrk(uplo, trans, n, k, alpha, a, lda, beta, c_o, n + 1) == 0
    assert mb.syrk(uplo, trans, n, k, alpha, a, lda, beta, c_g, n + 1, mode=mode) == 0
    A = oracle.op(oracle.view(a, *((n, k) if trans == "N" else (k, n)), lda), trans).astype(np.float64)
    ref = alpha * A @ A.T + beta * oracle.view(c, n, n, n + 1).astype(np.float64)
    mask = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    g, o = oracle.view(c_g, n, n, n + 1), oracle.view(c_o, n, n, n + 1)
    den = np.max(np.abs(ref[mask]))
    t = tol_mode(mode, k)
    assert np.max(np.abs(g[mask] - ref[mask])) / den < t
    assert np.max(np.abs(g[mask] - o[mask])) / den < t + tol32(k)
    np.testing.assert_array_equal(g[~mask], oracle.view(c, n, n, n + 1)[~mask])
    np.testing.assert_array_equal(c_g[n:], c[n:])


# ---- Ozaki dgemm --------------------------------------------------------------------
@pytest.mark.parametrize("slices", [4, 6, 7, 8])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
def test_ozaki_dgemm_parity(oracle, slices, ta, tb):
    m, n, k = 300, 200, 700
    g, o, ref, c0, c_gpu = _gemm(oracle, np.float64, mb.OZAKI, ta, tb, m, n, k, 1.5, 0.5, pad=(2, 3, 1),
                                 slices=slices)
    t = tol_oz(slices, k)
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, o) < t + tol64(k)
    np.testing.assert_array_equal(c_gpu[m:], c0[m:])


@pytest.mark.parametrize("slices", [7, 8])
def test_ozaki_scaled_rows(oracle, slices):
    """Rows scaled by 2^[-20, 20]: per-row / per-column power-of-two scaling keeps
    the int8 slices exact relative to each row's maximum."""
    g, _, ref, _, _ = _gemm(oracle, np.float64, mb.OZAKI, "N", "N", 256, 192, 512, 1.0, 0.0, slices=slices,
                            scaled=True)
    assert oracle.max_rel_err(g, ref) < 64 * 2.0 ** (-(8 * slices - 2)) + tol64(512)


def test_ozaki_s8_at_least_as_accurate_as_plain_fp64(oracle):
    g, _, ref, _, _ = _gemm(oracle, np.float64, mb.OZAKI, "N", "N", 256, 256, 2048, 1.0, 0.0, slices=8, seed=4)
    gp, _, ref2, _, _ = _gemm(oracle, np.float64, mb.PLAIN, "N", "N", 256, 256, 2048, 1.0, 0.0, seed=4)
    assert oracle.max_rel_err(g, ref) <= oracle.max_rel_err(gp, ref2)


def test_ozaki_int32_chunking_long_k(oracle):
    """k beyond the int32-exact range of one pass (16384 for 8 slices) is split
    into chunks accumulated in fp64."""
    g, _, ref, _, _ = _gemm(oracle, np.float64, mb.OZAKI, "T", "N", 64, 40, 17000, 1.0, 0.25, slices=8)
    assert oracle.max_rel_err(g, ref) < tol_oz(8, 17000)


def test_ozaki_zero_rows_and_columns(oracle):
    rng = np.random.default_rng(13)
    m, n, k = 130, 70, 96
    a = rand(rng, (m, k), np.float64)
    b = rand(rng, (k, n), np.float64)
    a[5, :] = 0.0
    b[:, 9] = 0.0
    c = np.zeros((m, n), order="F")
    mb.gemm("N", "N", m, n, k, 1.0, a, m, b, k, 0.0, c, m, mode=mb.OZAKI, slices=8)
    assert np.all(c[5, :] == 0.0) and np.all(c[:, 9] == 0.0)
    assert oracle.max_rel_err(c, a @ b) < tol_oz(8, k)


# ---- trsm with split / Ozaki trailing updates ------------------------------------------
@pytest.mark.parametrize("dt,mode", [(np.float32, mb.BF16X3), (np.float32, mb.BF16X6), (np.float64, mb.OZAKI)],
                         ids=["f32-bf16x3", "f32-bf16x6", "f64-ozaki"])
@pytest.mark.parametrize("side,uplo,ta", [("L", "L", "N"), ("L", "U", "N"), ("L", "L", "T"), ("L", "U", "T"),
                                          ("R", "U", "N"), ("R", "L", "T")])
@pytest.mark.parametrize("refine", [0, 1])
def test_trsm_modes(oracle, dt, mode, side, uplo, ta, refine):
    rng = np.random.default_rng(14)
    m, n, alpha = 300, 200, 0.5
    a, b, lda, ldb = tri_system(rng, side, m, n, dt, ld_pad=1)
    ref = oracle.trsm_f64(side, uplo, ta, "N", m, n, alpha, a, lda, b, ldb)
    x = b.copy(order="F")
    assert mb.trsm(side, uplo, ta, "N", m, n, alpha, a, lda, x, ldb, mode=mode, slices=8, refine=refine) == 0
    x_o = b.copy(order="F")
    oracle.trsm(side, uplo, ta, "N", m, n, alpha, a, lda, x_o, ldb)
    na = m if side == "L" else n
    t = tol_mode(mode, na) * 4
    g = oracle.view(x, m, n, ldb)
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, oracle.view(x_o, m, n, ldb).astype(np.float64)) < t + 4 * (
        tol32(na) if dt == np.float32 else tol64(na))


def test_dtrsm_configuration3_shape_small(oracle):
    """Left / Lower / NoTrans / NonUnit with the configuration-3 input distribution
    (off-diagonal N(0,1)/sqrt(n), diagonal n + |N(0,1)|), at 1024 for test time."""
    rng = np.random.default_rng(15)
    m = n = 1024
    a, b, lda, ldb = tri_system(rng, "L", m, n, np.float64)
    ref = oracle.trsm_f64("L", "L", "N", "N", m, n, 1.0, a, lda, b, ldb)
    errs = {}
    for label, kw in (("plain", {}), ("ozaki", {"mode": mb.OZAKI, "slices": 8}),
                      ("ozaki_ir", {"mode": mb.OZAKI, "slices": 6, "refine": 1})):
        x = b.copy(order="F")
        assert mb.trsm("L", "L", "N", "N", m, n, 1.0, a, lda, x, ldb, **kw) == 0
        errs[label] = oracle.max_rel_err(x, ref)
    assert errs["plain"] < tol64(m) * 4
    assert errs["ozaki"] < tol_oz(8, m) * 4
    assert errs["ozaki_ir"] < tol_oz(8, m) * 4
