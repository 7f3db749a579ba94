"""Parity of the level-2 gemv and trsv kernels with the reference's algorithms.

Every case runs the same seeded inputs through (a) the library's C ABI on the
GPU, (b) the oracle's restatement of the reference routine on the CPU
(src/level2/gemv.mojo:23-212, src/level2/trsv.mojo:20-214) and (c) float64
numpy / scipy.  Tolerance (normwise max relative error against float64, k = the
reduction length): 1e-6 sqrt(max(k, 16)) for float32, 4e-16 sqrt(max(k, 16))
for float64, each times 4 (trsv: times 8, the substitution's error grows with
the chain); GPU and oracle agree within twice that.  Vector elements between
the strided entries are NaN and must stay NaN.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import mojoblas_b200 as mb
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "level2_known_answers.json").read_text())


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()
    mb.load()


def tol(dt, k):
    return (1e-6 if dt == np.float32 else 4e-16) * np.sqrt(max(k, 16)) * 4


@pytest.mark.parametrize("case", GOLDEN["cases"], ids=[c["test"] for c in GOLDEN["cases"]])
def test_known_answers_on_gpu(case):
    """The reference's own gemv / trsv known answers through the C ABI."""
    dt = np.float32 if case["dtype"] == "float32" else np.float64
    bufs = {k: np.array(v, dtype=dt) for k, v in case["inputs"].items()}
    args = [bufs[a["array"]] if isinstance(a, dict) else a for a in case["call"]["args"]]
    fn = {"gemv": mb.gemv, "trsv": mb.trsv}[case["call"]["routine"]]
    assert fn(*args) == 0
    for a in case["asserts"]:
        got = float(bufs[a["array"]][a["index"]])
        atol = a["atol"] if a["atol"] is not None else 1e-8
        assert abs(got - a["expected"]) <= atol + 1e-5 * abs(a["expected"]), (case["test"], a, got)


def strided(rng, n, inc, dt, scale=1.0):
    buf = np.full(max(1, 1 + (n - 1) * abs(inc)), np.nan, dtype=dt)
    start = 0 if inc > 0 else (1 - n) * inc
    buf[start + np.arange(n) * inc] = (scale * rng.uniform(-1, 1, n)).astype(dt)
    return buf


def gaps(buf, n, inc):
    mask = np.ones(buf.size, bool)
    mask[(0 if inc > 0 else (1 - n) * inc) + np.arange(n) * inc] = False
    return buf[mask]


# ---- gemv --------------------------------------------------------------------------
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
@pytest.mark.parametrize("incx,incy", [(1, 1), (3, 1), (1, -2), (-1, 2)])
@pytest.mark.parametrize("m,n,alpha,beta", [(37, 50, 1.5, 0.5), (5000, 40, -1.0, 0.0), (40, 5000, 2.0, 1.0),
                                            (2049, 1537, 0.75, -0.5), (1, 1, 1.0, 0.0)])
def test_gemv(oracle, dt, trans, incx, incy, m, n, alpha, beta):
    """Shapes reach the single-pass kernels and both split-and-finish paths (long rows of
    columns for NoTrans, long columns for Trans), with unit, strided and negative
    increments and beta 0 (y not read), 1 and other."""
    rng = np.random.default_rng(m + 7 * n + incx)
    lda = m + 3
    a = np.asfortranarray(rng.uniform(-1, 1, (lda, n)).astype(dt))
    lenx, leny = (n, m) if trans == "N" else (m, n)
    x = strided(rng, lenx, incx, dt)
    y = strided(rng, leny, incy, dt)
    ref = oracle.gemv_f64(trans, m, n, alpha, a, lda, x, incx, beta, y, incy)
    y_orc = y.copy()
    assert oracle.gemv(trans, m, n, alpha, a, lda, x, incx, beta, y_orc, incy) == 0
    got = y.copy()
    if beta == 0.0:
        got[(0 if incy > 0 else (1 - leny) * incy) + np.arange(leny) * incy] = np.nan  # not read
    assert mb.gemv(trans, m, n, alpha, a, lda, x, incx, beta, got, incy) == 0
    g = oracle.vec(got, leny, incy)
    t = tol(dt, lenx)
    assert np.all(np.isfinite(g))
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, oracle.vec(y_orc, leny, incy).astype(np.float64)) < 2 * t
    assert np.all(np.isnan(gaps(got, leny, incy)))


def test_gemv_alpha_zero_and_zero_entries(oracle):
    """alpha == 0 scales y by beta without reading A or x (gemv.mojo:107-129); zero entries of
    x skip their columns, so an infinite column under a zero x stays out (NoTrans)."""
    y = np.arange(5, dtype=np.float64)
    a = np.full((5, 3), np.nan, order="F")
    assert mb.gemv("N", 5, 3, 0.0, a, 5, np.full(3, np.nan), 1, 2.0, y, 1) == 0
    np.testing.assert_array_equal(y, 2.0 * np.arange(5))
    a = np.asfortranarray(np.random.default_rng(3).uniform(-1, 1, (5, 3)))
    a[:, 1] = np.inf
    x = np.array([1.0, 0.0, -2.0])
    y = np.zeros(5)
    assert mb.gemv("N", 5, 3, 1.0, a, 5, x, 1, 0.0, y, 1) == 0
    np.testing.assert_allclose(y, a[:, 0] - 2.0 * a[:, 2], rtol=1e-15)


# ---- trsv --------------------------------------------------------------------------
def tri_matrix(rng, n, dt, diag):
    a = rng.standard_normal((n + 2, n)) / np.sqrt(n)
    a[np.arange(n), np.arange(n)] = 2.0 + np.abs(rng.standard_normal(n))
    if diag == "U":
        a /= 4.0  # keeps the unit-diagonal system well conditioned
    return np.asfortranarray(a.astype(dt))


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("incx", [1, 3, -2])
@pytest.mark.parametrize("n", [1, 63, 64, 65, 200, 1000])
def test_trsv(oracle, dt, uplo, trans, diag, incx, n):
    """n below, at and above one 64-row block, several blocks with a short last one
    (forward and backward solve order), strided and negative increments; the triangle
    that must not be read is NaN."""
    rng = np.random.default_rng(n + 11 * abs(incx))
    a = tri_matrix(rng, n, dt, diag)
    lda = n + 2
    x = strided(rng, n, incx, dt)
    ref = oracle.trsv_f64(uplo, trans, diag, n, a, lda, x, incx)
    x_orc = x.copy()
    assert oracle.trsv(uplo, trans, diag, n, a, lda, x_orc, incx) == 0
    junk = np.triu(np.ones((n, n), bool), 1) if uplo == "L" else np.tril(np.ones((n, n), bool), -1)
    if diag == "U":
        junk |= np.eye(n, dtype=bool)
    a[:n][junk] = np.nan
    got = x.copy()
    assert mb.trsv(uplo, trans, diag, n, a, lda, got, incx) == 0
    g = oracle.vec(got, n, incx)
    t = tol(dt, n) * 2
    assert np.all(np.isfinite(g))
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, oracle.vec(x_orc, n, incx).astype(np.float64)) < 2 * t
    assert np.all(np.isnan(gaps(got, n, incx)))


def test_trsv_zero_right_hand_side_entries(oracle):
    """NoTrans skips zero entries of x (trsv.mojo:96-155): leading zeros of b stay exact
    zeros, and an infinite entry below a zero pivot does not reach the solution."""
    rng = np.random.default_rng(5)
    n = 300
    a = tri_matrix(rng, n, np.float64, "N")
    x = rng.uniform(-1, 1, n)
    x[:130] = 0.0
    a[100, 3] = np.inf  # column 3 is multiplied by x_3 == 0 only
    got = x.copy()
    assert mb.trsv("L", "N", "N", n, a, n + 2, got, 1) == 0
    assert np.all(got[:130] == 0.0) and np.all(np.isfinite(got))
    want = x.copy()
    assert oracle.trsv("L", "N", "N", n, a, n + 2, want, 1) == 0
    assert oracle.max_rel_err(got, want) < tol(np.float64, n) * 4


def test_level2_device_pointers(oracle):
    """Device-resident operands (no staging) at larger sizes: dgemv 4096 x 3000 both
    ways, dtrsv of order 4100 (65 blocks, the last one short) forward and backward."""
    torch = need_gpu()
    rng = np.random.default_rng(8)
    m, n = 4096, 3000
    a = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    ad = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()
    for trans, lx, ly in (("N", n, m), ("T", m, n)):
        x = rng.uniform(-1, 1, lx)
        y = rng.uniform(-1, 1, ly)
        xd, yd = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
        assert mb.gemv(trans, m, n, 1.25, ad, m, xd, 1, 0.5, yd, 1) == 0
        torch.cuda.synchronize()
        ref = oracle.gemv_f64(trans, m, n, 1.25, a, m, x, 1, 0.5, y, 1)
        assert oracle.max_rel_err(yd.cpu().numpy(), ref) < tol(np.float64, lx)
    n = 4100
    t = tri_matrix(rng, n, np.float64, "N")
    td = torch.from_numpy(np.ascontiguousarray(t.T)).cuda()
    for uplo in ("L", "U"):
        b = rng.uniform(-1, 1, n)
        bd = torch.from_numpy(b.copy()).cuda()
        assert mb.trsv(uplo, "N", "N", n, td, n + 2, bd, 1) == 0
        torch.cuda.synchronize()
        ref = oracle.trsv_f64(uplo, "N", "N", n, t, n + 2, b, 1)
        assert oracle.max_rel_err(bd.cpu().numpy(), ref) < tol(np.float64, n) * 2
