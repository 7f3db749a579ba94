"""Device-resident operands that start one element past an aligned address, with
odd leading dimensions: the layout a caller gets when it passes a sub-matrix
(A + 1, lda = m + 3) of a larger device allocation.

Every kernel that reads the caller's memory with 16-byte accesses checks the
address and the leading dimension first and falls back to element accesses,
and the TMA copies only read the library's own split / slice planes; these
cases reach the fallbacks of each routine and precision mode.  Padding rows
(between the matrix and its leading dimension) and the element in front of
each operand hold NaN: BLAS leaves them unreferenced, so the results must stay
finite and the NaN must stay in place.  Tolerances are the parity tests' own
(normwise max relative error against float64): 4e-6 sqrt(max(k, 16)) for
plain float32 and BF16x6, 4e-5 for BF16x3, 1.6e-15 sqrt(max(k, 16)) for
plain float64 and Ozaki with the default 7 slices; solves twice that.
"""
import numpy as np
import pytest

import mojoblas_b200 as mb
from tests.gpu_util import need_gpu, rand, tri_system

pytestmark = pytest.mark.gpu

OFF = 1  # elements: 4 or 8 bytes past the allocation's alignment


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()
    mb.load()


def tol(dt, k, mode=mb.PLAIN):
    if mode == mb.BF16X3:
        return 4e-5
    return (1e-6 if dt == np.float32 else 4e-16) * np.sqrt(max(k, 16)) * 4


class Dev:
    """A column-major (rows, cols) matrix with leading dimension ld at OFF elements
    into a NaN-filled device buffer; rows rows..ld-1 of every column are NaN."""

    def __init__(self, a, rows):
        torch = need_gpu()
        self.ld, self.cols = a.shape
        self.rows = rows
        host = np.array(a, order="F", copy=True)
        host[rows:, :] = np.nan
        self.buf = torch.full((OFF + self.ld * self.cols,), float("nan"),
                              dtype=torch.float32 if a.dtype == np.float32 else torch.float64, device="cuda")
        self.buf[OFF:] = torch.from_numpy(host.reshape(-1, order="F").copy()).cuda()
        self.view = self.buf[OFF:]

    def host(self):
        need_gpu().cuda.synchronize()
        b = self.buf.cpu().numpy()
        assert np.isnan(b[:OFF]).all()  # nothing written in front of the operand
        full = b[OFF:].reshape(self.cols, self.ld).T
        assert np.isnan(full[self.rows:, :]).all()  # padding rows untouched
        return np.array(full[: self.rows, :], dtype=np.float64)


MODES = [(np.float32, mb.PLAIN), (np.float32, mb.BF16X3), (np.float32, mb.BF16X6),
         (np.float64, mb.PLAIN), (np.float64, mb.OZAKI)]
MODE_IDS = ["s-plain", "s-bf16x3", "s-bf16x6", "d-plain", "d-ozaki"]


@pytest.mark.parametrize("dt,mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T")])
def test_gemm_offset_operands(oracle, dt, mode, ta, tb):
    m, n, k = 259, 133, 197
    rng = np.random.default_rng(11)
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    a, b, c = rand(rng, (ra + 3, ca), dt), rand(rng, (rb + 5, cb), dt), rand(rng, (m + 1, n), dt)
    A, B, C = Dev(a, ra), Dev(b, rb), Dev(c, m)
    ref = oracle.gemm_f64(ta, tb, m, n, k, 1.25, a, ra + 3, b, rb + 5, -0.5, c, m + 1)
    assert mb.gemm(ta, tb, m, n, k, 1.25, A.view, A.ld, B.view, B.ld, -0.5, C.view, C.ld, mode=mode) == 0
    g = C.host()
    assert np.isfinite(g).all()
    assert oracle.max_rel_err(g, ref) < tol(dt, k, mode)


def test_sgemm_offset_operands_large():
    """m n k = 2^30 with a k-contiguous op(A): the plain float32 path transposes A into
    its workspace (element reads from the offset source) before the 16-byte tile copies."""
    m = n = k = 1024
    rng = np.random.default_rng(12)
    a, b = rand(rng, (k + 3, m), np.float32), rand(rng, (k + 1, n), np.float32)
    c = np.zeros((m + 1, n), np.float32, order="F")
    A, B, C = Dev(a, k), Dev(b, k), Dev(c, m)
    assert mb.gemm("T", "N", m, n, k, 1.0, A.view, A.ld, B.view, B.ld, 0.0, C.view, C.ld) == 0
    ref = a[:k].astype(np.float64).T @ b[:k].astype(np.float64)
    g = C.host()
    assert oracle_err(g, ref) < tol(np.float32, k)


def oracle_err(x, ref):
    return float(np.max(np.abs(x - ref)) / np.max(np.abs(ref)))


@pytest.mark.parametrize("dt,mode", [MODES[0], MODES[2], MODES[3], MODES[4]],
                         ids=["s-plain", "s-bf16x6", "d-plain", "d-ozaki"])
@pytest.mark.parametrize("uplo,trans", [("L", "N"), ("U", "T")])
def test_syrk_offset_operands(dt, mode, uplo, trans):
    n, k = 203, 150
    rng = np.random.default_rng(13)
    ra, ca = (n, k) if trans == "N" else (k, n)
    a, c = rand(rng, (ra + 3, ca), dt), rand(rng, (n + 1, n), dt)
    A, C = Dev(a, ra), Dev(c, n)
    assert mb.syrk(uplo, trans, n, k, 0.75, A.view, A.ld, 1.5, C.view, C.ld, mode=mode) == 0
    op = a[:ra].astype(np.float64)
    op = op if trans == "N" else op.T
    ref = 0.75 * op @ op.T + 1.5 * c[:n].astype(np.float64)
    mask = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    g = C.host()
    assert np.isfinite(g).all()
    assert np.max(np.abs(g[mask] - ref[mask])) / np.max(np.abs(ref[mask])) < tol(dt, k, mode)
    np.testing.assert_array_equal(g[~mask], c[:n].astype(np.float64)[~mask])  # other triangle untouched


@pytest.mark.parametrize("dt,mode", [MODES[0], MODES[2], MODES[3], MODES[4]],
                         ids=["s-plain", "s-bf16x6", "d-plain", "d-ozaki"])
@pytest.mark.parametrize("side,uplo,ta", [("L", "L", "N"), ("L", "U", "T"), ("R", "U", "N"), ("R", "L", "T")])
def test_trsm_offset_operands(oracle, dt, mode, side, uplo, ta):
    m, n = 150, 90
    rng = np.random.default_rng(14)
    a, b, lda, ldb = tri_system(rng, side, m, n, dt, ld_pad=3)
    na = lda - 3
    ref = oracle.trsm_f64(side, uplo, ta, "N", m, n, 2.0, a, lda, b, ldb)
    A, B = Dev(a, na), Dev(b, m)
    assert mb.trsm(side, uplo, ta, "N", m, n, 2.0, A.view, A.ld, B.view, B.ld, mode=mode) == 0
    g = B.host()
    assert np.isfinite(g).all()
    assert oracle.max_rel_err(g, ref) < 2 * tol(dt, na, mode)


@pytest.mark.parametrize("dt,mode", [MODES[0], MODES[2], MODES[3], MODES[4]],
                         ids=["s-plain", "s-bf16x6", "d-plain", "d-ozaki"])
def test_symm_trmm_offset_operands(oracle, dt, mode):
    m, n = 150, 90
    rng = np.random.default_rng(15)
    a, b, c = rand(rng, (m + 3, m), dt), rand(rng, (m + 1, n), dt), rand(rng, (m + 5, n), dt)
    A, B, C = Dev(a, m), Dev(b, m), Dev(c, m)
    ref = oracle.symm_f64("L", "U", m, n, 0.5, a, m + 3, b, m + 1, 2.0, c, m + 5)
    assert mb.symm("L", "U", m, n, 0.5, A.view, A.ld, B.view, B.ld, 2.0, C.view, C.ld, mode=mode) == 0
    g = C.host()
    assert np.isfinite(g).all()
    assert oracle.max_rel_err(g, ref) < tol(dt, m, mode)
    ref = oracle.trmm_f64("L", "L", "N", "N", m, n, 1.5, a, m + 3, b, m + 1)
    B2 = Dev(b, m)
    assert mb.trmm("L", "L", "N", "N", m, n, 1.5, A.view, A.ld, B2.view, B2.ld, mode=mode) == 0
    g = B2.host()
    assert np.isfinite(g).all()
    assert oracle.max_rel_err(g, ref) < tol(dt, m, mode)


class DevVec:
    """An n-vector with increment inc at OFF elements into a NaN-filled device buffer."""

    def __init__(self, v):
        torch = need_gpu()
        self.n = v.size
        self.buf = torch.full((OFF + v.size,), float("nan"),
                              dtype=torch.float32 if v.dtype == np.float32 else torch.float64, device="cuda")
        self.buf[OFF:] = torch.from_numpy(v.copy()).cuda()
        self.view = self.buf[OFF:]

    def host(self):
        need_gpu().cuda.synchronize()
        b = self.buf.cpu().numpy()
        assert np.isnan(b[:OFF]).all()
        return np.array(b[OFF:], dtype=np.float64)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("lda_pad", [3, 4])
def test_gemv_offset_operands(oracle, dt, trans, lda_pad):
    """lda_pad 4 keeps lda % 4 == 0 for an even m, so only the address rules out 16-byte loads."""
    m, n = 3000, 700
    rng = np.random.default_rng(16)
    a = rand(rng, (m + lda_pad, n), dt)
    lenx, leny = (n, m) if trans == "N" else (m, n)
    x, y = rng.uniform(-1, 1, lenx).astype(dt), rng.uniform(-1, 1, leny).astype(dt)
    A, X, Y = Dev(a, m), DevVec(x), DevVec(y)
    ref = oracle.gemv_f64(trans, m, n, 1.25, a, m + lda_pad, x, 1, 0.5, y, 1)
    assert mb.gemv(trans, m, n, 1.25, A.view, A.ld, X.view, 1, 0.5, Y.view, 1) == 0
    g = Y.host()
    assert np.isfinite(g).all()
    assert oracle.max_rel_err(g, ref) < tol(dt, lenx)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("uplo,trans", [("L", "N"), ("U", "T")])
def test_trsv_offset_operands(oracle, dt, uplo, trans):
    n = 300
    rng = np.random.default_rng(17)
    a = rng.standard_normal((n + 3, n)) / np.sqrt(n)
    a[np.arange(n), np.arange(n)] = 2.0 + np.abs(rng.standard_normal(n))
    a = np.asfortranarray(a.astype(dt))
    x = rng.uniform(-1, 1, n).astype(dt)
    A, X = Dev(a, n), DevVec(x)
    ref = oracle.trsv_f64(uplo, trans, "N", n, a, n + 3, x, 1)
    assert mb.trsv(uplo, trans, "N", n, A.view, A.ld, X.view, 1) == 0
    g = X.host()
    assert np.isfinite(g).all()
    assert oracle.max_rel_err(g, ref) < 2 * tol(dt, n)
