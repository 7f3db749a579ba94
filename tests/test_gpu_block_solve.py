"""Parity of the fused diagonal-block trsm kernel (block_solve_kernel).

The kernel solves diagonal blocks of up to `trsm_block_rows` rows in one launch
(64-row substitution sub-blocks with their updates in shared memory).  By
default it runs only with at least `trsm_block_min_cols` right-hand sides; these
tests lower that threshold so that small, ragged systems reach it, and check
every side / uplo / trans / diag case against the float64 oracle, the oracle's
restatement of the reference routine (src/level3/trsm.mojo:20-275), and the
64-row leaf path of the same library.  Tolerance as in test_gpu_plain.py.
"""
import numpy as np
import pytest

import mojoblas_b200 as mb
from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu, tri_system

pytestmark = pytest.mark.gpu


def tol(dt, k):
    return (1e-6 if dt == np.float32 else 4e-16) * np.sqrt(max(k, 16))


@pytest.fixture(scope="module")
def lib():
    need_gpu()
    mb.load()
    return L.load()


@pytest.fixture
def block_path(lib):
    """Fused blocks of up to 512 rows for any number of right-hand sides; restores the table."""
    old = {k: lib.mbg_get_tuning(k.encode()) for k in ("trsm_block_rows", "trsm_block_min_cols")}
    assert lib.mbg_set_tuning(b"trsm_block_rows", 512) == 0
    assert lib.mbg_set_tuning(b"trsm_block_min_cols", 1) == 0
    yield lib
    for k, v in old.items():
        assert lib.mbg_set_tuning(k.encode(), v) == 0


def solve(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb, **kw):
    x = b.copy(order="F")
    assert mb.trsm(side, uplo, ta, diag, m, n, alpha, a, lda, x, ldb, **kw) == 0
    return x


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("na,nrhs", [(65, 17), (300, 40), (512, 16), (1000, 33)])
def test_block_solve_all_cases(oracle, block_path, dt, side, uplo, ta, diag, na, nrhs):
    """na = order of A (one sub-block plus one row; ragged 300; exactly 512; 1000 = recursion
    over two fused blocks, the second ragged); nrhs ragged against the 16-column strips."""
    rng = np.random.default_rng(21)
    m, n = (na, nrhs) if side == "L" else (nrhs, na)
    alpha = 0.75
    a, b, lda, ldb = tri_system(rng, side, m, n, dt, ld_pad=3)
    if diag == "U":
        a = np.asfortranarray((a / na).astype(dt))
    junk = np.triu(np.ones((na, na), bool), 1) if uplo == "L" else np.tril(np.ones((na, na), bool), -1)
    a[:na][junk] = np.nan  # the unreferenced triangle must not be read
    a_clean = np.nan_to_num(a)
    ref = oracle.trsm_f64(side, uplo, ta, diag, m, n, alpha, a_clean, lda, b, ldb)
    x_gpu = solve(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb)
    x_orc = b.copy(order="F")
    assert oracle.trsm(side, uplo, ta, diag, m, n, alpha, a, lda, x_orc, ldb) == 0
    g = oracle.view(x_gpu, m, n, ldb)
    t = tol(dt, na) * 4
    assert np.all(np.isfinite(g))
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, oracle.view(x_orc, m, n, ldb).astype(np.float64)) < 2 * t
    np.testing.assert_array_equal(x_gpu[m:], b[m:])  # padding rows untouched
    # the 64-row leaf path of the same library agrees
    assert block_path.mbg_set_tuning(b"trsm_block_rows", 0) == 0
    x_leaf = solve(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb)
    assert block_path.mbg_set_tuning(b"trsm_block_rows", 512) == 0
    assert oracle.max_rel_err(g, oracle.view(x_leaf, m, n, ldb).astype(np.float64)) < 2 * t


@pytest.mark.parametrize("rows", [128, 256, 1024])
def test_block_rows_setting(oracle, block_path, rows):
    """Every block size the tuning table allows gives the same solution (dtrsm L/L/N/N)."""
    assert block_path.mbg_set_tuning(b"trsm_block_rows", rows) == 0
    rng = np.random.default_rng(22)
    m, n = 1100, 70
    a, b, lda, ldb = tri_system(rng, "L", m, n, np.float64)
    ref = oracle.trsm_f64("L", "L", "N", "N", m, n, 1.0, a, lda, b, ldb)
    x = solve("L", "L", "N", "N", m, n, 1.0, a, lda, b, ldb)
    assert oracle.max_rel_err(x, ref) < tol(np.float64, m) * 4


def test_block_solve_zero_columns_and_pivots(oracle, block_path):
    """Zero right-hand-side columns stay zero and zero pivots are skipped as in the
    reference (src/level3/trsm.mojo:130-148): an infinite entry of A under a zero
    pivot does not reach the solution."""
    rng = np.random.default_rng(23)
    m, n = 200, 20
    a, b, lda, ldb = tri_system(rng, "L", m, n, np.float64)
    b[:, 3] = 0.0
    b[:70, 5] = 0.0           # leading zeros: the first 70 pivots of column 5 are zero
    a[10, 0] = np.inf         # below the zero pivot x_0 of column 5 (and of column 3)
    x = solve("L", "L", "N", "N", m, n, 1.0, a, lda, b, ldb)
    assert np.all(x[:m, 3] == 0.0)
    assert np.all(x[:70, 5] == 0.0)
    assert np.all(np.isfinite(x[:m, 5]))
    x_orc = b.copy(order="F")
    assert oracle.trsm("L", "L", "N", "N", m, n, 1.0, a, lda, x_orc, ldb) == 0
    assert oracle.max_rel_err(x[:m, 5], x_orc[:m, 5]) < tol(np.float64, m) * 8


@pytest.mark.parametrize("dt,mode", [(np.float32, mb.BF16X6), (np.float64, mb.OZAKI)], ids=["bf16x6", "ozaki"])
def test_block_solve_with_split_updates(oracle, block_path, dt, mode):
    """Fused diagonal blocks with the split / Ozaki gemm updates between them."""
    rng = np.random.default_rng(24)
    m, n = 1536, 48
    a, b, lda, ldb = tri_system(rng, "L", m, n, dt)
    ref = oracle.trsm_f64("L", "L", "N", "N", m, n, 1.0, a, lda, b, ldb)
    x = solve("L", "L", "N", "N", m, n, 1.0, a, lda, b, ldb, mode=mode, slices=8)
    t = (1e-6 if dt == np.float32 else 4e-16) * np.sqrt(m) * 4
    assert oracle.max_rel_err(x, ref) < t
