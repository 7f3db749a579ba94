"""The split / Ozaki trsm with inverted diagonal blocks.

With a split (BF16x3 / BF16x6) or Ozaki mode and at least `trsm_inverse_min_cols`
right-hand sides, the blocked solve inverts each 512-row diagonal block of op(A)
once in the input precision (fused block solves of the identity, one launch) and
applies every inverse as one split / Ozaki product, with the same recursive
split / Ozaki updates between the blocks as the substitution path.  Checked here:
  * every side / uplo / trans / diag combination at ragged sizes (several
    diagonal blocks, a short last one, padded leading dimensions), against the
    float64 solve and the oracle's restatement of the reference's trsm
    (src/level3/trsm.mojo:20-275), and that the inverted-block path really ran;
  * the same accuracy as the substitution leaves on the trsm configuration's
    system, and, against an extended-precision checker, no worse than a small
    factor of the plain FP64 solve on systems with ill-conditioned diagonal
    blocks (cond about 1e6 and 1e18).
Tolerances are those of tests/test_gpu_tc.py (TOL32 / TOL_X3 / TOL_OZ, times 4
as for the substitution path's trsm tests).
"""
import ctypes as C

import numpy as np
import pytest

import mojoblas_b200 as mb
from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu, tri_system
from tests.test_gpu_tc import tol32, tol64, tol_mode

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    need_gpu()
    mb.load()
    return L.load()


def _ran_inverse(lib, call):
    """Runs call() with kernel timing on; True if the inverted-block launch ran."""
    lib.mbg_prof_enable(1)
    lib.mbg_prof_reset()
    try:
        st = call()
        tot, cnt = C.c_double(), C.c_int64()
        lib.mbg_prof_query(b"trsm_block_invert", C.byref(tot), C.byref(cnt))
    finally:
        lib.mbg_prof_enable(0)
    return st, cnt.value > 0


CASES = [(s, u, t, d) for s in "LR" for u in "LU" for t in "NT" for d in "NU"]


@pytest.mark.parametrize("dt,mode", [(np.float32, mb.BF16X3), (np.float32, mb.BF16X6), (np.float64, mb.OZAKI)],
                         ids=["f32-bf16x3", "f32-bf16x6", "f64-ozaki"])
@pytest.mark.parametrize("side,uplo,ta,diag", CASES, ids=["".join(c) for c in CASES])
def test_inverse_blocks_all_variants(oracle, lib, dt, mode, side, uplo, ta, diag):
    rng = np.random.default_rng(21)
    na, nrhs = 1100, 300  # blocks of 512, 512, 76
    m, n = (na, nrhs) if side == "L" else (nrhs, na)
    alpha = 0.5
    a, b, lda, ldb = tri_system(rng, side, m, n, dt, ld_pad=3)
    ref = oracle.trsm_f64(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb)
    x = b.copy(order="F")
    st, ran = _ran_inverse(lib, lambda: mb.trsm(side, uplo, ta, diag, m, n, alpha, a, lda, x, ldb, mode=mode,
                                                slices=7))
    assert st == 0 and ran
    x_o = b.copy(order="F")
    oracle.trsm(side, uplo, ta, diag, m, n, alpha, a, lda, x_o, ldb)
    t = tol_mode(mode, na, slices=7) * 4
    g = oracle.view(x, m, n, ldb)
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, oracle.view(x_o, m, n, ldb).astype(np.float64)) < t + 4 * (
        tol32(na) if dt == np.float32 else tol64(na))
    # padding rows between m and ldb are untouched
    np.testing.assert_array_equal(x[m:], b[m:])


def test_inverse_blocks_match_substitution_accuracy(oracle, lib):
    """The trsm configuration's system (order 2048, 512 right-hand sides): inverted
    blocks and substitution leaves reach the same error against the float64 solve."""
    rng = np.random.default_rng(22)
    m, n = 2048, 512
    a, b, lda, ldb = tri_system(rng, "L", m, n, np.float64)
    ref = oracle.trsm_f64("L", "L", "N", "N", m, n, 1.0, a, lda, b, ldb)
    errs = {}
    for label, cols in (("inverse", 256), ("substitution", 0)):
        assert lib.mbg_set_tuning(b"trsm_inverse_min_cols", cols) == 0
        try:
            x = b.copy(order="F")
            st, ran = _ran_inverse(lib, lambda: mb.trsm("L", "L", "N", "N", m, n, 1.0, a, lda, x, ldb,
                                                        mode=mb.OZAKI, slices=7))
        finally:
            lib.mbg_set_tuning(b"trsm_inverse_min_cols", 256)
        assert st == 0 and ran == (label == "inverse")
        errs[label] = oracle.max_rel_err(x, ref)
    assert errs["inverse"] < 4 * tol64(m) and errs["substitution"] < 4 * tol64(m)
    assert errs["inverse"] <= 2 * errs["substitution"] + 1e-16, errs


@pytest.mark.parametrize("case", ["moderate", "ill"])
def test_inverse_blocks_ill_conditioned(oracle, lib, case):
    """Lower triangles with O(1) off-diagonal entries: the diagonal blocks' condition
    numbers are about 1e6 ("moderate": diagonal 4 + |N(0,1)|) and 1e18 ("ill":
    diagonal 1 + |N(0,1)|).  Error against an extended-precision substitution: the
    Ozaki solve with inverted blocks stays within 4x the plain FP64 solve's."""
    rng = np.random.default_rng(23)
    n, nrhs = 1024, 256
    a = np.tril(rng.standard_normal((n, n)), -1)
    a[np.arange(n), np.arange(n)] = (4.0 if case == "moderate" else 1.0) + np.abs(rng.standard_normal(n))
    a = np.asfortranarray(a)
    b = np.asfortranarray(rng.standard_normal((n, nrhs)))
    ref = oracle.trsm_lower_longdouble(a, b)
    errs = {}
    for label, kw in (("plain", {}), ("ozaki_inverse", {"mode": mb.OZAKI, "slices": 7})):
        x = b.copy(order="F")
        st, ran = _ran_inverse(lib, lambda: mb.trsm("L", "L", "N", "N", n, nrhs, 1.0, a, n, x, n, **kw))
        assert st == 0 and ran == (label != "plain")
        den = float(np.max(np.abs(ref)))
        errs[label] = float(np.max(np.abs(x.astype(np.longdouble) - ref))) / den
    assert errs["ozaki_inverse"] <= 4 * errs["plain"] + 4e-16, errs


@pytest.mark.parametrize("dt,mode", [(np.float32, mb.BF16X6), (np.float64, mb.OZAKI)], ids=["f32-bf16x6", "f64-ozaki"])
@pytest.mark.parametrize("side,uplo,ta", [("L", "L", "N"), ("L", "U", "T"), ("R", "U", "N")])
def test_inverse_blocks_of_256_rows(oracle, lib, dt, mode, side, uplo, ta):
    """Tuning key trsm_inverse_block = 256: diagonal blocks of 256 rows (five blocks and a
    short one at 1300 rows), the same tolerances as the 512-row blocks."""
    default = lib.mbg_get_tuning(b"trsm_inverse_block")
    rng = np.random.default_rng(23)
    na, nrhs = 1300, 300
    m, n = (na, nrhs) if side == "L" else (nrhs, na)
    a, b, lda, ldb = tri_system(rng, side, m, n, dt, ld_pad=2)
    ref = oracle.trsm_f64(side, uplo, ta, "N", m, n, 1.5, a, lda, b, ldb)
    x = b.copy(order="F")
    try:
        assert lib.mbg_set_tuning(b"trsm_inverse_block", 256) == 0
        assert lib.mbg_set_tuning(b"trsm_inverse_block", 300) != 0  # only 256 or 512
        st, ran = _ran_inverse(lib, lambda: mb.trsm(side, uplo, ta, "N", m, n, 1.5, a, lda, x, ldb, mode=mode,
                                                    slices=7))
    finally:
        lib.mbg_set_tuning(b"trsm_inverse_block", default)
    assert st == 0 and ran
    assert oracle.max_rel_err(oracle.view(x, m, n, ldb), ref) < tol_mode(mode, na, slices=7) * 4
    np.testing.assert_array_equal(x[m:], b[m:])
