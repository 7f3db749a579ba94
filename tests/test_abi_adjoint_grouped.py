"""CPU-side argument checks of the entry points without a reference counterpart:
the gemm / trsm adjoints and the grouped plans.  Each invalid argument is
reported with its Netlib-style position before any pointer is read or any
device work starts (so null or unused buffers are fine here):

* gemm adjoint: gemm's numbering for 1..10 (src/level3/gemm.mojo:179-213), then
  ldg 12, ldda 14, lddb 16 (mode / slices not counted);
* trsm adjoint: trsm's numbering for 1..9 (src/level3/trsm.mojo:62-89), then
  ldx 11, ldg 13, lddb 15, ldda 17;
* grouped plans: the first invalid problem's gemm / trsm number, with the
  problem's index in mbg_last_error; sgemm plans take MBG_MODE_PLAIN, BF16X3 and
  BF16X6, strsm plans MBG_MODE_PLAIN.
"""
import ctypes as C

import numpy as np
import pytest

from mojoblas_b200 import _lib as L

BUF = np.zeros(64, dtype=np.float32)
DBUF = np.zeros(64, dtype=np.float64)
P = BUF.ctypes.data  # a real host address, never read by the checks below
DP = DBUF.ctypes.data


@pytest.fixture(scope="module")
def lib():
    return L.load()


# (ta, tb, m, n, k, lda, ldb, ldg, da?, ldda, db?, lddb) -> info
GEMM_ADJ = [
    (("X", "N", 2, 2, 2, 2, 2, 2, 1, 2, 1, 2), 1),
    (("N", "q", 2, 2, 2, 2, 2, 2, 1, 2, 1, 2), 2),
    (("N", "N", -1, 2, 2, 2, 2, 2, 1, 2, 1, 2), 3),
    (("N", "N", 2, -1, 2, 2, 2, 2, 1, 2, 1, 2), 4),
    (("N", "N", 2, 2, -1, 2, 2, 2, 1, 2, 1, 2), 5),
    (("N", "N", 3, 2, 2, 2, 2, 3, 1, 3, 1, 2), 8),
    (("T", "N", 2, 2, 3, 2, 3, 2, 1, 3, 1, 3), 8),
    (("N", "N", 2, 2, 3, 2, 2, 2, 1, 2, 1, 3), 10),
    (("N", "N", 3, 2, 2, 3, 2, 2, 1, 3, 1, 2), 12),
    (("N", "N", 3, 2, 2, 3, 2, 3, 1, 2, 1, 2), 14),
    (("N", "T", 2, 3, 2, 2, 3, 2, 1, 2, 1, 2), 16),
]


@pytest.mark.parametrize("args,info", GEMM_ADJ)
def test_gemm_adjoint_info(lib, args, info):
    ta, tb, m, n, k, lda, ldb, ldg, da, ldda, db, lddb = args
    st = lib.mbg_sgemm_adjoint(L.MODE_PLAIN, ta.encode(), tb.encode(), m, n, k, 1.0, P, lda, P, ldb, P, ldg,
                               P if da else None, ldda, P if db else None, lddb)
    assert st == info
    st = lib.mbg_dgemm_adjoint(L.MODE_OZAKI, 7, ta.encode(), tb.encode(), m, n, k, 1.0, DP, lda, DP, ldb, DP, ldg,
                               DP if da else None, ldda, DP if db else None, lddb)
    assert st == info


def test_gemm_adjoint_null_output_skips_its_check(lib):
    """ldda is only checked when dA is requested (and lddb only with dB)."""
    st = lib.mbg_sgemm_adjoint(L.MODE_PLAIN, b"N", b"N", 3, 2, 2, 1.0, P, 3, P, 2, P, 3, None, 1, P, 1)
    assert st == 16  # lddb < k, dA skipped
    st = lib.mbg_sgemm_adjoint(L.MODE_PLAIN, b"N", b"N", 3, 2, 2, 1.0, P, 3, P, 2, P, 3, P, 1, None, 1)
    assert st == 14


def test_adjoint_modes_rejected(lib):
    assert lib.mbg_sgemm_adjoint(L.MODE_OZAKI, b"N", b"N", 2, 2, 2, 1.0, P, 2, P, 2, P, 2, P, 2, P, 2) < 0
    assert lib.mbg_strsm_adjoint(L.MODE_OZAKI, b"L", b"L", b"N", b"N", 2, 2, 1.0, P, 2, P, 2, P, 2, P, 2, P, 2) < 0


# (side, uplo, ta, diag, m, n, lda, ldx, ldg, lddb, da?, ldda) -> info
TRSM_ADJ = [
    (("X", "L", "N", "N", 2, 2, 2, 2, 2, 2, 1, 2), 1),
    (("L", "X", "N", "N", 2, 2, 2, 2, 2, 2, 1, 2), 2),
    (("L", "L", "X", "N", 2, 2, 2, 2, 2, 2, 1, 2), 3),
    (("L", "L", "N", "X", 2, 2, 2, 2, 2, 2, 1, 2), 4),
    (("L", "L", "N", "N", -1, 2, 2, 2, 2, 2, 1, 2), 5),
    (("L", "L", "N", "N", 2, -1, 2, 2, 2, 2, 1, 2), 6),
    (("L", "L", "N", "N", 3, 2, 2, 3, 3, 3, 1, 3), 9),
    (("R", "L", "N", "N", 2, 3, 2, 2, 2, 2, 1, 3), 9),
    (("L", "L", "N", "N", 3, 2, 3, 2, 3, 3, 1, 3), 11),
    (("L", "L", "N", "N", 3, 2, 3, 3, 2, 3, 1, 3), 13),
    (("L", "L", "N", "N", 3, 2, 3, 3, 3, 2, 1, 3), 15),
    (("L", "L", "N", "N", 3, 2, 3, 3, 3, 3, 1, 2), 17),
]


@pytest.mark.parametrize("args,info", TRSM_ADJ)
def test_trsm_adjoint_info(lib, args, info):
    side, uplo, ta, diag, m, n, lda, ldx, ldg, lddb, da, ldda = args
    ch = [x.encode() for x in (side, uplo, ta, diag)]
    st = lib.mbg_strsm_adjoint(L.MODE_PLAIN, *ch, m, n, 1.0, P, lda, P, ldx, P, ldg, P, lddb,
                               P if da else None, ldda)
    assert st == info
    st = lib.mbg_dtrsm_adjoint(L.MODE_PLAIN, 0, *ch, m, n, 1.0, DP, lda, DP, ldx, DP, ldg, DP, lddb,
                               DP if da else None, ldda)
    assert st == info


def test_trsm_adjoint_empty_is_a_quick_return(lib):
    assert lib.mbg_strsm_adjoint(L.MODE_PLAIN, b"L", b"L", b"N", b"N", 0, 5, 1.0, None, 1, None, 1, None, 1,
                                 None, 1, None, 1) == 0
    assert lib.mbg_dtrsm_adjoint(L.MODE_PLAIN, 0, b"R", b"U", b"T", b"U", 4, 0, 1.0, None, 4, None, 4, None, 4,
                                 None, 4, None, 4) == 0


def sgemm_problems(bad_index, **bad):
    probs = (L.SgemmProblem * 3)()
    for i, q in enumerate(probs):
        vals = dict(trans_a=b"N", trans_b=b"N", m=2, n=2, k=2, alpha=1.0, beta=0.0, a=None, lda=2, b=None, ldb=2,
                    c=None, ldc=2)
        if i == bad_index:
            vals.update(bad)
        for key, v in vals.items():
            setattr(q, key, v)
    return probs


@pytest.mark.parametrize("bad,info", [
    (dict(trans_a=b"X"), 1), (dict(trans_b=b"z"), 2), (dict(m=-1), 3), (dict(n=-1), 4), (dict(k=-1), 5),
    (dict(m=3, ldc=3), 8), (dict(k=3, lda=3), 10), (dict(m=3, lda=3), 13),
])
def test_grouped_sgemm_plan_reports_first_invalid_problem(lib, bad, info):
    # problems are checked in order, arguments before pointers (device pointers only), so the invalid
    # problem goes first: the null pointers of the others would be reported before it otherwise
    plan = C.c_void_p()
    probs = sgemm_problems(0, **bad)
    assert lib.mbg_sgemm_grouped_plan(L.MODE_PLAIN, 3, probs, C.byref(plan)) == info
    assert not plan.value  # no plan is made
    assert "problem 0" in L.last_error()


def strsm_problems(bad_index, **bad):
    probs = (L.StrsmProblem * 2)()
    for i, q in enumerate(probs):
        vals = dict(side=b"L", uplo=b"L", trans_a=b"N", diag=b"N", m=4, n=3, alpha=1.0, a=None, lda=4, b=None,
                    ldb=4)
        if i == bad_index:
            vals.update(bad)
        for key, v in vals.items():
            setattr(q, key, v)
    return probs


@pytest.mark.parametrize("bad,info", [
    (dict(side=b"X"), 1), (dict(uplo=b"X"), 2), (dict(trans_a=b"X"), 3), (dict(diag=b"X"), 4), (dict(m=-1), 5),
    (dict(n=-1), 6), (dict(lda=3), 9), (dict(ldb=3), 11),
])
def test_grouped_strsm_plan_reports_first_invalid_problem(lib, bad, info):
    plan = C.c_void_p()
    probs = strsm_problems(0, **bad)
    assert lib.mbg_strsm_grouped_plan(L.MODE_PLAIN, 2, probs, C.byref(plan)) == info
    assert not plan.value
    assert "problem 0" in L.last_error()


def test_grouped_plan_rejects_host_pointers(lib):
    plan = C.c_void_p()
    assert lib.mbg_sgemm_grouped_plan(L.MODE_PLAIN, 3, sgemm_problems(-1), C.byref(plan)) < 0
    assert "problem 0" in L.last_error() and "device only" in L.last_error()


def test_grouped_plan_modes(lib):
    plan = C.c_void_p()
    # the split modes pass the mode check and reach the per-problem checks (host pointers here)
    assert lib.mbg_sgemm_grouped_plan(L.MODE_BF16X6, 3, sgemm_problems(-1), C.byref(plan)) < 0
    assert "device only" in L.last_error()
    assert lib.mbg_sgemm_grouped_plan(L.MODE_OZAKI, 3, sgemm_problems(-1), C.byref(plan)) == L.MBG_ERR_INVALID_MODE
    assert lib.mbg_strsm_grouped_plan(L.MODE_OZAKI, 2, strsm_problems(-1), C.byref(plan)) < 0
    assert lib.mbg_sgemm_grouped_plan(L.MODE_PLAIN, -1, None, C.byref(plan)) < 0
