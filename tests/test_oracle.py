"""Pins the CPU oracle before anything is compared against it.

1. Every gemm / syrk / trsm known answer in the reference's own level-3 tests
   (mojoBLAS tests/test_level3.mojo, extracted into tests/golden/) must come out
   of the oracle's restatement of the reference's algorithms.
2. On seeded random inputs (numpy default_rng seeds 0..4), the restatement
   agrees with an independent float64 computation (numpy / scipy) for every
   transpose, side, uplo and diag mode, and for each dispatch path (naive, v3,
   v7, v11).
3. The reference's two documented quirks reproduce only with BUG_COMPAT.
"""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).parent / "golden" / "level3_known_answers.json"
CASES = [c for c in json.loads(GOLDEN.read_text())["cases"]
         if c["call"]["routine"] in ("gemm", "syrk", "trsm")]


def _run_case(orc, case, flags):
    dt = np.float32 if case["dtype"] == "float32" else np.float64
    bufs = {k: np.array(v, dtype=dt) for k, v in case["inputs"].items()}
    args = [bufs[a["array"]] if isinstance(a, dict) else a for a in case["call"]["args"]]
    fn = {"gemm": orc.gemm, "syrk": orc.syrk, "trsm": orc.trsm}[case["call"]["routine"]]
    if case["call"]["routine"] == "syrk":
        info = fn(*args)
    else:
        info = fn(*args, flags=flags)
    return info, bufs


def test_golden_case_count():
    # 8 gemm, 5 syrk, 6 trsm known answers in the reference's level-3 tests
    names = [c["call"]["routine"] for c in CASES]
    assert names.count("gemm") == 8 and names.count("syrk") == 5 and names.count("trsm") == 6


@pytest.mark.parametrize("flags", [0, 1], ids=["netlib", "bug_compat"])
@pytest.mark.parametrize("case", CASES, ids=[c["test"] for c in CASES])
def test_oracle_matches_reference_known_answers(oracle, case, flags):
    info, bufs = _run_case(oracle, case, flags)
    assert info == 0
    for a in case["asserts"]:
        got = float(bufs[a["array"]][a["index"]])
        exp = a["expected"]
        atol = a["atol"] if a["atol"] is not None else 1e-8
        # Mojo's assert_almost_equal: |got-exp| <= atol + rtol*|exp|, rtol 1e-5
        assert abs(got - exp) <= atol + 1e-5 * abs(exp), (case["test"], a, got)


def _rand(rng, shape, dt):
    return np.asfortranarray(rng.uniform(-1, 1, size=shape).astype(dt))


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T"), ("C", "n")])
@pytest.mark.parametrize("m,n,k,alpha,beta", [(37, 29, 53, 1.5, 0.5), (64, 70, 1030, -0.75, 0.0),
                                               (5, 3, 0, 2.0, 3.0), (9, 600, 17, 1.0, 1.0)])
@pytest.mark.parametrize("seed", range(5))
def test_oracle_gemm_vs_float64(oracle, dt, ta, tb, m, n, k, alpha, beta, seed):
    rng = np.random.default_rng(seed)
    lda = (m if ta in "Nn" else k) + 3
    ldb = (k if tb in "Nn" else n) + 2
    ldc = m + 1
    a = _rand(rng, (lda, m if ta not in "Nn" else k), dt)
    b = _rand(rng, (ldb, k if tb not in "Nn" else n), dt)
    c = _rand(rng, (ldc, n), dt)
    ref = oracle.gemm_f64(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    c0 = c.copy()
    assert oracle.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) == 0
    tol = 1e-5 if dt == np.float32 else 1e-13
    assert oracle.max_rel_err(oracle.view(c, m, n, ldc), ref) < tol
    # rows m..ldc-1 (padding) untouched
    np.testing.assert_array_equal(c[m:], c0[m:])


def test_oracle_v7_alpha_quirk(oracle):
    """float64 NN with n >= 512 goes to gemm_v7, which drops alpha in the reference."""
    rng = np.random.default_rng(2)
    m, n, k = 33, 512, 40
    a, b = _rand(rng, (m, k), np.float64), _rand(rng, (k, n), np.float64)
    ref = oracle.gemm_f64("N", "N", m, n, k, 2.5, a, m, b, k, 0.0, a, m)
    c1 = np.zeros((m, n), order="F")
    oracle.gemm("N", "N", m, n, k, 2.5, a, m, b, k, 0.0, c1, m, flags=0)
    assert oracle.max_rel_err(c1, ref) < 1e-14
    c2 = np.zeros((m, n), order="F")
    oracle.gemm("N", "N", m, n, k, 2.5, a, m, b, k, 0.0, c2, m, flags=oracle.BUG_COMPAT)
    assert oracle.max_rel_err(c2, ref / 2.5) < 1e-14


def test_oracle_info_codes(oracle):
    z = np.zeros(16, dtype=np.float32)
    assert oracle.gemm("X", "N", 2, 2, 2, 1.0, z, 2, z, 2, 0.0, z, 2) == 1
    assert oracle.gemm("N", "Q", 2, 2, 2, 1.0, z, 2, z, 2, 0.0, z, 2) == 2
    assert oracle.gemm("N", "T", -1, 2, 2, 1.0, z, 2, z, 2, 0.0, z, 2) == 3
    assert oracle.gemm("T", "N", 2, 2, 2, 1.0, z, 1, z, 2, 0.0, z, 2) == 8
    assert oracle.gemm("N", "T", 2, 2, 2, 1.0, z, 2, z, 1, 0.0, z, 2) == 10
    assert oracle.gemm("N", "T", 2, 2, 2, 1.0, z, 2, z, 2, 0.0, z, 1) == 13
    assert oracle.syrk("X", "N", 2, 2, 1.0, z, 2, 0.0, z, 2) == 1
    assert oracle.syrk("L", "N", 2, 2, 1.0, z, 1, 0.0, z, 2) == 7
    assert oracle.trsm("L", "L", "N", "X", 2, 2, 1.0, z, 2, z, 2) == 4
    assert oracle.trsm("R", "L", "N", "N", 2, 3, 1.0, z, 2, z, 2) == 9
    assert oracle.trsm("L", "L", "N", "N", 3, 2, 1.0, z, 3, z, 2) == 11


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("seed", range(5))
def test_oracle_syrk_vs_float64(oracle, dt, uplo, trans, seed):
    rng = np.random.default_rng(seed)
    n, k, alpha, beta = 45, 31, 1.25, -0.5
    lda = (n if trans == "N" else k) + 2
    a = _rand(rng, (lda, k if trans == "N" else n), dt)
    c = _rand(rng, (n + 1, n), dt)
    A = oracle.op(oracle.view(a, *((n, k) if trans == "N" else (k, n)), lda), trans).astype(np.float64)
    ref = alpha * A @ A.T + beta * oracle.view(c, n, n, n + 1).astype(np.float64)
    c0 = c.copy()
    assert oracle.syrk(uplo, trans, n, k, alpha, a, lda, beta, c, n + 1) == 0
    got = oracle.view(c, n, n, n + 1)
    mask = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    tol = 1e-5 if dt == np.float32 else 1e-13
    assert np.max(np.abs(got[mask] - ref[mask])) / np.max(np.abs(ref[mask])) < tol
    np.testing.assert_array_equal(got[~mask], oracle.view(c0, n, n, n + 1)[~mask])


def _tri_problem(rng, side, m, n, dt):
    na = m if side == "L" else n
    a = rng.standard_normal((na + 2, na)) / np.sqrt(na)
    a[np.arange(na), np.arange(na)] = na + np.abs(rng.standard_normal(na))  # diagonally dominant
    b = rng.standard_normal((m + 1, n))
    return np.asfortranarray(a.astype(dt)), np.asfortranarray(b.astype(dt)), na + 2, m + 1


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("seed", range(5))
def test_oracle_trsm_vs_float64(oracle, dt, side, uplo, ta, diag, seed):
    rng = np.random.default_rng(seed)
    m, n, alpha = 23, 19, 0.75
    a, b, lda, ldb = _tri_problem(rng, side, m, n, dt)
    if diag == "U":  # keep the unit-diagonal system well conditioned
        a = np.asfortranarray((a / (m if side == "L" else n)).astype(dt))
    ref = oracle.trsm_f64(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb)
    x = b.copy(order="F")
    assert oracle.trsm(side, uplo, ta, diag, m, n, alpha, a, lda, x, ldb) == 0
    tol = 2e-6 if dt == np.float32 else 1e-13
    assert oracle.max_rel_err(oracle.view(x, m, n, ldb), ref) < tol
    if side == "R" and ta == "T":
        # the reference's right/trans branches solve with A, not A^T
        xb = b.copy(order="F")
        oracle.trsm(side, uplo, ta, diag, m, n, alpha, a, lda, xb, ldb, flags=oracle.BUG_COMPAT)
        ref_quirk = oracle.trsm_f64(side, uplo, "N", diag, m, n, alpha, a, lda, b, ldb)
        assert oracle.max_rel_err(oracle.view(xb, m, n, ldb), ref_quirk) < tol
