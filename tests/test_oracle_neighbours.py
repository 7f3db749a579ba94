"""Pins the oracle's symm / syr2k / trmm restatements before the GPU routines are
compared against them.

1. Every symm / syr2k / trmm known answer in the reference's own level-3 tests
   (mojoBLAS tests/test_level3.mojo, extracted into tests/golden/) comes out of
   the restatement (src/level3/symm.mojo:20-241, syr2k.mojo:20-190,
   trmm.mojo:20-305).
2. On seeded random inputs the restatement agrees with an independent float64
   computation for every side / uplo / trans / diag, alpha and beta case.
3. Info numbering and quick returns follow the reference.
4. The reference's left-side symm drops alpha * sum_i A(i,l) B(i,j) from C(l,j)
   when B(l,j) == 0 (symm.mojo:113, :131); that reproduces only with BUG_COMPAT.
"""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).parent / "golden" / "level3_known_answers.json"
CASES = [c for c in json.loads(GOLDEN.read_text())["cases"]
         if c["call"]["routine"] in ("symm", "syr2k", "trmm")]


def test_golden_case_count():
    # 6 trmm, 4 symm, 2 syr2k known answers in the reference's level-3 tests
    names = [c["call"]["routine"] for c in CASES]
    assert names.count("trmm") == 6 and names.count("symm") == 4 and names.count("syr2k") == 2


@pytest.mark.parametrize("flags", [0, 1], ids=["netlib", "bug_compat"])
@pytest.mark.parametrize("case", CASES, ids=[c["test"] for c in CASES])
def test_oracle_matches_reference_known_answers(oracle, case, flags):
    dt = np.float32 if case["dtype"] == "float32" else np.float64
    bufs = {k: np.array(v, dtype=dt) for k, v in case["inputs"].items()}
    args = [bufs[a["array"]] if isinstance(a, dict) else a for a in case["call"]["args"]]
    routine = case["call"]["routine"]
    if routine == "symm":
        info = oracle.symm(*args, flags=flags)
    else:
        info = {"syr2k": oracle.syr2k, "trmm": oracle.trmm}[routine](*args)
    assert info == 0
    for a in case["asserts"]:
        got = float(bufs[a["array"]][a["index"]])
        exp = a["expected"]
        atol = a["atol"] if a["atol"] is not None else 1e-8
        # Mojo's assert_almost_equal: |got-exp| <= atol + rtol*|exp|, rtol 1e-5
        assert abs(got - exp) <= atol + 1e-5 * abs(exp), (case["test"], a, got)


def _rand(rng, shape, dt):
    return np.asfortranarray(rng.uniform(-1, 1, size=shape).astype(dt))


def _tol(dt):
    return 1e-5 if dt == np.float32 else 1e-13


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("m,n,alpha,beta", [(37, 29, 1.5, 0.5), (70, 65, -0.75, 0.0), (9, 80, 1.0, 1.0)])
def test_oracle_symm_vs_float64(oracle, dt, side, uplo, m, n, alpha, beta):
    rng = np.random.default_rng(11)
    na = m if side == "L" else n
    lda, ldb, ldc = na + 2, m + 3, m + 1
    a = _rand(rng, (lda, na), dt)
    b = _rand(rng, (ldb, n), dt)
    c = _rand(rng, (ldc, n), dt)
    ref = oracle.symm_f64(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc)
    c0 = c.copy()
    assert oracle.symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c, ldc) == 0
    assert oracle.max_rel_err(oracle.view(c, m, n, ldc), ref) < _tol(dt)
    np.testing.assert_array_equal(c[m:], c0[m:])


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T", "c"])
@pytest.mark.parametrize("n,k,alpha,beta", [(45, 31, 1.25, -0.5), (70, 3, 1.0, 0.0), (8, 100, -2.0, 1.0)])
def test_oracle_syr2k_vs_float64(oracle, dt, uplo, trans, n, k, alpha, beta):
    rng = np.random.default_rng(12)
    rows, cols = (n, k) if trans == "N" else (k, n)
    lda, ldb, ldc = rows + 1, rows + 2, n + 1
    a = _rand(rng, (lda, cols), dt)
    b = _rand(rng, (ldb, cols), dt)
    c = _rand(rng, (ldc, n), dt)
    ref = oracle.syr2k_f64(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    c0 = c.copy()
    assert oracle.syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc) == 0
    got = oracle.view(c, n, n, ldc)
    mask = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    assert np.max(np.abs(got[mask] - ref[mask])) / np.max(np.abs(ref[mask])) < _tol(dt)
    np.testing.assert_array_equal(got[~mask], oracle.view(c0, n, n, ldc)[~mask])


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("alpha", [0.75, 1.0])
def test_oracle_trmm_vs_float64(oracle, dt, side, uplo, ta, diag, alpha):
    rng = np.random.default_rng(13)
    m, n = 23, 70  # n >= 64 reaches the parallel column loop
    na = m if side == "L" else n
    lda, ldb = na + 2, m + 1
    a = _rand(rng, (lda, na), dt)
    b = _rand(rng, (ldb, n), dt)
    b[3, 5] = 0.0  # a zero entry reaches the zero skips
    ref = oracle.trmm_f64(side, uplo, ta, diag, m, n, alpha, a, lda, b, ldb)
    x = b.copy(order="F")
    assert oracle.trmm(side, uplo, ta, diag, m, n, alpha, a, lda, x, ldb) == 0
    assert oracle.max_rel_err(oracle.view(x, m, n, ldb), ref) < _tol(dt)
    np.testing.assert_array_equal(x[m:], b[m:])


def test_oracle_neighbour_info_and_quick_returns(oracle):
    z = np.zeros(16, dtype=np.float64)
    assert oracle.symm("X", "U", 2, 2, 1.0, z, 2, z, 2, 0.0, z, 2) == 1
    assert oracle.symm("L", "X", 2, 2, 1.0, z, 2, z, 2, 0.0, z, 2) == 2
    assert oracle.symm("L", "U", -1, 2, 1.0, z, 2, z, 2, 0.0, z, 2) == 3
    assert oracle.symm("L", "U", 2, -1, 1.0, z, 2, z, 2, 0.0, z, 2) == 4
    assert oracle.symm("R", "U", 2, 3, 1.0, z, 2, z, 2, 0.0, z, 2) == 7
    assert oracle.symm("L", "U", 2, 2, 1.0, z, 2, z, 1, 0.0, z, 2) == 9
    assert oracle.symm("L", "U", 2, 2, 1.0, z, 2, z, 2, 0.0, z, 1) == 12
    assert oracle.syr2k("X", "N", 2, 2, 1.0, z, 2, z, 2, 0.0, z, 2) == 1
    assert oracle.syr2k("U", "X", 2, 2, 1.0, z, 2, z, 2, 0.0, z, 2) == 2
    assert oracle.syr2k("U", "N", -1, 2, 1.0, z, 2, z, 2, 0.0, z, 2) == 3
    assert oracle.syr2k("U", "N", 2, -1, 1.0, z, 2, z, 2, 0.0, z, 2) == 4
    assert oracle.syr2k("U", "T", 2, 3, 1.0, z, 2, z, 3, 0.0, z, 2) == 7
    assert oracle.syr2k("U", "N", 2, 2, 1.0, z, 2, z, 1, 0.0, z, 2) == 9
    assert oracle.syr2k("U", "N", 2, 2, 1.0, z, 2, z, 2, 0.0, z, 1) == 12
    assert oracle.trmm("X", "U", "N", "N", 2, 2, 1.0, z, 2, z, 2) == 1
    assert oracle.trmm("L", "X", "N", "N", 2, 2, 1.0, z, 2, z, 2) == 2
    assert oracle.trmm("L", "U", "X", "N", 2, 2, 1.0, z, 2, z, 2) == 3
    assert oracle.trmm("L", "U", "N", "X", 2, 2, 1.0, z, 2, z, 2) == 4
    assert oracle.trmm("L", "U", "N", "N", -1, 2, 1.0, z, 2, z, 2) == 5
    assert oracle.trmm("L", "U", "N", "N", 2, -1, 1.0, z, 2, z, 2) == 6
    assert oracle.trmm("R", "U", "N", "N", 2, 3, 1.0, z, 2, z, 2) == 9
    assert oracle.trmm("L", "U", "N", "N", 3, 2, 1.0, z, 3, z, 2) == 11
    # alpha == 0 and beta == 1: C untouched, even NaN (symm.mojo:88, syr2k.mojo:95)
    c = np.full(4, np.nan)
    assert oracle.symm("L", "U", 2, 2, 0.0, z, 2, z, 2, 1.0, c, 2) == 0
    assert oracle.syr2k("L", "N", 2, 2, 0.0, z, 2, z, 2, 1.0, c, 2) == 0
    assert np.all(np.isnan(c))
    # trmm with alpha == 0 writes zeros, NaN included (trmm.mojo:94-98)
    b = np.full(4, np.nan)
    assert oracle.trmm("L", "U", "N", "N", 2, 2, 0.0, z, 2, b, 2) == 0
    assert np.all(b == 0.0)
    # syr2k with beta == 0 clears the triangle, NaN included, and leaves the other one
    c = np.full(4, np.nan)
    assert oracle.syr2k("L", "N", 2, 2, 0.0, z, 2, z, 2, 0.0, c, 2) == 0
    assert c[0] == 0 and c[1] == 0 and c[3] == 0 and np.isnan(c[2])


@pytest.mark.parametrize("uplo", ["U", "L"])
def test_oracle_symm_zero_skip_quirk(oracle, uplo):
    rng = np.random.default_rng(14)
    m, n = 12, 3
    a = _rand(rng, (m, m), np.float64)
    b = _rand(rng, (m, n), np.float64)
    b[5, 1] = 0.0
    ref = oracle.symm_f64("L", uplo, m, n, 1.0, a, m, b, m, 0.0, b, m)
    c1 = np.zeros((m, n), order="F")
    assert oracle.symm("L", uplo, m, n, 1.0, a, m, b, m, 0.0, c1, m) == 0
    assert oracle.max_rel_err(c1, ref) < 1e-14
    c2 = np.zeros((m, n), order="F")
    assert oracle.symm("L", uplo, m, n, 1.0, a, m, b, m, 0.0, c2, m, flags=oracle.BUG_COMPAT) == 0
    # only C(5,1) differs: the quirk drops sum_i A(i,5) B(i,1) over the stored part of column 5
    diff = np.abs(c2 - ref) > 1e-12
    assert diff[5, 1] and diff.sum() == 1
    A = oracle.sym(a, uplo)
    rows = np.arange(5) if uplo == "U" else np.arange(6, m)
    np.testing.assert_allclose(c2[5, 1], ref[5, 1] - A[rows, 5] @ b[rows, 1], rtol=1e-12)
