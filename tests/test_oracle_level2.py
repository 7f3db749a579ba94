"""Pins the oracle's gemv / trsv restatements (src/level2/gemv.mojo:23-212,
src/level2/trsv.mojo:20-214) before the GPU routines are compared against them.

1. Every gemv / trsv known answer in the reference's own level-2 tests
   (tests/test_level2.mojo, tests/test_level2_extended.mojo, extracted into
   tests/golden/level2_known_answers.json) comes out of the restatement.
2. On seeded inputs the restatement agrees with float64 numpy / scipy for every
   trans / uplo / diag case and for unit, strided and negative increments.
3. Info numbering and quick returns follow the reference, including gemv's
   upper-case-only trans argument.
"""
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).parent / "golden" / "level2_known_answers.json"
CASES = json.loads(GOLDEN.read_text())["cases"]


def test_golden_case_count():
    names = [c["call"]["routine"] for c in CASES]
    assert names.count("gemv") == 8 and names.count("trsv") == 5


@pytest.mark.parametrize("case", CASES, ids=[c["test"] for c in CASES])
def test_oracle_matches_reference_known_answers(oracle, case):
    dt = np.float32 if case["dtype"] == "float32" else np.float64
    bufs = {k: np.array(v, dtype=dt) for k, v in case["inputs"].items()}
    args = [bufs[a["array"]] if isinstance(a, dict) else a for a in case["call"]["args"]]
    fn = {"gemv": oracle.gemv, "trsv": oracle.trsv}[case["call"]["routine"]]
    assert fn(*args) == 0
    for a in case["asserts"]:
        got = float(bufs[a["array"]][a["index"]])
        atol = a["atol"] if a["atol"] is not None else 1e-8
        assert abs(got - a["expected"]) <= atol + 1e-5 * abs(a["expected"]), (case["test"], a, got)


def strided(rng, n, inc, dt):
    """A buffer holding an n-vector with increment inc, filler NaN between its elements."""
    buf = np.full(max(1, 1 + (n - 1) * abs(inc)), np.nan, dtype=dt)
    start = 0 if inc > 0 else (1 - n) * inc
    buf[start + np.arange(n) * inc] = rng.uniform(-1, 1, n).astype(dt)
    return buf


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("trans", ["N", "T", "C"])
@pytest.mark.parametrize("incx,incy", [(1, 1), (2, 1), (1, -3), (-2, 2)])
@pytest.mark.parametrize("m,n,alpha,beta", [(37, 300, 1.5, 0.5), (300, 19, -1.0, 0.0), (5, 7, 2.0, 1.0)])
def test_oracle_gemv_vs_float64(oracle, dt, trans, incx, incy, m, n, alpha, beta):
    rng = np.random.default_rng(31)
    lda = m + 2
    a = np.asfortranarray(rng.uniform(-1, 1, (lda, n)).astype(dt))
    lenx, leny = (n, m) if trans == "N" else (m, n)
    x = strided(rng, lenx, incx, dt)
    y = strided(rng, leny, incy, dt)
    ref = oracle.gemv_f64(trans, m, n, alpha, a, lda, x, incx, beta, y, incy)
    got = y.copy()
    assert oracle.gemv(trans, m, n, alpha, a, lda, x, incx, beta, got, incy) == 0
    g = oracle.vec(got, leny, incy)
    tol = 1e-5 if dt == np.float32 else 1e-13
    assert oracle.max_rel_err(g, ref) < tol
    mask = np.ones(got.size, bool)
    mask[(0 if incy > 0 else (1 - leny) * incy) + np.arange(leny) * incy] = False
    assert np.all(np.isnan(got[mask]))  # the gaps between y's elements are untouched


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("incx", [1, 3, -2])
def test_oracle_trsv_vs_float64(oracle, dt, uplo, trans, diag, incx):
    rng = np.random.default_rng(32)
    n = 70
    a = rng.standard_normal((n + 1, n)) / np.sqrt(n)
    a[np.arange(n), np.arange(n)] = 2.0 + np.abs(rng.standard_normal(n))
    if diag == "U":
        a /= n
    a = np.asfortranarray(a.astype(dt))
    x = strided(rng, n, incx, dt)
    ref = oracle.trsv_f64(uplo, trans, diag, n, a, n + 1, x, incx)
    got = x.copy()
    assert oracle.trsv(uplo, trans, diag, n, a, n + 1, got, incx) == 0
    tol = 2e-6 if dt == np.float32 else 1e-13
    assert oracle.max_rel_err(oracle.vec(got, n, incx), ref) < tol


def test_oracle_level2_info_and_quick_returns(oracle):
    z = np.zeros(16)
    assert oracle.gemv("n", 2, 2, 1.0, z, 2, z, 1, 0.0, z, 1) == 1  # upper case only
    assert oracle.gemv("X", 2, 2, 1.0, z, 2, z, 1, 0.0, z, 1) == 1
    assert oracle.gemv("N", -1, 2, 1.0, z, 2, z, 1, 0.0, z, 1) == 2
    assert oracle.gemv("N", 2, -1, 1.0, z, 2, z, 1, 0.0, z, 1) == 3
    assert oracle.gemv("N", 3, 2, 1.0, z, 2, z, 1, 0.0, z, 1) == 6
    assert oracle.gemv("N", 2, 2, 1.0, z, 2, z, 0, 0.0, z, 1) == 8
    assert oracle.gemv("N", 2, 2, 1.0, z, 2, z, 1, 0.0, z, 0) == 11
    assert oracle.trsv("X", "N", "N", 2, z, 2, z, 1) == 1
    assert oracle.trsv("U", "X", "N", 2, z, 2, z, 1) == 2
    assert oracle.trsv("U", "N", "X", 2, z, 2, z, 1) == 3
    assert oracle.trsv("U", "N", "N", -1, z, 2, z, 1) == 4
    assert oracle.trsv("U", "N", "N", 3, z, 2, z, 1) == 6
    assert oracle.trsv("U", "N", "N", 2, z, 2, z, 0) == 8
    y = np.full(3, np.nan)
    assert oracle.gemv("T", 2, 3, 0.0, z, 2, z, 1, 1.0, y, 1) == 0  # alpha 0, beta 1: y untouched
    assert np.all(np.isnan(y))
    assert oracle.gemv("T", 2, 3, 0.0, z, 2, z, 1, 0.0, y, 1) == 0  # beta 0: zeros, NaN included
    assert np.all(y == 0.0)
