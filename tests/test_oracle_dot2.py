"""Pins the oracle's compensated float64 checker (oracle/dot2.cpp) before the GPU
tests use it: every element it returns is within a few units in the last place
of the exact value (rational arithmetic with fractions.Fraction), including
products whose terms cancel to far below their size, where a float64 dot
product loses all its digits; and op(A) / op(B) follow the Netlib transposes."""
from fractions import Fraction

import numpy as np
import pytest

U = 2.0 ** -53


def exact_rows(opa, opb, rows):
    out = np.empty((len(rows), opb.shape[1]))
    for r, i in enumerate(rows):
        for j in range(opb.shape[1]):
            out[r, j] = float(sum(Fraction(float(x)) * Fraction(float(y)) for x, y in zip(opa[i], opb[:, j])))
    return out


def test_cancellation_beyond_float64(oracle):
    """x . y = 1 exactly, with terms of size 1e16: float64 sums to 0, the checker to 1."""
    a = np.array([[1e16, 1.0, -1e16]], order="F")  # 1 x 3
    b = np.ones((3, 1), order="F")
    assert (a @ b)[0, 0] == 0.0
    got = oracle.gemm_rows_dot2("N", "N", 1, 3, a, 1, b, 3, [0])
    assert got[0, 0] == 1.0


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_matches_exact_arithmetic(oracle, ta, tb):
    rng = np.random.default_rng(40)
    m, n, k = 9, 6, 150
    opa = rng.uniform(-1, 1, (m, k)) * 2.0 ** rng.integers(-30, 31, (m, k))
    opb = rng.uniform(-1, 1, (k, n)) * 2.0 ** rng.integers(-30, 31, (k, n))
    opa[:, 0] = 2.0 ** 40
    opb[0, :] = 1.0
    opa[:, 1] = -(2.0 ** 40)  # the two leading terms cancel exactly
    opb[1, :] = 1.0
    a = np.asfortranarray(opa if ta == "N" else opa.T)
    b = np.asfortranarray(opb if tb == "N" else opb.T)
    rows = [0, 3, 8]
    got = oracle.gemm_rows_dot2(ta, tb, n, k, a, a.shape[0], b, b.shape[0], rows)
    want = exact_rows(opa, opb, rows)
    mag = np.abs(opa[rows]) @ np.abs(opb)  # sum |a_l b_l| per element
    # Dot2 bound: u |s| + gamma_k^2 sum |a b|, gamma_k = k u / (1 - k u)
    gamma = k * U / (1 - k * U)
    assert np.all(np.abs(got - want) <= 2 * U * np.abs(want) + 2 * gamma ** 2 * mag)
    # a plain float64 product misses by far more here: the check can tell the two apart
    plain = opa[rows] @ opb
    assert np.max(np.abs(plain - want) / np.abs(want)) > 100 * np.max(np.abs(got - want) / np.abs(want))
