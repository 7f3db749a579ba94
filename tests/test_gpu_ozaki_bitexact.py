"""The GPU's Ozaki dgemm equals the oracle's step-by-step restatement of the same
scheme (oracle.ozaki_gemm_emulated) bit for bit: the int32 slice products are
exact and the epilogue's fp64 operations are restated in the kernel's order, so
no tolerance is needed.  Covers one-pass (s <= 4) and two-pass (s > 4) slice
counts, every transpose pair, ragged tiles, a zero row (exponent 0), rows scaled
by 2^[-20, 20], alpha != 1 and beta = 0 (C is not read: it starts as NaN)."""
import numpy as np
import pytest

import mojoblas_b200 as mb
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()
    mb.load()


@pytest.mark.parametrize("s", [2, 4, 5, 7, 8])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
@pytest.mark.parametrize("m,n,k,scaled", [(96, 80, 300, False), (130, 257, 1000, True)])
def test_ozaki_bit_exact(oracle, s, ta, tb, m, n, k, scaled):
    rng = np.random.default_rng(m + n + k + s)
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ra + 1, ca)))
    b = np.asfortranarray(rng.uniform(-1, 1, (rb + 2, cb)))
    if scaled:  # rows of op(A) and the k rows of op(B) by 2^u, u in [-20, 20]
        su, sv = 2.0 ** rng.integers(-20, 21, m), 2.0 ** rng.integers(-20, 21, k)
        if ta == "N":
            a[:m, :] *= su[:, None]
        else:
            a[:, :m] *= su[None, :]
        if tb == "N":
            b[:k, :] *= sv[:, None]
        else:
            b[:, :k] *= sv[None, :]
    if ta == "N":  # one all-zero row of op(A)
        a[3, :] = 0.0
    else:
        a[:, 3] = 0.0
    c = np.full((m, n), np.nan, order="F")
    assert mb.gemm(ta, tb, m, n, k, 1.25, a, ra + 1, b, rb + 2, 0.0, c, m, mode=mb.OZAKI, slices=s) == 0
    want = oracle.ozaki_gemm_emulated(ta, tb, m, n, k, 1.25, a, ra + 1, b, rb + 2, s)
    assert np.array_equal(c, want), (np.max(np.abs(c - want)), np.sum(c != want))
