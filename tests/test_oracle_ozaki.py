"""Pins the oracle's restatement of the Ozaki scheme (oracle.ozaki_gemm_emulated),
which the GPU tests compare with the library bit for bit, against independent
references on the CPU:

* every transpose pair agrees with a float64 product to float64 accuracy at 7
  slices, and an all-zero row gives exact zeros;
* against compensated (Dot2) products, the error falls by about 2^-8 per added
  slice and stays within the truncation bound: each operand keeps 8s - 2 bits
  of its row's (column's) scale, so |error| <= 2 k 2^-(8s-2) max|A| max|B|
  per element, relative to max|C|.
"""
import numpy as np
import pytest


def case(rng, ta, tb, m, n, k):
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    a = np.asfortranarray(rng.uniform(-1, 1, (ra + 1, ca)))
    b = np.asfortranarray(rng.uniform(-1, 1, (rb + 2, cb)))
    return a, ra + 1, b, rb + 2


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("T", "N"), ("N", "T"), ("T", "T")])
def test_transposes_and_zero_row(oracle, ta, tb):
    rng = np.random.default_rng(61)
    m, n, k = 37, 29, 55
    a, lda, b, ldb = case(rng, ta, tb, m, n, k)
    if ta == "N":
        a[3, :] = 0.0
    else:
        a[:, 3] = 0.0
    ref = oracle.gemm_f64(ta, tb, m, n, k, 1.25, a, lda, b, ldb, 0.0, np.zeros((m, n), order="F"), m)
    got = oracle.ozaki_gemm_emulated(ta, tb, m, n, k, 1.25, a, lda, b, ldb, 7)
    assert oracle.max_rel_err(got, ref) < 4e-15
    assert np.all(got[3] == 0.0)


def test_error_per_slice(oracle):
    rng = np.random.default_rng(62)
    m, n, k = 96, 80, 300
    a, lda, b, ldb = case(rng, "N", "N", m, n, k)
    ref = oracle.gemm_rows_dot2("N", "N", n, k, a, lda, b, ldb, np.arange(m))
    errs = []
    for s in range(2, 9):
        got = oracle.ozaki_gemm_emulated("N", "N", m, n, k, 1.0, a, lda, b, ldb, s)
        err = oracle.max_rel_err(got, ref)
        bound = 2 * k * 2.0 ** -(8 * s - 2) / np.max(np.abs(ref))  # max|A|, max|B| <= 1
        assert err <= bound + 4 * 2.0 ** -53, (s, err, bound)
        errs.append(err)
    for s in range(2, 7):  # about 2^-8 per slice until the fp64 epilogue's own rounding is reached
        assert errs[s - 1] < errs[s - 2] / 64, errs
    assert errs[-2] < 2 * 2.0 ** -53 and errs[-1] < 2 * 2.0 ** -53  # 7 and 8 slices: at fp64 rounding
