"""The benchmark workloads at their full sizes, checked through properties that do
not need a full float64 product:

* sampled rows (columns for trsm) against float64 numpy / scipy on the same inputs,
  and for dgemm against the oracle's compensated product (exact to about 2^-106);
* row and column checksums, C 1 = op(A) (op(B) 1) and 1^T C = (1^T op(A)) op(B),
  formed in float64 from matrix-vector products (every element of C enters);
* the metric's fixed-error condition: each split / Ozaki form's error is at or
  below the plain kernel's on the same inputs;
* entries the routine must not write (syrk's other triangle) keep their values.

Workloads: sgemm NT and TN at M = N = K = 8192 (plain FP32, BF16x3, BF16x6),
dgemm NN at 4096^3 (plain FP64, Ozaki with the default 7 slices), dtrsm
Left/Lower/NoTrans/NonUnit at 4096^2 with the trsm configuration's inputs
(off-diagonal N(0,1)/sqrt(n), diagonal n + |N(0,1)|, B N(0,1)) and ssyrk
Lower/NoTrans at N = 8192, K = 2048.  Inputs uniform[-1, 1) unless stated, from
seeded torch generators on the device.  Tolerances (normwise relative):
1e-6 sqrt(k) for float32 plain and BF16x6, 1.5e-5 for BF16x3, 4e-16 sqrt(k)
for float64, each times 4.
"""
import numpy as np
import pytest

import mojoblas_b200 as mb
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    t = need_gpu()
    mb.load()
    return t


def col_major(torch, rows, cols, gen, dtype):
    """rows x cols column-major matrix, uniform[-1, 1) (a cols x rows row-major tensor)."""
    return torch.rand((cols, rows), generator=gen, device="cuda", dtype=dtype).mul_(2).sub_(1)


def host64(t):
    """The column-major matrix a device tensor holds, as a float64 (rows, cols) array."""
    return t.double().cpu().numpy().T


def rel(x, ref):
    return float(np.max(np.abs(x - ref)) / np.max(np.abs(ref)))


def tol32(k):
    return 4e-6 * np.sqrt(k)


def tol64(k):
    return 1.6e-15 * np.sqrt(k)


@pytest.fixture(scope="module")
def sgemm_8192(torch):
    n = 8192
    g = torch.Generator(device="cuda")
    g.manual_seed(21)
    A = col_major(torch, n, n, g, torch.float32)
    B = col_major(torch, n, n, g, torch.float32)
    C = torch.empty((n, n), device="cuda", dtype=torch.float32)
    rows = np.sort(np.random.default_rng(22).choice(n, 128, replace=False))
    return n, A, B, C, rows, host64(A), host64(B)


@pytest.mark.parametrize("ta,tb", [("N", "T"), ("T", "N")])
def test_sgemm_8192_split_forms(torch, sgemm_8192, ta, tb):
    n, A, B, C, rows, a, b = sgemm_8192
    opA = a if ta == "N" else a.T
    opB = b if tb == "N" else b.T
    ref = opA[rows, :] @ opB
    ones = np.ones(n)
    row_sums, col_sums = opA @ (opB @ ones), (ones @ opA) @ opB
    errs = {}
    for name, mode in (("plain", mb.PLAIN), ("bf16x3", mb.BF16X3), ("bf16x6", mb.BF16X6)):
        C.fill_(float("nan"))  # beta = 0: C must not be read
        assert mb.gemm(ta, tb, n, n, n, 1.0, A, n, B, n, 0.0, C, n, mode=mode) == 0
        c = host64(C)
        assert np.isfinite(c).all(), name
        errs[name] = rel(c[rows, :], ref)
        assert rel(c.sum(axis=1), row_sums) < (1.5e-5 if mode == mb.BF16X3 else tol32(n)), name
        assert rel(c.sum(axis=0), col_sums) < (1.5e-5 if mode == mb.BF16X3 else tol32(n)), name
    assert errs["plain"] < tol32(n)
    assert errs["bf16x3"] < 1.5e-5
    assert errs["bf16x6"] <= errs["plain"], errs  # the fixed-error condition of the metric


def test_dgemm_4096_ozaki(torch, oracle):
    """The sampled rows' reference is the oracle's compensated product, accurate well
    below a float64 GEMM's own rounding, so the two forms' errors are measured, not
    the reference's."""
    n = 4096
    g = torch.Generator(device="cuda")
    g.manual_seed(23)
    A = col_major(torch, n, n, g, torch.float64)
    B = col_major(torch, n, n, g, torch.float64)
    C = torch.empty((n, n), device="cuda", dtype=torch.float64)
    a, b = host64(A), host64(B)
    rows = np.sort(np.random.default_rng(24).choice(n, 32, replace=False))
    ref = oracle.gemm_rows_dot2("N", "N", n, n, a, n, b, n, rows)
    ones = np.ones(n)
    row_sums = a @ (b @ ones)
    errs = {}
    for name, mode in (("plain", mb.PLAIN), ("ozaki", mb.OZAKI)):
        assert mb.gemm("N", "N", n, n, n, 1.0, A, n, B, n, 0.0, C, n, mode=mode) == 0
        c = host64(C)
        errs[name] = rel(c[rows, :], ref)
        assert rel(c.sum(axis=1), row_sums) < tol64(n), name
    assert errs["plain"] < tol64(n)
    assert errs["ozaki"] <= errs["plain"], errs
    # 7 slices keep 54 bits of each scaled operand: within a few units of 2^-53 of max|C|
    assert errs["ozaki"] < 16 * 2.0 ** -53, errs


def test_dtrsm_4096_configuration_inputs(torch):
    import scipy.linalg as sl
    n = 4096
    g = torch.Generator(device="cuda")
    g.manual_seed(25)
    A = torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64) / np.sqrt(n)
    A.diagonal().copy_(n + torch.randn(n, generator=g, device="cuda", dtype=torch.float64).abs())
    B0 = torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64)
    L = np.tril(host64(A))
    b = host64(B0)
    cols = np.sort(np.random.default_rng(26).choice(n, 128, replace=False))
    ref = sl.solve_triangular(L, b[:, cols], lower=True)
    errs = {}
    for name, mode in (("plain", mb.PLAIN), ("ozaki", mb.OZAKI)):
        X = B0.clone()
        assert mb.trsm("L", "L", "N", "N", n, n, 1.0, A, n, X, n, mode=mode) == 0
        x = host64(X)
        errs[name] = rel(x[:, cols], ref)
        # backward error of every column: ||L x - b|| / (||L|| ||x|| + ||b||), float64 residual
        r = L @ x - b
        bwd = np.abs(r).max(axis=0) / (np.abs(L).sum(axis=1).max() * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
        assert bwd.max() < 1e-15, name
    assert errs["plain"] < 2 * tol64(n)
    assert errs["ozaki"] <= 2 * errs["plain"], errs


def test_ssyrk_8192x2048(torch):
    n, k = 8192, 2048
    g = torch.Generator(device="cuda")
    g.manual_seed(27)
    A = col_major(torch, n, k, g, torch.float32)
    C = torch.empty((n, n), device="cuda", dtype=torch.float32)
    a = host64(A)
    rows = np.sort(np.random.default_rng(28).choice(n, 128, replace=False))
    ref = a[rows, :] @ a.T
    lower = np.arange(n)[None, :] <= rows[:, None]
    errs = {}
    for name, mode in (("plain", mb.PLAIN), ("bf16x6", mb.BF16X6)):
        C.fill_(7.0)
        assert mb.syrk("L", "N", n, k, 1.0, A, n, 0.0, C, n, mode=mode) == 0
        c = host64(C)[rows, :]
        errs[name] = float(np.max(np.abs(c - ref)[lower]) / np.max(np.abs(ref[lower])))
        assert np.all(c[~lower] == 7.0), name  # the upper triangle is not written
    assert errs["plain"] < tol32(k)
    assert errs["bf16x6"] <= errs["plain"], errs
