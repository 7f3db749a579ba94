"""Parity of the plain FP32 / FP64 CUDA kernels with the reference's algorithms.

Every case runs the same seeded inputs through (a) the library's C ABI on the
GPU, (b) the oracle's restatement of the reference routine on the CPU and (c) a
float64 numpy/scipy computation.  Tolerance (max relative error, normwise
max|X - X64| / max|X64|):
    float32:  TOL32(k) = 1e-6 * sqrt(max(k, 16))   (k = reduction length)
    float64:  TOL64(k) = 4e-16 * sqrt(max(k, 16))
GPU and oracle must each be within the tolerance of float64 and within twice
the tolerance of each other.  Integer-valued known answers must be exact.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import mojoblas_b200 as mb
from tests.gpu_util import need_gpu, rand, tri_system

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "level3_known_answers.json").read_text())


def tol(dt, k):
    return (1e-6 if dt == np.float32 else 4e-16) * np.sqrt(max(k, 16))


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()
    mb.load()


# ---- the reference's own known answers, through the C ABI ------------------------
CASES = [c for c in GOLDEN["cases"] if c["call"]["routine"] in ("gemm", "syrk", "trsm")]


@pytest.mark.parametrize("case", CASES, ids=[c["test"] for c in CASES])
def test_known_answers_on_gpu(case):
    dt = np.float32 if case["dtype"] == "float32" else np.float64
    bufs = {k: np.array(v, dtype=dt) for k, v in case["inputs"].items()}
    args = [bufs[a["array"]] if isinstance(a, dict) else a for a in case["call"]["args"]]
    fn = {"gemm": mb.gemm, "syrk": mb.syrk, "trsm": mb.trsm}[case["call"]["routine"]]
    assert fn(*args) == 0
    for a in case["asserts"]:
        got = float(bufs[a["array"]][a["index"]])
        atol = a["atol"] if a["atol"] is not None else 1e-8
        assert abs(got - a["expected"]) <= atol + 1e-5 * abs(a["expected"]), (case["test"], a, got)


# ---- gemm ----------------------------------------------------------------------------
def _gemm_case(oracle, dt, ta, tb, m, n, k, alpha, beta, pad=(0, 0, 0), seed=0, flags=0):
    rng = np.random.default_rng(seed)
    lda = (m if ta in "Nn" else k) + pad[0]
    ldb = (k if tb in "Nn" else n) + pad[1]
    ldc = m + pad[2]
    a = rand(rng, (lda, k if ta in "Nn" else m), dt)
    b = rand(rng, (ldb, n if tb in "Nn" else k), dt)
    c = rand(rng, (ldc, n), dt)
    ref64 = oracle.gemm_f64(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    c_orc = c.copy(order="F")
    assert oracle.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c_orc, ldc, flags=flags) == 0
    c_gpu = c.copy(order="F")
    assert mb.gemm(ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c_gpu, ldc) == 0
    return a, b, c, c_orc, c_gpu, ref64, ldc


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T"), ("c", "C")])
@pytest.mark.parametrize("m,n,k,alpha,beta,pad", [
    (512, 512, 512, 1.5, 0.5, (0, 0, 0)),      # configuration 1 shape and scalars
    (129, 67, 300, -0.75, 0.0, (3, 1, 5)),     # ragged tiles, padded leading dims
    (1, 1, 1, 2.0, 1.0, (0, 0, 0)),
    (300, 17, 1, 1.0, -2.0, (1, 0, 2)),
    (64, 640, 1031, 0.5, 1.0, (0, 7, 0)),      # float64: the v7 path in the reference
])
def test_gemm_parity(oracle, dt, ta, tb, m, n, k, alpha, beta, pad):
    _, _, c0, c_orc, c_gpu, ref64, ldc = _gemm_case(oracle, dt, ta, tb, m, n, k, alpha, beta, pad)
    t = tol(dt, k)
    g = oracle.view(c_gpu, m, n, ldc)
    o = oracle.view(c_orc, m, n, ldc)
    assert oracle.max_rel_err(g, ref64) < t
    assert oracle.max_rel_err(o, ref64) < t
    assert oracle.max_rel_err(g, o.astype(np.float64)) < 2 * t
    # padding rows between m and ldc are never written
    np.testing.assert_array_equal(c_gpu[m:], c0[m:])


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("alpha,beta,k", [(0.0, 0.0, 5), (0.0, 2.5, 5), (1.0, 0.0, 0), (1.5, -1.0, 0),
                                          (0.0, 1.0, 9)])
def test_gemm_alpha_zero_or_k_zero(oracle, dt, alpha, beta, k):
    """alpha == 0 or k == 0: C := beta*C (beta == 0 writes zeros, even over NaN)."""
    rng = np.random.default_rng(5)
    m, n = 37, 23
    a = rand(rng, (m, max(k, 1)), dt)
    b = rand(rng, (max(k, 1), n), dt)
    c = rand(rng, (m, n), dt)
    if beta == 0.0:
        c[3, 4] = np.nan
    c_orc, c_gpu = c.copy(order="F"), c.copy(order="F")
    assert oracle.gemm("N", "N", m, n, k, alpha, a, m, b, max(k, 1), beta, c_orc, m) == 0
    assert mb.gemm("N", "N", m, n, k, alpha, a, m, b, max(k, 1), beta, c_gpu, m) == 0
    np.testing.assert_array_equal(c_gpu, c_orc)


def test_gemm_v7_alpha_divergence_documented(oracle):
    """The reference's float64 NN n>=512 kernel drops alpha; the library applies it
    (Netlib).  With alpha == 1 — the configuration-2 value — both agree."""
    rng = np.random.default_rng(6)
    m, n, k = 96, 512, 80
    a, b = rand(rng, (m, k), np.float64), rand(rng, (k, n), np.float64)
    for alpha in (1.0, 3.0):
        c_q = np.zeros((m, n), order="F")
        oracle.gemm("N", "N", m, n, k, alpha, a, m, b, k, 0.0, c_q, m, flags=oracle.BUG_COMPAT)
        c_g = np.zeros((m, n), order="F")
        mb.gemm("N", "N", m, n, k, alpha, a, m, b, k, 0.0, c_g, m)
        if alpha == 1.0:
            assert oracle.max_rel_err(c_g, c_q) < tol(np.float64, k)
        else:
            assert oracle.max_rel_err(c_g, alpha * c_q) < tol(np.float64, k)


def test_gemm_device_pointers_torch(oracle):
    torch = need_gpu()
    rng = np.random.default_rng(7)
    m, n, k = 300, 200, 100
    a, b, c = rand(rng, (m, k), np.float32), rand(rng, (n, k), np.float32), rand(rng, (m, n), np.float32)
    ref = oracle.gemm_f64("N", "T", m, n, k, 1.25, a, m, b, n, 0.5, c, m)
    da = torch.from_numpy(a.T.copy()).cuda().T  # column-major storage on the device
    db = torch.from_numpy(b.T.copy()).cuda().T
    dc = torch.from_numpy(c.T.copy()).cuda().T
    assert mb.gemm("N", "T", m, n, k, 1.25, da, m, db, n, 0.5, dc, m) == 0
    got = dc.cpu().numpy()
    assert oracle.max_rel_err(got, ref) < tol(np.float32, k)


# ---- syrk ----------------------------------------------------------------------------
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,k,alpha,beta", [(300, 129, 1.0, 0.0), (257, 64, -0.5, 1.5), (5, 3, 2.0, 1.0)])
def test_syrk_parity(oracle, dt, uplo, trans, n, k, alpha, beta):
    rng = np.random.default_rng(8)
    lda = (n if trans == "N" else k) + 1
    a = rand(rng, (lda, k if trans == "N" else n), dt)
    c = rand(rng, (n + 2, n), dt)
    c_orc, c_gpu = c.copy(order="F"), c.copy(order="F")
    assert oracle.syrk(uplo, trans, n, k, alpha, a, lda, beta, c_orc, n + 2) == 0
    assert mb.syrk(uplo, trans, n, k, alpha, a, lda, beta, c_gpu, n + 2) == 0
    A = oracle.op(oracle.view(a, *((n, k) if trans == "N" else (k, n)), lda), trans).astype(np.float64)
    ref = alpha * A @ A.T + beta * oracle.view(c, n, n, n + 2).astype(np.float64)
    mask = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    g, o = oracle.view(c_gpu, n, n, n + 2), oracle.view(c_orc, n, n, n + 2)
    t = tol(dt, k)
    den = np.max(np.abs(ref[mask]))
    assert np.max(np.abs(g[mask] - ref[mask])) / den < t
    assert np.max(np.abs(g[mask] - o[mask])) / den < 2 * t
    # the other triangle and the padding rows are untouched
    np.testing.assert_array_equal(g[~mask], oracle.view(c, n, n, n + 2)[~mask])
    np.testing.assert_array_equal(c_gpu[n:], c[n:])


# ---- trsm ----------------------------------------------------------------------------
@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("m,n,alpha", [(200, 70, 0.75), (64, 33, 1.0), (5, 130, -2.0)])
def test_trsm_parity_all_modes(oracle, dt, side, uplo, ta, diag, m, n, alpha):
    rng = np.random.default_rng(9)
    a, b, lda, ldb = tri_system(rng, side, m, n, dt, ld_pad=3)
    na = m if side == "L" else n
    if diag == "U":  # unit diagonal: shrink the off-diagonal part to stay well conditioned
        a = np.asfortranarray((a / na).astype(dt))
    # garbage in the unreferenced triangle must not matter
    junk = np.triu(np.ones((na, na), bool), 1) if uplo == "L" else np.tril(np.ones((na, na), bool), -1)
    a[:na][junk] = np.nan
    ref = oracle.trsm_f64(side, uplo, ta, diag, m, n, alpha, np.nan_to_num(a), lda, b, ldb)
    x_orc, x_gpu = b.copy(order="F"), b.copy(order="F")
    assert oracle.trsm(side, uplo, ta, diag, m, n, alpha, a, lda, x_orc, ldb) == 0
    assert mb.trsm(side, uplo, ta, diag, m, n, alpha, a, lda, x_gpu, ldb) == 0
    g, o = oracle.view(x_gpu, m, n, ldb), oracle.view(x_orc, m, n, ldb)
    t = tol(dt, na) * 4
    assert np.all(np.isfinite(g))
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, o.astype(np.float64)) < 2 * t
    np.testing.assert_array_equal(x_gpu[m:], b[m:])


def test_trsm_right_trans_divergence_documented(oracle):
    """The reference solves X*A = B for side='R', trans='T'; the library solves
    X*A^T = B as Netlib defines.  The oracle reproduces both."""
    rng = np.random.default_rng(10)
    m, n = 40, 30
    a, b, lda, ldb = tri_system(rng, "R", m, n, np.float64)
    x_ref_quirk = b.copy(order="F")
    oracle.trsm("R", "U", "T", "N", m, n, 1.0, a, lda, x_ref_quirk, ldb, flags=oracle.BUG_COMPAT)
    x_netlib = b.copy(order="F")
    oracle.trsm("R", "U", "T", "N", m, n, 1.0, a, lda, x_netlib, ldb)
    x_gpu = b.copy(order="F")
    mb.trsm("R", "U", "T", "N", m, n, 1.0, a, lda, x_gpu, ldb)
    assert oracle.max_rel_err(x_gpu, x_netlib) < 1e-13
    assert oracle.max_rel_err(x_gpu, x_ref_quirk) > 1e-6


def test_workspace_allocation_failure_is_reported():
    """A failed device allocation surfaces as MBG_ERR_ALLOC (injected on the host)."""
    from mojoblas_b200 import _lib as L
    lib = L.load()
    lib.mbg_release_workspace()
    a = np.ones((64, 64), np.float32, order="F")
    c = np.zeros((64, 64), np.float32, order="F")
    lib.mbg_debug_fail_alloc(1)
    try:
        with pytest.raises(mb.MbgError) as ei:
            mb.gemm("N", "N", 64, 64, 64, 1.0, a, 64, a, 64, 0.0, c, 64)
        assert ei.value.status == L.MBG_ERR_ALLOC
    finally:
        lib.mbg_debug_fail_alloc(0)
    assert mb.gemm("N", "N", 64, 64, 64, 1.0, a, 64, a, 64, 0.0, c, 64) == 0
    assert np.all(c == 64.0)


def test_bounded_wait_expires_and_context_survives():
    """A kernel wait that can never be satisfied gives up after its limit (50 ms
    here), reports MBG_ERR_TIMEOUT, and the library keeps working afterwards."""
    from mojoblas_b200 import _lib as L
    lib = L.load()
    assert lib.mbg_debug_wait_probe(50_000_000) == L.MBG_ERR_TIMEOUT
    assert "bounded wait expired" in L.last_error()
    a = np.ones((32, 32), np.float32, order="F")
    c = np.zeros((32, 32), np.float32, order="F")
    assert mb.gemm("N", "N", 32, 32, 32, 1.0, a, 32, a, 32, 0.0, c, 32, mode=mb.BF16X6) == 0
    assert np.all(c == 32.0)


def test_peak_probes_are_plausible():
    """The probe kernels run and report throughputs in a plausible range for a B200."""
    import ctypes as C
    from mojoblas_b200 import _lib as L
    lib = L.load()
    v = [C.c_double() for _ in range(4)]
    assert lib.mbg_probe_peaks(*[C.byref(x) for x in v]) == 0, L.last_error()
    fp32, fp64, bf16, int8 = (x.value for x in v)
    assert 20 < fp32 < 200 and 5 < fp64 < 100 and 300 < bf16 < 5000 and 600 < int8 < 10000, (fp32, fp64, bf16, int8)
