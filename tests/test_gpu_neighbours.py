"""Parity of symm, syr2k and trmm (the routines next to the gemm / syrk / trsm hot
path, on the same GEMM kernels) with the reference's algorithms.

Every case runs the same seeded inputs through (a) the library's C ABI on the
GPU, (b) the oracle's restatement of the reference routine on the CPU
(src/level3/symm.mojo:20-241, syr2k.mojo:20-190, trmm.mojo:20-305) and (c) a
float64 numpy computation.  Tolerance (normwise max relative error against
float64, k = the reduction length):
    plain float32, BF16x6:  1e-6 * sqrt(max(k, 16))
    BF16x3:                 1e-5 (two bf16 terms keep ~2^-17 per product at any k)
    plain float64, Ozaki (the default 7 slices):  4e-16 * sqrt(max(k, 16))
each times 4; GPU and oracle agree within twice that.  Entries that the routine
must not read (the other triangle of A, the diagonal of a unit triangle) are
NaN, and entries it must not write (padding rows, the other triangle of C) are
compared bit for bit.
"""
import json
from pathlib import Path

import numpy as np
import pytest

import mojoblas_b200 as mb
from tests.gpu_util import need_gpu, rand

pytestmark = pytest.mark.gpu

GOLDEN = json.loads((Path(__file__).parent / "golden" / "level3_known_answers.json").read_text())


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()
    mb.load()


def tol(dt, k, mode=mb.PLAIN):
    if mode == mb.BF16X3:
        return 1e-5 * 4
    return (1e-6 if dt == np.float32 else 4e-16) * np.sqrt(max(k, 16)) * 4


MODES = [(np.float32, mb.PLAIN), (np.float32, mb.BF16X3), (np.float32, mb.BF16X6),
         (np.float64, mb.PLAIN), (np.float64, mb.OZAKI)]
MODE_IDS = ["f32", "bf16x3", "bf16x6", "f64", "ozaki"]

CASES = [c for c in GOLDEN["cases"] if c["call"]["routine"] in ("symm", "syr2k", "trmm")]


@pytest.mark.parametrize("case", CASES, ids=[c["test"] for c in CASES])
def test_known_answers_on_gpu(case):
    """The reference's own symm / syr2k / trmm known answers through the C ABI."""
    dt = np.float32 if case["dtype"] == "float32" else np.float64
    bufs = {k: np.array(v, dtype=dt) for k, v in case["inputs"].items()}
    args = [bufs[a["array"]] if isinstance(a, dict) else a for a in case["call"]["args"]]
    fn = {"symm": mb.symm, "syr2k": mb.syr2k, "trmm": mb.trmm}[case["call"]["routine"]]
    assert fn(*args) == 0
    for a in case["asserts"]:
        got = float(bufs[a["array"]][a["index"]])
        atol = a["atol"] if a["atol"] is not None else 1e-8
        assert abs(got - a["expected"]) <= atol + 1e-5 * abs(a["expected"]), (case["test"], a, got)


def _blank_other_triangle(a, na, uplo, diag="N"):
    """NaN in the triangle of A that the routine must not read (and on a unit diagonal)."""
    keep = np.tril(np.ones((na, na), bool)) if uplo == "L" else np.triu(np.ones((na, na), bool))
    if diag == "U":
        keep &= ~np.eye(na, dtype=bool)
    a[:na, :na][~keep] = np.nan


# ---- symm ----------------------------------------------------------------------------
@pytest.mark.parametrize("dt,mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("m,n,alpha,beta", [(130, 70, 1.5, 0.5), (33, 300, -0.75, 0.0), (257, 129, 1.0, 1.0)])
def test_symm(oracle, dt, mode, side, uplo, m, n, alpha, beta):
    rng = np.random.default_rng(m + 3 * n)
    na = m if side == "L" else n
    lda, ldb, ldc = na + 3, m + 1, m + 2
    a = rand(rng, (lda, na), dt)
    b = rand(rng, (ldb, n), dt)
    c = rand(rng, (ldc, n), dt)
    ref = oracle.symm_f64(side, uplo, m, n, alpha, np.nan_to_num(a), lda, b, ldb, beta, c, ldc)
    c_orc = c.copy(order="F")
    assert oracle.symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, c_orc, ldc) == 0
    _blank_other_triangle(a, na, uplo)
    if beta == 0.0:
        c[:m] = np.nan  # beta == 0: C is not read
    got = c.copy(order="F")
    assert mb.symm(side, uplo, m, n, alpha, a, lda, b, ldb, beta, got, ldc, mode=mode) == 0
    g = oracle.view(got, m, n, ldc)
    t = tol(dt, na, mode)
    assert np.all(np.isfinite(g))
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, oracle.view(c_orc, m, n, ldc).astype(np.float64)) < 2 * t
    np.testing.assert_array_equal(got[m:], c[m:])


def test_symm_zero_entries_of_b(oracle):
    """B with exact zeros: the full product (Netlib), not the reference's zero skip
    (symm.mojo:113, :131), which the oracle reproduces only with BUG_COMPAT."""
    rng = np.random.default_rng(7)
    m, n = 96, 40
    a = rand(rng, (m, m), np.float64)
    b = rand(rng, (m, n), np.float64)
    b[::7, ::3] = 0.0
    ref = oracle.symm_f64("L", "U", m, n, 1.0, a, m, b, m, 0.0, b, m)
    got = np.zeros((m, n), order="F")
    assert mb.symm("L", "U", m, n, 1.0, a, m, b, m, 0.0, got, m) == 0
    assert oracle.max_rel_err(got, ref) < tol(np.float64, m)
    quirk = np.zeros((m, n), order="F")
    oracle.symm("L", "U", m, n, 1.0, a, m, b, m, 0.0, quirk, m, flags=oracle.BUG_COMPAT)
    assert oracle.max_rel_err(quirk, ref) > 1e-3


# ---- syr2k ---------------------------------------------------------------------------
@pytest.mark.parametrize("dt,mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("trans", ["N", "T"])
@pytest.mark.parametrize("n,k,alpha,beta", [(130, 70, 1.25, -0.5), (300, 33, 1.0, 0.0), (65, 257, -2.0, 1.0)])
def test_syr2k(oracle, dt, mode, uplo, trans, n, k, alpha, beta):
    rng = np.random.default_rng(n + 5 * k)
    rows, cols = (n, k) if trans == "N" else (k, n)
    lda, ldb, ldc = rows + 1, rows + 2, n + 3
    a = rand(rng, (lda, cols), dt)
    b = rand(rng, (ldb, cols), dt)
    c = rand(rng, (ldc, n), dt)
    ref = oracle.syr2k_f64(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c, ldc)
    c_orc = c.copy(order="F")
    assert oracle.syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, c_orc, ldc) == 0
    mask = np.tril(np.ones((n, n), bool)) if uplo == "L" else np.triu(np.ones((n, n), bool))
    if beta == 0.0:
        c[:n][mask] = np.nan  # beta == 0: the triangle is not read
    got = c.copy(order="F")
    assert mb.syr2k(uplo, trans, n, k, alpha, a, lda, b, ldb, beta, got, ldc, mode=mode) == 0
    g = oracle.view(got, n, n, ldc)
    t = tol(dt, 2 * k, mode)
    assert np.all(np.isfinite(g[mask]))
    den = np.max(np.abs(ref[mask]))
    assert np.max(np.abs(g[mask] - ref[mask])) / den < t
    assert np.max(np.abs(g[mask] - oracle.view(c_orc, n, n, ldc)[mask])) / den < 2 * t
    np.testing.assert_array_equal(g[~mask], oracle.view(c, n, n, ldc)[~mask])  # other triangle untouched
    np.testing.assert_array_equal(got[n:], c[n:])


# ---- trmm ----------------------------------------------------------------------------
@pytest.mark.parametrize("dt,mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("side", ["L", "R"])
@pytest.mark.parametrize("uplo", ["U", "L"])
@pytest.mark.parametrize("ta", ["N", "T"])
@pytest.mark.parametrize("diag", ["N", "U"])
@pytest.mark.parametrize("na,nb,alpha", [(200, 37, 0.75), (1000, 70, -1.5), (700, 5, 2.0), (129, 600, 1.0)])
def test_trmm(oracle, dt, mode, side, uplo, ta, diag, na, nb, alpha):
    """na = order of A, nb = the other dimension of B.  The product runs as one GEMM
    whose tiles skip the zero half of the triangle: ragged orders (200, 700, 129 =
    one row of tiles plus one), 1000 with several tile rows, and thin (5) or wide
    (600) B, so both tile sizes and every band (left / right, lower / upper) run."""
    rng = np.random.default_rng(na + nb)
    m, n = (na, nb) if side == "L" else (nb, na)
    lda, ldb = na + 2, m + 1
    a = rand(rng, (lda, na), dt)
    b = rand(rng, (ldb, n), dt)
    ref = oracle.trmm_f64(side, uplo, ta, diag, m, n, alpha, np.nan_to_num(a), lda, b, ldb)
    x_orc = b.copy(order="F")
    assert oracle.trmm(side, uplo, ta, diag, m, n, alpha, a, lda, x_orc, ldb) == 0
    _blank_other_triangle(a, na, uplo, diag)
    got = b.copy(order="F")
    assert mb.trmm(side, uplo, ta, diag, m, n, alpha, a, lda, got, ldb, mode=mode) == 0
    g = oracle.view(got, m, n, ldb)
    t = tol(dt, na, mode)
    assert np.all(np.isfinite(g))
    assert oracle.max_rel_err(g, ref) < t
    assert oracle.max_rel_err(g, oracle.view(x_orc, m, n, ldb).astype(np.float64)) < 2 * t
    np.testing.assert_array_equal(got[m:], b[m:])


def test_trmm_alpha_zero_writes_zeros():
    """alpha == 0 sets B to zero, NaN included, without reading A (trmm.mojo:94-98)."""
    b = np.full((5, 4), np.nan, order="F")
    a = np.full((5, 5), np.nan, order="F")
    assert mb.trmm("L", "U", "N", "N", 5, 4, 0.0, a, 5, b, 5) == 0
    assert np.all(b == 0.0)


def test_device_pointers(oracle):
    """Device-resident operands (the fast path), trmm with a 2100-order triangle."""
    torch = need_gpu()
    rng = np.random.default_rng(9)
    m, n = 2100, 300
    a = rand(rng, (m, m), np.float32)
    b = rand(rng, (m, n), np.float32)
    ref = oracle.trmm_f64("L", "L", "N", "N", m, n, 1.0, a, m, b, m)
    ad = torch.from_numpy(np.ascontiguousarray(a.T)).cuda()  # column-major storage of A
    bd = torch.from_numpy(np.ascontiguousarray(b.T)).cuda()
    assert mb.trmm("L", "L", "N", "N", m, n, 1.0, ad, m, bd, m) == 0
    torch.cuda.synchronize()
    got = bd.cpu().numpy().T
    assert oracle.max_rel_err(got, ref) < tol(np.float32, m)
    # symm and syr2k on the same device buffers
    c = torch.zeros((n, m), dtype=torch.float32, device="cuda")
    assert mb.symm("L", "L", m, n, 1.0, ad, m, ad[:n], m, 0.0, c, m) == 0
    torch.cuda.synchronize()
    bsrc = np.ascontiguousarray(a[:, :n])
    ref_s = oracle.symm_f64("L", "L", m, n, 1.0, a, m, np.asfortranarray(bsrc), m, 0.0, bsrc, m)
    assert oracle.max_rel_err(c.cpu().numpy().T, ref_s) < tol(np.float32, m)
