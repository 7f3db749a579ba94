"""Complex gemm (mbg_cgemm / mbg_zgemm and their _ex forms) in every precision mode.

The reference has no complex routines (complex dtypes are on its roadmap,
README.md:152), so the checker is numpy's complex128 product of the same
inputs: max relative error (normwise) within the real kernels' tolerances at
reduction length 2k (tests/test_gpu_tc.py: TOL32, TOL_X3, TOL_OZ, TOL64), for
every trans pair including the conjugate transpose, complex alpha / beta,
padded leading dimensions, host and device buffers, beta = 0 with NaN in C,
and the quick returns (alpha = 0 scales C by beta; m or n = 0 leaves C alone).
"""
import numpy as np
import pytest

import mojoblas_b200 as mb
from tests.gpu_util import need_gpu
from tests.test_gpu_tc import TOL_X3, tol32, tol64, tol_oz

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu():
    need_gpu()
    mb.load()


def crand(rng, shape, dt):
    x = rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)
    return np.asfortranarray(x.astype(dt))


def op(x, t):
    return x if t == "N" else (x.T if t == "T" else x.conj().T)


def tol(dt, mode, k):
    if dt == np.complex64:
        return {mb.PLAIN: tol32(2 * k), mb.BF16X3: TOL_X3, mb.BF16X6: tol32(2 * k)}[mode]
    return {mb.PLAIN: tol64(2 * k), mb.OZAKI: tol_oz(7, 2 * k)}[mode]


CASES = [(np.complex64, mb.PLAIN), (np.complex64, mb.BF16X3), (np.complex64, mb.BF16X6),
         (np.complex128, mb.PLAIN), (np.complex128, mb.OZAKI)]


@pytest.mark.parametrize("dt,mode", CASES, ids=["c-plain", "c-bf16x3", "c-bf16x6", "z-plain", "z-ozaki"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("C", "N"), ("N", "C"), ("T", "C"), ("C", "T")])
def test_complex_gemm(dt, mode, ta, tb):
    rng = np.random.default_rng(40)
    m, n, k = 150, 97, 203
    alpha, beta = 0.75 - 0.5j, -0.25 + 1.0j
    ra, ca = (m, k) if ta == "N" else (k, m)
    rb, cb = (k, n) if tb == "N" else (n, k)
    a = crand(rng, (ra + 2, ca), dt)
    b = crand(rng, (rb + 1, cb), dt)
    c = crand(rng, (m + 3, n), dt)
    ref = alpha * (op(a[:ra].astype(np.complex128), ta) @ op(b[:rb].astype(np.complex128), tb)) \
        + beta * c[:m].astype(np.complex128)
    got = c.copy(order="F")
    assert mb.gemm(ta, tb, m, n, k, alpha, a, ra + 2, b, rb + 1, beta, got, m + 3, mode=mode, slices=7) == 0
    err = float(np.max(np.abs(got[:m] - ref)) / np.max(np.abs(ref)))
    assert err < tol(dt, mode, k), err
    np.testing.assert_array_equal(got[m:], c[m:])


@pytest.mark.parametrize("dt,mode", [(np.complex64, mb.BF16X6), (np.complex128, mb.OZAKI)])
def test_complex_gemm_device_buffers_beta_zero(dt, mode):
    torch = need_gpu()
    rng = np.random.default_rng(41)
    m, n, k = 300, 260, 128
    a, b = crand(rng, (m, k), dt), crand(rng, (k, n), dt)
    tdt = torch.complex64 if dt == np.complex64 else torch.complex128
    da = torch.from_numpy(np.ascontiguousarray(a.T)).to("cuda")  # column-major storage as (cols, rows)
    db = torch.from_numpy(np.ascontiguousarray(b.T)).to("cuda")
    dc = torch.full((n, m), complex("nan"), dtype=tdt, device="cuda")
    assert mb.gemm("N", "N", m, n, k, 1.0, da, m, db, k, 0.0, dc, m, mode=mode, slices=7) == 0
    got = dc.cpu().numpy().T
    ref = a.astype(np.complex128) @ b.astype(np.complex128)
    err = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
    assert np.all(np.isfinite(got)) and err < tol(dt, mode, k), err


def test_complex_gemm_quick_returns_and_info(capsys):
    rng = np.random.default_rng(42)
    a, b = crand(rng, (8, 8), np.complex128), crand(rng, (8, 8), np.complex128)
    c0 = crand(rng, (8, 8), np.complex128)
    c = c0.copy(order="F")
    assert mb.gemm("N", "N", 8, 8, 8, 0.0, a, 8, b, 8, 2j, c, 8) == 0  # alpha = 0: C := beta C
    np.testing.assert_allclose(c, 2j * c0, rtol=0, atol=0)
    c = c0.copy(order="F")
    assert mb.gemm("N", "N", 0, 8, 8, 1.0, a, 8, b, 8, 2j, c, 8) == 0  # m = 0: nothing touched
    np.testing.assert_array_equal(c, c0)
    assert mb.gemm("X", "N", 8, 8, 8, 1.0, a, 8, b, 8, 0.0, c, 8) == 1
    assert mb.gemm("N", "C", 8, 8, 8, 1.0, a, 8, b, 7, 0.0, c, 8) == 10
    assert "gemm: Info 10" in capsys.readouterr().out
