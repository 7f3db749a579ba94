"""Pageable host operands with odd leading dimensions, through the page-locked
bounce-buffer staging (several 32 MiB chunks per operand here).

A caller of the reference passes plain host allocations (BLASPtr); the library
copies them through a ring of page-locked buffers, packed and unpacked by host
threads while the DMAs of the neighbouring chunks run.  Results must equal the
same call on device pointers bit for bit (the kernels see the same operands),
and the padding rows between m and ld must come back untouched, both on the
pipelined gemm path (large calls, C returned block by block by a helper
thread) and on the plain staging path (trsm, smaller gemm).
"""
import numpy as np
import pytest

from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = need_gpu()
    return torch, L.load()


def dev_copy(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x.T)).to("cuda")  # column-major storage as (cols, rows)


@pytest.mark.parametrize("m,n,k,pipelined", [(1024, 4100, 4096, True), (1500, 1300, 2100, False)])
@pytest.mark.parametrize("beta", [0.0, 0.75])
def test_pageable_gemm_odd_ld(env, m, n, k, pipelined, beta):
    torch, lib = env
    rng = np.random.default_rng(51)
    lda, ldb, ldc = m + 3, k + 5, m + 7
    a = np.asfortranarray(rng.uniform(-1, 1, (lda, k)).astype(np.float32))
    b = np.asfortranarray(rng.uniform(-1, 1, (ldb, n)).astype(np.float32))
    c0 = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)).astype(np.float32))
    da, db, dc = dev_copy(torch, a), dev_copy(torch, b), dev_copy(torch, c0)
    args = (L.MODE_BF16X6, b"N", b"N", m, n, k, 1.25)
    assert lib.mbg_sgemm_ex(*args, da.data_ptr(), lda, db.data_ptr(), ldb, beta, dc.data_ptr(), ldc) == 0
    torch.cuda.synchronize()
    want = dc.cpu().numpy().T
    c = c0.copy(order="F")
    assert lib.mbg_sgemm_ex(*args, a.ctypes.data, lda, b.ctypes.data, ldb, beta, c.ctypes.data, ldc) == 0, \
        L.last_error()
    np.testing.assert_array_equal(c[:m], want[:m])
    np.testing.assert_array_equal(c[m:], c0[m:])  # padding rows untouched


def test_pageable_trsm_odd_ld_multi_chunk(env):
    torch, lib = env
    rng = np.random.default_rng(52)
    m, n = 3000, 3000  # B is 72 MB of float64: three bounce-buffer chunks each way
    lda, ldb = m + 1, m + 3
    a = rng.standard_normal((lda, m)) / np.sqrt(m)
    a[np.arange(m), np.arange(m)] = m + np.abs(rng.standard_normal(m))
    a = np.asfortranarray(a)
    b0 = np.asfortranarray(rng.standard_normal((ldb, n)))
    da, db = dev_copy(torch, a), dev_copy(torch, b0)
    args = (L.MODE_OZAKI, 7, 0, b"L", b"L", b"N", b"N", m, n, 1.0)
    assert lib.mbg_dtrsm_ex(*args, da.data_ptr(), lda, db.data_ptr(), ldb) == 0
    torch.cuda.synchronize()
    want = db.cpu().numpy().T
    b = b0.copy(order="F")
    assert lib.mbg_dtrsm_ex(*args, a.ctypes.data, lda, b.ctypes.data, ldb) == 0, L.last_error()
    np.testing.assert_array_equal(b[:m], want[:m])
    np.testing.assert_array_equal(b[m:], b0[m:])
