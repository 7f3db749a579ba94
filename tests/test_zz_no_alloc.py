"""mbg_sgemm_ex_noalloc: the split-precision sgemm for callers that cannot let a
library allocate device memory (a host framework that owns a fixed device-memory
budget, a latency-critical loop where cudaMalloc / cudaFree may synchronise the
device, or code inside an allocator's out-of-memory handling).

Its result must equal the allocating entry point mbg_sgemm_ex's bit for bit
with the same mode on the same device inputs (the same pre-pass and tcgen05
kernels run on the same planes, only the planes' address differs), and stay
within the float32 tolerance of the other GPU tests against a float64 product,
on two calls in a row (the second reuses the fixed scratch array the first one
filled).  This file is collected last on purpose.

The device-memory check covers the library's own allocations.  The first launch
of a kernel in a process makes CUDA's lazy module loading map that kernel's code
(2 MiB was measured when the wide split kernel first ran inside the measured
call).  A small warm-up call in each mode therefore runs before the measured
calls, as a caller that must see no device-memory change would make one (or set
CUDA_MODULE_LOADING=EAGER).
"""
import ctypes as C

import numpy as np
import pytest

from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu


def tol32(k):
    return 1e-6 * np.sqrt(max(k, 16))  # the float32 tolerance of the GPU parity tests


def _col_major(torch, rows, cols, seed):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.rand((cols, rows), generator=g, device="cuda", dtype=torch.float32) * 2 - 1


def _call(fn, mode, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc):
    return fn(mode, ta.encode(), tb.encode(), m, n, k, alpha, a.data_ptr(), lda, b.data_ptr(), ldb, beta,
              c.data_ptr(), ldc)


def test_noalloc_matches_allocating_entry_point_twice():
    torch = need_gpu()
    lib = L.load()
    lib.mbg_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))
    for mode in (L.MODE_BF16X3, L.MODE_BF16X6):  # warm-up: the kernels' code loaded
        w = _col_major(torch, 64, 64, 1)
        cw = w.clone()
        assert _call(lib.mbg_sgemm_ex_noalloc, mode, "N", "N", 64, 64, 64, 1.0, w, 64, w, 64, 0.0, cw, 64) == 0, \
            L.last_error()
    torch.cuda.synchronize()
    cases = [  # two calls in a row, different shapes, modes and transposes
        (L.MODE_BF16X3, "N", "T", 1000, 700, 900, 1.5, 0.5),
        (L.MODE_BF16X6, "T", "N", 513, 1024, 2048, -1.0, 0.0),
    ]
    for i, (mode, ta, tb, m, n, k, alpha, beta) in enumerate(cases):
        lda = m if ta == "N" else k
        ldb = k if tb == "N" else n
        a = _col_major(torch, lda, k if ta == "N" else m, 10 + i)
        b = _col_major(torch, ldb, n if tb == "N" else k, 20 + i)
        c0 = _col_major(torch, m, n, 30 + i)
        c_ref, c_new = c0.clone(), c0.clone()
        st = _call(lib.mbg_sgemm_ex, mode, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c_ref, m)
        assert st == 0, L.last_error()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        st = _call(lib.mbg_sgemm_ex_noalloc, mode, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, c_new, m)
        assert st == 0, L.last_error()
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        assert free_before - free_after < (2 << 20), "the no-allocation entry point allocated device memory"
        assert torch.equal(c_new, c_ref), (i, float((c_new - c_ref).abs().max()))
        # and within the float32 tolerance of the float64 product
        A = a.double().T[:m, :k] if ta == "N" else a.double().T[:k, :m].T
        B = b.double().T[:k, :n] if tb == "N" else b.double().T[:n, :k].T
        ref = alpha * (A @ B) + beta * c0.double().T
        diff = float((c_new.double().T - ref).abs().max() / ref.abs().max())
        assert diff <= tol32(k), (i, diff)


def test_noalloc_wait_flag_reported_once_in_async_mode():
    """An expired wait in the no-allocation kernels (planted in the flag from the
    host; no kernel is made to wait) is reported by the next mbg_synchronize() as
    MBG_ERR_TIMEOUT exactly once, then cleared."""
    torch = need_gpu()
    lib = L.load()
    lib.mbg_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))
    lib.mbg_set_sync(0)
    try:
        assert lib.mbg_synchronize() == 0
        assert lib.mbg_debug_set_noalloc_error(1) == 0
        assert lib.mbg_synchronize() == L.MBG_ERR_TIMEOUT
        assert "site 77" in L.last_error()
        assert lib.mbg_synchronize() == 0
    finally:
        lib.mbg_set_sync(1)
    # synchronous mode: the next call itself reports it, and only once
    n = 64
    a = torch.ones((n, n), device="cuda", dtype=torch.float32)
    c = torch.zeros_like(a)
    assert lib.mbg_debug_set_noalloc_error(1) == 0
    st = _call(lib.mbg_sgemm_ex_noalloc, L.MODE_BF16X3, "N", "N", n, n, n, 1.0, a, n, a, n, 0.0, c, n)
    assert st == L.MBG_ERR_TIMEOUT
    st = _call(lib.mbg_sgemm_ex_noalloc, L.MODE_BF16X3, "N", "N", n, n, n, 1.0, a, n, a, n, 0.0, c, n)
    assert st == 0 and float(c[0, 0]) == n


def test_noalloc_rejects_oversized_and_host_operands():
    torch = need_gpu()
    lib = L.load()
    n = 4096  # BF16x3 needs 2 * (4096 + 4096) * 4096 * 2 bytes = 128 MiB > 32 MiB
    a = torch.zeros((n, n), device="cuda", dtype=torch.float32)
    st = _call(lib.mbg_sgemm_ex_noalloc, L.MODE_BF16X3, "N", "N", n, n, n, 1.0, a, n, a, n, 0.0, a, n)
    assert st == L.MBG_ERR_SCRATCH_LIMIT
    assert "limit" in L.last_error()
    h = np.zeros((64, 64), np.float32, order="F")
    st = lib.mbg_sgemm_ex_noalloc(L.MODE_BF16X3, b"N", b"N", 64, 64, 64, 1.0, h.ctypes.data, 64,
                                  h.ctypes.data, 64, 0.0, h.ctypes.data, 64)
    assert st == L.MBG_ERR_UNSUPPORTED
    st = lib.mbg_sgemm_ex_noalloc(L.MODE_PLAIN, b"N", b"N", 64, 64, 64, 1.0, h.ctypes.data, 64,
                                  h.ctypes.data, 64, 0.0, h.ctypes.data, 64)
    assert st == L.MBG_ERR_INVALID_MODE
    assert lib.mbg_sgemm_ex_noalloc(L.MODE_BF16X3, b"N", b"N", 64, 64, 64, 1.0, h.ctypes.data, 63,
                                    h.ctypes.data, 64, 0.0, h.ctypes.data, 64) == 8
