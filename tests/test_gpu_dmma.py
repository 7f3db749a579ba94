"""Copy paths of the plain GEMM kernels: FP64 on the tensor pipe (gemm_dmma_kernel) and
FP32 128-tiles on the CUDA cores (gemm_f32_kernel).

Operands that are 16-byte aligned with even leading dimensions are staged 16
bytes at a time (pairs along the contiguous index, the last pair of a ragged
edge half zero-filled); any other operand element by element.  Device buffers
with chosen leading dimensions and base offsets reach each path; ragged m, n, k
reach the edges.  Checked against float64 numpy within the plain FP64
tolerance 4e-16 sqrt(k) (normwise max relative error), with alpha/beta as the
reference's gemm applies them (src/level3/gemm.mojo:56-377).
"""
import numpy as np
import pytest

from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    torch = need_gpu()
    lib = L.load()
    assert lib.mbg_get_tuning(b"plain_fp64_simt") == 0
    return torch, lib


def dev_matrix(torch, host, ld, offset):
    """Column-major device copy of `host` with leading dimension ld, starting `offset` doubles in."""
    rows, cols = host.shape
    buf = torch.full((offset + ld * cols + 2,), float("nan"), dtype=torch.float64, device="cuda")
    view = buf[offset:offset + ld * cols].view(cols, ld)
    view[:, :rows] = torch.from_numpy(np.ascontiguousarray(host.T))
    return buf, view


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("m,n,k", [(130, 70, 45), (129, 67, 33), (300, 520, 257), (64, 64, 64)])
@pytest.mark.parametrize("path", ["vec16", "odd_ld", "offset"])
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.5])
def test_dgemm_tensor_pipe(env, ta, tb, m, n, k, path, beta):
    torch, lib = env
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    a = rng.uniform(-1, 1, (ar, ac))
    b = rng.uniform(-1, 1, (br, bc))
    c = rng.uniform(-1, 1, (m, n))
    pad = {"vec16": (2 - ar % 2) % 2, "odd_ld": 1 - ar % 2, "offset": (2 - ar % 2) % 2}[path]
    padb = {"vec16": (2 - br % 2) % 2, "odd_ld": 1 - br % 2, "offset": (2 - br % 2) % 2}[path]
    off = 1 if path == "offset" else 0
    lda, ldb, ldc = ar + pad, br + padb, m + 1
    abuf, _ = dev_matrix(torch, a, lda, off)
    bbuf, _ = dev_matrix(torch, b, ldb, off)
    cbuf, cview = dev_matrix(torch, c, ldc, 0)
    alpha = 1.25
    st = lib.mbg_dgemm(ta.encode(), tb.encode(), m, n, k, alpha, abuf.data_ptr() + 8 * off, lda,
                       bbuf.data_ptr() + 8 * off, ldb, beta, cbuf.data_ptr(), ldc)
    assert st == 0, L.last_error()
    torch.cuda.synchronize()
    got = cview[:, :m].T.cpu().numpy()
    opa = a if ta == "N" else a.T
    opb = b if tb == "N" else b.T
    ref = alpha * (opa @ opb) + beta * c
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < 4e-16 * np.sqrt(max(k, 16)) * 4
    # the padding rows of C are untouched
    assert torch.isnan(cview[:, m:]).all()


def test_dsyrk_tensor_pipe_triangle(env):
    """dsyrk through the triangular tile schedule: one triangle written, the other untouched."""
    torch, lib = env
    rng = np.random.default_rng(5)
    n, k = 300, 130
    a = rng.uniform(-1, 1, (n, k))
    c = rng.uniform(-1, 1, (n, n))
    abuf, _ = dev_matrix(torch, a, n, 0)
    cbuf, cview = dev_matrix(torch, c, n, 0)
    assert lib.mbg_dsyrk(b"L", b"N", n, k, 0.5, abuf.data_ptr(), n, 2.0, cbuf.data_ptr(), n) == 0
    torch.cuda.synchronize()
    got = cview.T.cpu().numpy()
    ref = 0.5 * a @ a.T + 2.0 * c
    low = np.tril(np.ones((n, n), bool))
    assert np.max(np.abs(got[low] - ref[low])) / np.max(np.abs(ref[low])) < 4e-16 * np.sqrt(k) * 4
    np.testing.assert_array_equal(got[~low], c[~low])


@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N"), ("T", "T")])
@pytest.mark.parametrize("m,n,k", [(2200, 2180, 33), (2304, 2304, 64), (2177, 2201, 130), (300, 521, 257)])
@pytest.mark.parametrize("path", ["vec16", "odd_ld", "offset"])
@pytest.mark.parametrize("beta", [0.0, 1.0, 0.5])
def test_sgemm_pipelined_copy_paths(env, ta, tb, m, n, k, path, beta):
    """Plain FP32 128-tiles (cp.async pipeline): 16-byte copies need an operand contiguous along
    m (n), a 16-byte aligned base and ld % 4 == 0; every other operand is copied element-wise.
    Three sizes give at least two waves of 128 x 128 tiles, the last one the 64 x 64 tiles of
    smaller launches, all with ragged edges in m, n and k; tolerance 1e-6 sqrt(k)."""
    torch, lib = env
    rng = np.random.default_rng(m + 5 * n + 11 * k)
    ar, ac = (m, k) if ta == "N" else (k, m)
    br, bc = (k, n) if tb == "N" else (n, k)
    a = rng.uniform(-1, 1, (ar, ac)).astype(np.float32)
    b = rng.uniform(-1, 1, (br, bc)).astype(np.float32)
    c = rng.uniform(-1, 1, (m, n)).astype(np.float32)

    def ld_for(rows):
        return {"vec16": -(-rows // 4) * 4, "odd_ld": rows + (1 - rows % 2), "offset": -(-rows // 4) * 4}[path]

    off = 1 if path == "offset" else 0
    lda, ldb, ldc = ld_for(ar), ld_for(br), m + 3

    def dev(host, ld, o):
        rows, cols = host.shape
        buf = torch.full((o + ld * cols + 4,), float("nan"), dtype=torch.float32, device="cuda")
        view = buf[o:o + ld * cols].view(cols, ld)
        view[:, :rows] = torch.from_numpy(np.ascontiguousarray(host.T))
        return buf, view

    abuf, _ = dev(a, lda, off)
    bbuf, _ = dev(b, ldb, off)
    cbuf, cview = dev(c, ldc, 0)
    assert lib.mbg_set_tuning(b"plain_fp32_staged", 0) == 0
    st = lib.mbg_sgemm(ta.encode(), tb.encode(), m, n, k, 0.75, abuf.data_ptr() + 4 * off, lda,
                       bbuf.data_ptr() + 4 * off, ldb, beta, cbuf.data_ptr(), ldc)
    assert st == 0, L.last_error()
    torch.cuda.synchronize()
    got = cview[:, :m].T.cpu().numpy().astype(np.float64)
    opa = (a if ta == "N" else a.T).astype(np.float64)
    opb = (b if tb == "N" else b.T).astype(np.float64)
    ref = 0.75 * (opa @ opb) + beta * c.astype(np.float64)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < 1e-6 * np.sqrt(max(k, 16)) * 4
    assert torch.isnan(cview[:, m:]).all()
