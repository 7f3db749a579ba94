"""Large gemm calls with host operands take the pipelined host path: C is cut into
column blocks whose host <-> device copies overlap the arithmetic of the others.
Every element is computed by the same kernel arithmetic as in a call on device
pointers (the blocks start at multiples of 256 columns, and each element's sum
does not depend on the blocking), so the results must be bit-identical to the
device-pointer call, for pageable and pinned host memory, every precision mode,
and beta == 0 (C not read) or beta != 0 (C copied in block by block).
"""
import numpy as np
import pytest

from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu

M, N, K = 1024, 4100, 4096  # m n k >= 2^34 and n >= 4096: the pipelined path; 4100 leaves a ragged block


@pytest.fixture(scope="module")
def env():
    torch = need_gpu()
    return torch, L.load()


@pytest.mark.parametrize("dt,mode", [(np.float32, L.MODE_PLAIN), (np.float32, L.MODE_BF16X6),
                                     (np.float64, L.MODE_PLAIN), (np.float64, L.MODE_OZAKI)],
                         ids=["f32-plain", "f32-bf16x6", "f64-plain", "f64-ozaki"])
@pytest.mark.parametrize("ta,tb", [("N", "N"), ("N", "T"), ("T", "N")])
@pytest.mark.parametrize("beta", [0.0, 0.5])
@pytest.mark.parametrize("memory", ["pageable", "pinned"])
def test_pipelined_host_gemm_matches_device_call(env, dt, mode, ta, tb, beta, memory):
    torch, lib = env
    rng = np.random.default_rng(17)
    ar, ac = (M, K) if ta == "N" else (K, M)
    br, bc = (K, N) if tb == "N" else (N, K)
    a = np.asfortranarray(rng.uniform(-1, 1, (ar, ac)).astype(dt))
    b = np.asfortranarray(rng.uniform(-1, 1, (br, bc)).astype(dt))
    c0 = np.asfortranarray(rng.uniform(-1, 1, (M, N)).astype(dt))

    def call(pa, pb, pc):
        if dt == np.float32:
            return lib.mbg_sgemm_ex(mode, ta.encode(), tb.encode(), M, N, K, 1.5, pa, ar, pb, br, beta, pc, M)
        return lib.mbg_dgemm_ex(mode, 8, ta.encode(), tb.encode(), M, N, K, 1.5, pa, ar, pb, br, beta, pc, M)

    # reference: the same call on device pointers (one launch over all of C)
    da = torch.from_numpy(a.T.copy()).to("cuda")  # column-major storage as (cols, rows) row-major
    db = torch.from_numpy(b.T.copy()).to("cuda")
    dc = torch.from_numpy(c0.T.copy()).to("cuda")
    assert call(da.data_ptr(), db.data_ptr(), dc.data_ptr()) == 0, L.last_error()
    torch.cuda.synchronize()
    want = dc.cpu().numpy().T

    if memory == "pageable":
        ha, hb, hc = a.copy(order="F"), b.copy(order="F"), c0.copy(order="F")
        st = call(ha.ctypes.data, hb.ctypes.data, hc.ctypes.data)
        got = hc
    else:
        ta_ = torch.from_numpy(a.T.copy()).pin_memory()
        tb_ = torch.from_numpy(b.T.copy()).pin_memory()
        tc_ = torch.from_numpy(c0.T.copy()).pin_memory()
        st = call(ta_.data_ptr(), tb_.data_ptr(), tc_.data_ptr())
        got = tc_.numpy().T
    assert st == 0, L.last_error()
    np.testing.assert_array_equal(got, want)
