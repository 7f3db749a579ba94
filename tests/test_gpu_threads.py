"""Calls from two host threads, each on its own stream (mbg_set_thread_stream).

Each thread runs a loop of device-pointer calls (BF16x6 sgemm, Ozaki dgemm,
blocked dtrsm) on its own operands and stream while the other thread does the
same; ctypes releases the interpreter lock for the duration of each foreign
call, so the two threads' calls really overlap on the host and the GPU.  The
library's kernels are deterministic, so every result must equal, bit for bit,
the result of the same call made alone from one thread beforehand; and the
workspace pools are per stream, so the two threads never share a block that
is still in use.
"""
import ctypes as C
import threading

import pytest

from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu


def _col(torch, rows, cols, seed, dtype):
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.rand((cols, rows), generator=g, device="cuda", dtype=dtype) * 2 - 1


def _problem(torch, seed):
    """Operands of one thread: sgemm NT 768 x 640 x 1024, dgemm NN 512^3, dtrsm L/L/N/N 640 x 300."""
    p = {"a": _col(torch, 768, 1024, seed, torch.float32), "b": _col(torch, 640, 1024, seed + 1, torch.float32),
         "c": torch.empty((640, 768), device="cuda", dtype=torch.float32),
         "da": _col(torch, 512, 512, seed + 2, torch.float64), "db": _col(torch, 512, 512, seed + 3, torch.float64),
         "dc": torch.empty((512, 512), device="cuda", dtype=torch.float64),
         "ta": _col(torch, 640, 640, seed + 4, torch.float64) / 640, "tb0": _col(torch, 640, 300, seed + 5,
                                                                                    torch.float64)}
    p["ta"].diagonal().add_(640.0)  # column-major storage: the diagonal is the tensor's diagonal
    p["tb"] = torch.empty_like(p["tb0"])
    return p


def _run(lib, p):
    """One round of the three calls; returns the statuses."""
    st = [lib.mbg_sgemm_ex(L.MODE_BF16X6, b"N", b"T", 768, 640, 1024, 1.0, p["a"].data_ptr(), 768,
                           p["b"].data_ptr(), 640, 0.0, p["c"].data_ptr(), 768),
          lib.mbg_dgemm_ex(L.MODE_OZAKI, 7, b"N", b"N", 512, 512, 512, 1.0, p["da"].data_ptr(), 512,
                           p["db"].data_ptr(), 512, 0.0, p["dc"].data_ptr(), 512)]
    p["tb"].copy_(p["tb0"])
    st.append(lib.mbg_dtrsm_ex(L.MODE_OZAKI, 7, 0, b"L", b"L", b"N", b"N", 640, 300, 1.0, p["ta"].data_ptr(), 640,
                               p["tb"].data_ptr(), 640))
    return st


def test_two_host_threads_on_two_streams():
    torch = need_gpu()
    lib = L.load()
    probs = [_problem(torch, 100), _problem(torch, 200)]
    expect = []
    for p in probs:  # each problem alone, from this thread, on the default stream
        assert _run(lib, p) == [0, 0, 0], L.last_error()
        torch.cuda.synchronize()
        expect.append({k: p[k].clone() for k in ("c", "dc", "tb")})
    errors = []
    barrier = threading.Barrier(2)

    def worker(i):
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                lib.mbg_set_thread_stream(1, C.c_void_p(s.cuda_stream))
                lib.mbg_set_sync(1)
                barrier.wait()
                for it in range(12):
                    for k in ("c", "dc"):
                        probs[i][k].fill_(float("nan"))
                    st = _run(lib, probs[i])
                    if st != [0, 0, 0]:
                        errors.append((i, it, st, L.last_error()))
                        return
                    s.synchronize()
                    for k, v in expect[i].items():
                        if not torch.equal(probs[i][k], v):
                            errors.append((i, it, k, float((probs[i][k] - v).abs().max())))
                            return
                assert lib.mbg_get_stream() == s.cuda_stream
                lib.mbg_set_thread_stream(0, None)
        except Exception as e:  # reported below, from the main thread
            errors.append((i, repr(e)))

    threads = [threading.Thread(target=worker, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
