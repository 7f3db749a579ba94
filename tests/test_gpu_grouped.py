"""Grouped (batched) sgemm / strsm plans against the float64 oracle and the
reference's algorithms, problem by problem.

Tolerance: TOL32(k) = 1e-6 * sqrt(max(k, 16)) normwise per problem, as for the
single-problem plain kernels; trsm uses 4 * TOL32(n).  Each plan is executed
twice (graph replay) and both results are checked.
"""
import ctypes as C

import numpy as np
import pytest

import mojoblas_b200 as mb
from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu

pytestmark = pytest.mark.gpu


def tol32(k):
    return 1e-6 * np.sqrt(max(k, 16))


def log_uniform(rng, lo, hi, size):
    return np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), size))).astype(int)


class DeviceArena:
    """Column-major matrices carved out of one device buffer."""

    def __init__(self, torch, arrays):
        self.torch = torch
        offs, total = [], 0
        for a in arrays:
            offs.append(total)
            total += (a.size + 63) // 64 * 64
        host = np.zeros(max(total, 1), np.float32)
        for a, o in zip(arrays, offs):
            host[o:o + a.size] = a.reshape(-1, order="F")
        self.host = host
        self.buf = torch.from_numpy(host).cuda()
        self.offs = offs
        self.base = self.buf.data_ptr()

    def ptr(self, i):
        return self.base + 4 * self.offs[i]

    def get(self, i, shape):
        n = shape[0] * shape[1]
        flat = self.buf[self.offs[i]:self.offs[i] + n].cpu().numpy()
        return flat.reshape(shape, order="F")


def test_grouped_sgemm_uneven_batch(oracle):
    torch = need_gpu()
    lib = L.load()
    rng = np.random.default_rng(21)
    count = 300
    ms, ns, ks = (log_uniform(rng, 16, 300, count) for _ in range(3))
    ks[:5] = 0          # k == 0: C := beta*C
    ms[5] = 1
    tas = rng.choice(list("NT"), count)
    tbs = rng.choice(list("NT"), count)
    alphas = rng.uniform(-2, 2, count).astype(np.float32)
    alphas[6] = 0.0     # alpha == 0
    betas = np.where(rng.random(count) < 0.5, 0.0, rng.uniform(-1, 1, count)).astype(np.float32)
    arrays, meta = [], []
    for i in range(count):
        m, n, k, ta, tb = ms[i], ns[i], ks[i], tas[i], tbs[i]
        a = rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)).astype(np.float32)
        b = rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)).astype(np.float32)
        c = rng.uniform(-1, 1, (m, n)).astype(np.float32)
        arrays += [np.asfortranarray(a), np.asfortranarray(b), np.asfortranarray(c)]
        meta.append((m, n, k, ta, tb, a.shape[0], b.shape[0]))
    arena = DeviceArena(torch, arrays)
    probs = (L.SgemmProblem * count)()
    for i, (m, n, k, ta, tb, lda, ldb) in enumerate(meta):
        probs[i] = L.SgemmProblem(ta.encode(), tb.encode(), m, n, k, float(alphas[i]), float(betas[i]),
                                  arena.ptr(3 * i), max(lda, 1), arena.ptr(3 * i + 1), max(ldb, 1),
                                  arena.ptr(3 * i + 2), m)
    plan = C.c_void_p()
    assert lib.mbg_sgemm_grouped_plan(L.MODE_PLAIN, count, probs, C.byref(plan)) == 0, L.last_error()
    try:
        for rep in range(2):
            if rep == 1:  # restore C and replay the same graph
                arena.buf.copy_(torch.from_numpy(arena.host).cuda())
            assert lib.mbg_plan_execute(plan) == 0, L.last_error()
            torch.cuda.synchronize()
            for i, (m, n, k, ta, tb, lda, ldb) in enumerate(meta):
                a, b, c = arrays[3 * i], arrays[3 * i + 1], arrays[3 * i + 2]
                got = arena.get(3 * i + 2, (m, n))
                ref = oracle.gemm_f64(ta, tb, m, n, k, alphas[i], a, max(lda, 1), b, max(ldb, 1), betas[i], c, m)
                c_orc = c.copy(order="F")
                oracle.gemm(ta, tb, m, n, k, alphas[i], a, max(lda, 1), b, max(ldb, 1), betas[i], c_orc, m)
                assert oracle.max_rel_err(got, ref) < tol32(k), (i, m, n, k, ta, tb)
                assert oracle.max_rel_err(got, c_orc.astype(np.float64)) < 2 * tol32(k), i
    finally:
        lib.mbg_plan_destroy(plan)


def test_grouped_strsm_uneven_batch(oracle):
    torch = need_gpu()
    lib = L.load()
    rng = np.random.default_rng(22)
    count = 200
    ns = log_uniform(rng, 8, 256, count)
    nrhs = rng.integers(1, 65, count)
    uplos = rng.choice(list("LU"), count)
    transes = rng.choice(list("NT"), count)
    diags = rng.choice(list("NU"), count)
    alphas = rng.uniform(0.5, 2, count).astype(np.float32)
    arrays = []
    for i in range(count):
        n = ns[i]
        a = rng.standard_normal((n, n)) / np.sqrt(n)
        a[np.arange(n), np.arange(n)] = n + np.abs(rng.standard_normal(n))
        if diags[i] == "U":
            a = a / n
        junk = np.triu(np.ones((n, n), bool), 1) if uplos[i] == "L" else np.tril(np.ones((n, n), bool), -1)
        a[junk] = 1e30  # never read
        arrays += [np.asfortranarray(a.astype(np.float32)),
                   np.asfortranarray(rng.standard_normal((n, nrhs[i])).astype(np.float32))]
    arena = DeviceArena(torch, arrays)
    probs = (L.StrsmProblem * count)()
    for i in range(count):
        probs[i] = L.StrsmProblem(b"L", uplos[i].encode(), transes[i].encode(), diags[i].encode(), int(ns[i]),
                                  int(nrhs[i]), float(alphas[i]), arena.ptr(2 * i), int(ns[i]),
                                  arena.ptr(2 * i + 1), int(ns[i]))
    plan = C.c_void_p()
    assert lib.mbg_strsm_grouped_plan(L.MODE_PLAIN, count, probs, C.byref(plan)) == 0, L.last_error()
    try:
        assert lib.mbg_plan_execute(plan) == 0, L.last_error()
        torch.cuda.synchronize()
        for i in range(count):
            n, r = int(ns[i]), int(nrhs[i])
            a, b = arrays[2 * i], arrays[2 * i + 1]
            got = arena.get(2 * i + 1, (n, r))
            ref = oracle.trsm_f64("L", uplos[i], transes[i], diags[i], n, r, alphas[i],
                                  np.where(np.abs(a) > 1e29, 0, a).astype(np.float32), n, b, n)
            x_orc = b.copy(order="F")
            oracle.trsm("L", uplos[i], transes[i], diags[i], n, r, alphas[i], a, n, x_orc, n)
            assert oracle.max_rel_err(got, ref) < 4 * tol32(n), (i, n, r, uplos[i], transes[i], diags[i])
            assert oracle.max_rel_err(got, x_orc.astype(np.float64)) < 8 * tol32(n), i
    finally:
        lib.mbg_plan_destroy(plan)


def test_grouped_invalid_problem_reports_info():
    torch = need_gpu()
    lib = L.load()
    buf = torch.zeros(64, device="cuda")
    probs = (L.SgemmProblem * 2)()
    probs[0] = L.SgemmProblem(b"N", b"N", 4, 4, 4, 1.0, 0.0, buf.data_ptr(), 4, buf.data_ptr(), 4, buf.data_ptr(), 4)
    probs[1] = L.SgemmProblem(b"N", b"N", 4, 4, 4, 1.0, 0.0, buf.data_ptr(), 3, buf.data_ptr(), 4, buf.data_ptr(), 4)
    plan = C.c_void_p()
    assert lib.mbg_sgemm_grouped_plan(L.MODE_PLAIN, 2, probs, C.byref(plan)) == 8
    assert "problem 1" in L.last_error()
    h = np.zeros(16, np.float32)
    probs[1] = L.SgemmProblem(b"N", b"N", 4, 4, 4, 1.0, 0.0, h.ctypes.data, 4, buf.data_ptr(), 4, buf.data_ptr(), 4)
    assert lib.mbg_sgemm_grouped_plan(L.MODE_PLAIN, 2, probs, C.byref(plan)) == L.MBG_ERR_UNSUPPORTED
    tp = (L.StrsmProblem * 1)()
    tp[0] = L.StrsmProblem(b"R", b"L", b"N", b"N", 4, 4, 1.0, buf.data_ptr(), 4, buf.data_ptr(), 4)
    assert lib.mbg_strsm_grouped_plan(L.MODE_PLAIN, 1, tp, C.byref(plan)) == L.MBG_ERR_UNSUPPORTED
    assert lib.mbg_sgemm_grouped(L.MODE_PLAIN, 0, None) == 0
