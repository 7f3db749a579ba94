"""Grouped plans at the batched configuration's full counts, every problem checked.

4096 independent sgemm problems (m, n, k each log-uniform over 16..512, entries
uniform[-1, 1), mixed transposes, alpha and beta drawn per problem) in the plain
(FP32 CUDA cores) and the split (BF16x6 / BF16x3, tensor cores) forms, and 2048
lower-triangular strsm problems (n log-uniform 8..256, nrhs uniform 1..64,
diagonally dominant A): every result against the float64 product / solve of the
same inputs (normwise per problem: TOL32(k) = 1e-6 sqrt(max(k, 16)) for plain and
BF16x6, TOL_X3 = 1.5e-5 for BF16x3, 4 TOL32(n) for the solves).  The split plan is
replayed twice from its CUDA graph.  A per-class tile entry of the tuning table
(the split form's 64-column tiles for a class that defaults to 128) is checked to
take effect without changing the results beyond the tolerance.
"""
import ctypes as C

import numpy as np
import pytest

from mojoblas_b200 import _lib as L
from tests.gpu_util import need_gpu
from tests.test_gpu_grouped import DeviceArena, log_uniform

pytestmark = pytest.mark.gpu

TOL_X3 = 1.5e-5


def tol32(k):
    return 1e-6 * np.sqrt(max(k, 16))


def sgemm_batch(rng, count):
    ms, ns, ks = (log_uniform(rng, 16, 512, count) for _ in range(3))
    tas, tbs = rng.choice(list("NT"), count), rng.choice(list("NT"), count)
    alphas = rng.uniform(-2, 2, count).astype(np.float32)
    betas = np.where(rng.random(count) < 0.5, 0.0, rng.uniform(-1, 1, count)).astype(np.float32)
    arrays, meta = [], []
    for i in range(count):
        m, n, k, ta, tb = int(ms[i]), int(ns[i]), int(ks[i]), tas[i], tbs[i]
        arrays += [np.asfortranarray(rng.uniform(-1, 1, (m, k) if ta == "N" else (k, m)).astype(np.float32)),
                   np.asfortranarray(rng.uniform(-1, 1, (k, n) if tb == "N" else (n, k)).astype(np.float32)),
                   np.asfortranarray(rng.uniform(-1, 1, (m, n)).astype(np.float32))]
        meta.append((m, n, k, ta, tb))
    return arrays, meta, alphas, betas


def run_sgemm_plan(torch, lib, mode, arrays, meta, alphas, betas, reps=1):
    count = len(meta)
    arena = DeviceArena(torch, arrays)
    probs = (L.SgemmProblem * count)()
    for i, (m, n, k, ta, tb) in enumerate(meta):
        probs[i] = L.SgemmProblem(ta.encode(), tb.encode(), m, n, k, float(alphas[i]), float(betas[i]),
                                  arena.ptr(3 * i), arrays[3 * i].shape[0], arena.ptr(3 * i + 1),
                                  arrays[3 * i + 1].shape[0], arena.ptr(3 * i + 2), m)
    plan = C.c_void_p()
    assert lib.mbg_sgemm_grouped_plan(mode, count, probs, C.byref(plan)) == 0, L.last_error()
    outs = []
    try:
        for rep in range(reps):
            if rep:
                arena.buf.copy_(torch.from_numpy(arena.host).cuda())
            assert lib.mbg_plan_execute(plan) == 0, L.last_error()
            torch.cuda.synchronize()
            outs.append([arena.get(3 * i + 2, (m, n)) for i, (m, n, k, ta, tb) in enumerate(meta)])
    finally:
        lib.mbg_plan_destroy(plan)
    return outs


def check_sgemm(outs, arrays, meta, alphas, betas, tol):
    worst = 0.0
    for got_all in outs:
        for i, (m, n, k, ta, tb) in enumerate(meta):
            a, b, c = (x.astype(np.float64) for x in arrays[3 * i:3 * i + 3])
            ref = alphas[i] * ((a if ta == "N" else a.T) @ (b if tb == "N" else b.T)) + betas[i] * c
            err = float(np.max(np.abs(got_all[i] - ref)) / max(np.max(np.abs(ref)), 1e-30))
            assert err < tol(k), (i, m, n, k, ta, tb, err)
            worst = max(worst, err / tol(k))
    return worst


@pytest.mark.parametrize("mode", [L.MODE_PLAIN, L.MODE_BF16X6, L.MODE_BF16X3], ids=["plain", "bf16x6", "bf16x3"])
def test_grouped_sgemm_full_count(mode):
    torch = need_gpu()
    lib = L.load()
    rng = np.random.default_rng(61)
    arrays, meta, alphas, betas = sgemm_batch(rng, 4096)
    outs = run_sgemm_plan(torch, lib, mode, arrays, meta, alphas, betas, reps=2 if mode != L.MODE_PLAIN else 1)
    tol = (lambda k: TOL_X3) if mode == L.MODE_BF16X3 else tol32
    check_sgemm(outs, arrays, meta, alphas, betas, tol)


def test_grouped_sgemm_tile_table_entry():
    torch = need_gpu()
    lib = L.load()
    rng = np.random.default_rng(62)
    arrays, meta, alphas, betas = sgemm_batch(rng, 300)
    keys = [f"grouped_tc_bn_{a}{b}_c{c}".encode() for a in "NT" for b in "NT" for c in range(5)]
    try:
        for key in keys:  # every class on 64-column tiles (the default is 128 above n = 64)
            assert lib.mbg_set_tuning(key, 64) == 0
            assert lib.mbg_get_tuning(key) == 64
        outs = run_sgemm_plan(torch, lib, L.MODE_BF16X6, arrays, meta, alphas, betas)
    finally:
        for key in keys:
            lib.mbg_set_tuning(key, 0)
    check_sgemm(outs, arrays, meta, alphas, betas, tol32)
    assert lib.mbg_set_tuning(b"grouped_tc_bn_NN_c5", 64) != 0  # no class 5
    assert lib.mbg_set_tuning(b"grouped_simt_tile_NT_c1", 96) != 0  # 64 or 128 only


def test_grouped_strsm_full_count():
    torch = need_gpu()
    lib = L.load()
    rng = np.random.default_rng(63)
    count = 2048
    ns = log_uniform(rng, 8, 256, count)
    nrhs = rng.integers(1, 65, count)
    arrays = []
    for i in range(count):
        n = int(ns[i])
        a = rng.standard_normal((n, n)) / np.sqrt(n)
        a[np.arange(n), np.arange(n)] = n + np.abs(rng.standard_normal(n))
        arrays += [np.asfortranarray(np.tril(a).astype(np.float32)),
                   np.asfortranarray(rng.standard_normal((n, int(nrhs[i]))).astype(np.float32))]
    arena = DeviceArena(torch, arrays)
    probs = (L.StrsmProblem * count)()
    for i in range(count):
        n = int(ns[i])
        probs[i] = L.StrsmProblem(b"L", b"L", b"N", b"N", n, int(nrhs[i]), 1.0, arena.ptr(2 * i), n,
                                  arena.ptr(2 * i + 1), n)
    plan = C.c_void_p()
    assert lib.mbg_strsm_grouped_plan(L.MODE_PLAIN, count, probs, C.byref(plan)) == 0, L.last_error()
    try:
        assert lib.mbg_plan_execute(plan) == 0, L.last_error()
        torch.cuda.synchronize()
    finally:
        lib.mbg_plan_destroy(plan)
    import scipy.linalg as sl
    for i in range(count):
        n, r = int(ns[i]), int(nrhs[i])
        a, b = arrays[2 * i].astype(np.float64), arrays[2 * i + 1].astype(np.float64)
        ref = sl.solve_triangular(a, b, lower=True)
        got = arena.get(2 * i + 1, (n, r))
        err = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
        assert err < 4 * tol32(n), (i, n, r, err)


@pytest.mark.parametrize("mode", [L.MODE_BF16X6, L.MODE_BF16X3], ids=["bf16x6", "bf16x3"])
def test_grouped_split_padded_and_misaligned(mode):
    """The split form's copy paths: leading dimensions past the stored rows (by 0..5
    floats, so some are multiples of four and some not), base addresses 0..3 floats
    past a 256-byte boundary (16-byte copies only where both allow), k not a multiple
    of the 32-deep slab (zero-filled tails), m and n not multiples of the tile (padding
    rows), both transposes.  The padding between the stored rows and ld must come back
    untouched in C."""
    torch = need_gpu()
    lib = L.load()
    rng = np.random.default_rng(77)
    count = 160
    dims = np.array([1, 3, 31, 32, 33, 63, 64, 65, 127, 128, 129, 200, 257, 300])
    meta, host_parts, offs, total = [], [], [], 0

    def place(x):
        nonlocal total
        start = (total + 63) // 64 * 64 + int(rng.integers(0, 4))  # 0..3 floats past a 256-byte boundary
        offs.append(start)
        host_parts.append((start, x))
        total = start + x.size

    for i in range(count):
        m, n, k = (int(v) for v in rng.choice(dims, 3))
        ta, tb = rng.choice(list("NT"), 2)
        ra, ca = (m, k) if ta == "N" else (k, m)
        rb, cb = (k, n) if tb == "N" else (n, k)
        lda, ldb, ldc = ra + int(rng.integers(0, 6)), rb + int(rng.integers(0, 6)), m + int(rng.integers(0, 6))
        a = np.asfortranarray(rng.uniform(-1, 1, (lda, ca)).astype(np.float32))
        b = np.asfortranarray(rng.uniform(-1, 1, (ldb, cb)).astype(np.float32))
        c = np.asfortranarray(rng.uniform(-1, 1, (ldc, n)).astype(np.float32))
        for x in (a, b, c):
            place(x.reshape(-1, order="F"))
        meta.append((m, n, k, ta, tb, lda, ldb, ldc, a, b, c, float(rng.uniform(-2, 2)),
                     float(rng.choice([0.0, 0.5]))))
    host = np.zeros(total + 64, np.float32)
    for start, x in host_parts:
        host[start:start + x.size] = x
    buf = torch.from_numpy(host).cuda()
    base = buf.data_ptr()
    probs = (L.SgemmProblem * count)()
    for i, (m, n, k, ta, tb, lda, ldb, ldc, a, b, c, al, be) in enumerate(meta):
        probs[i] = L.SgemmProblem(ta.encode(), tb.encode(), m, n, k, al, be, base + 4 * offs[3 * i], lda,
                                  base + 4 * offs[3 * i + 1], ldb, base + 4 * offs[3 * i + 2], ldc)
    plan = C.c_void_p()
    assert lib.mbg_sgemm_grouped_plan(mode, count, probs, C.byref(plan)) == 0, L.last_error()
    try:
        assert lib.mbg_plan_execute(plan) == 0, L.last_error()
        torch.cuda.synchronize()
    finally:
        lib.mbg_plan_destroy(plan)
    out = buf.cpu().numpy()
    tol = (lambda k: TOL_X3) if mode == L.MODE_BF16X3 else tol32
    for i, (m, n, k, ta, tb, lda, ldb, ldc, a, b, c, al, be) in enumerate(meta):
        got = out[offs[3 * i + 2]:offs[3 * i + 2] + ldc * n].reshape((ldc, n), order="F")
        a64, b64 = a[:(m if ta == "N" else k)].astype(np.float64), b[:(k if tb == "N" else n)].astype(np.float64)
        ref = al * ((a64 if ta == "N" else a64.T) @ (b64 if tb == "N" else b64.T)) + be * c[:m].astype(np.float64)
        err = float(np.max(np.abs(got[:m] - ref)) / max(np.max(np.abs(ref)), 1e-30))
        assert err < tol(k), (i, m, n, k, ta, tb, lda, ldb, err)
        np.testing.assert_array_equal(got[m:], c[m:])
