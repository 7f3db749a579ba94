"""Benchmark: TFLOP/s at fixed FP64-oracle error, split-precision tensor-core
GEMM vs the plain FP32/FP64 kernels, on the large-GEMM workload:

    sgemm NT and TN, M = N = K = 8192, float32, alpha = 1, beta = 0,
    entries uniform[-1, 1) from a seeded generator (synthetic, as the
    reference publishes no dataset), plus dgemm NN 4096^3 (plain FP64 vs
    Ozaki int8 slices) reported beside it.

One step = one NT and one TN sgemm 8192^3 in the split-precision mode (BF16x6
by default: the mode whose error is at or below the plain FP32 kernel's at
K = 8192).  `value` is whole-job TFLOP/s (2*M*N*K per call) with inputs
resident in HBM (each input is 256 MiB, larger than the 126 MB L2); `e2e` is
the same metric through the C ABI with pinned host buffers, so every step
includes the host->device copies of A and B and the device->host copy of C.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank runs an independent replica (the path has no
data exchange) and rank 0 prints the line; time is the max over ranks.
`--impl reference` times the reference's own algorithm for the same calls
(mojoBLAS gemm -> _gemm_naive for NT/TN, restated in C++ with OpenMP) on the
host cores, on a bounded column sample of each call.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

N_S = 8192      # sgemm size
N_D = 4096      # dgemm size
FLOPS_S = 2.0 * N_S ** 3
FLOPS_D = 2.0 * N_D ** 3
SAMPLE_ROWS = 256  # rows of C checked against the float64 oracle


# DRAM bytes of one tc_gemm_bf16x6 launch at M = N = K = 8192 (NT), measured with
# ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum (one pass, full size):
# 3.43 GB read + 0.267 GB written.  Algorithmic: 3 bf16 planes of A and of B
# (2 x 3 x 8192^2 x 2 B) read once, C (8192^2 x 4 B) written once.
TRAFFIC_BF16X6_8192 = 3.43e9 + 0.267e9
PLANES_BF16X6_8192 = 2 * 3 * 8192 * 8192 * 2 + 8192 * 8192 * 4


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d["hbm_gbs"], "bf16": d["bf16_tflops"], "bf16_sustained": d["bf16_tflops_sustained"],
                "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16": 1590.0, "bf16_sustained": 1400.0, "source": "fallback"}


class Clocks:
    """nvidia-smi sampling during the timed region."""
    Q = ("timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.dev = device
        self.proc = None
        self.window = None  # (t0, t1) host wall-clock of the timed region

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        import datetime
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = []
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                ts = datetime.datetime.strptime(f[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                pw = float(f[3]) if f[3] not in ("", "[N/A]", "N/A") else float("nan")
                rows.append((ts, float(f[1]), float(f[2]), f[5:9], pw))
            except ValueError:
                continue
        inside = [r for r in rows if self.window and self.window[0] <= r[0] <= self.window[1]]
        use = inside or rows
        if not use:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        reasons = sorted({nm for r in use for nm, v in zip(names, r[3]) if v.lower() == "active"})
        pw = [r[4] for r in use if r[4] == r[4]]
        return {"sm_mhz": float(np.median([r[1] for r in use])), "sm_max_mhz": use[-1][2], "reasons": reasons,
                "power_w": round(float(np.median(pw)), 1) if pw else None,
                "samples": len(use), "samples_in_timed_region": len(inside)}


def col_major(torch, rows, cols, gen, dtype, device):
    """rows x cols column-major matrix (stored as a cols x rows row-major tensor)."""
    t = torch.rand((cols, rows), generator=gen, dtype=torch.float64 if dtype == "f64" else torch.float32,
                   device=device)
    return t.mul_(2).sub_(1)


def max_over_ranks(value: float, dist, device="cpu") -> float:
    """The slowest rank's time: every rank contributes its own measurement and all
    receive the maximum (all_reduce MAX; NCCL on GPUs, gloo in the CPU tests)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def ref_rows(ta, tb, a, b, rows):
    """float64 oracle rows of C = op(A) op(B) (a, b: column-major torch tensors)."""
    A = a.double().cpu().numpy().T  # A[i, l]
    B = b.double().cpu().numpy().T
    opA = A if ta == "N" else A.T
    opB = B if tb == "N" else B.T
    return opA[rows, :] @ opB


def compensated_rows(a, b, count, seed):
    """`count` sampled rows of A B (NN, column-major float64 device tensors) from the
    oracle's compensated dot products: accurate to about 2^-106, so a float64 GEMM's own
    rounding error shows against it (a float64 numpy product has errors of that size)."""
    import oracle as orc
    n = a.shape[0]
    rows = np.sort(np.random.default_rng(seed).choice(n, count, replace=False))
    A, B = a.cpu().numpy().T, b.cpu().numpy().T  # column-major (n x n) views
    return orc.gemm_rows_dot2("N", "N", n, n, A, n, B, n, rows), rows


def rows_error(c, ref, rows):
    """max|C - C64| / max|C64| on the sampled rows."""
    got = c.double().cpu().numpy().T[rows, :]
    return float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))


def dtrsm_leg(torch, lib, L, stream, n, g, variants):
    """Left/Lower/NoTrans/NonUnit dtrsm of order n with n right-hand sides (A off-diagonal
    N(0,1)/sqrt(n), diagonal n + |N(0,1)|, B N(0,1)): CUDA-event time of each variant
    (label, mode, slices, refinement steps) and its float64-oracle error on 128 sampled
    columns of X (scipy's triangular solve)."""
    import scipy.linalg as sl
    A = torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64) / np.sqrt(n)
    A.diagonal().copy_(n + torch.randn(n, generator=g, device="cuda", dtype=torch.float64).abs())
    B0 = torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64)
    X = torch.empty_like(B0)
    cols = np.random.default_rng(5).choice(n, 128, replace=False)
    L_ = np.tril(A.cpu().numpy().T)  # column-major view: A[i, l]
    Xref = sl.solve_triangular(L_, B0.cpu().numpy().T[:, cols], lower=True)
    del L_

    def tcall(md, s_, r_):
        X.copy_(B0)
        st = lib.mbg_dtrsm_ex(md, s_, r_, b"L", b"L", b"N", b"N", n, n, 1.0, A.data_ptr(), n, X.data_ptr(), n)
        if st:
            raise RuntimeError(f"dtrsm failed {st}: {L.last_error()}")

    tr = {}
    for label, md, s_, r_ in variants:
        tcall(md, s_, r_)
        torch.cuda.synchronize()
        got = X.cpu().numpy().T[:, cols]
        err = float(np.max(np.abs(got - Xref)) / np.max(np.abs(Xref)))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 3
        e0.record(stream)
        for _ in range(reps):
            tcall(md, s_, r_)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        tr[label] = {"tflops": round(n ** 3 / (ms * 1e-3) / 1e12, 2), "ms": round(ms, 3), "fp64_err": err}
        if md != L.MODE_PLAIN:  # where one call's time goes: device time of each library kernel kind
            lib.mbg_prof_enable(1)
            lib.mbg_prof_reset()
            tcall(md, s_, r_)
            torch.cuda.synchronize()
            parts = {}
            for kname in ("tc_gemm_ozaki", "tc_gemm_bf16", "ozaki_slice", "ozaki_exponent", "split_bf16",
                          "trsm_block_invert", "trsm_block_solve", "trsm_diag"):
                tot, cnt = C.c_double(), C.c_int64()
                lib.mbg_prof_query(kname.encode(), C.byref(tot), C.byref(cnt))
                if cnt.value:
                    parts[kname] = {"ms": round(tot.value, 3), "launches": int(cnt.value)}
            lib.mbg_prof_enable(0)
            tr[label]["kernel_ms"] = parts
    del A, B0, X
    return tr


def run_cfg3(torch, lib, L, stream):
    """Blocked trsm (Left/Lower/NoTrans/NonUnit, 4096^2 float64, A off-diagonal
    N(0,1)/sqrt(4096), diagonal 4096 + |N(0,1)|, B N(0,1); and the same at order 8192,
    the size the split forms' 3x target is stated at) and syrk (Lower/NoTrans, N = 8192,
    K = 2048, float32, A uniform[-1,1)), plain vs split / Ozaki, with the float64-oracle
    error on sampled columns (trsm) / rows (syrk)."""
    out = {}
    g = torch.Generator(device="cuda")
    g.manual_seed(99)
    out["dtrsm_LLNN_4096"] = dtrsm_leg(torch, lib, L, stream, 4096, g, (
        ("plain_fp64", L.MODE_PLAIN, 0, 0), ("ozaki_s7", L.MODE_OZAKI, 7, 0), ("ozaki_s4_ir1", L.MODE_OZAKI, 4, 1)))
    out["dtrsm_LLNN_8192"] = dtrsm_leg(torch, lib, L, stream, 8192, g, (
        ("plain_fp64", L.MODE_PLAIN, 0, 0), ("ozaki_s7", L.MODE_OZAKI, 7, 0)))
    out["dtrsm_note"] = ("flops m^2 n; each timed call includes a device copy restoring B "
                         "(128 MiB at 4096, 512 MiB at 8192)")

    nn, kk = 8192, 2048
    As = torch.rand((kk, nn), generator=g, device="cuda", dtype=torch.float32) * 2 - 1  # column-major n x k
    Cs = torch.zeros((nn, nn), device="cuda", dtype=torch.float32)
    rows = np.sort(np.random.default_rng(6).choice(nn, 128, replace=False))
    Ah = As.double().cpu().numpy().T  # n x k
    ref = Ah[rows, :] @ Ah.T  # rows of A A^T
    mask = np.arange(nn)[None, :] <= rows[:, None]  # lower triangle of those rows
    sy = {}
    for label, md in (("plain_fp32", L.MODE_PLAIN), ("bf16x3", L.MODE_BF16X3), ("bf16x6", L.MODE_BF16X6)):
        def scall():
            st = lib.mbg_ssyrk_ex(md, b"L", b"N", nn, kk, 1.0, As.data_ptr(), nn, 0.0, Cs.data_ptr(), nn)
            if st:
                raise RuntimeError(f"ssyrk failed {st}: {L.last_error()}")
        scall()
        torch.cuda.synchronize()
        got = Cs.double().cpu().numpy().T[rows, :]
        err = float(np.max(np.abs((got - ref)[mask])) / np.max(np.abs(ref[mask])))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            scall()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        sy[label] = {"tflops": round(nn * (nn + 1) * kk / (ms * 1e-3) / 1e12, 2), "ms": round(ms, 3),
                     "fp64_err": err}
    out["ssyrk_LN_8192x2048"] = sy
    out["ssyrk_note"] = "flops n(n+1)k (the reference plot uses n^3 at n = k)"
    return out


def run_neighbours(torch, lib, L, stream):
    """symm, syr2k and trmm at the configuration sizes of the hot path: symm (Left, Upper)
    with A symmetric and B uniform[-1,1) at M = N = 4096 (float32 and float64); syr2k
    (Lower, NoTrans) at N = 8192, K = 2048 float32; trmm (Left, Lower, NoTrans, NonUnit)
    at M = N = 4096 with the trsm configuration's triangle (float64 and float32).  Plain
    vs split / Ozaki, with the float64-oracle error on 128 sampled columns (rows for
    syr2k).  Flops: symm 2 m^2 n, syr2k 2 n(n+1) k, trmm m^2 n."""
    out = {}
    g = torch.Generator(device="cuda")
    g.manual_seed(77)
    cols = np.sort(np.random.default_rng(8).choice(4096, 128, replace=False))

    def timed(call, flops):
        call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        return {"tflops": round(flops / (ms * 1e-3) / 1e12, 2), "ms": round(ms, 3)}

    def check(st, what):
        if st:
            raise RuntimeError(f"{what} failed {st}: {L.last_error()}")

    def kernel_ms(call, names):
        # device time of each library kernel in one call (CUDA events around every launch)
        import ctypes as C
        lib.mbg_prof_enable(1)
        lib.mbg_prof_reset()
        call()
        torch.cuda.synchronize()
        out_ms = {}
        for nm in names:
            tot, cnt = C.c_double(0), C.c_int64(0)
            lib.mbg_prof_query(nm.encode(), C.byref(tot), C.byref(cnt))
            if cnt.value:
                out_ms[nm] = round(tot.value, 4)
        lib.mbg_prof_enable(0)
        return out_ms

    trmm_kernels = ("copy", "trsm_tri_dense", "trmm_diag", "split_bf16", "tc_gemm_bf16x6", "ozaki_exponent",
                    "ozaki_slice", "tc_gemm_ozaki", "gemm_f32", "gemm_dmma_f64")

    n = 4096
    for dt, tname, modes in ((torch.float32, "s", (("plain_fp32", L.MODE_PLAIN, 0), ("bf16x6", L.MODE_BF16X6, 0))),
                             (torch.float64, "d", (("plain_fp64", L.MODE_PLAIN, 0), ("ozaki_s7", L.MODE_OZAKI, 7)))):
        A = torch.rand((n, n), generator=g, device="cuda", dtype=dt) * 2 - 1
        B = torch.rand((n, n), generator=g, device="cuda", dtype=dt) * 2 - 1
        C = torch.empty_like(B)
        An = A.double().cpu().numpy().T
        Asym = np.triu(An) + np.triu(An, 1).T
        ref = Asym @ B.double().cpu().numpy().T[:, cols]
        res = {}
        for label, md, sl in modes:
            def call():
                args = (b"L", b"U", n, n, 1.0, A.data_ptr(), n, B.data_ptr(), n, 0.0, C.data_ptr(), n)
                check(lib.mbg_ssymm_ex(md, *args) if tname == "s" else lib.mbg_dsymm_ex(md, sl, *args), "symm")
            r = timed(call, 2.0 * n ** 3)
            got = C.double().cpu().numpy().T[:, cols]
            r["fp64_err"] = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
            res[label] = r
        out[f"{tname}symm_LU_4096"] = res

        # trmm with the trsm configuration's triangle: off-diagonal N(0,1)/sqrt(n), diagonal n + |N(0,1)|
        T = torch.randn((n, n), generator=g, device="cuda", dtype=dt) / np.sqrt(n)
        T.diagonal().copy_(n + torch.randn(n, generator=g, device="cuda", dtype=dt).abs())
        B0 = torch.randn((n, n), generator=g, device="cuda", dtype=dt)
        ref = np.tril(T.double().cpu().numpy().T) @ B0.double().cpu().numpy().T[:, cols]
        res = {}
        for label, md, sl in modes:
            def call():
                C.copy_(B0)
                args = (b"L", b"L", b"N", b"N", n, n, 1.0, T.data_ptr(), n, C.data_ptr(), n)
                check(lib.mbg_strmm_ex(md, *args) if tname == "s" else lib.mbg_dtrmm_ex(md, sl, *args), "trmm")
            r = timed(call, 1.0 * n ** 3)
            got = C.double().cpu().numpy().T[:, cols]
            r["fp64_err"] = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
            r["kernels_ms"] = kernel_ms(call, trmm_kernels)
            res[label] = r
        out[f"{tname}trmm_LLNN_4096"] = res
        del A, B, C, T, B0

    nn, kk = 8192, 2048
    A = torch.rand((kk, nn), generator=g, device="cuda", dtype=torch.float32) * 2 - 1  # column-major n x k
    B = torch.rand((kk, nn), generator=g, device="cuda", dtype=torch.float32) * 2 - 1
    C = torch.zeros((nn, nn), device="cuda", dtype=torch.float32)
    rows = np.sort(np.random.default_rng(9).choice(nn, 128, replace=False))
    Ah, Bh = A.double().cpu().numpy().T, B.double().cpu().numpy().T
    ref = Ah[rows] @ Bh.T + Bh[rows] @ Ah.T
    mask = np.arange(nn)[None, :] <= rows[:, None]
    res = {}
    for label, md in (("plain_fp32", L.MODE_PLAIN), ("bf16x3", L.MODE_BF16X3), ("bf16x6", L.MODE_BF16X6)):
        def call():
            check(lib.mbg_ssyr2k_ex(md, b"L", b"N", nn, kk, 1.0, A.data_ptr(), nn, B.data_ptr(), nn, 0.0,
                                    C.data_ptr(), nn), "syr2k")
        r = timed(call, 2.0 * nn * (nn + 1) * kk)
        got = C.double().cpu().numpy().T[rows]
        r["fp64_err"] = float(np.max(np.abs((got - ref)[mask])) / np.max(np.abs(ref[mask])))
        res[label] = r
    out["ssyr2k_LN_8192x2048"] = res
    out["note"] = ("flops: symm 2 m^2 n, trmm m^2 n (each timed trmm call includes a device copy restoring B), "
                   "syr2k 2 n(n+1) k")
    del A, B, C
    return out


def run_complex(torch, lib, L, stream):
    """Complex gemm NN (C := A B, alpha = 1, beta = 0; real and imaginary parts uniform[-1, 1)):
    cgemm at 4096^3 (plain FP32 vs BF16x6) and zgemm at 2048^3 (plain FP64 vs Ozaki 7 slices),
    8 m n k real flops per call, error against complex128 numpy on 64 sampled rows."""
    out = {}
    g = torch.Generator(device="cuda")
    g.manual_seed(55)
    for name, nn, tdt, legs in (("cgemm_NN_4096", 4096, torch.complex64,
                                 (("plain_fp32", L.MODE_PLAIN, 0), ("bf16x6", L.MODE_BF16X6, 0))),
                                ("zgemm_NN_2048", 2048, torch.complex128,
                                 (("plain_fp64", L.MODE_PLAIN, 0), ("ozaki_s7", L.MODE_OZAKI, 7)))):
        rt = torch.float32 if tdt == torch.complex64 else torch.float64
        A = torch.complex(torch.rand((nn, nn), generator=g, device="cuda", dtype=rt) * 2 - 1,
                          torch.rand((nn, nn), generator=g, device="cuda", dtype=rt) * 2 - 1)
        B = torch.complex(torch.rand((nn, nn), generator=g, device="cuda", dtype=rt) * 2 - 1,
                          torch.rand((nn, nn), generator=g, device="cuda", dtype=rt) * 2 - 1)
        Cc = torch.empty_like(A)
        rows = np.random.default_rng(9).choice(nn, 64, replace=False)
        Ah = A.cpu().numpy().T.astype(np.complex128)  # column-major storage: tensor [col][row]
        ref = Ah[rows, :] @ B.cpu().numpy().T.astype(np.complex128)
        al = np.array([1.0, 0.0], np.float32 if tdt == torch.complex64 else np.float64)
        be = np.zeros(2, al.dtype)
        res = {}
        for label, md, s_ in legs:
            def call():
                args = (b"N", b"N", nn, nn, nn, al.ctypes.data, A.data_ptr(), nn, B.data_ptr(), nn, be.ctypes.data,
                        Cc.data_ptr(), nn)
                st = lib.mbg_cgemm_ex(md, *args) if tdt == torch.complex64 else lib.mbg_zgemm_ex(md, s_, *args)
                if st:
                    raise RuntimeError(f"{name} failed {st}: {L.last_error()}")
            call()
            torch.cuda.synchronize()
            got = Cc.cpu().numpy().T[rows, :]
            err = float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(3):
                call()
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 3
            res[label] = {"tflops": round(8.0 * nn ** 3 / (ms * 1e-3) / 1e12, 2), "ms": round(ms, 3),
                          "fp64_err": err}
        out[name] = res
        del A, B, Cc
    out["note"] = "flops 8 m n k (four real products per complex multiply-add); the real embedding (4M)"
    return out


def run_level2(torch, lib, L, stream):
    """gemv (NoTrans and Trans, 8192 x 8192, float32 and float64, alpha 1.5, beta 0.5, uniform[-1,1)) and
    trsv (Lower / Upper, NoTrans, order 4096, the trsm configuration's triangle scaled to a vector), device
    resident.  Bytes per call: gemv m n + m + 2n (x read, y read and written) elements; trsv n(n+1)/2 + 2n.
    A is 256 / 512 MiB for gemv (larger than L2); the 4096-order triangle (32 / 64 MiB) fits in L2, so each
    trsv call is preceded by a 256 MiB L2 flush."""
    out = {}
    pk = peaks()
    g = torch.Generator(device="cuda")
    g.manual_seed(55)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")

    def timed(call, nbytes, reps=5, flush_l2=False):
        call()
        torch.cuda.synchronize()
        tot = 0.0
        for _ in range(reps):
            if flush_l2:
                flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        ms = tot / reps
        gbs = nbytes / (ms * 1e-3) / 1e9
        return {"gbs": round(gbs, 1), "ms": round(ms, 4), "hbm_frac": round(gbs / pk["hbm_gbs"], 3)}

    m = n = 8192
    for dt, tn in ((torch.float32, "s"), (torch.float64, "d")):
        esz = 4 if dt == torch.float32 else 8
        A = torch.rand((n, m), generator=g, device="cuda", dtype=dt) * 2 - 1  # column-major m x n
        x = torch.rand(max(m, n), generator=g, device="cuda", dtype=dt) * 2 - 1
        y0 = torch.rand(max(m, n), generator=g, device="cuda", dtype=dt) * 2 - 1
        y = y0.clone()
        Ah = A.double().cpu().numpy().T
        fn = lib.mbg_sgemv if tn == "s" else lib.mbg_dgemv
        for trans in ("N", "T"):
            def call():
                st = fn(trans.encode(), m, n, 1.5, A.data_ptr(), m, x.data_ptr(), 1, 0.5, y.data_ptr(), 1)
                if st:
                    raise RuntimeError(f"gemv failed {st}: {L.last_error()}")
            y.copy_(y0)
            call()
            torch.cuda.synchronize()
            op = Ah if trans == "N" else Ah.T
            ref = 1.5 * op @ x.double().cpu().numpy()[:op.shape[1]] + 0.5 * y0.double().cpu().numpy()[:op.shape[0]]
            err = float(np.max(np.abs(y.double().cpu().numpy()[:op.shape[0]] - ref)) / np.max(np.abs(ref)))
            r = timed(call, esz * (m * n + m + 2 * n))
            r["fp64_err"] = err
            out[f"{tn}gemv_{trans}_8192"] = r
        del A, Ah

    nt = 4096
    for dt, tn in ((torch.float32, "s"), (torch.float64, "d")):
        esz = 4 if dt == torch.float32 else 8
        T = torch.randn((nt, nt), generator=g, device="cuda", dtype=dt) / np.sqrt(nt)
        T.diagonal().copy_(2.0 + torch.randn(nt, generator=g, device="cuda", dtype=dt).abs())
        b0 = torch.randn(nt, generator=g, device="cuda", dtype=dt)
        xb = b0.clone()
        Th = T.double().cpu().numpy().T
        fn = lib.mbg_strsv if tn == "s" else lib.mbg_dtrsv
        import scipy.linalg as sla
        for uplo in ("L", "U"):
            def call():
                xb.copy_(b0)
                st = fn(uplo.encode(), b"N", b"N", nt, T.data_ptr(), nt, xb.data_ptr(), 1)
                if st:
                    raise RuntimeError(f"trsv failed {st}: {L.last_error()}")
            call()
            torch.cuda.synchronize()
            tri = np.tril(Th) if uplo == "L" else np.triu(Th)
            ref = sla.solve_triangular(tri, b0.double().cpu().numpy(), lower=uplo == "L")
            err = float(np.max(np.abs(xb.double().cpu().numpy() - ref)) / np.max(np.abs(ref)))
            r = timed(call, esz * (nt * (nt + 1) // 2 + 2 * nt), flush_l2=True)
            r["fp64_err"] = err
            out[f"{tn}trsv_{uplo}N_4096"] = r
        del T
    out["note"] = ("GB/s = algorithmic bytes / CUDA-event time; each timed trsv call includes a 16 / 32 KiB "
                   "device copy restoring b; hbm_frac against the " + pk["source"] + " HBM copy bandwidth")
    del flush
    return out


def run_cfg4(torch, lib, L, stream):
    """Batched: 4096 sgemm problems (m, n, k log-uniform 16..512, NN, uniform[-1,1))
    and 2048 lower-triangular strsm problems (n log-uniform 8..256, nrhs uniform
    1..64, A diagonally dominant as in the trsm configuration, B N(0,1)), each in
    one graph-replayed persistent launch (sgemm in the plain form and in the split
    BF16x6 / BF16x3 forms on the tensor cores); float64-oracle error on 64 sampled
    problems of each."""
    from mojoblas_b200.autotune import log_uniform, sgemm_batch
    out = {}
    buf, probs, (m, n, k, offs), flops = sgemm_batch(torch, L, 4096, seed=41)
    reps = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sample = np.random.default_rng(3).choice(len(probs), 64, replace=False)

    def grouped(mode):
        """CUDA-event time of one plan execution (mean of reps graph replays) and the
        float64-oracle error on the sampled problems."""
        plan = C.c_void_p()
        if lib.mbg_sgemm_grouped_plan(mode, len(probs), probs, C.byref(plan)):
            raise RuntimeError(L.last_error())
        try:
            lib.mbg_plan_execute(plan)
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(reps):
                lib.mbg_plan_execute(plan)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_ = e0.elapsed_time(e1) / reps
        finally:
            lib.mbg_plan_destroy(plan)
        host = buf.cpu().numpy()
        errs_ = []
        for i in sample:
            o, mi, ni, ki = int(offs[i]), int(m[i]), int(n[i]), int(k[i])
            a = host[o:o + mi * ki].reshape((mi, ki), order="F").astype(np.float64)
            b = host[o + mi * ki:o + mi * ki + ki * ni].reshape((ki, ni), order="F").astype(np.float64)
            c = host[o + mi * ki + ki * ni:o + mi * ki + ki * ni + mi * ni].reshape((mi, ni), order="F")
            ref = a @ b
            errs_.append(float(np.max(np.abs(c - ref)) / np.max(np.abs(ref))))
        return ms_, max(errs_)

    ms, err_plain = grouped(L.MODE_PLAIN)
    ms_x6, err_x6 = grouped(L.MODE_BF16X6)
    ms_x3, err_x3 = grouped(L.MODE_BF16X3)
    # the same problems as 4096 separate library calls (what a caller without batching does)
    lib.mbg_set_sync(0)
    e0.record(stream)
    for i in range(len(probs)):
        q = probs[i]
        lib.mbg_sgemm(b"N", b"N", q.m, q.n, q.k, 1.0, q.a, q.lda, q.b, q.ldb, 0.0, q.c, q.ldc)
    e1.record(stream)
    torch.cuda.synchronize()
    loop_ms = e0.elapsed_time(e1)
    out["grouped_sgemm_4096"] = {"tflops": round(flops / ms / 1e9, 2), "ms": round(ms, 4),
                                 "looped_calls_ms": round(loop_ms, 3), "max_fp64_err_64_sampled": err_plain,
                                 "tile": int(lib.mbg_get_tuning(b"grouped_gemm_tile"))}
    out["grouped_sgemm_4096_bf16x6"] = {"tflops": round(flops / ms_x6 / 1e9, 2), "ms": round(ms_x6, 4),
                                        "speedup_vs_plain_grouped": round(ms / ms_x6, 2),
                                        "max_fp64_err_64_sampled": err_x6}
    out["grouped_sgemm_4096_bf16x3"] = {"tflops": round(flops / ms_x3 / 1e9, 2), "ms": round(ms_x3, 4),
                                        "max_fp64_err_64_sampled": err_x3}
    del buf

    rng = np.random.default_rng(42)
    cnt = 2048
    ns = log_uniform(rng, 8, 256, cnt)
    rh = rng.integers(1, 65, cnt)
    a_offs, b_offs, tot = [], [], 0
    for i in range(cnt):
        a_offs.append(tot); tot += int(ns[i] * ns[i] + 63) // 64 * 64
        b_offs.append(tot); tot += int(ns[i] * rh[i] + 63) // 64 * 64
    hostbuf = np.zeros(tot, np.float32)
    for i in range(cnt):
        ni = int(ns[i])
        a = rng.standard_normal((ni, ni)) / np.sqrt(ni)
        a[np.arange(ni), np.arange(ni)] = ni + np.abs(rng.standard_normal(ni))
        hostbuf[a_offs[i]:a_offs[i] + ni * ni] = np.tril(a).reshape(-1, order="F")
        hostbuf[b_offs[i]:b_offs[i] + ni * int(rh[i])] = rng.standard_normal(ni * int(rh[i]))
    dbuf = torch.from_numpy(hostbuf).cuda()
    base = dbuf.data_ptr()
    tp = (L.StrsmProblem * cnt)()
    for i in range(cnt):
        tp[i] = L.StrsmProblem(b"L", b"L", b"N", b"N", int(ns[i]), int(rh[i]), 1.0, base + 4 * a_offs[i],
                               int(ns[i]), base + 4 * b_offs[i], int(ns[i]))
    plan = C.c_void_p()
    if lib.mbg_strsm_grouped_plan(L.MODE_PLAIN, cnt, tp, C.byref(plan)):
        raise RuntimeError(L.last_error())
    lib.mbg_plan_execute(plan)  # solves once; check that result
    torch.cuda.synchronize()
    res = dbuf.cpu().numpy()
    import scipy.linalg as sl
    terr = []
    for i in np.random.default_rng(4).choice(cnt, 64, replace=False):
        ni, ri = int(ns[i]), int(rh[i])
        a = hostbuf[a_offs[i]:a_offs[i] + ni * ni].reshape((ni, ni), order="F").astype(np.float64)
        b = hostbuf[b_offs[i]:b_offs[i] + ni * ri].reshape((ni, ri), order="F").astype(np.float64)
        x = res[b_offs[i]:b_offs[i] + ni * ri].reshape((ni, ri), order="F")
        ref = sl.solve_triangular(a, b, lower=True)
        terr.append(float(np.max(np.abs(x - ref)) / np.max(np.abs(ref))))
    orig = torch.from_numpy(hostbuf).cuda()
    e0.record(stream)
    for _ in range(reps):  # restore B, then solve
        dbuf.copy_(orig)
        lib.mbg_plan_execute(plan)
    e1.record(stream)
    torch.cuda.synchronize()
    both = e0.elapsed_time(e1) / reps
    e0.record(stream)
    for _ in range(reps):
        dbuf.copy_(orig)
    e1.record(stream)
    torch.cuda.synchronize()
    tms = both - e0.elapsed_time(e1) / reps  # the restoring copy's time taken out
    lib.mbg_plan_destroy(plan)
    tflop = float(np.sum(ns.astype(np.float64) ** 2 * rh))
    tbytes = float(np.sum(4.0 * (ns * (ns + 1) / 2 + 2 * ns * rh)))
    out["grouped_strsm_2048"] = {"tflops": round(tflop / tms / 1e9, 3), "gbs": round(tbytes / tms / 1e6, 1),
                                 "ms": round(tms, 4), "bytes": tbytes,
                                 "hbm_frac": round(tbytes / tms / 1e6 / peaks()["hbm_gbs"], 3),
                                 "max_fp64_err_64_sampled": max(terr)}
    return out


def run_cfg5(torch, lib, L, stream):
    """Adjoints at the configuration-5 sizes, float32 kernels: trsm with L 2048^2
    lower and diagonally dominant, B 2048 x 512 N(0,1), X = L^-1 B, G N(0,1)
    (dB = L^-T G, dL = -tril(dB X^T)); gemm C = A B, A 3072 x 1024, B 1024 x 2048
    uniform[-1,1) (dA = G B^T, dB = A^T G).  Checked by central finite differences
    in float64 along 64 random directions, the function evaluated with the
    library's plain FP64 kernels."""
    out = {}
    g = torch.Generator(device="cuda")
    g.manual_seed(55)
    n, r = 2048, 512
    Ld = torch.randn((n, n), generator=g, device="cuda", dtype=torch.float64) / np.sqrt(n)
    Ld.diagonal().copy_(n + torch.randn(n, generator=g, device="cuda", dtype=torch.float64).abs())
    Ld = torch.tril(Ld.T).T.contiguous()  # column-major lower triangle (row-major upper storage)
    Bd = torch.randn((r, n), generator=g, device="cuda", dtype=torch.float64)
    Gd = torch.randn((r, n), generator=g, device="cuda", dtype=torch.float64)
    Lf, Bf, Gf = Ld.float(), Bd.float(), Gd.float()
    Xd = Bd.clone()
    lib.mbg_dtrsm(b"L", b"L", b"N", b"N", n, r, 1.0, Ld.data_ptr(), n, Xd.data_ptr(), n)
    Xf = Xd.float()

    def f(Lp, Bp):  # <G, L^-1 B> in float64 with the plain FP64 trsm
        Y = Bp.clone()
        lib.mbg_dtrsm(b"L", b"L", b"N", b"N", n, r, 1.0, Lp.data_ptr(), n, Y.data_ptr(), n)
        return float((Gd * Y).sum())

    lower = torch.tril(torch.ones((n, n), device="cuda", dtype=torch.float64)).T  # storage mask
    res = {}
    for label, md in (("plain", L.MODE_PLAIN), ("bf16x6", L.MODE_BF16X6)):
        dB = torch.zeros_like(Bf)
        dL = torch.zeros_like(Lf)

        def call():
            st = lib.mbg_strsm_adjoint(md, b"L", b"L", b"N", b"N", n, r, 1.0, Lf.data_ptr(), n, Xf.data_ptr(), n,
                                       Gf.data_ptr(), n, dB.data_ptr(), n, dL.data_ptr(), n)
            if st:
                raise RuntimeError(f"strsm_adjoint {st}: {L.last_error()}")
        call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(5):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 5
        gg = torch.Generator(device="cuda")
        gg.manual_seed(7)
        worst = worst_fd = 0.0
        h = 1e-4
        for _ in range(64):
            eL = torch.randn((n, n), generator=gg, device="cuda", dtype=torch.float64) * lower
            eB = torch.randn((r, n), generator=gg, device="cuda", dtype=torch.float64)
            fd = (f(Ld + h * eL, Bd + h * eB) - f(Ld - h * eL, Bd - h * eB)) / (2 * h)
            ad = float((dL.double() * eL).sum() + (dB.double() * eB).sum())
            scale = float((dL.double() * lower).norm() * eL.norm() + dB.double().norm() * eB.norm())
            worst = max(worst, abs(fd - ad) / scale)
            worst_fd = max(worst_fd, abs(fd - ad) / max(abs(fd), 1e-300))
        flops = 2.0 * n * n * r  # dB: n^2 r, masked dL: n^2 r
        res[label] = {"ms": round(ms, 3), "tflops": round(flops / ms / 1e9, 2),
                      "fd_max_rel_discrepancy_64_dirs": worst, "fd_max_rel_to_fd_64_dirs": worst_fd}
    out["strsm_adjoint_2048x512"] = res
    del Ld, Bd, Gd, Lf, Bf, Gf, Xd, Xf, lower

    m, k, nn = 3072, 1024, 2048
    Ad = torch.rand((k, m), generator=g, device="cuda", dtype=torch.float64) * 2 - 1  # column-major m x k
    Bd = torch.rand((nn, k), generator=g, device="cuda", dtype=torch.float64) * 2 - 1  # column-major k x nn
    Gd = torch.randn((nn, m), generator=g, device="cuda", dtype=torch.float64)
    Af, Bf, Gf = Ad.float(), Bd.float(), Gd.float()
    Cd = torch.empty_like(Gd)

    def fg(Ap, Bp):
        lib.mbg_dgemm(b"N", b"N", m, nn, k, 1.0, Ap.data_ptr(), m, Bp.data_ptr(), k, 0.0, Cd.data_ptr(), m)
        return float((Gd * Cd).sum())

    res = {}
    for label, md in (("plain", L.MODE_PLAIN), ("bf16x6", L.MODE_BF16X6)):
        dA = torch.zeros_like(Af)
        dB = torch.zeros_like(Bf)

        def call():
            st = lib.mbg_sgemm_adjoint(md, b"N", b"N", m, nn, k, 1.0, Af.data_ptr(), m, Bf.data_ptr(), k,
                                       Gf.data_ptr(), m, dA.data_ptr(), m, dB.data_ptr(), k)
            if st:
                raise RuntimeError(f"sgemm_adjoint {st}: {L.last_error()}")
        call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(5):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 5
        gg = torch.Generator(device="cuda")
        gg.manual_seed(8)
        worst = worst_fd = 0.0
        h = 1e-3
        for _ in range(64):
            eA = torch.randn(Ad.shape, generator=gg, device="cuda", dtype=torch.float64)
            eB = torch.randn(Bd.shape, generator=gg, device="cuda", dtype=torch.float64)
            fd = (fg(Ad + h * eA, Bd + h * eB) - fg(Ad - h * eA, Bd - h * eB)) / (2 * h)
            ad = float((dA.double() * eA).sum() + (dB.double() * eB).sum())
            scale = float(dA.double().norm() * eA.norm() + dB.double().norm() * eB.norm())
            worst = max(worst, abs(fd - ad) / scale)
            worst_fd = max(worst_fd, abs(fd - ad) / max(abs(fd), 1e-300))
        flops = 2.0 * (2.0 * m * nn * k)
        res[label] = {"ms": round(ms, 3), "tflops": round(flops / ms / 1e9, 2),
                      "fd_max_rel_discrepancy_64_dirs": worst, "fd_max_rel_to_fd_64_dirs": worst_fd}
    out["sgemm_adjoint_3072x1024x2048"] = res
    out["note"] = ("discrepancy = |FD - <grad, dir>| / (|grad| |dir|), FD in float64 with the plain FP64 kernels; "
                   "trsm flops 2 n^2 nrhs (dB + triangle-only dL), gemm 2 x 2mnk")
    return out


def leg_fractions(dg, cfg3, cfg4, cfg5, probes, pk):
    """Each leg's achieved rate over the peak of the pipe that bounds it: the measured
    bf16 burst for split-precision tensor work (P bf16 products per FP32 product), the
    run's own probes for the FP32 / FP64 pipes and the int8 tensor pipe (28 int8 products
    per FP64 product at 7 slices), the measured HBM copy for the batched trsm."""
    out = {}
    f32, f64, i8 = probes.get("fp32_fma_tflops"), probes.get("fp64_fma_tflops"), probes.get("int8_mma_tops")

    def put(key, value, peak, note):
        if value is not None and peak:
            out[key] = {"frac": round(value / peak, 3), "peak": round(peak, 1), "bound": note}
    if dg:
        put("dgemm_plain_fp64", dg["plain_fp64"]["tflops"], f64, "fp64 pipe (probe)")
        put("dgemm_ozaki_s7_int8", 28 * dg["ozaki_s7"]["tflops"], i8, "int8 tensor pipe (probe), whole call")
    sy = cfg3.get("ssyrk_LN_8192x2048", {}) if cfg3 else {}
    if sy:
        put("ssyrk_plain_fp32", sy["plain_fp32"]["tflops"], f32, "fp32 pipe (probe)")
        put("ssyrk_bf16x6_tensor", 6 * sy["bf16x6"]["tflops"], pk["bf16"], "bf16 tensor pipe (measured burst)")
    tr = cfg3.get("dtrsm_LLNN_4096", {}) if cfg3 else {}
    if tr:
        put("dtrsm_plain_fp64", tr["plain_fp64"]["tflops"], f64, "fp64 pipe (probe); diagonal blocks latency-bound")
    tr8 = cfg3.get("dtrsm_LLNN_8192", {}) if cfg3 else {}
    if tr8 and "ozaki_s7" in tr8:
        put("dtrsm_8192_ozaki_s7_int8", 28 * tr8["ozaki_s7"]["tflops"], i8,
            "int8 tensor pipe (probe), whole call (m^2 n flops; the inverted-block leaves add m nb n)")
    if cfg4:
        put("grouped_sgemm_fp32", cfg4["grouped_sgemm_4096"]["tflops"], f32, "fp32 pipe (probe)")
        gx = cfg4.get("grouped_sgemm_4096_bf16x6")
        if gx:
            put("grouped_sgemm_bf16x6_tensor", 6 * gx["tflops"], pk["bf16"],
                "bf16 tensor pipe (measured burst); useful flops only (tile padding not counted)")
        g = cfg4.get("grouped_strsm_2048")
        if g:
            put("grouped_strsm_hbm", g["gbs"], pk["hbm_gbs"], "HBM (measured copy); latency-bound")
    ga = (cfg5 or {}).get("sgemm_adjoint_3072x1024x2048")
    if ga:
        put("sgemm_adjoint_bf16x6_tensor", 6 * ga["bf16x6"]["tflops"], pk["bf16"], "bf16 tensor pipe (measured burst)")
    ta_ = (cfg5 or {}).get("strsm_adjoint_2048x512")
    if ta_ and "bf16x6" in ta_:
        put("strsm_adjoint_bf16x6_tensor", 6 * ta_["bf16x6"]["tflops"], pk["bf16"],
            "bf16 tensor pipe (measured burst), whole call (inverted diagonal blocks, masked dL product)")
        put("strsm_adjoint_plain_fp32", ta_["plain"]["tflops"] if "plain" in ta_ else None, f32,
            "fp32 pipe (probe)")
    return out


def run_ours(args, rank, world, dist):
    import torch
    import mojoblas_b200 as mb
    from mojoblas_b200 import _lib as L

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    lib = L.load()
    stream = torch.cuda.current_stream()
    lib.mbg_set_stream(C.c_void_p(stream.cuda_stream))
    lib.mbg_set_sync(0)
    mode = {"bf16x3": L.MODE_BF16X3, "bf16x6": L.MODE_BF16X6}[args.mode]
    nprod = 3 if args.mode == "bf16x3" else 6

    g = torch.Generator(device="cuda")
    g.manual_seed(1234 + rank)
    A = col_major(torch, N_S, N_S, g, "f32", "cuda")
    B = col_major(torch, N_S, N_S, g, "f32", "cuda")
    Cm = torch.empty((N_S, N_S), dtype=torch.float32, device="cuda")
    n = N_S

    def call(md, ta, tb, c=Cm):
        st = lib.mbg_sgemm_ex(md, ta.encode(), tb.encode(), n, n, n, 1.0, A.data_ptr(), n, B.data_ptr(), n,
                              0.0, c.data_ptr(), n)
        if st:
            raise RuntimeError(f"mbg_sgemm_ex({md}) failed: {st} {L.last_error()}")

    def step(md):
        call(md, "N", "T")
        call(md, "T", "N")

    window = [None, None]

    def timed(md, steps, warmup):
        for _ in range(warmup):
            step(md)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        lib.mbg_prof_reset()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        window[0] = time.time()
        e0.record(stream)
        for _ in range(steps):
            step(md)
        e1.record(stream)
        torch.cuda.synchronize()
        window[1] = time.time()
        launches = int(lib.mbg_launch_count())
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, dist, "cuda")
        return ms, launches

    # ---- headline: split-precision sgemm ----
    clocks = Clocks(dev)
    with clocks:
        time.sleep(0.3)  # let the sampler start before the timed region
        ms, launches = timed(mode, args.steps, args.warmup)
    clocks.window = tuple(window)
    value = world * 2 * FLOPS_S / (ms * 1e-3) / 1e12

    # per-kernel timing of the dominant kernel (CUDA events around each launch)
    lib.mbg_prof_enable(1)
    lib.mbg_prof_reset()
    for _ in range(max(2, args.steps // 2)):
        step(mode)
    torch.cuda.synchronize()
    kname = b"tc_gemm_" + args.mode.encode()
    tot, cnt = C.c_double(), C.c_int64()
    lib.mbg_prof_query(kname, C.byref(tot), C.byref(cnt))
    k_ms = tot.value / max(cnt.value, 1)
    lib.mbg_prof_query(b"split_bf16", C.byref(tot), C.byref(cnt))
    split_ms = tot.value / max(cnt.value, 1)
    lib.mbg_prof_enable(0)

    # ---- errors against the float64 oracle (sampled rows) ----
    rs = np.random.default_rng(7).choice(N_S, SAMPLE_ROWS, replace=False)
    errs, refs = {}, {}
    Cp = torch.empty_like(Cm)
    for ta, tb in (("N", "T"), ("T", "N")):
        refs[ta + tb] = ref_rows(ta, tb, A, B, rs)
        call(mode, ta, tb)
        call(L.MODE_PLAIN, ta, tb, Cp)
        torch.cuda.synchronize()
        errs[ta + tb] = {args.mode: rows_error(Cm, refs[ta + tb], rs),
                         "plain_fp32": rows_error(Cp, refs[ta + tb], rs)}
    del Cp

    # ---- second input set: rows of op(A) and of op(B) (the k dimension) scaled by 2^u,
    #      u uniform integer in [-20, 20]; errors only ----
    su = torch.exp2(torch.randint(-20, 21, (n,), generator=g, device="cuda").double()).float()
    sv = torch.exp2(torch.randint(-20, 21, (n,), generator=g, device="cuda").double()).float()
    As, Bs = torch.empty_like(A), torch.empty_like(B)
    Cs = torch.empty_like(Cm)
    for ta, tb in (("N", "T"), ("T", "N")):
        # storage is column-major: tensor [col][row]; op(A) rows = A rows ("N") or A columns ("T")
        As.copy_(A * su[None, :] if ta == "N" else A * su[:, None])
        Bs.copy_(B * sv[:, None] if tb == "T" else B * sv[None, :])
        ref = ref_rows(ta, tb, As, Bs, rs)
        for label, md in (("plain_fp32", L.MODE_PLAIN), ("bf16x3", L.MODE_BF16X3), ("bf16x6", L.MODE_BF16X6)):
            st = lib.mbg_sgemm_ex(md, ta.encode(), tb.encode(), n, n, n, 1.0, As.data_ptr(), n, Bs.data_ptr(), n,
                                  0.0, Cs.data_ptr(), n)
            if st:
                raise RuntimeError(L.last_error())
            torch.cuda.synchronize()
            errs.setdefault(ta + tb + "_scaled_rows", {})[label] = rows_error(Cs, ref, rs)
    del As, Bs, Cs

    # ---- plain FP32 for the same step ----
    ms_plain, _ = timed(L.MODE_PLAIN, max(2, args.steps // 4), 1)
    plain_tflops = world * 2 * FLOPS_S / (ms_plain * 1e-3) / 1e12

    # ---- the other split mode, for reference ----
    other = "bf16x3" if args.mode == "bf16x6" else "bf16x6"
    other_mode = L.MODE_BF16X3 if other == "bf16x3" else L.MODE_BF16X6
    ms_other, _ = timed(other_mode, max(2, args.steps // 2), 1)
    for ta, tb in (("N", "T"), ("T", "N")):
        call(other_mode, ta, tb)
        torch.cuda.synchronize()
        errs[ta + tb][other] = rows_error(Cm, refs[ta + tb], rs)

    # ---- dgemm 4096^3 NN: plain FP64 vs Ozaki ----
    dg, dg8 = {}, {}
    if not args.skip_dgemm:
        Ad = col_major(torch, N_D, N_D, g, "f64", "cuda")
        Bd = col_major(torch, N_D, N_D, g, "f64", "cuda")
        Cd = torch.empty((N_D, N_D), dtype=torch.float64, device="cuda")
        rsd = np.random.default_rng(8).choice(N_D, SAMPLE_ROWS, replace=False)
        refd = ref_rows("N", "N", Ad, Bd, rsd)
        refc, rsc = compensated_rows(Ad, Bd, 32, 11)

        def dcall(md, s):
            st = lib.mbg_dgemm_ex(md, s, b"N", b"N", N_D, N_D, N_D, 1.0, Ad.data_ptr(), N_D, Bd.data_ptr(), N_D,
                                  0.0, Cd.data_ptr(), N_D)
            if st:
                raise RuntimeError(f"mbg_dgemm_ex failed: {st} {L.last_error()}")

        for label, md, s in (("plain_fp64", L.MODE_PLAIN, 0), ("ozaki_s7", L.MODE_OZAKI, 7),
                             ("ozaki_s8", L.MODE_OZAKI, 8)):
            for _ in range(2):
                dcall(md, s)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            reps = 3
            e0.record(stream)
            for _ in range(reps):
                dcall(md, s)
            e1.record(stream)
            torch.cuda.synchronize()
            dms = e0.elapsed_time(e1) / reps
            dg[label] = {"tflops": round(FLOPS_D / (dms * 1e-3) / 1e12, 2), "ms": round(dms, 3),
                         "fp64_err": rows_error(Cd, refd, rsd),
                         "err_vs_compensated": rows_error(Cd, refc, rsc)}
            if md == L.MODE_OZAKI:  # kernel-only time (CUDA events around the tcgen05 launch)
                lib.mbg_prof_enable(1)
                lib.mbg_prof_reset()
                dcall(md, s)
                torch.cuda.synchronize()
                tot, cnt = C.c_double(), C.c_int64()
                lib.mbg_prof_query(b"tc_gemm_ozaki", C.byref(tot), C.byref(cnt))
                lib.mbg_prof_enable(0)
                dg[label]["kernel_ms"] = round(tot.value / max(cnt.value, 1), 3)
        sud = torch.exp2(torch.randint(-20, 21, (N_D,), generator=g, device="cuda").double())
        svd = torch.exp2(torch.randint(-20, 21, (N_D,), generator=g, device="cuda").double())
        Ad.mul_(sud[None, :])  # rows of A (NN)
        Bd.mul_(svd[None, :])  # rows of B = the k dimension
        refd = ref_rows("N", "N", Ad, Bd, rsd)
        for label, md, s_ in (("plain_fp64", L.MODE_PLAIN, 0), ("ozaki_s7", L.MODE_OZAKI, 7),
                              ("ozaki_s8", L.MODE_OZAKI, 8)):
            dcall(md, s_)
            torch.cuda.synchronize()
            dg[label]["fp64_err_scaled_rows"] = rows_error(Cd, refd, rsd)
        del Ad, Bd, Cd

        # the size the split forms' 3x target is stated at: M = N = K = 8192, plain FP64 vs Ozaki s = 7
        n8 = 2 * N_D
        Ad = col_major(torch, n8, n8, g, "f64", "cuda")
        Bd = col_major(torch, n8, n8, g, "f64", "cuda")
        Cd = torch.empty((n8, n8), dtype=torch.float64, device="cuda")
        rs8 = np.random.default_rng(10).choice(n8, 128, replace=False)
        ref8 = ref_rows("N", "N", Ad, Bd, rs8)
        refc8, rsc8 = compensated_rows(Ad, Bd, 32, 12)
        for label, md, s in (("plain_fp64", L.MODE_PLAIN, 0), ("ozaki_s7", L.MODE_OZAKI, 7)):
            def call8():
                st = lib.mbg_dgemm_ex(md, s, b"N", b"N", n8, n8, n8, 1.0, Ad.data_ptr(), n8, Bd.data_ptr(), n8,
                                      0.0, Cd.data_ptr(), n8)
                if st:
                    raise RuntimeError(f"mbg_dgemm_ex failed: {st} {L.last_error()}")
            call8()
            torch.cuda.synchronize()
            err = rows_error(Cd, ref8, rs8)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(3):
                call8()
            e1.record(stream)
            torch.cuda.synchronize()
            ms8 = e0.elapsed_time(e1) / 3
            dg8[label] = {"tflops": round(2.0 * n8 ** 3 / (ms8 * 1e-3) / 1e12, 2), "ms": round(ms8, 3),
                          "fp64_err": err, "err_vs_compensated": rows_error(Cd, refc8, rsc8)}
        del Ad, Bd, Cd

    # ---- own peak probes (FMA loops, back-to-back tcgen05.mma) ----
    pv = [C.c_double() for _ in range(4)]
    probes = {}
    if lib.mbg_probe_peaks(*[C.byref(x) for x in pv]) == 0:
        probes = {"fp32_fma_tflops": round(pv[0].value, 1), "fp64_fma_tflops": round(pv[1].value, 1),
                  "bf16_mma_tflops": round(pv[2].value, 1), "int8_mma_tops": round(pv[3].value, 1)}
        probes["plain_fp32_frac"] = round(plain_tflops / pv[0].value, 3)
        if dg:
            probes["plain_fp64_frac"] = round(dg["plain_fp64"]["tflops"] / pv[1].value, 3)
            probes["ozaki_s7_int8_frac"] = round(28 * FLOPS_D / (dg["ozaki_s7"]["kernel_ms"] * 1e-3) / 1e12
                                                 / pv[3].value, 3) if dg["ozaki_s7"].get("kernel_ms") else None

    # ---- context: the vendor library's plain FP32 / FP64 GEMM on the same sizes ----
    ctx = {}
    if not args.skip_context:
        prev = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = False  # true FP32 arithmetic
        for label, dtype, nn, flops in (("torch_matmul_fp32_8192", torch.float32, N_S, FLOPS_S),
                                        ("torch_matmul_fp64_4096", torch.float64, N_D, FLOPS_D)):
            xa = torch.rand((nn, nn), device="cuda", dtype=dtype)
            xb = torch.rand((nn, nn), device="cuda", dtype=dtype)
            for _ in range(2):
                torch.matmul(xa, xb)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(3):
                torch.matmul(xa, xb)
            e1.record()
            torch.cuda.synchronize()
            tms = e0.elapsed_time(e1) / 3
            ctx[label] = {"tflops": round(flops / (tms * 1e-3) / 1e12, 2), "ms": round(tms, 3)}
            del xa, xb
        torch.backends.cuda.matmul.allow_tf32 = prev

    # ---- configuration 3: blocked dtrsm 4096^2 and ssyrk 8192 x 2048 ----
    cfg3 = {} if args.skip_cfg3 else run_cfg3(torch, lib, L, stream)
    cfg4 = {} if args.skip_cfg4 else run_cfg4(torch, lib, L, stream)
    cfg5 = {} if args.skip_cfg5 else run_cfg5(torch, lib, L, stream)
    neighbours = {} if args.skip_neighbours else run_neighbours(torch, lib, L, stream)
    level2 = {} if args.skip_level2 else run_level2(torch, lib, L, stream)
    cplx = {} if args.skip_complex else run_complex(torch, lib, L, stream)

    # ---- e2e through the C ABI with pinned host buffers ----
    hA = A.cpu().pin_memory()
    hB = B.cpu().pin_memory()
    hC = torch.empty((N_S, N_S), dtype=torch.float32).pin_memory()
    lib.mbg_set_sync(1)

    def e2e_step():
        for ta, tb in (("N", "T"), ("T", "N")):
            st = lib.mbg_sgemm_ex(mode, ta.encode(), tb.encode(), n, n, n, 1.0, hA.data_ptr(), n, hB.data_ptr(), n,
                                  0.0, hC.data_ptr(), n)
            if st:
                raise RuntimeError(f"e2e call failed: {st} {L.last_error()}")
        return float(hC[0, 0])  # host read of the result

    e2e_step()
    if dist:
        dist.barrier()
    e2e_steps = max(10, args.steps // 2)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps, dist, "cuda")

    # the same through ordinary (pageable) host buffers, as a mojoBLAS caller passes them: the
    # library stages them through its page-locked bounce buffers
    pA = np.asfortranarray(hA.numpy().T)  # column-major n x n
    pB = np.asfortranarray(hB.numpy().T)
    pC = np.zeros((n, n), np.float32, order="F")

    def e2e_step_pageable():
        for ta, tb in (("N", "T"), ("T", "N")):
            st = lib.mbg_sgemm_ex(mode, ta.encode(), tb.encode(), n, n, n, 1.0, pA.ctypes.data, n, pB.ctypes.data,
                                  n, 0.0, pC.ctypes.data, n)
            if st:
                raise RuntimeError(f"e2e (pageable) call failed: {st} {L.last_error()}")
        return float(pC[0, 0])

    e2e_step_pageable()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step_pageable()
    e2e_pg_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps, dist, "cuda")
    del pA, pB, pC
    lib.mbg_set_sync(0)
    e2e_value = world * 2 * FLOPS_S / (e2e_ms * 1e-3) / 1e12
    bytes_in = 2 * 2 * N_S * N_S * 4  # A and B per call, two calls
    bytes_out = 2 * N_S * N_S * 4

    pk = peaks()
    achieved_tensor = nprod * FLOPS_S / (k_ms * 1e-3) / 1e12
    out = {
        "metric": "TFLOP/s at fixed FP64-oracle error (split-precision tensor-core sgemm vs plain FP32)",
        "value": round(value, 2),
        "unit": "TFLOP/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 (bf16 split terms, fp32 accumulation)",
        "data": "synthetic: uniform[-1,1) seeded (torch.Generator 1234+rank)",
        "config": {"workload": "large_gemm: sgemm NT + TN, M=N=K=8192, alpha=1, beta=0",
                   "mode": args.mode, "l2": "inputs larger than L2 (256 MiB each)",
                   "parallelism": f"replicas x{world}"},
        "plain_fp32_tflops": round(plain_tflops, 2),
        "speedup_vs_plain": round(value / plain_tflops, 2),
        f"{other}_tflops": round(world * 2 * FLOPS_S / (ms_other * 1e-3) / 1e12, 2),
        "fp64_oracle_error": errs,
        # the metric's "fixed error" condition: a split mode qualifies when its error is at or below plain
        # FP32's on every input set measured (uniform and scaled rows, NT and TN)
        "error_at_or_below_plain_fp32": {m_: all(v[m_] <= v["plain_fp32"] for v in errs.values() if m_ in v)
                                         for m_ in ("bf16x3", "bf16x6")},
        "error_metric": f"max|C-C64|/max|C64| over {SAMPLE_ROWS} sampled rows, C64 = float64 numpy",
        "dgemm_4096": dg,
        "dgemm_8192": dg8,
        "context_vendor_plain_gemm": ctx,
        "probe_peaks": probes,
        "cfg3": cfg3,
        "cfg4_batched": cfg4,
        "cfg5_adjoints": cfg5,
        "symm_syr2k_trmm": neighbours,
        "gemv_trsv": level2,
        "complex_gemm": cplx,
        "roofline_fractions": leg_fractions(dg, cfg3, cfg4, cfg5, probes, pk),
        "e2e": {"value": round(e2e_value, 2), "unit": "TFLOP/s", "h2d_bytes_per_step": bytes_in,
                "d2h_bytes_per_step": bytes_out, "ms_per_step": round(e2e_ms, 2), "host_memory": "pinned",
                "steps": e2e_steps},
        "e2e_pageable": {"value": round(world * 2 * FLOPS_S / (e2e_pg_ms * 1e-3) / 1e12, 2), "unit": "TFLOP/s",
                         "h2d_bytes_per_step": bytes_in, "d2h_bytes_per_step": bytes_out,
                         "ms_per_step": round(e2e_pg_ms, 2), "steps": e2e_steps,
                         "host_memory": "pageable numpy buffers, staged through page-locked bounce buffers",
                         "vs_pinned_time": round(e2e_pg_ms / e2e_ms, 2)},
        "gpu_launches": launches,
        "roofline": {"bound": "tensor", "kernel": kname.decode(),
                     "achieved": round(achieved_tensor, 1), "peak": pk["bf16"], "unit": "TFLOP/s",
                     "frac": round(achieved_tensor / pk["bf16"], 3),
                     # dram__bytes_read.sum + dram__bytes_write.sum of one full-size launch (8192^3 NT, bf16x6)
                     # from a single-pass ncu capture
                     "traffic": TRAFFIC_BF16X6_8192 if args.mode == "bf16x6" else None,
                     "traffic_unit": "bytes per launch",
                     "note": f"bf16 tensor flops = {nprod} products x 2MNK per launch / mean launch time "
                             f"({k_ms:.3f} ms); peak = {pk['source']} bf16 burst; traffic = "
                             f"{TRAFFIC_BF16X6_8192 / 1e9:.2f} GB against {PLANES_BF16X6_8192 / 1e9:.2f} GB of bf16 "
                             f"planes + C: the planes are re-read across output tiles",
                     "split_prepass_ms": round(split_ms, 3)},
        "clocks": clocks.summary(),
    }
    out["targets"] = targets_summary(value, plain_tflops, errs, args.mode, dg, dg8, cfg3)
    return out


def targets_summary(split_tflops, plain_tflops, errs, mode, dg, dg8, cfg3):
    """The 3x-at-equal-error targets, one compact entry per operation: plain and split /
    Ozaki TFLOP/s, their ratio, and the float64-oracle error of each (the maximum over
    the input sets measured).  Printed as the line's last key."""
    def entry(p_tf, s_tf, e_p, e_s, form):
        return {"form": form, "plain_tflops": p_tf, "split_tflops": s_tf,
                "ratio": round(s_tf / p_tf, 2) if p_tf else None,
                "err_plain": float(f"{e_p:.2g}") if e_p is not None else None,
                "err_split": float(f"{e_s:.2g}") if e_s is not None else None}
    t = {"sgemm_NT_TN_8192": entry(round(plain_tflops, 1), round(split_tflops, 1),
                                   max(v["plain_fp32"] for v in errs.values()),
                                   max(v[mode] for v in errs.values() if mode in v), mode)}

    def from_legs(legs, plain_key, split_key, err_key):
        if not legs or plain_key not in legs or split_key not in legs:
            return None
        p, q = legs[plain_key], legs[split_key]
        return entry(p["tflops"], q["tflops"], p.get(err_key), q.get(err_key), split_key)
    for name, legs, ek in (("dgemm_NN_4096", dg, "err_vs_compensated"), ("dgemm_NN_8192", dg8, "err_vs_compensated"),
                           ("dtrsm_LLNN_4096", cfg3.get("dtrsm_LLNN_4096"), "fp64_err"),
                           ("dtrsm_LLNN_8192", cfg3.get("dtrsm_LLNN_8192"), "fp64_err")):
        e = from_legs(legs, "plain_fp64", "ozaki_s7", ek)
        if e is not None:
            t[name] = e
    return t


_CPU_DATA = {}


def cpu_sample_cols(threads: int) -> int:
    """Columns of C in one CPU sample: at least the reference's parallel threshold (64,
    gemm.mojo:255 / :276, restated at oracle/ref_level3.cpp PAR_THRESHOLD), so the sampled
    _gemm_naive call takes the same multi-threaded branch as the full 8192-column call,
    and four columns per thread so the dynamic schedule keeps every thread busy."""
    return max(64, 4 * threads)


def run_cpu_baseline(args, threads=None, rows=None, calls=("NT", "TN")):
    """Reference algorithm (oracle restatement of _gemm_naive NT/TN) on host cores,
    over a bounded sample of each 8192^3 call in `calls`: rows 0..rows-1 of the first
    cpu_sample_cols(threads) columns of C (the reference parallelises over columns).
    Only full-height columns give the full call's rate: shorter ones keep more of A
    in cache (4096 rows already run 1.6x faster per flop).  `cores` is the thread
    count the oracle reports for the sampled call's column loop."""
    import oracle as orc
    nth = threads or os.cpu_count() or 1
    orc.set_threads(nth)
    n = N_S
    rows = n if rows is None else min(rows, n)
    if "ab" not in _CPU_DATA:
        rng = np.random.default_rng(1234)
        _CPU_DATA["ab"] = (np.asfortranarray(rng.uniform(-1, 1, (n, n)).astype(np.float32)),
                           np.asfortranarray(rng.uniform(-1, 1, (n, n)).astype(np.float32)))
    a, b = _CPU_DATA["ab"]
    cols = cpu_sample_cols(nth)
    c = np.zeros((n, cols), np.float32, order="F")
    used = []

    def sample(ta, tb):
        t0 = time.perf_counter()
        orc.gemm_naive(ta, tb, rows, cols, n, 1.0, a, n, b, n, 0.0, c, n)
        dt = time.perf_counter() - t0
        used.append(orc.naive_threads())
        return dt
    secs = sum(sample(cl[0], cl[1]) for cl in calls)
    flops = 2.0 * rows * n * cols * len(calls)
    cores = min(used)
    return {"value": flops / secs / 1e12, "unit": "TFLOP/s", "cores": cores, "kind": "port",
            "sample": f"rows 0..{rows - 1} x columns 0..{cols - 1} of C for {' and '.join(calls)} {n}^3 "
                      f"(2*{rows}*{n}*{cols} flop each), float32, mojoBLAS _gemm_naive restated "
                      f"(oracle/ref_level3.cpp), OpenMP, {cores} threads in the column loop",
            "seconds": round(secs, 3), "flops": flops, "columns": cols, "threads_used": cores}


def run_cpu_context_numpy(cols=512, min_seconds=1.0):
    """Context beside the CPU baseline: numpy's float32 matmul (the BLAS numpy ships) on the
    same 8192 x 8192 operands, columns 0..cols-1 of C for the NT and TN calls, repeated until
    min_seconds have passed (mean rate); threads as the BLAS library reports them."""
    n = N_S
    if "ab" not in _CPU_DATA:
        rng = np.random.default_rng(1234)
        _CPU_DATA["ab"] = (np.asfortranarray(rng.uniform(-1, 1, (n, n)).astype(np.float32)),
                           np.asfortranarray(rng.uniform(-1, 1, (n, n)).astype(np.float32)))
    a, b = _CPU_DATA["ab"]
    calls = {"NT": lambda: a @ b[:cols, :].T, "TN": lambda: a.T @ b[:, :cols]}
    for f in calls.values():
        f()  # warm-up: thread pool start, first touch of the result
    secs, reps = 0.0, 0
    while secs < min_seconds or reps < 2:
        for f in calls.values():
            t0 = time.perf_counter()
            f()
            secs += time.perf_counter() - t0
        reps += 1
    flops = 2.0 * n * n * cols * len(calls) * reps
    lib = {}
    try:
        from threadpoolctl import threadpool_info
        blas = [i for i in threadpool_info() if i.get("user_api") == "blas"]
        if blas:
            lib = {"library": f"{blas[0].get('internal_api')} {blas[0].get('version')}",
                   "threads": blas[0].get("num_threads")}
    except Exception as e:  # context only: a missing introspection module is reported, not fatal
        lib = {"library": f"unknown ({type(e).__name__})"}
    return {"value": round(flops / secs / 1e12, 3), "unit": "TFLOP/s", "kind": "numpy matmul (context)",
            "sample": f"columns 0..{cols - 1} of C for NT and TN 8192^3, float32, mean over {reps} repetitions",
            "seconds": round(secs, 3), **lib}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="bf16x6", choices=["bf16x3", "bf16x6"])
    ap.add_argument("--skip-dgemm", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-cfg3", action="store_true")
    ap.add_argument("--skip-cfg4", action="store_true")
    ap.add_argument("--skip-cfg5", action="store_true")
    ap.add_argument("--skip-neighbours", action="store_true")
    ap.add_argument("--skip-level2", action="store_true")
    ap.add_argument("--skip-complex", action="store_true")
    ap.add_argument("--skip-context", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        # each step is a bounded sample of the workload: 64 full-height columns of C (four per
        # thread above 16 threads) of the NT call (even steps, well under a second) or the TN call
        # (odd steps, about 4-10 s: the reference's TN loop reads A with a stride of lda), so K
        # steps plus W short warm-up samples stay within a few minutes
        for _ in range(args.warmup):
            run_cpu_baseline(args, rows=min(512, N_S))
        flops = secs = 0.0
        info = None
        for i in range(args.steps):
            info = run_cpu_baseline(args, calls=("NT",) if i % 2 == 0 else ("TN",))
            flops += info["flops"]
            secs += info["flops"] / (info["value"] * 1e12)  # the step's time, unrounded
        v = flops / secs / 1e12
        cols = info["columns"]
        info.update(sample=f"per step: rows 0..{N_S - 1} x columns 0..{cols - 1} of C of the NT (even steps) or TN "
                           f"(odd steps) {N_S}^3 call (2*{N_S}*{N_S}*{cols} flop), float32, mojoBLAS _gemm_naive "
                           f"restated (oracle/ref_level3.cpp), OpenMP, {info['cores']} threads in the column loop",
                    seconds=round(secs, 2), flops=flops)
        line = {"impl": "reference", "metric": "TFLOP/s at fixed FP64-oracle error (split-precision tensor-core "
                "sgemm vs plain FP32)", "value": v, "unit": "TFLOP/s", "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(1e3 * secs / args.steps, 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic: uniform[-1,1) seeded",
                "config": {"workload": "large_gemm: sgemm NT + TN, M=N=K=8192, alpha=1, beta=0"},
                "cpu_baseline": {**info, "value": v},
                "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    out = run_ours(args, rank, world, dist)
    if rank == 0 and not args.skip_cpu:
        cb = run_cpu_baseline(args)
        out["cpu_baseline"] = cb
        out["cpu_context_numpy"] = run_cpu_context_numpy()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        out["targets"] = out.pop("targets")  # last key: it stays in a truncated tail of the output
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
