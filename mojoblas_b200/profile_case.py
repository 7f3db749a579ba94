"""Run one library routine on cuda:0 a few times — the command profilers wrap.

    python mojoblas_b200/profile_case.py --op sgemm --mode bf16x6 --m 4096 --n 4096 --k 8192
    python mojoblas_b200/profile_case.py --op dgemm --mode ozaki --slices 8 --m 2048 --n 2048 --k 4096
    python mojoblas_b200/profile_case.py --op dtrsm --mode ozaki --m 4096 --n 4096
    python mojoblas_b200/profile_case.py --op strmm --mode bf16x6 --m 4096 --n 4096
    python mojoblas_b200/profile_case.py --op dgemv --ta N --m 8192 --n 8192
    python mojoblas_b200/profile_case.py --op dgemm --mode ozaki --slices 7 --pair 1 --m 4096 --n 4096 --k 4096
    python mojoblas_b200/profile_case.py --op grouped_sgemm --mode bf16x6
    python mojoblas_b200/profile_case.py --op zgemm --mode ozaki --slices 7 --m 2048 --n 2048 --k 2048
    python mojoblas_b200/profile_case.py --op strsm_adjoint --mode bf16x6 --m 2048 --n 512
    python mojoblas_b200/profile_case.py --op sgemm_adjoint --mode bf16x6 --m 3072 --n 2048 --k 1024

Inputs are uniform[-1, 1) (trsm, trmm: diagonally dominant lower triangle), device
resident; each rep is one call through the C ABI.  Prints the mean CUDA-event
time per call.
"""
from __future__ import annotations

import argparse
import ctypes as C
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--op", choices=["sgemm", "dgemm", "cgemm", "zgemm", "ssyrk", "dtrsm", "strsm", "grouped_sgemm",
                                     "grouped_strsm",
                                     "strmm", "dtrmm", "ssymm", "dsymm", "ssyr2k", "dsyr2k",
                                     "sgemv", "dgemv", "strsv", "dtrsv", "strsm_adjoint", "sgemm_adjoint"],
                    default="sgemm")
    ap.add_argument("--mode", choices=["plain", "bf16x3", "bf16x6", "ozaki"], default="bf16x6")
    ap.add_argument("--slices", type=int, default=8)
    ap.add_argument("--refine", type=int, default=0)
    ap.add_argument("--ta", default="N")
    ap.add_argument("--tb", default="T")
    ap.add_argument("--m", type=int, default=4096)
    ap.add_argument("--n", type=int, default=4096)
    ap.add_argument("--k", type=int, default=8192)
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--beta", type=float, default=0.0, help="gemm: C := A B + beta C (1: the trsm update form)")
    ap.add_argument("--pair", type=int, default=-1, help="Ozaki kernel: 1 CTA pairs, 0 one CTA per tile")
    a = ap.parse_args()

    import torch
    from mojoblas_b200 import _lib as L
    lib = L.load()
    torch.cuda.set_device(0)
    lib.mbg_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))
    lib.mbg_set_sync(0)
    mode = {"plain": L.MODE_PLAIN, "bf16x3": L.MODE_BF16X3, "bf16x6": L.MODE_BF16X6, "ozaki": L.MODE_OZAKI}[a.mode]
    if a.pair >= 0:
        assert lib.mbg_set_tuning(b"ozaki_cta_pair", a.pair) == 0
    dt = torch.float64 if a.op[0] in "dz" else torch.float32
    g = torch.Generator(device="cuda")
    g.manual_seed(0)

    def cm(rows, cols):  # column-major rows x cols
        return torch.rand((cols, rows), generator=g, device="cuda", dtype=dt) * 2 - 1

    if a.op == "grouped_sgemm":  # 4096 problems, m, n, k log-uniform 16..512
        from mojoblas_b200.autotune import sgemm_batch
        buf, probs, _, _ = sgemm_batch(torch, L, 4096, seed=41)
        plan = C.c_void_p()
        assert lib.mbg_sgemm_grouped_plan(mode, len(probs), probs, C.byref(plan)) == 0, L.last_error()

        def call():
            return lib.mbg_plan_execute(plan)
    elif a.op == "grouped_strsm":  # 2048 lower solves, n log-uniform 8..256, nrhs 1..64
        import numpy as np
        from mojoblas_b200.autotune import log_uniform
        rng = np.random.default_rng(42)
        ns, rh = log_uniform(rng, 8, 256, 2048), rng.integers(1, 65, 2048)
        sizes = [int(x * x) for x in ns] + [int(x * y) for x, y in zip(ns, rh)]
        tot = sum((v + 63) // 64 * 64 for v in sizes)
        buf = torch.randn(tot, generator=g, device="cuda") * 0.01
        probs = (L.StrsmProblem * 2048)()
        off = 0
        base = buf.data_ptr()
        for i in range(2048):
            ai = off
            off += (int(ns[i] * ns[i]) + 63) // 64 * 64
            bi = off
            off += (int(ns[i] * rh[i]) + 63) // 64 * 64
            buf[ai:ai + int(ns[i] * ns[i]):int(ns[i]) + 1] = float(ns[i])  # dominant diagonal
            probs[i] = L.StrsmProblem(b"L", b"L", b"N", b"N", int(ns[i]), int(rh[i]), 1.0, base + 4 * ai,
                                      int(ns[i]), base + 4 * bi, int(ns[i]))
        plan = C.c_void_p()
        assert lib.mbg_strsm_grouped_plan(L.MODE_PLAIN, 2048, probs, C.byref(plan)) == 0, L.last_error()

        def call():
            return lib.mbg_plan_execute(plan)
    elif a.op in ("sgemm", "dgemm"):
        lda = a.m if a.ta == "N" else a.k
        ldb = a.k if a.tb == "N" else a.n
        A, B, Cm = cm(lda, a.k if a.ta == "N" else a.m), cm(ldb, a.n if a.tb == "N" else a.k), cm(a.m, a.n)

        def call():
            if a.op == "sgemm":
                return lib.mbg_sgemm_ex(mode, a.ta.encode(), a.tb.encode(), a.m, a.n, a.k, 1.0, A.data_ptr(), lda,
                                        B.data_ptr(), ldb, a.beta, Cm.data_ptr(), a.m)
            return lib.mbg_dgemm_ex(mode, a.slices, a.ta.encode(), a.tb.encode(), a.m, a.n, a.k, 1.0, A.data_ptr(),
                                    lda, B.data_ptr(), ldb, a.beta, Cm.data_ptr(), a.m)
    elif a.op in ("cgemm", "zgemm"):  # complex, interleaved (re, im): a real buffer of twice the rows
        lda = a.m if a.ta == "N" else a.k
        ldb = a.k if a.tb == "N" else a.n
        A, B, Cm = cm(2 * lda, a.k if a.ta == "N" else a.m), cm(2 * ldb, a.n if a.tb == "N" else a.k), cm(2 * a.m, a.n)
        import numpy as np
        al = np.array([1.0, 0.0], np.float64 if a.op == "zgemm" else np.float32)
        be = np.zeros(2, al.dtype)

        def call():
            args = (a.ta.encode(), a.tb.encode(), a.m, a.n, a.k, al.ctypes.data, A.data_ptr(), lda, B.data_ptr(), ldb,
                    be.ctypes.data, Cm.data_ptr(), a.m)
            if a.op == "cgemm":
                return lib.mbg_cgemm_ex(mode, *args)
            return lib.mbg_zgemm_ex(mode, a.slices, *args)
    elif a.op == "ssyrk":
        A, Cm = cm(a.n, a.k), cm(a.n, a.n)

        def call():
            return lib.mbg_ssyrk_ex(mode, b"L", b"N", a.n, a.k, 1.0, A.data_ptr(), a.n, 0.0, Cm.data_ptr(), a.n)
    elif a.op in ("sgemv", "dgemv"):  # y = 1.5 op(A) x + 0.5 y, A m x n, op by --ta
        A, x, y = cm(a.m, a.n), cm(max(a.m, a.n), 1), cm(max(a.m, a.n), 1)

        def call():
            args = (a.ta.encode(), a.m, a.n, 1.5, A.data_ptr(), a.m, x.data_ptr(), 1, 0.5, y.data_ptr(), 1)
            return lib.mbg_sgemv(*args) if a.op == "sgemv" else lib.mbg_dgemv(*args)
    elif a.op in ("strsv", "dtrsv"):  # Lower, NoTrans, NonUnit, order --m, diagonally dominant
        A = torch.randn((a.m, a.m), generator=g, device="cuda", dtype=dt) / a.m ** 0.5
        A.diagonal().copy_(2.0 + torch.rand(a.m, generator=g, device="cuda", dtype=dt))
        b0 = torch.randn(a.m, generator=g, device="cuda", dtype=dt)
        xb = b0.clone()

        def call():
            xb.copy_(b0)
            args = (b"L", b"N", b"N", a.m, A.data_ptr(), a.m, xb.data_ptr(), 1)
            return lib.mbg_strsv(*args) if a.op == "strsv" else lib.mbg_dtrsv(*args)
    elif a.op == "strsm_adjoint":  # L (m x m lower, dominant diagonal), X and G m x n: dB, dL
        import numpy as np
        Lm = torch.randn((a.m, a.m), generator=g, device="cuda") / np.sqrt(a.m)
        Lm.diagonal().add_(a.m)
        Lm = torch.tril(Lm.T).T.contiguous()
        X, G = cm(a.m, a.n), cm(a.m, a.n)
        dB, dL = torch.zeros_like(X), torch.zeros_like(Lm)

        def call():
            return lib.mbg_strsm_adjoint(mode, b"L", b"L", b"N", b"N", a.m, a.n, 1.0, Lm.data_ptr(), a.m, X.data_ptr(),
                                         a.m, G.data_ptr(), a.m, dB.data_ptr(), a.m, dL.data_ptr(), a.m)
    elif a.op == "sgemm_adjoint":  # C = A B (A m x k, B k x n, NN): dA = G B^T, dB = A^T G
        A, B, G = cm(a.m, a.k), cm(a.k, a.n), cm(a.m, a.n)
        dA, dB = torch.zeros_like(A), torch.zeros_like(B)

        def call():
            return lib.mbg_sgemm_adjoint(mode, b"N", b"N", a.m, a.n, a.k, 1.0, A.data_ptr(), a.m, B.data_ptr(), a.k,
                                         G.data_ptr(), a.m, dA.data_ptr(), a.m, dB.data_ptr(), a.k)
    elif a.op in ("ssymm", "dsymm"):  # Left, Upper: C (m x n) = A (m x m, symmetric) B
        A, B, Cm = cm(a.m, a.m), cm(a.m, a.n), cm(a.m, a.n)

        def call():
            args = (b"L", b"U", a.m, a.n, 1.0, A.data_ptr(), a.m, B.data_ptr(), a.m, 0.0, Cm.data_ptr(), a.m)
            return lib.mbg_ssymm_ex(mode, *args) if a.op == "ssymm" else lib.mbg_dsymm_ex(mode, a.slices, *args)
    elif a.op in ("ssyr2k", "dsyr2k"):  # Lower, NoTrans: A, B n x k
        A, B, Cm = cm(a.n, a.k), cm(a.n, a.k), cm(a.n, a.n)

        def call():
            args = (b"L", b"N", a.n, a.k, 1.0, A.data_ptr(), a.n, B.data_ptr(), a.n, 0.0, Cm.data_ptr(), a.n)
            return lib.mbg_ssyr2k_ex(mode, *args) if a.op == "ssyr2k" else lib.mbg_dsyr2k_ex(mode, a.slices, *args)
    else:
        m = a.m
        A = torch.randn((m, m), generator=g, device="cuda", dtype=dt) / m ** 0.5
        A.diagonal().copy_(m + torch.rand(m, generator=g, device="cuda", dtype=dt))
        B0 = torch.randn((a.n, m), generator=g, device="cuda", dtype=dt)
        X = B0.clone()

        def call():
            X.copy_(B0)
            if a.op in ("strmm", "dtrmm"):  # Left, Lower, NoTrans, NonUnit
                args = (b"L", b"L", b"N", b"N", m, a.n, 1.0, A.data_ptr(), m, X.data_ptr(), m)
                return lib.mbg_strmm_ex(mode, *args) if a.op == "strmm" else lib.mbg_dtrmm_ex(mode, a.slices, *args)
            if a.op == "dtrsm":
                return lib.mbg_dtrsm_ex(mode, a.slices, a.refine, b"L", b"L", b"N", b"N", m, a.n, 1.0, A.data_ptr(),
                                        m, X.data_ptr(), m)
            return lib.mbg_strsm_ex(mode, a.refine, b"L", b"L", b"N", b"N", m, a.n, 1.0, A.data_ptr(), m,
                                    X.data_ptr(), m)

    st = call()
    assert st == 0, L.last_error()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        st = call()
        assert st == 0, L.last_error()
    e1.record()
    torch.cuda.synchronize()
    print(f"{a.op} {a.mode} m={a.m} n={a.n} k={a.k}: {e0.elapsed_time(e1) / a.reps:.3f} ms per call")


if __name__ == "__main__":
    main()
