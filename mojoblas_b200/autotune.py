"""Autotuner: sweeps the library's tunable choices on the current GPU and writes
the fastest into a tuning table that libmojoblas_gpu.so loads with
mbg_load_tuning (mojoblas_b200.load_tuning applies it from Python).

    python -m mojoblas_b200.autotune [--out mojoblas_b200/tuning_b200.json]

Keys swept:
  grouped_gemm_tile  64 or 128 — tile edge of grouped sgemm plans, timed on a
                     batch of 4096 problems with m, n, k log-uniform in 16..512
                     (the batched configuration's distribution);
  trsm_tc_min_k      128 .. 1024 — the reduction length below which the
                     blocked trsm's off-diagonal updates stay on the plain
                     kernel, timed on dtrsm 4096^2 with 8-slice Ozaki updates.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))

DEFAULT_OUT = Path(__file__).resolve().parent / "tuning_b200.json"


def log_uniform(rng, lo, hi, size):
    return np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), size))).astype(np.int64)


def sgemm_batch(torch, L, count=4096, seed=0):
    """count problems NN, m, n, k log-uniform 16..512, uniform[-1,1) data on the device."""
    rng = np.random.default_rng(seed)
    m, n, k = (log_uniform(rng, 16, 512, count) for _ in range(3))
    sizes = m * k + k * n + m * n
    offs = np.concatenate([[0], np.cumsum((sizes + 63) // 64 * 64)])
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    buf = torch.rand(int(offs[-1]), generator=g, device="cuda") * 2 - 1
    base = buf.data_ptr()
    probs = (L.SgemmProblem * count)()
    for i in range(count):
        pa = base + 4 * int(offs[i])
        pb = pa + 4 * int(m[i] * k[i])
        pc = pb + 4 * int(k[i] * n[i])
        probs[i] = L.SgemmProblem(b"N", b"N", int(m[i]), int(n[i]), int(k[i]), 1.0, 0.0, pa, int(m[i]), pb,
                                  int(k[i]), pc, int(m[i]))
    flops = float(np.sum(2.0 * m * n * k))
    return buf, probs, (m, n, k, offs), flops


def time_plan(torch, lib, plan, reps=20):
    lib.mbg_plan_execute(plan)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        lib.mbg_plan_execute(plan)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def tune(out: Path) -> dict:
    import torch
    from mojoblas_b200 import _lib as L
    lib = L.load()
    torch.cuda.set_device(0)
    lib.mbg_set_stream(C.c_void_p(torch.cuda.current_stream().cuda_stream))
    lib.mbg_set_sync(0)
    table, log = {}, {}

    buf, probs, _, flops = sgemm_batch(torch, L)
    best = None
    for tile in (64, 128):
        lib.mbg_set_tuning(b"grouped_gemm_tile", tile)
        plan = C.c_void_p()
        st = lib.mbg_sgemm_grouped_plan(L.MODE_PLAIN, len(probs), probs, C.byref(plan))
        if st:
            raise RuntimeError(L.last_error())
        ms = time_plan(torch, lib, plan)
        lib.mbg_plan_destroy(plan)
        log[f"grouped_gemm_tile={tile}"] = {"ms": round(ms, 4), "tflops": round(flops / ms / 1e9, 2)}
        if best is None or ms < best[1]:
            best = (tile, ms)
    table["grouped_gemm_tile"] = best[0]
    lib.mbg_set_tuning(b"grouped_gemm_tile", best[0])
    del buf

    n = 4096
    A = torch.randn(n, n, dtype=torch.float64, device="cuda") / n ** 0.5
    A.diagonal().copy_(n + torch.rand(n, dtype=torch.float64, device="cuda"))
    B0 = torch.randn(n, n, dtype=torch.float64, device="cuda")
    X = B0.clone()
    best = None
    for thr in (128, 256, 512, 1024):
        lib.mbg_set_tuning(b"trsm_tc_min_k", thr)

        def call():
            X.copy_(B0)
            st = lib.mbg_dtrsm_ex(L.MODE_OZAKI, 8, 0, b"L", b"L", b"N", b"N", n, n, 1.0, A.data_ptr(), n,
                                  X.data_ptr(), n)
            if st:
                raise RuntimeError(L.last_error())
        call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            call()
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 3
        log[f"trsm_tc_min_k={thr}"] = {"ms": round(ms, 3)}
        if best is None or ms < best[1]:
            best = (thr, ms)
    table["trsm_tc_min_k"] = best[0]
    lib.mbg_set_tuning(b"trsm_tc_min_k", best[0])

    doc = {**table, "_measurements": log, "_device": torch.cuda.get_device_name(0)}
    out.write_text(json.dumps(doc, indent=1) + "\n")
    return doc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(DEFAULT_OUT))
    args = ap.parse_args()
    print(json.dumps(tune(Path(args.out))))


if __name__ == "__main__":
    main()
