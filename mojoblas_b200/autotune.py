"""Autotuner: sweeps the library's tunable choices on the current GPU and writes
the fastest into a tuning table that libmojoblas_gpu.so loads with
mbg_load_tuning (mojoblas_b200.load_tuning applies it from Python).

    python -m mojoblas_b200.autotune [--out mojoblas_b200/tuning_b200.json]

Keys swept:
  grouped_simt_tile_<TT>_c<d>   per transposes TT (NN, NT, TN, TT) and size
  grouped_tc_bn_<TT>_c<d>       class d of max(m, n) (0: <= 32, 1: <= 64,
                     2: <= 128, 3: <= 256, 4: <= 512): the tile edge (64 / 128)
                     of the plain grouped sgemm and the tile width (64 / 128) of
                     the split (BF16x6, tensor-core) grouped sgemm, each timed on
                     a batch of problems of that class (m and n log-uniform within
                     the class, k log-uniform in 16..512, the batched
                     configuration's distribution);
  grouped_gemm_tile  the plain form's tile for classes without an entry: the
                     faster one on the whole configuration batch (4096 problems,
                     m, n, k log-uniform in 16..512);
  trsm_block_rows    0 (64-row leaves), 256, 512 — diagonal blocks solved in
  trsm_tc_min_k      one fused launch, and the reduction length below which
                     the blocked trsm's off-diagonal updates stay on the plain
                     kernel; swept jointly on dtrsm 4096^2 with Ozaki
                     updates (the blocked-trsm configuration);
  trsm_block_min_cols  the fewest right-hand sides for which the fused launch
                     beats the 64-row leaves, timed on dtrsm 4096 x nrhs;
  trsm_inverse_min_cols  the fewest right-hand sides for which the Ozaki trsm's
                     inverted diagonal blocks beat substitution leaves.
Labels in the measurement log avoid the key names, since the library's loader
reads the table as "key value" pairs.
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
ROUNDS = 5  # interleaved timing rounds per trsm candidate


def log_uniform(rng, lo, hi, size):
    return np.round(np.exp(rng.uniform(np.log(lo), np.log(hi), size))).astype(np.int64)


CLASS_BOUNDS = [(16, 32), (33, 64), (65, 128), (129, 256), (257, 512)]  # max(m, n) per size class


def sgemm_batch(torch, L, count=4096, seed=0, mn=(16, 512), trans=("N", "N")):
    """count problems, m, n log-uniform in mn, k log-uniform 16..512, transposes `trans`,
    uniform[-1,1) data on the device (leading dimensions the stored row counts)."""
    rng = np.random.default_rng(seed)
    m, n = (log_uniform(rng, mn[0], mn[1], count) for _ in range(2))
    k = log_uniform(rng, 16, 512, count)
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
        lda = int(m[i]) if trans[0] == "N" else int(k[i])
        ldb = int(k[i]) if trans[1] == "N" else int(n[i])
        probs[i] = L.SgemmProblem(trans[0].encode(), trans[1].encode(), int(m[i]), int(n[i]), int(k[i]), 1.0, 0.0,
                                  pa, lda, pb, ldb, pc, int(m[i]))
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

    def plan_ms(mode, probs):
        plan = C.c_void_p()
        st = lib.mbg_sgemm_grouped_plan(mode, len(probs), probs, C.byref(plan))
        if st:
            raise RuntimeError(L.last_error())
        try:
            return time_plan(torch, lib, plan)
        finally:
            lib.mbg_plan_destroy(plan)

    buf, probs, _, flops = sgemm_batch(torch, L)
    best = None
    for tile in (64, 128):
        lib.mbg_set_tuning(b"grouped_gemm_tile", tile)
        ms = plan_ms(L.MODE_PLAIN, probs)
        log[f"grouped sgemm tile {tile}"] = {"ms": round(ms, 4), "tflops": round(flops / ms / 1e9, 2)}
        if best is None or ms < best[1]:
            best = (tile, ms)
    table["grouped_gemm_tile"] = best[0]
    lib.mbg_set_tuning(b"grouped_gemm_tile", best[0])
    del buf

    # per transposes and size class: the plain form's tile edge, the split form's tile width
    for ta in "NT":
        for tb in "NT":
            for cls, bounds in enumerate(CLASS_BOUNDS):
                buf, probs, _, flops = sgemm_batch(torch, L, count=512, seed=100 + cls, mn=bounds, trans=(ta, tb))
                for prefix, mode, label in (("grouped_simt_tile", L.MODE_PLAIN, "plain"),
                                            ("grouped_tc_bn", L.MODE_BF16X6, "bf16x6")):
                    key = f"{prefix}_{ta}{tb}_c{cls}"
                    times = {}
                    for v in (64, 128):
                        lib.mbg_set_tuning(key.encode(), v)
                        times[v] = plan_ms(mode, probs)
                    choice = min(times, key=times.get)
                    table[key] = choice
                    lib.mbg_set_tuning(key.encode(), choice)
                    log[f"grouped sgemm {label} {ta}{tb} max(m,n) in {bounds}, tile 64 / 128"] = {
                        "ms": [round(times[64], 4), round(times[128], 4)],
                        "tflops": [round(flops / times[64] / 1e9, 2), round(flops / times[128] / 1e9, 2)]}
                del buf

    n = 4096
    A = torch.randn(n, n, dtype=torch.float64, device="cuda") / n ** 0.5
    A.diagonal().copy_(n + torch.rand(n, dtype=torch.float64, device="cuda"))
    B0 = torch.randn(n, n, dtype=torch.float64, device="cuda")
    X = B0.clone()

    def time_trsm(mode, nrhs, reps=3):
        def call():
            X[:nrhs].copy_(B0[:nrhs])  # column-major: the first nrhs columns
            st = lib.mbg_dtrsm_ex(mode, 7, 0, b"L", b"L", b"N", b"N", n, nrhs, 1.0, A.data_ptr(), n,
                                  X.data_ptr(), n)
            if st:
                raise RuntimeError(L.last_error())
        call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            call()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    lib.mbg_set_tuning(b"trsm_block_min_cols", 1)
    # the keys swept here govern the substitution path: the fused diagonal blocks' rows (the
    # plain solve's, and the split / Ozaki solves' below trsm_inverse_min_cols right-hand sides),
    # chosen on the plain FP64 solve; then the k from which the substitution path's updates
    # are split / Ozaki products, chosen on the Ozaki solve with the inverted-block path off.
    # Candidates are timed in interleaved rounds and ranked by their median, so that a clock
    # or power-cap drift during the sweep does not favour whichever ran first.
    lib.mbg_set_tuning(b"trsm_inverse_min_cols", 0)
    samples = {rows: [] for rows in (0, 256, 512)}
    for _ in range(ROUNDS):
        for rows in samples:
            lib.mbg_set_tuning(b"trsm_block_rows", rows)
            samples[rows].append(time_trsm(L.MODE_PLAIN, n))
    med = {rows: float(np.median(v)) for rows, v in samples.items()}
    for rows, ms in med.items():
        log[f"plain dtrsm 4096^2, fused rows {rows}"] = {"ms_median": round(ms, 3), "rounds": ROUNDS}
    rows_best = min(med, key=med.get)
    lib.mbg_set_tuning(b"trsm_block_rows", rows_best)
    samples = {thr: [] for thr in (256, 512, 1024)}
    for _ in range(ROUNDS):
        for thr in samples:
            lib.mbg_set_tuning(b"trsm_tc_min_k", thr)
            samples[thr].append(time_trsm(L.MODE_OZAKI, n))
    med = {thr: float(np.median(v)) for thr, v in samples.items()}
    for thr, ms in med.items():
        log[f"ozaki dtrsm 4096^2 (substitution), fused rows {rows_best}, split from k {thr}"] = {
            "ms_median": round(ms, 3), "rounds": ROUNDS}
    best = (rows_best, min(med, key=med.get))
    table["trsm_block_rows"], table["trsm_tc_min_k"] = best[0], best[1]
    lib.mbg_set_tuning(b"trsm_block_rows", best[0])
    lib.mbg_set_tuning(b"trsm_tc_min_k", best[1])

    # smallest right-hand-side count from which the fused blocks win (plain dtrsm 4096 x nrhs)
    min_cols = n  # fused blocks won at n right-hand sides in the sweep above
    if best[0] > 64:
        for nrhs in (2048, 1024, 512, 256, 128, 64):
            lib.mbg_set_tuning(b"trsm_block_rows", best[0])
            fused = time_trsm(L.MODE_PLAIN, nrhs)
            lib.mbg_set_tuning(b"trsm_block_rows", 0)
            leaves = time_trsm(L.MODE_PLAIN, nrhs)
            log[f"plain dtrsm 4096 x {nrhs}: fused vs leaves"] = {"ms": [round(fused, 3), round(leaves, 3)]}
            if fused <= leaves:
                min_cols = nrhs
            else:
                break
        lib.mbg_set_tuning(b"trsm_block_rows", best[0])
    table["trsm_block_min_cols"] = min_cols
    lib.mbg_set_tuning(b"trsm_block_min_cols", min_cols)

    # smallest right-hand-side count from which the Ozaki trsm's inverted diagonal blocks win
    inv_cols = 0
    for nrhs in (2048, 1024, 512, 256, 128, 64):
        lib.mbg_set_tuning(b"trsm_inverse_min_cols", 1)
        inv = time_trsm(L.MODE_OZAKI, nrhs)
        lib.mbg_set_tuning(b"trsm_inverse_min_cols", 0)
        sub = time_trsm(L.MODE_OZAKI, nrhs)
        log[f"ozaki dtrsm 4096 x {nrhs}: inverted blocks vs substitution"] = {"ms": [round(inv, 3), round(sub, 3)]}
        if inv <= sub:
            inv_cols = nrhs
        else:
            break
    table["trsm_inverse_min_cols"] = inv_cols
    lib.mbg_set_tuning(b"trsm_inverse_min_cols", inv_cols)

    # rows of the inverted diagonal blocks (Ozaki dtrsm 4096^2), interleaved rounds, medians
    if inv_cols:
        samples = {256: [], 512: []}
        for _ in range(ROUNDS):
            for blk in samples:
                lib.mbg_set_tuning(b"trsm_inverse_block", blk)
                samples[blk].append(time_trsm(L.MODE_OZAKI, n))
        med = {blk: float(np.median(v)) for blk, v in samples.items()}
        for blk, ms in med.items():
            log[f"ozaki dtrsm 4096^2, inverted blocks of {blk} rows"] = {"ms_median": round(ms, 3),
                                                                        "rounds": len(samples[blk])}
        table["trsm_inverse_block"] = min(med, key=med.get)
        lib.mbg_set_tuning(b"trsm_inverse_block", table["trsm_inverse_block"])

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
