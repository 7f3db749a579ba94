"""The reference arm of bench.py (`--impl reference`): the one JSON line it prints
carries the base contract's keys, `impl: "reference"`, a `cpu_baseline` whose
value is the line's, and an `e2e` with no host-device bytes; under torchrun only
rank 0 does work and prints.  The workload is shrunk (N_S = 256) so the arm runs
in well under a second; the code path is the one the full-size run takes."""
import json
import sys

import bench

KEYS = ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
        "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e")


def run_main(monkeypatch, capsys, argv, env=None):
    monkeypatch.setattr(bench, "N_S", 256)
    monkeypatch.setattr(bench, "_CPU_DATA", {})
    monkeypatch.setattr(sys, "argv", ["bench.py"] + argv)
    for k, v in (env or {}).items():
        monkeypatch.setenv(k, v)
    bench.main()
    return capsys.readouterr().out


def test_reference_arm_line(monkeypatch, capsys):
    out = run_main(monkeypatch, capsys, ["--impl", "reference", "--steps", "2", "--warmup", "1"],
                   env={"RANK": "0", "WORLD_SIZE": "1"})
    lines = [ln for ln in out.splitlines() if ln.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert all(k in d for k in KEYS), [k for k in KEYS if k not in d]
    assert d["impl"] == "reference"
    assert d["steps"] == 2 and d["warmup"] == 3  # at least three warm-up steps, whatever is asked
    assert d["value"] > 0 and d["higher_is_better"] is True and d["unit"] == "TFLOP/s"
    cb = d["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == d["value"] and "256^3" in cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("large_gemm")


def test_cpu_sample_reaches_the_parallel_branch():
    """The sampled _gemm_naive call has at least the reference's 64-column parallel
    threshold (gemm.mojo:255), so it runs multi-threaded like the full 8192-column call,
    and the line's `cores` is the thread count the oracle saw in the column loop."""
    import oracle as orc
    assert bench.cpu_sample_cols(1) >= 64 and bench.cpu_sample_cols(16) >= 64
    assert bench.cpu_sample_cols(32) == 128
    cb = bench.run_cpu_baseline(None, threads=2, rows=64, calls=("NT",))
    assert cb["columns"] >= 64
    assert cb["cores"] == cb["threads_used"] == 2, cb
    # below the threshold the restated loop stays serial, as the reference's does
    import numpy as np
    a = np.asfortranarray(np.ones((32, 32), np.float32))
    c = np.zeros((32, 16), np.float32, order="F")
    orc.set_threads(2)
    orc.gemm_naive("N", "N", 32, 16, 32, 1.0, a, 32, a, 32, 0.0, c, 32)
    assert orc.naive_threads() == 1


def test_reference_arm_other_ranks_do_nothing(monkeypatch, capsys):
    out = run_main(monkeypatch, capsys, ["--impl", "reference", "--steps", "1"],
                   env={"RANK": "1", "WORLD_SIZE": "2"})
    assert out == ""
