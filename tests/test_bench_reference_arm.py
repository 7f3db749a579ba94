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


def test_reference_arm_other_ranks_do_nothing(monkeypatch, capsys):
    out = run_main(monkeypatch, capsys, ["--impl", "reference", "--steps", "1"],
                   env={"RANK": "1", "WORLD_SIZE": "2"})
    assert out == ""
