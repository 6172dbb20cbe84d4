"""bench.py's stdout contract: one JSON line of at most a few KB, whatever the
run measured; curves and sweeps go to the side file.  Runs main() on a stub
measurement (no GPU)."""
import importlib
import io
import json
import os
import sys
from contextlib import redirect_stdout

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _big_result():
    curve = [{"ef": e, "bf_words": b, "recall_cal": 0.9, "qps": 1e6} for e in range(64, 1100, 4)
             for b in (256, 512, 1024)]
    line = {
        "metric": "QPS", "value": 6.6e6, "unit": "queries/s", "n_gpus": 1, "steps": 20,
        "warmup": 5, "ms_per_step": 1.5, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "w" * 100}, "recall_at_10": 0.951,
        "e2e": {"value": 5.9e6, "unit": "queries/s", "h2d_bytes_per_step": 1, "d2h_bytes_per_step": 1},
        "gpu_launches": 40, "roofline": {"bound": "hbm", "frac": 0.1}, "cpu_baseline": {"value": 1.0},
        "clocks": {"sm_mhz": 1965},
        "configs": {f"c{i}": {"curve": curve[:40]} for i in range(6)},
        "forms": {"plain": {"qps": 1e6}, "learned": {"qps": 6.6e6, "x": "y" * 3000}},
    }
    return line, {"plain_curve": curve, "kernel_ms": [1.0] * 1000}


def test_main_prints_one_short_parseable_line(tmp_path, monkeypatch):
    bench = importlib.import_module("bench")
    monkeypatch.setattr(bench, "run_ours", lambda args, ws, rank, local: _big_result())
    side = tmp_path / "details.json"
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.main(["--details", str(side)]) == 0
    lines = [l for l in buf.getvalue().splitlines() if l.strip()]
    assert len(lines) == 1
    assert len(lines[-1].encode()) <= 4096
    out = json.loads(lines[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "dtype", "config", "e2e", "roofline", "cpu_baseline",
                "clocks", "recall_at_10", "gpu_launches"):
        assert key in out, key
    details = json.loads(side.read_text())
    assert len(details["plain_curve"]) > 100          # the curves live in the side file
    assert details["line"]["value"] == out["value"]


def test_compact_line_keeps_small_lines_whole():
    bench = importlib.import_module("bench")
    small = {"metric": "m", "value": 1.0, "configs": {"a": [1, 2]}}
    assert json.loads(bench.compact_line(small)) == small
