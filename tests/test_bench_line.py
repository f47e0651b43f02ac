"""The bench's printed line (CPU): from a full line recorded by a run with
every section (`--steps 20 --warmup 5`; tests/data/bench_line_full.json), the
compacted line keeps every key of the bench contract and stays well under
the 3,000 characters of a log tail."""
import importlib.util
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    argv = sys.argv
    try:
        sys.argv = ["bench.py"]
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def test_compact_line_keeps_the_contract_and_fits():
    b = _bench()
    full = json.loads((ROOT / "tests" / "data" / "bench_line_full.json").read_text())
    line = b._compact(full)
    text = json.dumps(line)
    assert len(text) < 2950, len(text)
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "roofline", "cpu_baseline", "e2e", "clocks", "gpu_launches"):
        assert k in line, k
    assert "workload" in line["config"] and "l2" in line["config"]
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in line["roofline"], k
    for k in ("value", "unit", "cores", "kind", "sample"):
        assert k in line["cpu_baseline"], k
    for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"):
        assert k in line["e2e"], k
    assert line["higher_is_better"] is True and line["n_gpus"] == 1
    assert abs(line["roofline"]["frac"] - line["roofline"]["achieved"] / line["roofline"]["peak"]) < 1e-3
