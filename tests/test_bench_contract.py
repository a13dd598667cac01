"""bench.py's reference arm (the FP64 restatement of the timestep on the host
cores) prints one JSON line with the keys the bench contract names. The arm
needs no GPU; here it runs on two host threads."""
import contextlib
import importlib.util
import io
import json
import os
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    return bench


def test_reference_arm_prints_the_contract_line(monkeypatch):
    bench = load_bench()
    monkeypatch.setattr(bench.os, "cpu_count", lambda: 2)
    args = types.SimpleNamespace(gpus=1, steps=4, warmup=0, impl="reference")
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.reference_arm(args, 0)
    lines = out.getvalue().strip().splitlines()
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["unit"] == "sim-days/s" and line["value"] > 0 and line["higher_is_better"] is True
    assert line["n_gpus"] == 1 and line["steps"] == 4 and line["warmup"] == 0
    assert line["e2e"] == {"value": line["value"], "unit": "sim-days/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}
    cpu = line["cpu_baseline"]
    assert cpu["kind"] == "port" and cpu["cores"] == 2 and cpu["value"] == line["value"] and cpu["sample"]
    assert line["config"]["workload"] and line["config"]["planets"] == 2


def test_reference_arm_is_silent_on_other_ranks(monkeypatch):
    bench = load_bench()
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.reference_arm(types.SimpleNamespace(gpus=2, steps=4, warmup=0, impl="reference"), 1)
    assert out.getvalue() == ""
