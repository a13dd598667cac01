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
    assert cpu["cpu_model"] and cpu["host_threads"] >= 1
    assert line["config"]["workload"] and line["config"]["planets"] == 2


def test_reference_arm_is_silent_on_other_ranks():
    bench = load_bench()
    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.reference_arm(types.SimpleNamespace(gpus=2, steps=4, warmup=0, impl="reference"), 1)
    assert out.getvalue() == ""


def test_roofline_takes_the_dominant_hbm_kernel_and_its_committed_traffic():
    """roofline() times every kernel of PER_STEP, picks the HBM-bound one with
    the most time per step, and reports its algorithmic bytes over its launch
    time against the measured peak (or the fallback), with the DRAM traffic
    of its committed ncu summary."""
    bench = load_bench()
    times = {k: 0.01 for k in bench.PER_STEP}
    times["fourier_forward"] = 0.0175
    nbytes = 70123520.0

    class Engine:
        def time_kernel(self, kernel, reps):
            return times[kernel], nbytes

    top = max(bench.HBM_BOUND, key=lambda k: times[k] * bench.PER_STEP[k])
    r = bench.roofline(Engine(), {})
    assert r["kernel"] == top and r["bound"] == "hbm" and r["unit"] == "GB/s"
    assert r["peak"] == 6650.0 and r["peak_source"] == "fallback"
    assert abs(r["achieved"] - nbytes / (times[top] * 1e-3) / 1e9) < 0.1
    assert r["frac"] == round(r["achieved"] / r["peak"], 4)
    assert set(r["per_kernel_ms_x_launches_per_step"]) == set(bench.PER_STEP)
    measured = bench.roofline(Engine(), {"hbm_gbs": 7000.0})
    assert measured["peak"] == 7000.0 and measured["peak_source"] == "measured"
    traffic = bench.measured_traffic()
    for kernel in ("fourier_forward", "fourier_inverse", "sp2gp"):
        assert traffic.get(kernel, 0) > 0, kernel
    assert r["traffic"] == traffic.get(top)


def test_clock_summary_keeps_the_timed_region_and_its_reasons(tmp_path):
    """The clocks line is the median SM clock of the nvidia-smi rows inside the
    timed region, with every throttle reason seen Active there; a region
    shorter than the sampling interval takes the rows on either side."""
    import datetime
    bench = load_bench()
    base = datetime.datetime(2026, 1, 1, 12, 0, 0)

    def at(seconds):
        return base + datetime.timedelta(seconds=seconds)

    def row(seconds, mhz, power_cap=False):
        stamp = at(seconds).strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
        cap = "Active" if power_cap else "Not Active"
        return f"{stamp}, {mhz}, 1965, Not Active, Not Active, Not Active, {cap}"

    clocks = bench.Clocks(0)
    clocks.path = str(tmp_path / "clocks.csv")
    rows = [row(0.0, 1000), row(1.0, 1965), row(1.05, 1965, power_cap=True), row(1.10, 1800), row(2.0, 1000)]
    (tmp_path / "clocks.csv").write_text("\n".join(rows) + "\n")
    clocks.t0, clocks.t1 = at(0.5).timestamp(), at(1.5).timestamp()
    s = clocks.summary()
    assert s["sm_mhz"] == 1965 and s["sm_max_mhz"] == 1965 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"] and s["region_s"] == 1.0
    clocks.t0, clocks.t1 = at(1.2).timestamp(), at(1.3).timestamp()
    short = clocks.summary()
    assert short["samples"] == 2 and short["sm_mhz"] == 1800 and short["reasons"] == []


def test_profile_kernels_brackets_each_timed_launch():
    """bench.py --profile-kernels: each kernel's untimed launch runs outside
    the profiler range, its timed launch inside it, and one JSON line (not a
    bench line) reports the event times and the tuning."""
    bench = load_bench()
    events = []

    class Profiler:
        def start(self):
            events.append("start")

        def stop(self):
            events.append("stop")

    fake_torch = types.SimpleNamespace(
        cuda=types.SimpleNamespace(synchronize=lambda: None, profiler=Profiler()))

    class Engine:
        def time_kernel(self, kernel, reps):
            events.append(kernel)
            return 0.0123456, 1000.0

        def tuning(self):
            return {"fft_rows": 32}

    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.profile_kernels(fake_torch, Engine(), ["sp2gp", "calcgp"])
    assert events == ["sp2gp", "start", "sp2gp", "stop", "calcgp", "start", "calcgp", "stop"]
    line = json.loads(out.getvalue())
    assert "metric" not in line and line["tuning"] == {"fft_rows": 32}
    assert line["profile_kernels"]["calcgp"] == {"ms": 0.0123, "algorithmic_bytes": 1000.0}
