"""Benchmark: aggregate simulated days per second of the ExoPlaSim timestep at
T42 L10 (45-minute steps), batched over many planets on each GPU, with the
plain single-run figure, the split-precision (tensor-core Legendre) arm, the
T63 and mixed-resolution ensemble configurations and the served latency
sample beside it.

Default (our arm): python bench.py [--gpus N --steps K --warmup W]
  one process per GPU (torchrun for N > 1); every rank steps its own batch of
  seeded T42 L10 planets (no collective on the data path: planets are
  independent), timed on the device with CUDA events, max over ranks.
Reference arm: python bench.py --impl reference ...
  the reference's timestep restated in FP64 on the host cores (the oracle;
  the reference's own engines need WebGPU or Wasm and cannot run here),
  one planet per thread, on rank 0 only.
"""
from __future__ import annotations

import argparse
import datetime
import importlib
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sim-days/s T42L10 plain vs batched split-precision; served p50/p99 run latency"
STEP_MINUTES = 45.0
DAYS_PER_STEP = STEP_MINUTES / 1440.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=320, help="timed model steps (about 1 s at 128 planets)")
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--slots", type=int, default=128)
    ap.add_argument("--chunk", type=int, default=32, help="model steps per engine call (one CUDA graph)")
    ap.add_argument("--no-baseline", action="store_true", help="skip the timed CPU baseline sample")
    ap.add_argument("--no-served", action="store_true", help="skip the continuous-batching latency sample")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the split-precision, T63 and mixed-ensemble configurations")
    ap.add_argument("--served-seconds", type=float, default=30.0, help="serving window (config 5 asks 600 s)")
    ap.add_argument("--profile-kernels", default="",
                    help="comma-separated exogcm_time_kernel names: after the warm-up steps, launch each once "
                         "between cudaProfilerStart and cudaProfilerStop (for ncu --profile-from-start off), "
                         "print their CUDA-event times and exit; no bench line")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region.

    The sampler starts before the region and is waited for until its first
    row is written; rows are kept by their timestamps, those inside the
    region (or, for a region shorter than the 50 ms interval, the rows just
    before and after it)."""

    FIELDS = ("timestamp,clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"exogcm_clocks_{os.getpid()}.csv")
        self.t0 = self.t1 = None

    def _rows(self):
        try:
            text = open(self.path).read()
        except OSError:
            return []
        out = []
        for line in text.strip().splitlines():
            r = [x.strip() for x in line.split(",")]
            if len(r) < 7:
                continue
            try:
                stamp = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                out.append((stamp, float(r[1]), float(r[2]), r[3:7]))
            except ValueError:
                continue
        return out

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            deadline = time.time() + 5.0
            while not self._rows() and time.time() < deadline:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        self.t0 = time.time()
        return self

    def __exit__(self, *exc):
        self.t1 = time.time()
        if self.proc:
            deadline = time.time() + 1.0
            while time.time() < deadline and not any(r[0] > self.t1 for r in self._rows()):
                time.sleep(0.02)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        rows = self._rows()
        if not rows:
            return None
        inside = [r for r in rows if self.t0 <= r[0] <= self.t1]
        if not inside:
            before = [r for r in rows if r[0] < self.t0][-1:]
            after = [r for r in rows if r[0] > self.t1][:1]
            inside = before + after or rows[-1:]
        sm = sorted(r[1] for r in inside)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in inside:
            for name, v in zip(names, r[3]):
                if v == "Active":
                    reasons.add(name)
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": inside[0][2], "reasons": sorted(reasons),
                "samples": len(inside), "region_s": round(self.t1 - self.t0, 3)}


def make_planets(count, seed0=1000):
    planets = importlib.import_module("web-exoplasim_b200.planets")
    return [planets.make_planet(seed0 + i, truncation=42, levels=10) for i in range(count)]


# Launches of each timed kernel in one model step (engine.cu's step order),
# counting a surface-pressure launch (one plane per slot) as 1/L of a
# full-level launch; the timed launches are all full-level.
PER_STEP = {"fourier_inverse": 10.2, "sp2gp": 8.2, "fourier_forward": 16.1, "legendre_inverse": 0.1, "dv2uv": 5,
            "legendre_forward": 5.1, "uv2dv": 2, "qtend": 2, "swr": 1, "lwr_radstep": 1, "vdiff": 1, "kuo": 1,
            "rain_column": 1, "calcgp": 1, "spectrala": 1, "mkdheat": 3, "physics_in": 1, "physics_out": 1}


# Kernels whose bound is HBM bandwidth (transforms and elementwise dynamics);
# the column physics kernels are latency- and special-function-bound.
HBM_BOUND = ("fourier_inverse", "sp2gp", "fourier_forward", "legendre_inverse", "dv2uv", "legendre_forward", "uv2dv", "qtend",
             "calcgp", "spectrala", "mkdheat", "physics_in", "physics_out")


def measured_traffic():
    """DRAM bytes per launch (read + write) of the HBM-bound kernels at 128
    planets, from the committed data file profiles/dram_traffic.json (ncu
    captures; the file names them)."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            return {k: int(v) for k, v in json.load(f)["bytes_per_launch"].items()}
    except (OSError, ValueError, KeyError):
        return {}


def compulsory_bytes(truncation, levels):
    """The step's compulsory HBM traffic per planet: the state read and
    written once, 4 * 2 * [(8L + 2) NRSP + (7L + 36) NHOR] bytes (the 10
    spectral prognostics and about 37 grid fields of the reference's
    trajectory field list)."""
    nlat = {21: 32, 42: 64, 63: 96}[truncation]
    nrsp = (truncation + 1) * (truncation + 2)
    nhor = 2 * nlat * nlat
    return 4 * 2 * ((8 * levels + 2) * nrsp + (7 * levels + 36) * nhor)


def roofline(engine, peaks):
    """The dominant HBM-bound kernel's achieved bandwidth: algorithmic bytes
    per launch / mean device time per launch (CUDA events around 20 launches
    on the engine's stream). Dominant = largest launches-per-step x time
    among HBM_BOUND; every timed kernel's ms per step is listed."""
    out = {}
    for kernel in PER_STEP:
        ms, nbytes = engine.time_kernel(kernel, 20)
        out[kernel] = (ms, nbytes)
    top = max(HBM_BOUND, key=lambda k: out[k][0] * PER_STEP[k])
    ms, nbytes = out[top]
    achieved = nbytes / (ms * 1e-3) / 1e9
    peak = peaks.get("hbm_gbs", 6650.0)
    return {"kernel": top, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": measured_traffic().get(top),
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "ms_per_launch": round(ms, 4), "bytes_per_launch": nbytes,
            "per_kernel_ms_x_launches_per_step": {k: round(v[0] * PER_STEP[k], 3) for k, v in out.items()}}


def cpu_baseline_sample(planet_list, threads, steps):
    """The FP64 oracle stepping `threads` planets concurrently (one per
    thread; ctypes releases the GIL), `steps` main-loop steps each."""
    import oracle
    models = [oracle.model_for(p) for p in planet_list[:threads]]
    oracles = [oracle.Oracle(m) for m in models]
    for o in oracles:
        o.startup()

    def run(o):
        o.advance(steps)
    t0 = time.perf_counter()
    ts = [threading.Thread(target=run, args=(o,)) for o in oracles]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    dt = time.perf_counter() - t0
    return threads * steps * DAYS_PER_STEP / dt, dt


def timed_steps(engine, steps, chunk=32):
    """Device time (ms, CUDA events of exogcm_last_step_ms summed over the
    calls) of `steps` model steps in calls of at most `chunk` steps, after
    capturing each call's graph."""
    calls = []
    while steps > 0:
        calls.append(min(chunk, steps))
        steps -= calls[-1]
    for k in set(calls):
        engine.step(k, publish_every=1 << 20)
    total = 0.0
    for k in calls:
        engine.step(k, publish_every=1 << 20)
        total += engine.last_step_ms()
    return total


def engine_for(pkg, planet_list, mode):
    cfg = planet_list[0].config
    e = pkg.Engine(cfg["truncation"], cfg["layers"], len(planet_list), mode=mode)
    for s, p in enumerate(planet_list):
        e.configure(s, p)
    e.step(3)  # start-up steps
    e.step(4, publish_every=1 << 20)
    return e


def sim_days_per_s(planets_n, steps, minutes, ms):
    return planets_n * steps * minutes / 1440.0 / (ms / 1000.0)


def extra_configs(pkg, plist, steps):
    """The metric's other configurations on one GPU:
    split precision: the same 128 T42 L10 planets with every Legendre
      transform on the tensor cores (engine mode 2);
    single slot: one T42 L10 planet on the optimized path (mode 1);
    T63 L10 (30-minute steps): one planet on the split-precision path, and 32
      planets batched on both paths;
    mixed ensemble: 128 T21 L5 + 96 T42 L10 + 32 T63 L10 planets with the
      ensemble's seeded parameter draw, one simulated day (32, 32 and 48
      steps) per launch of one CUDA graph holding the three engines' batch
      graphs (exogcm_group_step), device-timed with CUDA events."""
    import torch
    planets = importlib.import_module("web-exoplasim_b200.planets")
    out = {}
    e = engine_for(pkg, plist, 2)
    ms = timed_steps(e, steps)
    out["split_precision"] = {"value": round(sim_days_per_s(len(plist), steps, 45.0, ms), 3), "unit": "sim-days/s",
                              "ms_per_step": round(ms / steps, 4), "mode": 2, "launches_per_step": e.graph_launches(1)}
    e.close()
    e = engine_for(pkg, plist[:1], 1)
    ms = timed_steps(e, 128)
    out["single_slot_optimized"] = {"value": round(sim_days_per_s(1, 128, 45.0, ms), 3), "unit": "sim-days/s",
                                    "ms_per_step": round(ms / 128, 4)}
    e.close()
    t63 = [planets.make_planet(3000 + i, truncation=63, levels=10, timestepMinutes=30.0) for i in range(32)]
    e = engine_for(pkg, t63[:1], 2)
    ms = timed_steps(e, 96)
    out["t63_single_split"] = {"value": round(sim_days_per_s(1, 96, 30.0, ms), 3), "unit": "sim-days/s",
                               "ms_per_step": round(ms / 96, 4)}
    e.close()
    for mode in (1, 2):
        e = engine_for(pkg, t63, mode)
        ms = timed_steps(e, 64)
        out[f"t63_32planets_mode{mode}"] = {"value": round(sim_days_per_s(32, 64, 30.0, ms), 3),
                                            "unit": "sim-days/s", "ms_per_step": round(ms / 64, 4)}
        e.close()
    groups = []
    for (tr, lv, n, minutes, seed) in ((21, 5, 128, 45.0, 41), (42, 10, 96, 45.0, 42), (63, 10, 32, 30.0, 43)):
        draws = planets.ensemble_parameters(seed, n)
        ps = []
        for i, d in enumerate(draws):
            d = dict(d)
            lf = d.pop("land_fraction")
            ps.append(planets.make_planet(seed * 1000 + i, truncation=tr, levels=lv, land_fraction=lf,
                                          timestepMinutes=minutes, **d))
        groups.append((engine_for(pkg, ps, 1), n, minutes, int(round(1440 / minutes))))
    engines = [e for e, *_ in groups]
    per_day = [d for *_, d in groups]
    pkg.group_step(engines, per_day)  # instantiates the group graph
    rounds = 3
    device_ms = 0.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(rounds):
        device_ms += pkg.group_step(engines, per_day)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    days = rounds * sum(n for _, n, _, _ in groups)
    unstable = sum(int(e.unstable().sum()) for e in engines)
    out["mixed_ensemble"] = {"value": round(days / (device_ms / 1000.0), 3), "unit": "sim-days/s",
                             "planets": "128 T21L5 + 96 T42L10 + 32 T63L10", "simulated_days": days,
                             "ms_per_simulated_day": round(device_ms / rounds, 3),
                             "wall_value": round(days / wall, 3), "unstable_planets": unstable,
                             "launch": "one CUDA graph per simulated day (exogcm_group_step): the three "
                                       "engines' 32, 32 and 48-step batch graphs as child nodes"}
    for e, *_ in groups:
        e.close()
    return out


def served_config5(seconds, budget_gb=40.0, seed=7):
    """Config 5's serving loop: Poisson arrivals at 20 runs/s of seeded
    planets, resolution uniform over T21/T42/T63 x L5/L10, duration uniform
    over 1-365 simulated days, admitted by HBM footprint into engine blocks
    within one byte budget, stepped with exogcm_step_async. The window is
    `seconds` (config 5 names 10 minutes); runs unfinished at its end count
    toward throughput by the steps they completed."""
    serving = importlib.import_module("web-exoplasim_b200.serving")
    planets = importlib.import_module("web-exoplasim_b200.planets")
    reqs = serving.poisson_requests(20.0, seconds, seed=seed, max_days=365.0, min_days=1.0)
    for r in reqs:
        r.planet = planets.make_planet(r.seed, truncation=r.truncation, levels=r.levels,
                                       timestepMinutes=serving.STEP_MINUTES[r.truncation])
    server = serving.Server(budget_bytes=budget_gb * 1e9, chunk=32, keep_results=False)
    prewarm_s = server.prewarm()  # one warm block per resolution before the window opens
    rep = server.run(reqs, window=seconds, drain=False)
    server.close()
    return {"p50_s": round(rep["p50_s"], 3), "p99_s": round(rep["p99_s"], 3), "completed": rep["completed"],
            "failed": rep["failed"], "sim_days_per_s": round(rep["sim_days_per_s"], 2), "requests": len(reqs),
            "arrival_rate_per_s": 20.0, "run_days": "1-365 (uniform)", "resolutions": "T21/T42/T63 x L5/L10",
            "window_s": round(rep["window_s"], 2), "queue_depth_mean": round(rep["queue_depth_mean"], 1),
            "queue_depth_max": rep["queue_depth_max"], "budget_gb": budget_gb, "slots": rep["slots"],
            "blocks_created": rep["blocks_created"], "blocks_destroyed": rep["blocks_destroyed"],
            "configure_ms_p50": rep["configure_ms_p50"] and round(rep["configure_ms_p50"], 2),
            "configure_ms_p99": rep["configure_ms_p99"] and round(rep["configure_ms_p99"], 2),
            "setup_on_device": rep["setup_on_device"], "prewarm_s": round(prewarm_s, 2)}


def admission_latency(pkg, repeats=5):
    """exogcm_configure wall time (FP64 set-up plus upload) of one planet at
    each resolution, with the heavy set-up loops on the host and on the
    device; the median of `repeats` configures of a fresh planet into slot 0
    of a 4-slot mode-1 engine whose shared tables are already built."""
    planets = importlib.import_module("web-exoplasim_b200.planets")
    out = {}
    for truncation in (21, 42, 63):
        plist = [planets.make_planet(500 + k, truncation=truncation, levels=10) for k in range(repeats + 1)]
        row = {}
        for where in ("host", "device"):
            e = pkg.Engine(truncation, 10, 4, mode=1)
            try:
                e.setup_on_device(where == "device")
                e.configure(1, plist[0])  # shared tables, autotuning, staging buffers
                times = []
                for p in plist[1:]:
                    t = time.perf_counter()
                    e.configure(0, p)
                    times.append(time.perf_counter() - t)
                row[where] = round(float(sorted(times)[len(times) // 2]) * 1e3, 2)
            finally:
                e.close()
        out[f"T{truncation}L10"] = row
    return {"unit": "ms per planet (median of %d)" % repeats, **out}


def cpu_model():
    """The host CPU's model name (/proc/cpuinfo), or the platform's processor string."""
    try:
        with open("/proc/cpuinfo") as f:
            for row in f:
                if row.startswith("model name"):
                    return row.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def reference_arm(args, rank):
    if rank != 0:
        return
    # one planet per host thread, capped so the set-up of the sample stays short
    cores = min(os.cpu_count() or 1, 32)
    planet_list = make_planets(cores, seed0=1000)
    sample_steps = max(4, args.steps // 4)
    value, dt = cpu_baseline_sample(planet_list, cores, sample_steps)
    line = {
        "metric": METRIC, "impl": "reference", "value": round(value, 4), "unit": "sim-days/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(DAYS_PER_STEP * cores / value * 1000, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "T42 L10 seeded planets, 45-minute steps, one planet per host thread",
                   "planets": cores, "seq_len": None},
        "cpu_baseline": {"value": round(value, 4), "unit": "sim-days/s", "cores": cores, "kind": "port",
                         "sample": f"{cores} planets x {sample_steps} main-loop steps after the 3 "
                                   f"start-up steps ({dt:.1f} s)",
                         "cpu_model": cpu_model(), "host_threads": os.cpu_count()},
        "e2e": {"value": round(value, 4), "unit": "sim-days/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's engines need WebGPU (graphics API, unavailable on this box) or its Wasm binary "
                "(closed); its timestep is timed as the FP64 restatement on the host cores",
    }
    print(json.dumps(line), flush=True)


def profile_kernels(torch, engine, names):
    """Each named kernel's launch through exogcm_time_kernel (its warm-up
    launch and one timed launch) inside a profiler range, so an ncu capture
    started with --profile-from-start off sees exactly those launches."""
    out = {}
    for k in names:
        engine.time_kernel(k, 1)  # untimed: shapes, caches
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        ms, nbytes = engine.time_kernel(k, 1)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        out[k] = {"ms": round(ms, 4), "algorithmic_bytes": nbytes}
    print(json.dumps({"profile_kernels": out, "tuning": engine.tuning()}), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    import torch
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist
    pkg = importlib.import_module("web-exoplasim_b200")
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    slots = args.slots
    chunk = max(1, min(args.chunk, 64))
    plist = make_planets(slots, seed0=1000 + rank * slots)
    engine = pkg.Engine(42, 10, slots, mode=1)
    for s, p in enumerate(plist):
        engine.configure(s, p)
    # start-up steps (3) then warm-up main steps
    engine.step(3)
    for _ in range(max(3, args.warmup)):
        engine.step(1)
    if args.profile_kernels:
        profile_kernels(torch, engine, args.profile_kernels.split(","))
        return
    calls = []
    remaining = args.steps
    while remaining > 0:
        calls.append(min(chunk, remaining))
        remaining -= calls[-1]
    for k in set(calls):
        engine.step(k, publish_every=1 << 20)  # capture each graph size before timing
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clocks:
        device_ms = 0.0
        for k in calls:
            engine.step(k, publish_every=1 << 20)
            device_ms += engine.last_step_ms()
    torch.cuda.synchronize()
    if pg:
        t = torch.tensor([device_ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        device_ms = float(t.item())
    value = world * slots * args.steps * DAYS_PER_STEP / (device_ms / 1000.0)

    # End to end through the C ABI: host values uploaded every call, a
    # snapshot published per slot every model day (32 steps) and read back to
    # host buffers, host wall clock around the calls. Days are submitted as
    # the reference's worker does (two batches in flight): exogcm_step_async
    # and a snapshot copy queued behind it, so the host computes the next
    # day's per-step values while the device runs the current one.
    publish = 32
    e2e_calls = max(4, args.steps // publish)  # several days, so each day's copy can overlap the next
    snap_floats = engine.field_size("snapshot")
    import numpy as np
    # every slot's published snapshot lands in pinned host memory; each day's
    # copy drains on the engine's copy stream while the next day computes, and
    # the last one is waited for inside the timed region
    host = torch.empty(slots * snap_floats, dtype=torch.float32, pin_memory=True).numpy()
    # one untimed day first: the first exogcm_snapshots_begin creates the copy
    # stream and allocates the device staging buffer (a warm-up, like the
    # device-timed steps')
    engine.step(publish, publish_every=publish)
    engine.snapshots_begin(host)
    engine.snapshots_wait()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_calls):
        engine.step_async(publish, publish_every=publish)
        engine.snapshots_begin(host)
    engine.snapshots_wait()
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_steps = e2e_calls * publish
    if pg:
        t = torch.tensor([e2e_s], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * slots * e2e_steps * DAYS_PER_STEP / e2e_s
    d2h_per_step = slots * snap_floats * 4 / publish
    h2d_per_step = slots * 96

    # plain single-run FP32 path: one planet, same kernels, one slot
    plain = pkg.Engine(42, 10, 1, mode=0)
    plain.configure(0, plist[0])
    plain.step(3)
    plain.step(8, publish_every=1 << 20)
    torch.cuda.synchronize()
    pms = 0.0
    for _ in range(4):
        plain.step(8, publish_every=1 << 20)
        pms += plain.last_step_ms()
    plain_value = 32 * DAYS_PER_STEP / (pms / 1000.0)
    plain.close()

    launches = engine.graph_launches(1) * args.steps
    roof = roofline(engine, peaks) if rank == 0 else None
    if roof is not None:
        # the path's roofline: the step's compulsory bytes over the step time
        b_min = compulsory_bytes(42, 10) * slots
        peak = peaks.get("hbm_gbs", 6650.0)
        roof["path"] = {"compulsory_bytes_per_step": b_min, "ms_per_step": round(device_ms / args.steps, 4),
                        "achieved": round(b_min / (device_ms / args.steps * 1e-3) / 1e9, 1), "peak": peak,
                        "frac": round(b_min / (device_ms / args.steps * 1e-3) / 1e9 / peak, 4)}
    tuning = engine.tuning()
    extra = None
    served = None
    if rank == 0 and world == 1:
        engine.close()
        engine = None
        # the extra configurations report an error in the line rather than
        # losing the headline when one of them fails
        if not args.no_extra:
            try:
                extra = extra_configs(pkg, plist, max(64, args.steps // 2))
            except Exception as exc:  # noqa: BLE001
                extra = {"extra_configs_error": f"{type(exc).__name__}: {exc}"}
        if not args.no_extra:
            try:
                extra = dict(extra or {}, admission=admission_latency(pkg))
            except Exception as exc:  # noqa: BLE001
                extra = dict(extra or {}, admission={"error": f"{type(exc).__name__}: {exc}"})
        if not args.no_served:
            try:
                served = served_config5(args.served_seconds)
            except Exception as exc:  # noqa: BLE001
                served = {"error": f"{type(exc).__name__}: {exc}"}
    cpu = None
    if rank == 0 and world == 1 and not args.no_baseline:
        v, dt = cpu_baseline_sample(plist, 1, 4)
        cpu = {"value": round(v, 5), "unit": "sim-days/s", "cores": 1, "kind": "port",
               "sample": f"1 T42 L10 planet, 4 FP64 main-loop steps after start-up ({dt:.1f} s)",
               "cpu_model": cpu_model(), "host_threads": os.cpu_count()}
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "sim-days/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(device_ms / args.steps, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "T42 L10 batched ensemble, 45-minute steps (seeded synthetic planet recipe, "
                                   "seeded per planet)", "planets_per_gpu": slots, "global_batch": slots * world,
                       "seq_len": None, "parallelism": f"planets sharded over {world} GPU(s), no collective",
                       "l2": "state of the batch (GBs) far above the 126 MB L2; no flush needed",
                       "path": "optimized FP32: FFT longitude transforms, latitude-pair SIMT Legendre (mode 1); "
                               "split_precision: Legendre transforms on tcgen05 in 3xTF32 (mode 2); "
                               "plain single run: mode 0"},
            "plain_single_run": {"value": round(plain_value, 3), "unit": "sim-days/s",
                                 "ms_per_step": round(pms / 32, 4)},
            "e2e": {"value": round(e2e_value, 3), "unit": "sim-days/s", "h2d_bytes_per_step": h2d_per_step,
                    "d2h_bytes_per_step": int(d2h_per_step)},
            "gpu_launches": launches,
            "roofline": roof, "cpu_baseline": cpu, "clocks": clocks.summary(),
            "served": served, "tuning": tuning,
        }
        if extra:
            line.update(extra)
        print(json.dumps(line), flush=True)
    if engine is not None:
        unstable = engine.unstable()
        if unstable.any() and rank == 0:
            print(json.dumps({"warning": f"{int(unstable.sum())} planets became unstable"}), file=sys.stderr)
        engine.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
