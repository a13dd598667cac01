"""Long runs against the FP64 oracle (fixtures from tests/golden/
make_long_runs.py, which documents them): T42 L10 over 30 simulated days and
T63 L10 over 10 (the north star's configs 2 and 3), judged per prognostic
field by the reference's V4 rule (scripts/exoplasim-webgpu/trajectory.mjs:
67-79: the RMS difference from the f64 run at most twice the sequential-f32
run's); and a one-year T21 ensemble's global annual means against the FP64
ensemble by the reference's climatology test
(scripts/exoplasim-wasm/compare-climate.mjs:13-16, 57-71: |difference of
means| <= k sigma sqrt(2 / N), sigma across the ensemble, k = 3 here, see
SIGMAS), where a field outside that threshold still passes if the GPU's mean
is no further from FP64 than twice the sequential-f32 oracle ensemble's."""
import os

import numpy as np
import pytest

from tests.golden import make_long_runs as gen
from tests.helpers import pkg, planets, rel_rms

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIELD_LABEL = {"st": "T", "sz": "vorticity", "sd": "divergence", "sq": "q", "sp": "ln ps"}
# compare-climate.mjs tests at 2 sigma (95 % per field) over years of one run;
# here the spread is that of six one-year runs from 0.1 K initial noise, and
# the sequential-f32 ensemble itself departs from FP64 by up to 0.68 of the
# 2-sigma threshold (air temperature), so a single FP32 realisation sits near
# it by chance: the test uses 3 sigma (99.7 % per field, seven fields).
SIGMAS = 3


def _engine_from_rounded_state(planet, mode, slots=1):
    m = gen.rounded_model(planet)
    e = pkg.Engine(planet.config["truncation"], planet.config["layers"], slots, mode=mode)
    for s in range(slots):
        e.configure(s, planet)
        for name, v in m["state"].items():
            e.write(s, name, np.asarray(v, dtype=np.float32))
    return e


def _run(e, steps):
    while steps > 0:
        k = min(64, steps)
        e.step(k)
        steps -= k


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["t42", "t63"])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_long_run_passes_v4(name, mode):
    spec = gen.LONG_RUNS[name]
    ref = np.load(os.path.join(HERE, "long_runs.npz"))
    p = planets.make_planet(spec["seed"], truncation=spec["truncation"], levels=10, timestepMinutes=spec["minutes"])
    e = _engine_from_rounded_state(p, mode)
    e.step(3)  # start-up steps
    _run(e, int(round(spec["days"] * 1440 / spec["minutes"])))
    assert not e.unstable().any()
    report = {}
    for k in gen.PROGNOSTIC:
        f64 = ref[f"{name}_f64_{k}"].astype(np.float64)
        gpu = rel_rms(e.read(0, k), f64)
        f32 = rel_rms(ref[f"{name}_f32_{k}"], f64)
        report[FIELD_LABEL[k]] = (float(f"{gpu:.3g}"), float(f"{f32:.3g}"))
        assert gpu <= 2 * f32, (k, gpu, f32)
    print(f"{name} mode {mode} after {spec['days']} days, relative RMS vs FP64 (GPU, sequential f32):", report)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2])
def test_one_year_t21_climatology_matches_fp64_ensemble(mode):
    clim = np.load(os.path.join(HERE, "climatology_t21.npz"))
    daily = clim["daily"]  # [seed][day][field], FP64 oracle
    seeds = [int(s) for s in clim["seeds"]]
    n = len(seeds)
    e = None
    for i, seed in enumerate(seeds):
        p = planets.make_planet(21, truncation=21, levels=10, noise_seed=seed)
        if e is None:
            e = pkg.Engine(21, 10, n, mode=mode)
        m = gen.rounded_model(p)
        e.configure(i, p)
        for name, v in m["state"].items():
            e.write(i, name, np.asarray(v, dtype=np.float32))
    e.step(3)
    weights = np.repeat(np.asarray(gen.rounded_model(planets.make_planet(21, truncation=21, levels=10))["weights"]),
                        64)
    gpu = np.zeros((n, gen.CLIMATE_DAYS, len(gen.CLIMATE_FIELDS)))
    for day in range(gen.CLIMATE_DAYS):
        e.step(32)
        for i in range(n):
            gpu[i, day] = _global_means(e, i, weights)
    assert not e.unstable().any()
    ref_annual = daily.mean(axis=1)  # [seed][field]
    f32_annual = clim["daily_f32"].mean(axis=1)
    gpu_annual = gpu.mean(axis=1)
    report = {}
    for f, name in enumerate(gen.CLIMATE_FIELDS):
        sigma = np.std(ref_annual[:, f], ddof=1)
        threshold = SIGMAS * sigma * np.sqrt(2 / n)
        diff = gpu_annual[:, f].mean() - ref_annual[:, f].mean()
        f32_diff = f32_annual[:, f].mean() - ref_annual[:, f].mean()
        report[name] = tuple(float(f"{x:.4g}") for x in (ref_annual[:, f].mean(), diff, threshold, f32_diff))
        # within the ensemble's sampling threshold, or no further from FP64
        # than twice the sequential-f32 build's own ensemble (V4's rule on
        # the annual means)
        assert abs(diff) <= max(threshold, 2 * abs(f32_diff)), (name, diff, threshold, f32_diff)
    print("one-year T21 global means (FP64 ensemble mean, GPU - FP64, 3 sigma sqrt(2/N), f32 - FP64):", report)


def _global_means(e, slot, w):
    L, nhor = 10, 2048
    dt = e.read(slot, "dt").reshape(L + 1, nhor)
    dlwfl = e.read(slot, "dlwfl").reshape(L + 1, nhor)
    dswfl = e.read(slot, "dswfl").reshape(L + 1, nhor)
    dcc = e.read(slot, "dcc").reshape(L + 1, nhor)
    fields = (dt[L], e.read(slot, "dtsa"), e.read(slot, "dprc") + e.read(slot, "dprl"), dcc[L], -dlwfl[0],
              dswfl[0] + dlwfl[0], e.read(slot, "dp"))
    return np.array([np.sum(f.astype(np.float64) * w) / np.sum(w) for f in fields])
