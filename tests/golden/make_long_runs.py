"""Generates the long-run fixtures (run on a CPU host; takes about 10 minutes
on 8 cores). Commit the .npz files it writes next to this script.

long_runs.npz -- the north star's configs 2 and 3 against the FP64 oracle:
  T42 L10, 45-minute step, 30 simulated days, planet seed 42, and
  T63 L10, 30-minute step, 10 simulated days, planet seed 63.
  Both oracles (f64 and sequential f32) start from the oracle's initial
  state rounded once to f32 and run the start-up steps then the days; the
  final spectral prognostics st, sz, sd, sq, sp of each are stored (f32).
  The GPU test starts from the same rounded state and judges each field by
  the reference's V4 rule (scripts/exoplasim-webgpu/trajectory.mjs:67-79):
  its RMS difference from f64 at most twice the f32 run's.

climatology_t21.npz -- a one-year T21 L10 ensemble: planet seed 21 with
  initial noise seeds 0..5, each run for 360 days by the FP64 oracle
  ("daily") and by the sequential-f32 oracle ("daily_f32"); the daily global
  means of surface temperature, 2 m air temperature, precipitation, total
  cloud cover, outgoing longwave, top-of-atmosphere net flux and surface
  pressure (the fields scripts/exoplasim-wasm/compare-climate.mjs:10-11
  compares) are stored per seed.

  python make_long_runs.py            # everything
  python make_long_runs.py f32-climate  # adds daily_f32 to an existing climatology_t21.npz
"""
import importlib
import multiprocessing as mp
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

HERE = os.path.dirname(os.path.abspath(__file__))
PROGNOSTIC = ("st", "sz", "sd", "sq", "sp")
LONG_RUNS = {"t42": dict(truncation=42, seed=42, minutes=45.0, days=30),
             "t63": dict(truncation=63, seed=63, minutes=30.0, days=10)}
CLIMATE_SEEDS = tuple(range(6))
CLIMATE_DAYS = 360
# snapshot slots (snapshot/wgsl/pack.wgsl order): surface T, 2 m air T,
# precipitation (convective + large-scale), total cloud cover, OLR, TOA net, ps
CLIMATE_FIELDS = ("surface_temperature", "air_temperature", "precipitation", "cloud_cover", "olr", "toa_net",
                  "surface_pressure")


def rounded_model(planet):
    import oracle
    m = oracle.model_for(planet)
    m["state"] = {k: np.asarray(v, dtype=np.float64).astype(np.float32).astype(np.float64)
                  for k, v in m["state"].items()}
    return m


def long_run(args):
    name, precision = args
    import oracle
    planets = importlib.import_module("web-exoplasim_b200.planets")
    spec = LONG_RUNS[name]
    p = planets.make_planet(spec["seed"], truncation=spec["truncation"], levels=10, timestepMinutes=spec["minutes"])
    o = oracle.Oracle(rounded_model(p), precision=precision)
    steps = int(round(spec["days"] * 1440 / spec["minutes"]))
    o.startup()
    o.advance(steps)
    return name, precision, {k: o.get(k).astype(np.float32) for k in PROGNOSTIC}


def global_means(o, nlat):
    """Area-weighted global means of the climatology fields from the oracle's
    state after a step (the quantities pack.wgsl publishes)."""
    nlon = 2 * nlat
    nhor = nlat * nlon
    w = np.repeat(np.asarray(o.model["weights"], dtype=np.float64), nlon)
    L = o.model["levels"]
    dt = o.get("dt").reshape(L + 1, nhor)
    dlwfl = o.get("dlwfl").reshape(L + 1, nhor)
    dswfl = o.get("dswfl").reshape(L + 1, nhor)
    fields = (dt[L], o.get("dtsa"), o.get("dprc") + o.get("dprl"), o.get("dcc").reshape(L + 1, nhor)[L],
              -dlwfl[0], dswfl[0] + dlwfl[0], o.get("dp"))
    return np.array([np.sum(f * w) / np.sum(w) for f in fields])


def climate_run(noise_seed, precision=64):
    import oracle
    planets = importlib.import_module("web-exoplasim_b200.planets")
    p = planets.make_planet(21, truncation=21, levels=10, noise_seed=noise_seed)
    o = oracle.Oracle(rounded_model(p), precision=precision)
    o.startup()
    daily = []
    for _ in range(CLIMATE_DAYS):
        o.advance(32)
        daily.append(global_means(o, 32))
    return noise_seed, np.array(daily)


def climate_run_f32(noise_seed):
    return climate_run(noise_seed, precision=32)


def add_f32_climate():
    path = os.path.join(HERE, "climatology_t21.npz")
    with mp.get_context("spawn").Pool(min(8, os.cpu_count() or 1)) as pool:
        clim32 = dict(pool.map(climate_run_f32, CLIMATE_SEEDS))
    old = dict(np.load(path))
    old["daily_f32"] = np.stack([clim32[s] for s in CLIMATE_SEEDS])
    np.savez_compressed(path, **old)


def main():
    if sys.argv[1:] == ["f32-climate"]:
        add_f32_climate()
        return
    ctx = mp.get_context("spawn")
    with ctx.Pool(min(8, os.cpu_count() or 1)) as pool:
        long_jobs = pool.map_async(long_run, [(n, prec) for n in LONG_RUNS for prec in (64, 32)])
        climate_jobs = pool.map_async(climate_run, CLIMATE_SEEDS)
        out = {}
        for name, precision, state in long_jobs.get():
            for k, v in state.items():
                out[f"{name}_f{precision}_{k}"] = v
        np.savez_compressed(os.path.join(HERE, "long_runs.npz"), **out)
        clim = dict(climate_jobs.get())
        clim32 = dict(pool.map(climate_run_f32, CLIMATE_SEEDS))
        np.savez_compressed(os.path.join(HERE, "climatology_t21.npz"),
                            daily=np.stack([clim[s] for s in CLIMATE_SEEDS]),
                            daily_f32=np.stack([clim32[s] for s in CLIMATE_SEEDS]),
                            seeds=np.array(CLIMATE_SEEDS), fields=np.array(CLIMATE_FIELDS))


if __name__ == "__main__":
    main()
