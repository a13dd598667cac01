"""Seeded synthetic planets: the inputs every run of this library is measured on.

The reference publishes no dataset for its timestep; the benchmark and the
parity tests run on planets generated here from a seed, following one recipe:

* land mask: random spherical-harmonic coefficients of total wavenumber
  n <= 10 (unit-variance Gaussian per coefficient), synthesised on the Gaussian
  grid and thresholded at the (1 - land fraction) quantile;
* orography: the positive part of that noise scaled to a 4 km maximum, as
  surface geopotential g*h (the 0129 boundary field of
  src/model/climate/gcm/boundary/index.ts:12-40);
* a 50 m slab ocean with a 288 K SST climatology and no sea ice;
* a resting isothermal 250 K atmosphere plus Gaussian temperature noise of
  0.1 K standard deviation per grid value, at 80 % relative humidity
  (saturation formula of setup/surface/index.ts:159-167).

Planet parameters default to the reference's page defaults
(src/model/climate/gcm/index.ts:4-44) with an Earth atmosphere of 1011 hPa
and 360 ppm CO2, no stellar spectrum, and a fixed orbit.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

EARTH_GAS_CONSTANT = 8314.46261815324 / 28.970253

BASE_CONFIG = dict(
    layers=10, truncation=21, radiusEarth=1.0, gravityMs2=9.80665, synchronous=False,
    substellarLongitudeDeg=180.0, oceanDepthM=50.0, fluxWm2=1367.0, starTemperatureK=0.0,
    yearDays=360, eccentricity=0.016715, rotationPeriodDays=1.0, obliquityDeg=23.44,
    fixedOrbit=True, keplerian=False, wetSoil=False, vegetation=2, initialGrowth=0.5,
    glaciersEnabled=True, glaciersMinDepthM=2.0, glaciersInitialHeightM=-1.0,
    physicsFilter=("gp", "exp", "sp"), timestepMinutes=45.0, pressureBar=1.011,
    gasConstant=EARTH_GAS_CONSTANT, co2Ppm=360.0, ozone=True, soilDepthScale=1.0, stormclim=False,
)

LATITUDES = {21: 32, 42: 64, 63: 96}


@dataclass
class Planet:
    """One seeded planet: its configuration and its grid-point inputs."""
    config: dict
    land_fraction: float
    boundary: dict = field(default_factory=dict)   # surface code -> grid field(s)
    t_grid: np.ndarray | None = None               # [levels, nhor] K
    q_grid: np.ndarray | None = None               # [levels, nhor] kg/kg
    seed: int = 0


def gaussian_sines(nlat: int) -> np.ndarray:
    x, _ = np.polynomial.legendre.leggauss(nlat)
    return -x  # north first


def _sh_noise(rng, nlat, nlon, nmax=10):
    """A smooth random field: real spherical harmonics up to total wavenumber
    nmax with unit-variance Gaussian coefficients, on the Gaussian grid."""
    from scipy.special import lpmv
    mu = gaussian_sines(nlat)
    lam = 2 * np.pi * np.arange(nlon) / nlon
    out = np.zeros((nlat, nlon))
    for n in range(nmax + 1):
        for m in range(n + 1):
            norm = math.sqrt((2 * n + 1) / (4 * math.pi) * math.factorial(n - m) / math.factorial(n + m))
            p = norm * lpmv(m, n, mu)
            a = rng.standard_normal()
            out += a * p[:, None] * np.cos(m * lam)[None, :]
            if m > 0:
                b = rng.standard_normal()
                out += b * p[:, None] * np.sin(m * lam)[None, :]
    return out.reshape(-1)


def sigma_levels(levels: int) -> np.ndarray:
    z = (np.arange(levels) + 1) / levels
    sigmah = 0.75 * z + 1.75 * z ** 3 - 1.5 * z ** 4
    prev = np.concatenate([[0.0], sigmah[:-1]])
    return 0.5 * (prev + sigmah)


def saturation(t, p, gascon):
    rdbrv = gascon / 461.51
    q = rdbrv * 610.78 * np.exp(17.2693882 * (t - 273.16) / (t - 35.86)) / p
    return q / (1 - (1 / rdbrv - 1) * q)


def make_planet(seed: int, truncation: int = 21, levels: int = 10, land_fraction: float = 0.3,
                noise_seed: int | None = None, **overrides) -> Planet:
    """The planet of `seed`. With `noise_seed` the initial temperature noise
    comes from that seed instead, so one terrain carries an ensemble of
    initial states (the climatology gate's control runs)."""
    cfg = dict(BASE_CONFIG)
    cfg.update(truncation=truncation, layers=levels)
    cfg.update(overrides)
    rng = np.random.default_rng(seed)
    nlat = LATITUDES[truncation]
    nlon = 2 * nlat
    noise = _sh_noise(rng, nlat, nlon)
    if land_fraction <= 0:
        mask = np.zeros_like(noise)
        oro = np.zeros_like(noise)
    else:
        threshold = np.quantile(noise, 1 - land_fraction)
        mask = (noise >= threshold).astype(float)
        height = np.maximum(noise - threshold, 0.0)
        top = height.max()
        oro = (height / top * 4000.0 if top > 0 else height) * cfg["gravityMs2"]
    nhor = nlat * nlon
    boundary = {172: mask, 129: oro, 169: np.full(nhor, 288.0), 210: np.zeros(nhor)}
    sigma = sigma_levels(levels)
    if noise_seed is not None:
        rng = np.random.default_rng([seed, noise_seed])
    t = 250.0 + 0.1 * rng.standard_normal((levels, nhor))
    p = sigma[:, None] * cfg["pressureBar"] * 1e5
    q = 0.8 * saturation(t, p, cfg["gasConstant"])
    return Planet(config=cfg, land_fraction=land_fraction, boundary=boundary, t_grid=t, q_grid=q, seed=seed)


def ensemble_parameters(seed: int, count: int):
    """The batched-ensemble parameter draw: rotation period log-uniform over
    0.25-100 days, stellar flux 0.5-1.5 x 1367 W/m2, surface pressure
    log-uniform 0.1-10 bar, CO2 log-uniform 1e-5 to 1e-1 volume fraction,
    land fraction uniform 0-0.6."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        out.append(dict(
            rotationPeriodDays=float(math.exp(rng.uniform(math.log(0.25), math.log(100.0)))),
            fluxWm2=float(rng.uniform(0.5, 1.5) * 1367.0),
            pressureBar=float(math.exp(rng.uniform(math.log(0.1), math.log(10.0)))),
            co2Ppm=float(math.exp(rng.uniform(math.log(1e-5), math.log(1e-1))) * 1e6),
            land_fraction=float(rng.uniform(0.0, 0.6)),
        ))
    return out
