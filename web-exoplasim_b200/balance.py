"""The energy-balance assessment of a run (ExoPlaSim's Model._isbalanced as
the reference restates it, src/model/climate/gcm/balance/index.ts:1-70): the
yearly global means of top-of-atmosphere net radiation and surface net heat
flux, which the engine's FP64 budgets provide (Engine.budgets), are reduced
to 10-year running means of their absolute values, least-squares slopes over
5 consecutive running means, and the mean of the last 30 slopes; the run is
balanced when both drifts are below 5e-4 W/m^2 per year."""
from __future__ import annotations

import math
from dataclasses import dataclass

RUNNING_MEAN_YEARS = 10
SLOPE_WINDOW = 5
SLOPES_AVERAGED = 30
THRESHOLD_W_M2_PER_YEAR = 5e-4
MINIMUM_YEARS = RUNNING_MEAN_YEARS + SLOPE_WINDOW - 1


@dataclass
class YearlyBalance:
    year: int
    toa_net_radiation: float
    surface_net_heat: float
    surface_temperature: float


@dataclass
class Assessment:
    status: str  # "spinning-up", "balanced" or "drifting"
    years_needed: int
    toa_drift_per_year: float
    surface_drift_per_year: float


def _mean(values):
    return sum(values) / len(values)


def _slope(values):
    x_mean = (len(values) + 1) / 2
    y_mean = _mean(values)
    num = den = 0.0
    for i, v in enumerate(values):
        x = i + 1 - x_mean
        num += x * (v - y_mean)
        den += x * x
    return num / den


def drift(series) -> float:
    running = [abs(_mean(series[end - RUNNING_MEAN_YEARS:end]))
               for end in range(RUNNING_MEAN_YEARS, len(series) + 1)]
    slopes = [_slope(running[end - SLOPE_WINDOW:end]) for end in range(SLOPE_WINDOW, len(running) + 1)]
    return abs(_mean(slopes[-SLOPES_AVERAGED:]))


def assess(years: list[YearlyBalance]) -> Assessment:
    if len(years) < MINIMUM_YEARS:
        return Assessment("spinning-up", MINIMUM_YEARS - len(years), math.nan, math.nan)
    toa = drift([y.toa_net_radiation for y in years])
    surface = drift([y.surface_net_heat for y in years])
    status = "balanced" if toa < THRESHOLD_W_M2_PER_YEAR and surface < THRESHOLD_W_M2_PER_YEAR else "drifting"
    return Assessment(status, 0, toa, surface)


def yearly_from_budgets(year: int, mean: dict) -> YearlyBalance:
    """A year's balance from the mean budgets over that year's publishing
    steps (Engine.budgets(slot, reset=True)['mean'] at the year's end)."""
    return YearlyBalance(year, mean["toa_net"], mean["surface_net"], mean["surface_temperature"])
