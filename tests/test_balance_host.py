"""The energy-balance assessment (balance.py) on synthetic yearly series: too
few years, a steady run, and a run whose balances still drift."""
import importlib
import math

balance = importlib.import_module("web-exoplasim_b200.balance")


def _years(toa, surf):
    return [balance.YearlyBalance(i + 1, t, s, 288.0) for i, (t, s) in enumerate(zip(toa, surf))]


def test_spinning_up_until_fourteen_years():
    a = balance.assess(_years([0.1] * 13, [0.1] * 13))
    assert a.status == "spinning-up" and a.years_needed == 1 and math.isnan(a.toa_drift_per_year)


def test_steady_balances_are_balanced():
    a = balance.assess(_years([0.3 + 1e-5 * (i % 2) for i in range(40)], [-0.2] * 40))
    assert a.status == "balanced" and a.toa_drift_per_year < balance.THRESHOLD_W_M2_PER_YEAR


def test_linear_drift_is_measured():
    # |running mean| of a 0.01 W/m^2 per year ramp grows at 0.01 per year
    toa = [1.0 + 0.01 * i for i in range(40)]
    a = balance.assess(_years(toa, [0.0] * 40))
    assert a.status == "drifting" and abs(a.toa_drift_per_year - 0.01) < 1e-12 and a.surface_drift_per_year == 0.0
