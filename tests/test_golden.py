"""Parity on the reference's packaged Earth climatologies (tests/golden/,
made by make_earth_climatology.py from public/gcm/t21/inputs.json): a
planet whose sea-surface temperature and ice-cover climatologies are the
Earth's monthly fields, so the month interpolation of the surface step and
the sea-ice and slab-ocean routines run on the reference's own data."""
import os

import numpy as np
import pytest

import oracle
from tests.helpers import pkg, planets, rel_rms
from tests.test_gpu_parity import STAGES, TRANSFORM_TOL, PHYSICS_TOL, PHYSICS_FIELDS, FLIPPED_COLUMNS

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "earth_t21_climatology.npz")


def climatology():
    return np.load(FIXTURE)


def earth_planet(seed=5, levels=10):
    p = planets.make_planet(seed, truncation=21, levels=levels)
    c = climatology()
    p.boundary[169] = c["sst"].astype(np.float64).reshape(-1)
    p.boundary[210] = c["ice"].astype(np.float64).reshape(-1)
    return p


def test_fixture_holds_twelve_months_of_the_packaged_inputs():
    c = climatology()
    assert c["sst"].shape == (12, 2048) and c["ice"].shape == (12, 2048)
    assert [int(d) // 100 % 100 for d in c["sst_dates"]] == list(range(14))
    assert 265.0 < c["sst"].min() and c["sst"].max() < 310.0
    assert c["ice"].max() > 50.0  # polar ice in percent
    assert c["source_sha256"].size == 32


def test_earth_climatology_setup_matches_oracle():
    p = earth_planet()
    m = oracle.model_for(p)
    for name, ref in m["state"].items():
        got = pkg.setup_preview(p, "state:" + name)
        ref = np.asarray(ref, dtype=float).reshape(-1)
        assert got.shape == ref.shape, name
        assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0), name
    for step in (0, 250, 5000):
        got = pkg.setup_preview(p, f"calendar:{step}")
        vals, cs = oracle.setup_f64.step_values(step, 0, m["calendar"])
        ref = np.concatenate([vals["radiation_step"], vals["surface_step"], vals["carbon_step"], [cs]])
        np.testing.assert_allclose(got[:14], ref, atol=1e-12)
    # the climatology reaches the model: ocean points below freezing carry ice
    assert np.asarray(m["state"]["xclicec"]).max() > 0.5


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_earth_climatology_stage_replay(mode):
    from tests.test_gpu_parity import _replay_errors
    worst = _replay_errors(earth_planet(), 21, 10, 6, mode)
    for name, (err, stage) in worst.items():
        tol = PHYSICS_TOL if name in PHYSICS_FIELDS else TRANSFORM_TOL
        assert err <= tol, f"{name} after {stage}: relative RMS {err:.3e} > {tol:g}"


@pytest.mark.gpu
def test_earth_climatology_one_day():
    p = earth_planet(seed=6)
    e = pkg.Engine(21, 10, 1, mode=1)
    e.configure(0, p)
    o = oracle.Oracle(oracle.model_for(p))
    e.step(3)
    o.startup()
    for _ in range(4):
        e.step(8)
        o.advance(8)
    errs = {n: rel_rms(e.read(0, n), o.get(n)) for n in ("st", "sz", "sd", "sq", "sp", "dt", "xicec", "xsst")}
    print("Earth climatology, 1 day vs FP64:", errs)
    assert errs["st"] < 5e-3 and errs["sz"] < 1e-3 and errs["sq"] < 5e-2 and errs["sp"] < 5e-2
    assert errs["dt"] < 1e-3 and errs["xsst"] < 1e-3
