"""Parity on the reference's packaged Earth climatologies (tests/golden/,
made by make_earth_climatology.py from public/gcm/t21/inputs.json): a
planet whose sea-surface temperature and ice-cover climatologies are the
Earth's monthly fields, so the month interpolation of the surface step and
the sea-ice and slab-ocean routines run on the reference's own data."""
import os

import numpy as np
import pytest

import oracle
from tests.helpers import pkg, planets

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
    """Every stage on the Earth SST and sea-ice climatology passes the
    reference's V3 gate (see tests/test_gpu_parity.py)."""
    from tests.test_gpu_parity import replay_v3
    verdicts = replay_v3(earth_planet(), 21, 10, 6, mode)
    failed = [(k, v) for k, v in verdicts.items() if not v["ok"]]
    assert not failed, failed[:5]


@pytest.mark.gpu
def test_earth_climatology_one_day():
    """One day on the Earth climatology (start-up included) by the reference's
    V4 gate against the FP64 and sequential-f32 oracles."""
    from tests.test_gpu_parity import v4_judge
    p = earth_planet(seed=6)
    m = oracle.model_for(p)
    m["state"] = {k: np.asarray(v, dtype=np.float64).astype(np.float32).astype(np.float64)
                  for k, v in m["state"].items()}
    e = pkg.Engine(21, 10, 1, mode=1)
    e.configure(0, p)
    for name, v in m["state"].items():
        e.write(0, name, v.astype(np.float32))
    o64, o32 = oracle.Oracle(m), oracle.Oracle(m, precision=32)
    e.step(3)
    e.step(32)
    for o in (o64, o32):
        o.advance(32)
    verdict = v4_judge(e, o64, o32, fields=("st", "sz", "sd", "sq", "sp", "dt", "xicec", "xsst", "xiced"))
    print("Earth climatology, 1 day (GPU, f32) vs FP64:", verdict)
    bad = {k: v for k, v in verdict.items() if not v[2]}
    assert not bad, bad
