"""The reference's text formats on the host (no device): .sra surface files
(setup/surface/index.ts:76-104, boundary/index.ts:46-79), namelists
(namelist/index.ts:40-243) and JavaScript number formatting, checked
against the reference's packaged T21 inputs (tests/golden/
reference_inputs_t21.json.gz) and by round trips into the engine's set-up."""
import gzip
import importlib
import json
import os

import numpy as np
import pytest

from tests.helpers import pkg, planets

formats = importlib.import_module("web-exoplasim_b200.formats")
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
POINTS = 2048


@pytest.fixture(scope="module")
def files():
    with gzip.open(os.path.join(GOLDEN, "reference_inputs_t21.json.gz"), "rt", encoding="utf-8") as f:
        return json.load(f)["files"]


def test_read_sra_matches_the_extracted_climatology(files):
    ref = np.load(os.path.join(GOLDEN, "earth_t21_climatology.npz"))
    for code, key in ((169, "sst"), (210, "ice")):
        name = formats.sra_name(32, code)
        months = formats.read_sra(files[name], POINTS, formats.MONTHS, name)
        assert months.shape == (14, POINTS)
        np.testing.assert_array_equal(months[1:13].astype(np.float32), ref[key])
        headers, _ = formats.sra_records(files[name], POINTS)
        np.testing.assert_array_equal(headers[:, 2], ref[key + "_dates"])


def test_read_sra_fills_fourteen_months():
    rng = np.random.default_rng(0)
    twelve = rng.normal(size=(12, 16))
    text = "".join(formats.write_sra(169, m, 4, 4) for m in twelve)
    got = formats.read_sra(text, 16)
    np.testing.assert_allclose(got[1:13], twelve, atol=5e-4)
    np.testing.assert_array_equal(got[0], got[12])
    np.testing.assert_array_equal(got[13], got[1])
    one = formats.read_sra(formats.write_sra(169, twelve[0], 4, 4), 16)
    assert (one == one[0]).all()
    with pytest.raises(ValueError, match="has 5 fields, expected 14"):
        formats.read_sra("".join(formats.write_sra(169, m, 4, 4) for m in twelve[:5]), 16, name="x")


def test_write_sra_layout():
    text = formats.write_sra(172, np.arange(10) * 0.5, 4, 2)
    lines = text.split("\n")
    assert lines[0] == "".join(" " + str(v).rjust(11) for v in (172, 0, 20240101, 0, 4, 2, 0, 0))
    assert lines[1] == "".join(" " + f"{v:.3f}".rjust(9) for v in np.arange(8) * 0.5)
    assert lines[2] == "     4.000     4.500" and text.endswith("\n")
    files = formats.boundary_files(32, np.zeros(POINTS), np.ones(POINTS))
    assert sorted(files) == ["N032_surf_0129.sra", "N032_surf_0172.sra"]


@pytest.mark.parametrize("value,places,text", [
    (0.0625, 3, "0.063"), (-0.0625, 3, "-0.063"), (1.0005, 3, "1.000"), (-0.0, 3, "0.000"),
    (-0.0001, 3, "-0.000"), (2.5, 0, "3"), (271.3595, 3, "271.360"), (12345.6785, 3, "12345.678")])
def test_to_fixed_follows_javascript(value, places, text):
    assert formats.to_fixed(value, places) == text


@pytest.mark.parametrize("value,text", [
    (1.0, "1"), (0.1, "0.1"), (1e21, "1e+21"), (1e20, "100000000000000000000"), (1e-7, "1e-7"),
    (1.5e-5, "0.000015"), (-2.5, "-2.5"), (6371220.0, "6371220"), (1 / 3, "0.3333333333333333"),
    (5e-324, "5e-324"), (1.7976931348623157e308, "1.7976931348623157e+308"), (123e-20, "1.23e-18"),
    (0.0, "0"), (-0.0, "0"), (100040.0, "100040")])
def test_js_number(value, text):
    assert formats.js_number(value) == text


def test_namelist_parse_apply_read(files):
    text = files["plasim_namelist"]
    values = formats.parse_namelist(text)
    assert values["MPSTEP"] == "30.0" and values["SEED"] == "14963991,2,3,4,5,6,7,8" and values["NSTPW"] == "160"
    edited = formats.apply_namelist(text, {"MPSTEP": "45", "FIXEDLON": "180"})
    after = formats.parse_namelist(edited)
    assert after["MPSTEP"] == "45" and after["FIXEDLON"] == "180"
    assert edited.rstrip().endswith("/END") and edited.count("MPSTEP") == 1
    read = formats.read_namelist(edited, {"mpstep": 30.0, "seed": [0] * 10, "nveg": 2, "absent": 7.5})
    assert read["mpstep"] == 45 and read["seed"][:8] == [14963991, 2, 3, 4, 5, 6, 7, 8] and read["seed"][8:] == [0, 0]
    assert read["nveg"] == 0 and read["absent"] == 7.5
    assert formats.namelist_number(" 1.5d-3 ") == pytest.approx(1.5e-3)


def test_edits_match_the_reference_rules():
    cfg = dict(planets.BASE_CONFIG, layers=5, rotationPeriodDays=2.0, yearDays=365, stormclim=True)
    e = formats.namelist_edits(cfg)
    assert e["planet_namelist"]["ROTSPD"] == "0.5" and e["planet_namelist"]["PLARAD"] == "6371220"
    assert e["plasim_namelist"]["N_DAYS_PER_YEAR"] == "180" and e["plasim_namelist"]["N_START_YEAR"] == "0"
    assert e["plasim_namelist"]["NSELA"] == "0" and e["plasim_namelist"]["NSTPW"] == "160"
    assert e["landmod_namelist"]["DSOILZ"] == "0.4,0.8,1.6,3.2,6.4"
    assert e["hurricane_namelist"] == {"NSTORMDIAG": "1", "HC_CAPTURE": "0"}
    with pytest.raises(ValueError, match="5 or 10"):
        formats.namelist_edits(dict(cfg, layers=7))


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_configuration_round_trips_through_namelists(files, seed):
    rng = np.random.default_rng(seed)
    cfg = dict(planets.BASE_CONFIG, truncation=21, layers=10, radiusEarth=float(rng.uniform(0.5, 2)),
               gravityMs2=float(rng.uniform(5, 20)), rotationPeriodDays=float(rng.choice([1.0, 3.0])),
               pressureBar=float(rng.uniform(0.5, 3)), co2Ppm=float(rng.uniform(100, 1000)),
               oceanDepthM=float(rng.uniform(10, 100)), stormclim=bool(seed % 2), glaciersEnabled=bool(seed % 2))
    named = formats.apply_edits({k: v for k, v in files.items() if k.endswith("_namelist")}, cfg)
    got, ignored = formats.config_from_namelists(named, 21, 10)
    for key, value in cfg.items():
        if isinstance(value, float):
            assert got[key] == pytest.approx(value, rel=1e-14), key
        else:
            assert got[key] == value, key
    assert ("planet_namelist", "MVELP") in ignored and ("plasim_namelist", "SEED") in ignored


def test_planet_from_files_sets_up_as_the_planet(files):
    p = planets.make_planet(5, truncation=21, levels=5)
    nlat = 32
    bd = dict(p.boundary)
    sst = np.asarray(bd[169]).reshape(-1, POINTS)
    run = {k: v for k, v in files.items() if k.endswith("_namelist")}
    run = formats.apply_edits(run, p.config)
    run.update(formats.boundary_files(nlat, bd[172], bd.get(129, np.zeros(POINTS))))
    run[formats.sra_name(nlat, 169)] = "".join(formats.write_sra(169, m, 2 * nlat, nlat) for m in sst)
    q, _ = formats.planet_from_files(run, 21, 5, p.t_grid, p.q_grid)
    # the same planet with the boundary as the files carry it (three decimals)
    p.boundary = dict(q.boundary)
    for name in ("state:st", "state:sq", "table:bm1", "table:sop", "state:dls", "state:xclsst2", "const:GA",
                 "const:PSURF", "const:GASCON"):
        a = pkg.setup_preview(p, name)
        b = pkg.setup_preview(q, name)
        np.testing.assert_allclose(b, a, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(a).max()), err_msg=name)


@pytest.mark.gpu
def test_planet_from_files_steps_as_the_planet(files):
    """A run's namelists and .sra files, read by planet_from_files, configure
    and step the engine exactly as the planet they were written from."""
    p = planets.make_planet(6, truncation=21, levels=10, stormclim=True)
    nlat = 32
    bd = dict(p.boundary)
    run = formats.apply_edits({k: v for k, v in files.items() if k.endswith("_namelist")}, p.config)
    run.update(formats.boundary_files(nlat, bd[172], bd.get(129, np.zeros(POINTS))))
    sst = np.asarray(bd[169]).reshape(-1, POINTS)
    run[formats.sra_name(nlat, 169)] = "".join(formats.write_sra(169, m, 2 * nlat, nlat) for m in sst)
    q, _ = formats.planet_from_files(run, 21, 10, p.t_grid, p.q_grid)
    p.boundary = dict(q.boundary)  # the boundary as the files carry it
    engines = [pkg.Engine(21, 10, 1, mode=1) for _ in range(2)]
    try:
        engines[0].configure(0, p)
        engines[1].configure(0, q)
        for e in engines:
            e.step(3)
            e.step(8)
        for name in ("st", "sz", "sd", "sq", "sp", "dt", "dq", "dp", "capen", "gpi"):
            np.testing.assert_array_equal(engines[1].read(0, name), engines[0].read(0, name), err_msg=name)
    finally:
        for e in engines:
            e.close()
