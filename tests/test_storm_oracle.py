"""The oracle's storm diagnostics (physics/storm/wgsl/storm.wgsl) on the
reference's synthetic columns (verify-storm.mjs:48-66): the sequential-f32
build within the reference's storm tolerance of the FP64 one, and the
documented sentinels and limits (docs/climate/exoplasim-stormclim.md:22-30)."""
import numpy as np
import pytest

import oracle
from tests.helpers import STORM_FIELDS, planets, storm_columns, storm_state, storm_within


def run_oracle(levels, rd, precision, enabled=True):
    p = planets.make_planet(11, truncation=21, levels=levels, stormclim=enabled)
    model = oracle.model_for(p)
    o = oracle.Oracle(model, precision=precision)
    sigma = model["tables"]["sigma"]
    rows = storm_columns(sigma, rd)
    nhor = 2 * 32 * 32
    for name, values in storm_state(rows, levels, nhor).items():
        o.set(name, values)
    o.set_const("GASCON", rd)
    o.run("storm")
    return rows, {name: o.get(name) for name in STORM_FIELDS}, model


@pytest.mark.parametrize("levels", [5, 10])
@pytest.mark.parametrize("rd", [287.0, 189.0])
def test_f32_oracle_within_storm_tolerance_of_f64(levels, rd):
    _, f64, _ = run_oracle(levels, rd, 64)
    _, f32, _ = run_oracle(levels, rd, 32)
    assert storm_within(f32, f64) == {}


@pytest.mark.parametrize("levels", [5, 10])
def test_storm_sentinels_and_limits(levels):
    rows, out, model = run_oracle(levels, 287.0, 64)
    n = len(rows)
    col = {row["climate"]: k for k, row in enumerate(rows)}
    # SST at or below 5 C, or a profile at or below 100 K: intensity -1 and
    # the environmental CAPE / neutral-buoyancy pressure left at -1.
    for climate in ("cold", "cold-profile"):
        h = col[climate]
        if climate == "cold-profile" and min(rows[h]["t"][:levels]) > 100:
            continue  # at L5 the top level (sigma above 1/30) stays above 100 K
        assert out["mpoti"][h] == -1 and out["capen"][h] == -1 and out["lnb"][h] == -1, climate
    # A dry parcel: zero CAPE and -1 neutral-buoyancy pressure.
    assert out["capen"][col["dry"]] == 0 and out["lnb"][col["dry"]] == -1
    # Equal wind speeds at both levels: no shear, hence VI = 0 and a zero
    # reduced intensity (the native discontinuity at VI = 0).
    assert out["shear"][col["zero-shear"]] == 0 and out["vrmpi"][col["zero-shear"]] == 0
    # Vorticity is gz * ww at the level nearest sigma 0.85, signed.
    ww = model["phases"][0]["WW"]
    assert out["laav"][col["reversed-vorticity"]] == pytest.approx(-1.2 * ww)
    assert out["laav"][col["tropical"]] == pytest.approx(1.2 * ww)
    # The warm tropical columns have a positive potential intensity and CAPE.
    for climate in ("tropical", "warm", "hot", "humid"):
        assert out["mpoti"][col[climate]] > 0 and out["capen"][col[climate]] >= 0, climate
    # Every column of the tiled grid repeats its climate's values.
    for name in STORM_FIELDS:
        v = out[name]
        assert np.array_equal(v[:n], v[n:2 * n]), name


def test_disabled_storm_leaves_the_fields():
    _, out, _ = run_oracle(5, 287.0, 64, enabled=False)
    for name in STORM_FIELDS:
        assert not out[name].any(), name
