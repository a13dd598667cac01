"""The format-21 checkpoint container (checkpoint/index.ts:14-164) on the
host: byte layout, JavaScript-compatible header, round trips and the
reference's rejections; a container of an engine slot restored into a
fresh engine steps on bit for bit (GPU)."""
import importlib
import json
import struct

import numpy as np
import pytest

from tests.helpers import field_names, pkg, planets

checkpoint = importlib.import_module("web-exoplasim_b200.checkpoint")
POINTS = 2048


def sample(layers=5, truncation=21, fmt=21, restart=b"GCM-WEBGPU-STATE\nrest"):
    points = 2 * checkpoint.LATITUDES[truncation] ** 2
    n = points * checkpoint.field_count(layers)
    cfg = checkpoint.gcm_config(dict(planets.BASE_CONFIG, layers=layers, truncation=truncation))
    date = {"year": 1, "month": 2, "day": 3, "hour": 4, "minute": 30}
    snap = {"layers": layers, "step": 96, "date": date, "values": np.arange(n, dtype=np.float32)}
    meta = {"format": fmt, "config": cfg, "precisionBytes": 4, "date": date, "step": 97}
    averager = {"current": {"year": 1, "month": 2, "sum": np.linspace(0, 1, n), "samples": 3, "last": snap},
                "months": [{"year": 1, "month": 1, "snapshot": snap}], "years": []}
    terrain = {"name": "Planet", "width": 8, "height": 4, "elevationM": np.zeros(32, np.float32),
               "land": np.ones(32, np.float32)}
    return meta, restart, {"targeting": None, "averager": averager, "snapshot": snap}, terrain


def test_layout_and_header():
    meta, restart, diag, terrain = sample()
    data = checkpoint.encode(meta, restart, diag, terrain)
    assert data.startswith(b"EXOPLASIM-CHECKPOINT\n")
    (hl,) = struct.unpack_from("<I", data, 21)
    header = data[25:25 + hl].decode()
    (ab,) = struct.unpack_from("<I", data, 25 + hl)
    # JSON.stringify's compact form; arrays replaced in the order met
    assert header.startswith('{"meta":{"format":21,"config":{"targetTemperatureK":null,"stormclim":false,')
    assert '"radiusEarth":1,' in header and '"gravityMs2":9.80665,' in header
    parsed = json.loads(header)
    n = 76 * POINTS
    # diagnostics = {targeting, averager, snapshot}: the averager's sum, its
    # last snapshot and its month come first, then the snapshot, the terrain
    avg = parsed["diagnostics"]["averager"]
    assert avg["current"]["sum"] == {"array": "Float64Array", "offset": 0, "bytes": n * 8}
    assert avg["current"]["last"]["values"] == {"array": "Float32Array", "offset": n * 8, "bytes": n * 4}
    assert avg["months"][0]["snapshot"]["values"]["offset"] == n * 12
    assert parsed["diagnostics"]["snapshot"]["values"] == {"array": "Float32Array", "offset": n * 16, "bytes": n * 4}
    assert parsed["terrain"]["land"] == {"array": "Float32Array", "offset": n * 20 + 128, "bytes": 128}
    assert ab == n * 20 + 2 * 32 * 4
    assert data[25 + hl + 4 + ab:] == restart


def test_round_trip():
    meta, restart, diag, terrain = sample(layers=10)
    got = checkpoint.decode(checkpoint.encode(meta, restart, diag, terrain))
    assert got["restart"] == restart and got["meta"] == json.loads(json.dumps(meta))
    np.testing.assert_array_equal(got["diagnostics"]["snapshot"]["values"], diag["snapshot"]["values"])
    assert got["diagnostics"]["averager"]["current"]["sum"].dtype == np.float64
    np.testing.assert_array_equal(got["diagnostics"]["averager"]["current"]["sum"],
                                  diag["averager"]["current"]["sum"])
    assert checkpoint.file_name(got["meta"]) == "exoplasim-t21-layers10-year0001-month02.ckpt"
    assert checkpoint.engine_of(got["meta"]) == "gpu"


def rewrite(data, edit):
    """The container with its JSON header edited and its length field kept right."""
    (hl,) = struct.unpack_from("<I", data, 21)
    header = edit(data[25:25 + hl].decode()).encode()
    return data[:21] + struct.pack("<I", len(header)) + header + data[25 + hl:]


@pytest.mark.parametrize("mutate,message", [
    (lambda d: b"X" + d[1:], "Not an ExoPlaSim checkpoint file"),
    (lambda d: d[:23], "Truncated ExoPlaSim checkpoint"),
    (lambda d: d.replace(b'"format":21', b'"format":19', 1), "Unsupported checkpoint format 19. Format 20 (CPU) or "
                                                            "21 (GPU) is required."),
    (lambda d: d.replace(b'"layers":5,"periapse', b'"layers":7,"periapse', 1), "Invalid checkpoint atmospheric"),
    (lambda d: rewrite(d, lambda h: h.replace('"offset":0,', '"offset":-4,', 1)), "Invalid checkpoint diagnostic"),
    (lambda d: rewrite(d, lambda h: h.replace('"offset":0,', '"offset":0.5,', 1)), "Invalid checkpoint diagnostic"),
])
def test_rejections(mutate, message):
    meta, restart, diag, terrain = sample()
    data = checkpoint.encode(meta, restart, diag, terrain)
    with pytest.raises(checkpoint.CheckpointError, match=message.replace("(", r"\(").replace(")", r"\)")):
        checkpoint.decode(mutate(data))


def test_rejects_mismatched_diagnostics_and_terrain():
    meta, restart, diag, terrain = sample()
    diag["snapshot"]["values"] = diag["snapshot"]["values"][:-1]
    with pytest.raises(checkpoint.CheckpointError, match="do not match the saved model resolution"):
        checkpoint.decode(checkpoint.encode(meta, restart, diag, terrain))
    meta, restart, diag, terrain = sample()
    terrain["land"] = terrain["land"] * 2
    with pytest.raises(checkpoint.CheckpointError, match="land coverage between 0 and 1"):
        checkpoint.decode(checkpoint.encode(meta, restart, diag, terrain))
    meta, restart, diag, terrain = sample()
    terrain["width"] = 6
    with pytest.raises(checkpoint.CheckpointError, match="full-world 2:1 raster"):
        checkpoint.decode(checkpoint.encode(meta, restart, diag, terrain))


def test_configuration_round_trip_and_atmosphere():
    cfg = dict(planets.BASE_CONFIG, pressureBar=2.5, gasConstant=300.0, co2Ppm=420.0, stormclim=True)
    back = checkpoint.flat_config(checkpoint.gcm_config(cfg))
    for k, v in back.items():
        if isinstance(v, float):
            assert v == pytest.approx(cfg[k], rel=1e-12), k
        else:
            assert v == cfg[k], k
    air = {"mode": "partialPressures", "partialPressures": dict.fromkeys(checkpoint.GAS_MOLAR_MASS),
           "pressureBar": None, "gasConstant": None, "ozone": True}
    air["partialPressures"].update(N2=0.78, O2=0.21, Ar=0.0093, CO2=0.0004)
    res = checkpoint.resolve_atmosphere(air)
    mass = (0.78 * 28.0134 + 0.21 * 31.9988 + 0.0093 * 39.948 + 0.0004 * 44.01) / 0.9997
    assert res["pressureBar"] == pytest.approx(0.9997)
    assert res["gasConstant"] == pytest.approx(checkpoint.UNIVERSAL_GAS_CONSTANT / mass)
    assert res["co2Ppm"] == pytest.approx(0.0004 / 0.9997 * 1e6)
    air["partialPressures"]["CO2"] = None
    assert checkpoint.resolve_atmosphere(air)["co2Ppm"] == 300
    air["mode"] = "pressureAndGasConstant"
    air["pressureBar"] = 0.5
    with pytest.raises(checkpoint.CheckpointError, match="exceed total surface pressure"):
        checkpoint.resolve_atmosphere(air)


@pytest.mark.gpu
def test_engine_container_restores_bit_for_bit():
    p = planets.make_planet(21, truncation=21, levels=5)
    e, f = pkg.Engine(21, 5, 1, mode=1), pkg.Engine(21, 5, 1, mode=1)
    try:
        e.configure(0, p)
        e.step(3)
        e.step(24, publish_every=24)
        data = checkpoint.save(e, 0, p)
        ckpt = checkpoint.decode(data)
        info = e.slot_info(0)
        assert ckpt["meta"]["step"] == info["step"] and ckpt["meta"]["date"] == e.date(0)
        back = checkpoint.flat_config(ckpt["meta"]["config"])
        assert back["rotationPeriodDays"] == p.config["rotationPeriodDays"] and back["layers"] == 5
        assert ckpt["diagnostics"]["snapshot"]["values"].size == 76 * e.nhor
        f.configure(0, p)
        f.step(3)
        checkpoint.load(f, 0, data)
        assert f.slot_info(0)["step"] == info["step"]
        e.step(16, publish_every=16)
        f.step(16, publish_every=16)
        import oracle
        for name in field_names(oracle.Oracle(oracle.model_for(p))):
            np.testing.assert_array_equal(f.read(0, name), e.read(0, name), err_msg=name)
    finally:
        e.close()
        f.close()
