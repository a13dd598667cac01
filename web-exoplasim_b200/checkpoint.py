"""The reference's checkpoint container (checkpoint/index.ts:14-164), format 21
for this GPU engine: the magic line, a uint32 header length, a JSON header
{meta, diagnostics, terrain} whose Float32/Float64 arrays are replaced by
{array, offset, bytes} descriptors, a uint32 byte count, the arrays, then the
engine's restart file unchanged (exogcm_checkpoint_save: the
GCM-WEBGPU-STATE format of checkpoint/restart/index.ts).

The header is written as JavaScript's JSON.stringify writes it (compact,
numbers in JavaScript's shortest form), so a container this module writes
reads in the reference and the other way round. ``decode`` accepts formats
20 (CPU) and 21 (GPU) and checks the diagnostics against the saved
resolution as the reference does; ``save`` and ``load`` connect it to an
engine slot.
"""
from __future__ import annotations

import json
import math
import struct

import numpy as np

from .formats import js_number

MAGIC = b"EXOPLASIM-CHECKPOINT\n"
FORMATS = {"cpu": 20, "gpu": 21}
GPU_PRECISION_BYTES = 4
HEADER_LENGTH_BYTES = 4
MAX_TERRAIN_PIXELS = 8_388_608   # terrain/index.ts:9
LATITUDES = {21: 32, 42: 64, 63: 96}

# atmosphere/index.ts:8-64: gas molar masses (g/mol) and the native values.
UNIVERSAL_GAS_CONSTANT = 8314.46261815324
NATIVE_PRESSURE_BAR = 1.011
NATIVE_MEAN_MOLAR_MASS = 28.970253
NATIVE_GAS_CONSTANT = UNIVERSAL_GAS_CONSTANT / NATIVE_MEAN_MOLAR_MASS
NATIVE_CO2_PPM = 300
GAS_MOLAR_MASS = {"H2": 2.01588, "He": 4.002602, "N2": 28.0134, "O2": 31.9988, "Ar": 39.948, "Ne": 20.1797,
                  "Kr": 83.798, "CO2": 44.01, "H2O": 18.01528}


class CheckpointError(ValueError):
    """A container the reference would reject, with its message."""


# ---------------------------------------------------------------- JSON
def _json(value, arrays: list) -> str:
    """JSON.stringify with the container's replacer: float arrays become
    descriptors in the order they are met, appended to `arrays`."""
    if isinstance(value, np.ndarray) and value.dtype in (np.float32, np.float64):
        kind = "Float32Array" if value.dtype == np.float32 else "Float64Array"
        raw = np.ascontiguousarray(value).astype(value.dtype.newbyteorder("<"), copy=False).tobytes()
        offset = sum(len(a) for a in arrays)
        arrays.append(raw)
        return _json({"array": kind, "offset": offset, "bytes": len(raw)}, arrays)
    if value is None:
        return "null"
    if isinstance(value, (bool, np.bool_)):
        return "true" if value else "false"
    if isinstance(value, (int, np.integer)):
        return js_number(float(value)) if abs(int(value)) >= 2 ** 53 else str(int(value))
    if isinstance(value, (float, np.floating)):
        return js_number(value) if math.isfinite(value) else "null"
    if isinstance(value, str):
        return json.dumps(value, ensure_ascii=False)
    if isinstance(value, dict):
        return "{" + ",".join(json.dumps(str(k), ensure_ascii=False) + ":" + _json(v, arrays)
                              for k, v in value.items()) + "}"
    if isinstance(value, (list, tuple)):
        return "[" + ",".join(_json(v, arrays) for v in value) + "]"
    raise TypeError(f"cannot write {type(value).__name__} into a checkpoint header")


def encode(meta: dict, restart: bytes, diagnostics: dict, terrain: dict) -> bytes:
    """checkpoint/index.ts:20-64 (encode)."""
    arrays: list[bytes] = []
    header = _json({"meta": meta, "diagnostics": diagnostics, "terrain": terrain}, arrays).encode("utf-8")
    blob = b"".join(arrays)
    return b"".join([MAGIC, struct.pack("<I", len(header)), header, struct.pack("<I", len(blob)), blob,
                     bytes(restart)])


def field_count(layers: int) -> int:
    """fields/index.ts:416-418: 51 surface fields plus five per layer."""
    return 51 + 5 * layers


def validate_terrain(terrain: dict) -> dict:
    """terrain/index.ts:11-48."""
    width, height = terrain.get("width"), terrain.get("height")
    if not (isinstance(height, int) and height >= 2 and width == 2 * height and width * height <= MAX_TERRAIN_PIXELS):
        raise CheckpointError("Terrain must be a full-world 2:1 raster, at least 4 × 2 and at most 4096 × 2048 pixels")
    elev, land = terrain.get("elevationM"), terrain.get("land")
    if not (isinstance(elev, np.ndarray) and elev.dtype == np.float32 and isinstance(land, np.ndarray)
            and land.dtype == np.float32 and elev.size == width * height and land.size == elev.size):
        raise CheckpointError("Terrain arrays do not match the image dimensions")
    if not (np.isfinite(elev).all() and np.isfinite(land).all() and (land >= 0).all() and (land <= 1).all()):
        raise CheckpointError("Terrain requires finite elevations and land coverage between 0 and 1")
    return terrain


def decode(data: bytes) -> dict:
    """checkpoint/index.ts:66-148 (decode): {meta, diagnostics, terrain,
    restart}, or CheckpointError with the reference's message."""
    data = bytes(data)
    if data[:len(MAGIC)] != MAGIC:
        raise CheckpointError("Not an ExoPlaSim checkpoint file")
    if len(data) < len(MAGIC) + HEADER_LENGTH_BYTES:
        raise CheckpointError("Truncated ExoPlaSim checkpoint")
    (header_length,) = struct.unpack_from("<I", data, len(MAGIC))
    header_start = len(MAGIC) + HEADER_LENGTH_BYTES
    header_end = header_start + header_length
    if header_end + HEADER_LENGTH_BYTES > len(data):
        raise CheckpointError("Truncated ExoPlaSim checkpoint")
    header = data[header_start:header_end].decode("utf-8")
    meta = json.loads(header)["meta"]
    if meta.get("format") not in FORMATS.values():
        raise CheckpointError(f"Unsupported checkpoint format {js_number(meta.get('format', float('nan')))}. "
                              f"Format {FORMATS['cpu']} (CPU) or {FORMATS['gpu']} (GPU) is required.")
    (array_bytes,) = struct.unpack_from("<I", data, header_end)
    array_start = header_end + HEADER_LENGTH_BYTES
    restart_start = array_start + array_bytes
    if restart_start >= len(data):
        raise CheckpointError("Truncated ExoPlaSim checkpoint")

    def revive(obj):
        if obj.get("array") in ("Float32Array", "Float64Array"):
            off, size = obj.get("offset"), obj.get("bytes")
            if not (isinstance(off, int) and isinstance(size, int) and off >= 0 and size >= 0
                    and off + size <= array_bytes):
                raise CheckpointError("Invalid checkpoint diagnostic array")
            dtype = np.dtype("<f4") if obj["array"] == "Float32Array" else np.dtype("<f8")
            if size % dtype.itemsize:
                raise CheckpointError("Invalid checkpoint diagnostic array")
            return np.frombuffer(data, dtype=dtype, count=size // dtype.itemsize, offset=array_start + off).copy()
        return obj

    parsed = json.loads(header, object_hook=revive)
    diagnostics, terrain = parsed["diagnostics"], parsed["terrain"]
    config = meta["config"]
    if config.get("layers") not in (5, 10):
        raise CheckpointError("Invalid checkpoint atmospheric layer count")
    if config.get("targetTemperatureK") is not None:
        raise CheckpointError("Checkpoints of temperature-targeted runs are not supported by this engine")
    averager = diagnostics["averager"]
    snapshots = [diagnostics["snapshot"]] + [m["snapshot"] for m in averager["months"]]
    if averager.get("current"):
        snapshots.append(averager["current"]["last"])
    points = 2 * LATITUDES[config["truncation"]] ** 2
    expected = points * field_count(config["layers"])
    if any(s["layers"] != config["layers"] or np.size(s["values"]) != expected for s in snapshots) or \
            (averager.get("current") and np.size(averager["current"]["sum"]) != expected):
        raise CheckpointError("Checkpoint diagnostics do not match the saved model resolution and atmospheric layers")
    return {"meta": meta, "diagnostics": diagnostics, "terrain": validate_terrain(terrain),
            "restart": data[restart_start:]}


def engine_of(meta: dict) -> str:
    return "gpu" if meta["format"] == FORMATS["gpu"] else "cpu"


def file_name(meta: dict) -> str:
    """checkpoint/index.ts:154-157."""
    d, c = meta["date"], meta["config"]
    return f"exoplasim-t{c['truncation']}-layers{c['layers']}-year{d['year']:04d}-month{d['month']:02d}.ckpt"


# ---------------------------------------------------------------- configuration
def resolve_atmosphere(atm: dict) -> dict:
    """atmosphere/index.ts:84-163 (resolve): pressure, gas constant and CO2
    of the reference's atmosphere settings."""
    specified = weighted = 0.0
    pressures = atm.get("partialPressures", {})
    for gas, mass in GAS_MOLAR_MASS.items():
        p = pressures.get(gas)
        if p is None:
            continue
        if not (math.isfinite(p) and p >= 0):
            raise CheckpointError(f"{gas} partial pressure must be finite and nonnegative.")
        specified += p
        weighted += p * mass
    pressure = specified or NATIVE_PRESSURE_BAR
    gascon = UNIVERSAL_GAS_CONSTANT / (weighted / specified) if specified > 0 else NATIVE_GAS_CONSTANT
    if atm.get("mode") == "pressureAndGasConstant":
        pressure = NATIVE_PRESSURE_BAR if atm.get("pressureBar") is None else atm["pressureBar"]
        gascon = NATIVE_GAS_CONSTANT if atm.get("gasConstant") is None else atm["gasConstant"]
    elif atm.get("mode") != "partialPressures":
        raise CheckpointError("Choose an atmosphere input mode.")
    if not (math.isfinite(pressure) and pressure > 0 and math.isfinite(gascon) and gascon > 0):
        raise CheckpointError("Total pressure and gas constant must be finite and positive.")
    if specified > pressure + 1e-12 * max(1.0, pressure):
        raise CheckpointError("The specified partial pressures exceed total surface pressure.")
    co2 = pressures.get("CO2")
    return {"pressureBar": pressure, "gasConstant": gascon,
            "co2Ppm": NATIVE_CO2_PPM if co2 is None else min(1.0, co2 / pressure) * 1e6}


def gcm_config(config: dict) -> dict:
    """The reference's GcmConfig (types.ts, key order of index.ts:4-43) for a
    planets configuration; its atmosphere as total pressure, gas constant
    and a CO2 partial pressure."""
    p = float(config["pressureBar"])
    return {
        "targetTemperatureK": None,
        "stormclim": bool(config.get("stormclim", False)),
        "atmosphere": {"mode": "pressureAndGasConstant",
                       "partialPressures": {g: (p * config["co2Ppm"] / 1e6 if g == "CO2" else None)
                                            for g in GAS_MOLAR_MASS},
                       "pressureBar": p, "gasConstant": float(config["gasConstant"]),
                       "ozone": bool(config["ozone"])},
        "layers": int(config["layers"]),
        "periapseLongitudeDeg": None, "keplerian": bool(config["keplerian"]), "initialMeanAnomalyDeg": None,
        "soilWaterCapacityM": None, "soilHeatCapacity": None, "soilDepthScale": float(config["soilDepthScale"]),
        "landAlbedo": None, "oceanAlbedo": None, "snowIceAlbedo": None,
        "radiusEarth": float(config["radiusEarth"]), "gravityMs2": float(config["gravityMs2"]),
        "synchronous": bool(config["synchronous"]), "substellarLongitudeDeg": float(config["substellarLongitudeDeg"]),
        "oceanDepthM": float(config["oceanDepthM"]), "fluxWm2": float(config["fluxWm2"]),
        "starTemperatureK": float(config["starTemperatureK"]), "yearDays": float(config["yearDays"]),
        "eccentricity": float(config["eccentricity"]), "rotationPeriodDays": float(config["rotationPeriodDays"]),
        "obliquityDeg": float(config["obliquityDeg"]), "fixedOrbit": bool(config["fixedOrbit"]),
        "wetSoil": bool(config["wetSoil"]), "vegetation": int(config["vegetation"]),
        "initialGrowth": float(config["initialGrowth"]),
        "glaciers": {"enabled": bool(config["glaciersEnabled"]), "minDepthM": float(config["glaciersMinDepthM"]),
                     "initialHeightM": float(config["glaciersInitialHeightM"])},
        "physicsFilter": list(config["physicsFilter"]),
        "timestepMinutes": float(config["timestepMinutes"]),
        "truncation": int(config["truncation"]),
        "earthSurfaceClimatology": bool(config.get("earthSurfaceClimatology", False)),
    }


def flat_config(gcm: dict) -> dict:
    """The planets configuration of a GcmConfig (the inverse of gcm_config;
    settings the engine does not take must be at their defaults)."""
    for key in ("periapseLongitudeDeg", "initialMeanAnomalyDeg", "soilWaterCapacityM", "soilHeatCapacity",
                "landAlbedo", "oceanAlbedo", "snowIceAlbedo", "targetTemperatureK"):
        if gcm.get(key) is not None:
            raise CheckpointError(f"{key} is not supported by this engine")
    atm = resolve_atmosphere(gcm["atmosphere"])
    g = gcm["glaciers"]
    out = {k: gcm[k] for k in ("layers", "truncation", "radiusEarth", "gravityMs2", "synchronous",
                               "substellarLongitudeDeg", "oceanDepthM", "fluxWm2", "starTemperatureK", "yearDays",
                               "eccentricity", "rotationPeriodDays", "obliquityDeg", "fixedOrbit", "keplerian",
                               "wetSoil", "vegetation", "initialGrowth", "timestepMinutes", "soilDepthScale",
                               "stormclim")}
    out.update(pressureBar=atm["pressureBar"], gasConstant=atm["gasConstant"], co2Ppm=atm["co2Ppm"],
               ozone=bool(gcm["atmosphere"]["ozone"]), glaciersEnabled=g["enabled"], glaciersMinDepthM=g["minDepthM"],
               glaciersInitialHeightM=g["initialHeightM"], physicsFilter=tuple(gcm["physicsFilter"]))
    return out


# ---------------------------------------------------------------- engine slots
def planet_terrain(planet) -> dict:
    """A terrain raster on the model grid for a planet without an image:
    elevation = surface geopotential / g, land = the land mask."""
    cfg = planet.config
    nlat = LATITUDES[cfg["truncation"]]
    points = 2 * nlat * nlat
    oro = planet.boundary.get(129)
    oro = np.zeros(points) if oro is None else np.asarray(oro, dtype=np.float64).reshape(points)
    land = np.clip(np.asarray(planet.boundary[172], dtype=np.float64).reshape(points), 0, 1)
    return {"name": "Planet", "width": 2 * nlat, "height": nlat,
            "elevationM": (oro / cfg["gravityMs2"]).astype(np.float32), "land": land.astype(np.float32)}


def save(engine, slot: int, planet, averager: dict | None = None, terrain: dict | None = None,
         snapshot: dict | None = None) -> bytes:
    """A format-21 container of an engine slot: its restart state, the
    planet's configuration, the last snapshot (the slot's published
    snapshot, else its packed snapshot field) and the averager."""
    cfg = planet.config
    info = engine.slot_info(slot)
    step = int(info["step"])
    if snapshot is None:
        pub_step, values = engine.snapshot(slot)
        if pub_step < 0:
            pub_step, values = step, engine.read(slot, "snapshot")
        snapshot = {"layers": int(cfg["layers"]), "step": int(pub_step), "date": engine.date(slot, pub_step),
                    "values": np.asarray(values, dtype=np.float32).reshape(-1)}
    meta = {"format": FORMATS["gpu"], "config": gcm_config(cfg), "precisionBytes": GPU_PRECISION_BYTES,
            "date": engine.date(slot, step), "step": step}
    diagnostics = {"targeting": None, "averager": averager or {"current": None, "months": [], "years": []},
                   "snapshot": snapshot}
    return encode(meta, engine.checkpoint_save(slot), diagnostics, terrain or planet_terrain(planet))


def load(engine, slot: int, data: bytes) -> dict:
    """Restores a format-21 container into a configured slot of the same
    resolution; returns its meta and diagnostics. A CPU-engine container
    (format 20) carries a native restart this engine cannot read."""
    ckpt = decode(data)
    if engine_of(ckpt["meta"]) != "gpu":
        raise CheckpointError("This checkpoint was not saved by the WebGPU model")
    engine.checkpoint_load(slot, ckpt["restart"])
    return ckpt
