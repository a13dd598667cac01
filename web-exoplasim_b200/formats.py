"""The reference's input formats on the host: ExoPlaSim ``.sra`` surface
files and Fortran namelist text, read into the engine's planet
configuration and boundary arrays, and written back.

- ``.sra``: an 8-integer header and NUGP values per record
  (setup/surface/index.ts:76-104 ``read``; boundary/index.ts:46-62 ``toSra``
  and 64-79 ``files``).
- namelists: ``KEY = value`` lines between a group header and ``/END``
  (namelist/index.ts:184-231 ``apply``, ``parse``, ``read``), and the edits
  a configuration makes to them (namelist/index.ts:40-182 ``edits``).
- ``planet_from_files``: a planets.Planet from a run directory's files (the
  namelists plus N<NLAT>_surf_<code>.sra), for exogcm_configure.

Numbers written into text follow JavaScript's Number-to-String and
``toFixed`` so files match the reference's byte for byte.
"""
from __future__ import annotations

import math
import re
from decimal import ROUND_HALF_UP, Decimal

import numpy as np

EARTH_RADIUS_M = 6371220.0       # namelist/index.ts:11
SECONDS_PER_DAY = 86400.0
NSTPW_WINDOW_MINUTES = 7200
SOIL_LAYER_DEPTHS_M = (0.4, 0.8, 1.6, 3.2, 6.4)
SRA_VALUES_PER_LINE = 8
MONTHS = 14                      # December before, the twelve months, January after
LAND_SEA_CODE, OROGRAPHY_CODE, SST_CODE, ICE_COVER_CODE = 172, 129, 169, 210
LATITUDES = {21: 32, 42: 64, 63: 96}

# namelist/index.ts:26-33.
FILTER_SWITCHES = {"gp": ("NGPTFILTER", "1"), "sp": ("NSPVFILTER", "1"), "none": ("NFILTER", "0"),
                   "cesaro": ("NFILTER", "1"), "exp": ("NFILTER", "2"), "lh": ("NFILTER", "3")}
VEGETATION_DEFAULTS = {"NCVEG": "1", "FORGROW": "1.0", "RINIDSC": "1.0", "RINIDMR": "2.0", "RINISOIL": "0.0",
                       "RINIVEG": "0.0"}


# ---------------------------------------------------------------- numbers
def js_number(x) -> str:
    """JavaScript's String(x) for a number (ECMAScript Number::toString):
    the shortest round-trip digits, plain between 1e-7 and 1e21."""
    x = float(x)
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "Infinity" if x > 0 else "-Infinity"
    if x == 0:
        return "0"
    sign = "-" if x < 0 else ""
    t = Decimal(repr(abs(x))).as_tuple()
    digits = "".join(map(str, t.digits)).rstrip("0")
    exponent = t.exponent + (len(t.digits) - len(digits))
    k = len(digits)
    n = k + exponent  # value = 0.digits x 10^n
    if k <= n <= 21:
        body = digits + "0" * (n - k)
    elif 0 < n <= 21:
        body = digits[:n] + "." + digits[n:]
    elif -6 < n <= 0:
        body = "0." + "0" * (-n) + digits
    else:
        e = n - 1
        body = (digits if k == 1 else digits[0] + "." + digits[1:]) + "e" + ("+" if e >= 0 else "-") + str(abs(e))
    return sign + body


def to_fixed(x, places: int) -> str:
    """JavaScript's x.toFixed(places): the exact binary value rounded half
    away from zero; -0 prints without a sign."""
    x = float(x)
    if x == 0:
        x = 0.0
    q = Decimal(x).quantize(Decimal(1).scaleb(-places), rounding=ROUND_HALF_UP)
    s = format(q, "f")
    return s


# ---------------------------------------------------------------- .sra
def sra_name(nlat: int, code: int) -> str:
    return f"N{nlat:03d}_surf_{code:04d}.sra"


def read_sra(text: str, points: int, months: int = MONTHS, name: str = "") -> np.ndarray:
    """setup/surface/index.ts:76-104 (get_surf_array): `months` fields of
    `points` values from records of 8 header integers and `points` values.
    Of 14 months, a file of 12 gains December before and January after, a
    file of 1 fills all 14."""
    tokens = np.array(text.split(), dtype=np.float64)
    record = 8 + points
    found = min(months, len(tokens) // record)
    out = np.zeros((months, points))
    for month in range(found):
        out[month] = tokens[month * record + 8:(month + 1) * record]
    if found == months:
        return out
    if found == 12 and months == MONTHS:
        out[1:13] = out[0:12].copy()
        out[13] = out[1]
        out[0] = out[12]
    elif found == 1 and months == MONTHS:
        out[1:] = out[0]
    else:
        raise ValueError(f"{name or 'surface file'} has {found} fields, expected {months}")
    return out


def sra_records(text: str, points: int) -> tuple[np.ndarray, np.ndarray]:
    """Every record of a .sra file as (headers [n][8] int, values [n][points])."""
    tokens = np.array(text.split(), dtype=np.float64)
    record = 8 + points
    n = len(tokens) // record
    rec = tokens[:n * record].reshape(n, record)
    return rec[:, :8].astype(np.int64), rec[:, 8:]


def write_sra(code: int, values, nlon: int, nlat: int) -> str:
    """boundary/index.ts:46-62 (toSra): one record, header
    [code, 0, 20240101, 0, NLON, NLAT, 0, 0] right-aligned in 11 columns,
    then eight values a line with three decimals in 9 columns."""
    header = "".join(" " + js_number(v).rjust(11) for v in (code, 0, 20240101, 0, nlon, nlat, 0, 0))
    vals = np.asarray(values, dtype=np.float64).reshape(-1)
    lines = [header]
    for start in range(0, len(vals), SRA_VALUES_PER_LINE):
        lines.append("".join(" " + to_fixed(v, 3).rjust(9) for v in vals[start:start + SRA_VALUES_PER_LINE]))
    return "\n".join(lines) + "\n"


def boundary_files(nlat: int, land_fraction, geopotential) -> dict:
    """boundary/index.ts:64-79 (files): the land mask and orography files."""
    nlon = 2 * nlat
    return {sra_name(nlat, LAND_SEA_CODE): write_sra(LAND_SEA_CODE, land_fraction, nlon, nlat),
            sra_name(nlat, OROGRAPHY_CODE): write_sra(OROGRAPHY_CODE, geopotential, nlon, nlat)}


# ---------------------------------------------------------------- namelists
_LINE = re.compile(r"^\s*([A-Za-z_][A-Za-z0-9_]*)\s*=\s*(.*?)\s*$")


def parse_namelist(text: str) -> dict:
    """namelist/index.ts:201-211: KEY = value lines, keys upper-cased,
    values as written (comma lists stay one string)."""
    out = {}
    for line in re.split(r"\r?\n", text or ""):
        m = _LINE.match(line)
        if m:
            out[m.group(1).upper()] = m.group(2)
    return out


def namelist_number(text: str) -> float:
    """namelist/index.ts:213-215: Fortran's d exponent read as e."""
    return float(re.sub(r"[dD]", "e", text.strip(), count=1))


def read_namelist(text: str, defaults: dict) -> dict:
    """namelist/index.ts:217-241: the defaults with every value the text
    sets; arrays are filled from the front."""
    values = parse_namelist(text or "")
    out = dict(defaults)
    for key, fallback in defaults.items():
        value = values.get(key.upper())
        if value is None:
            continue
        parts = [namelist_number(p) for p in value.split(",")]
        if isinstance(fallback, (list, tuple)):
            arr = list(fallback)
            for i, p in enumerate(parts):
                if i < len(arr):
                    arr[i] = p
                else:
                    arr.append(p)
            out[key] = arr
        else:
            out[key] = parts[0]
    return out


def apply_namelist(text: str, values: dict) -> str:
    """namelist/index.ts:184-196: replace each KEY's line, or add it before /END."""
    result = text
    for key, value in values.items():
        line = f" {key} = {value}"
        pattern = re.compile(rf"^\s*{re.escape(key)}\s*=.*$", re.I | re.M)
        if pattern.search(result):
            result = pattern.sub(lambda _m: line, result, count=1)
        else:
            result = re.sub(r"^\s*/END", lambda _m: f"{line}\n /END", result, count=1, flags=re.I | re.M)
    return result


def _flag(v) -> str:
    return "1" if v else "0"


def namelist_edits(config: dict) -> dict:
    """namelist/index.ts:40-182 (edits) for a planets configuration (its
    flat keys: pressureBar, gasConstant, co2Ppm and ozone resolved from the
    reference's atmosphere, glaciersEnabled/MinDepthM/InitialHeightM for
    its glaciers group)."""
    s = js_number
    if config["layers"] not in (5, 10):
        raise ValueError("Choose 5 or 10 atmospheric layers")
    planet = {"GA": s(config["gravityMs2"]), "PLARAD": s(config["radiusEarth"] * EARTH_RADIUS_M),
              "GSOL0": s(config["fluxWm2"]), "ECCEN": s(config["eccentricity"]), "OBLIQ": s(config["obliquityDeg"]),
              "NFIXORB": _flag(config["fixedOrbit"]), "NGENKEPLERIAN": _flag(config["keplerian"]),
              "GASCON": s(config["gasConstant"]), "SIDEREAL_YEAR": s(config["yearDays"] * SECONDS_PER_DAY)}
    tsm = config["timestepMinutes"]
    plasim = {"FIXEDLON": s(config["substellarLongitudeDeg"]), "N_DAYS_PER_YEAR": s(config["yearDays"]),
              "PSURF": s(config["pressureBar"] * 1e5), "NVEG": s(config["vegetation"]), "NEQSIG": "0",
              "MPSTEP": s(tsm), "NSTPW": s(math.floor(NSTPW_WINDOW_MINUTES / tsm)), "FILTERKAPPA": "8",
              "NFILTEREXP": "8", "LANDHOSKN0": "15"}
    if config["layers"] == 5:
        plasim["NSELA"] = "0"
    if config["rotationPeriodDays"] != 1:
        planet["ROTSPD"] = s(1 / config["rotationPeriodDays"])
        plasim["N_DAYS_PER_YEAR"] = s(max(math.floor(config["yearDays"] / config["rotationPeriodDays"] / 12 + 0.5),
                                          1) * 12)
    plasim["N_START_YEAR"] = "1" if plasim["N_DAYS_PER_YEAR"] == "365" else "0"
    for f in config["physicsFilter"]:
        key, value = FILTER_SWITCHES[f]
        plasim[key] = value
    scale = config.get("soilDepthScale", 1.0)
    if not (math.isfinite(scale) and scale > 0):
        raise ValueError("Soil depth, water capacity and heat capacity must be positive")
    land = {"NWETSOIL": _flag(config["wetSoil"]), "DSOILZ": ",".join(s(d * scale) for d in SOIL_LAYER_DEPTHS_M)}
    rad = {"NFIXED": _flag(config["synchronous"])}
    if config.get("starTemperatureK", 0) > 0:
        rad.update(NSTARTEMP="1", STARBBTEMP=s(config["starTemperatureK"]))
    rad.update(NO3=_flag(config["ozone"]), NRADINT="1", CO2=s(config["co2Ppm"]), NPBROADEN="1", NECHAM="1",
               NECHAM6="0")
    hurricane = {"NSTORMDIAG": _flag(config.get("stormclim", False)), "HC_CAPTURE": "0"}
    if config.get("stormCkcd"):
        hurricane["CKCD"] = s(config["stormCkcd"])
    if config.get("stormVithresh"):
        hurricane["VITHRESH"] = s(config["stormVithresh"])
    return {
        "planet_namelist": planet,
        "plasim_namelist": plasim,
        "radmod_namelist": rad,
        "landmod_namelist": land,
        "oceanmod_namelist": {"MLDEPTH": s(config["oceanDepthM"])},
        "vegmod_namelist": dict(VEGETATION_DEFAULTS, RINIDAGG=s(config["initialGrowth"])),
        "hurricane_namelist": hurricane,
        "glacier_namelist": {"NGLACIER": _flag(config["glaciersEnabled"]),
                             "GLACELIM": s(config["glaciersMinDepthM"]),
                             "ICESHEETH": s(config["glaciersInitialHeightM"])},
    }


def apply_edits(files: dict, config: dict) -> dict:
    """The namelist files with a configuration's edits applied (names the
    files lack are created as an empty group)."""
    out = dict(files)
    for name, values in namelist_edits(config).items():
        text = out.get(name, f" &{name.replace('_namelist', '_nl')}\n /END\n")
        out[name] = apply_namelist(text, values)
    return out


# The planet configuration keys the engine takes, from namelist values:
# (namelist, KEY, config key, conversion).
_FROM_NAMELIST = [
    ("planet_namelist", "GA", "gravityMs2", float),
    ("planet_namelist", "PLARAD", "radiusEarth", lambda v: v / EARTH_RADIUS_M),
    ("planet_namelist", "GSOL0", "fluxWm2", float),
    ("planet_namelist", "ECCEN", "eccentricity", float),
    ("planet_namelist", "OBLIQ", "obliquityDeg", float),
    ("planet_namelist", "NFIXORB", "fixedOrbit", lambda v: v != 0),
    ("planet_namelist", "NGENKEPLERIAN", "keplerian", lambda v: v != 0),
    ("planet_namelist", "GASCON", "gasConstant", float),
    ("planet_namelist", "SIDEREAL_YEAR", "yearDays", lambda v: v / SECONDS_PER_DAY),
    ("planet_namelist", "ROTSPD", "rotationPeriodDays", lambda v: 1 / v),
    ("plasim_namelist", "FIXEDLON", "substellarLongitudeDeg", float),
    ("plasim_namelist", "PSURF", "pressureBar", lambda v: v / 1e5),
    ("plasim_namelist", "NVEG", "vegetation", int),
    ("plasim_namelist", "MPSTEP", "timestepMinutes", float),
    ("radmod_namelist", "NFIXED", "synchronous", lambda v: v != 0),
    ("radmod_namelist", "NO3", "ozone", lambda v: v != 0),
    ("radmod_namelist", "CO2", "co2Ppm", float),
    ("landmod_namelist", "NWETSOIL", "wetSoil", lambda v: v != 0),
    ("oceanmod_namelist", "MLDEPTH", "oceanDepthM", float),
    ("vegmod_namelist", "RINIDAGG", "initialGrowth", float),
    ("hurricane_namelist", "NSTORMDIAG", "stormclim", lambda v: v != 0),
    ("hurricane_namelist", "CKCD", "stormCkcd", float),
    ("hurricane_namelist", "VITHRESH", "stormVithresh", float),
    ("glacier_namelist", "NGLACIER", "glaciersEnabled", lambda v: v != 0),
    ("glacier_namelist", "GLACELIM", "glaciersMinDepthM", float),
    ("glacier_namelist", "ICESHEETH", "glaciersInitialHeightM", float),
]
# Values the edits derive from the configuration: nothing more to read.
_DERIVED = {("plasim_namelist", k) for k in ("N_DAYS_PER_YEAR", "NSTPW", "N_START_YEAR", "NEQSIG", "NSELA",
                                             "FILTERKAPPA", "NFILTEREXP", "LANDHOSKN0")} | \
           {("radmod_namelist", k) for k in ("NRADINT", "NPBROADEN", "NECHAM", "NECHAM6")} | \
           {("hurricane_namelist", "HC_CAPTURE")} | {("vegmod_namelist", k) for k in VEGETATION_DEFAULTS}


def config_from_namelists(files: dict, truncation: int, layers: int, base: dict | None = None) -> tuple[dict, list]:
    """A planets configuration from namelist texts: `base` (the planets
    defaults) with every value the engine takes set from the files, and the
    list of (namelist, KEY) the engine does not take from them (their values
    stay the set-up's own)."""
    from . import planets  # noqa: PLC0415
    cfg = dict(base or planets.BASE_CONFIG)
    cfg.update(truncation=truncation, layers=layers)
    taken = set()
    values = {name: parse_namelist(text) for name, text in files.items() if name.endswith("_namelist")}
    for name, key, target, conv in _FROM_NAMELIST:
        raw = values.get(name, {}).get(key)
        if raw is None:
            continue
        cfg[target] = conv(namelist_number(raw.split(",")[0]))
        taken.add((name, key))
    plasim = values.get("plasim_namelist", {})
    if "ROTSPD" not in values.get("planet_namelist", {}) and "N_DAYS_PER_YEAR" in plasim \
            and "SIDEREAL_YEAR" not in values.get("planet_namelist", {}):
        cfg["yearDays"] = namelist_number(plasim["N_DAYS_PER_YEAR"])
    filters = []
    for key, kinds in (("NGPTFILTER", {"1": "gp"}), ("NFILTER", {"0": "none", "1": "cesaro", "2": "exp", "3": "lh"}),
                       ("NSPVFILTER", {"1": "sp"})):
        if key in plasim:
            taken.add(("plasim_namelist", key))
            kind = kinds.get(str(int(namelist_number(plasim[key]))))
            if kind:
                filters.append(kind)
    if any(k in plasim for k in ("NGPTFILTER", "NFILTER", "NSPVFILTER")):
        cfg["physicsFilter"] = tuple(filters)
    land = values.get("landmod_namelist", {})
    if "DSOILZ" in land:
        cfg["soilDepthScale"] = namelist_number(land["DSOILZ"].split(",")[0]) / SOIL_LAYER_DEPTHS_M[0]
        taken.add(("landmod_namelist", "DSOILZ"))
    rad = values.get("radmod_namelist", {})
    if "NSTARTEMP" in rad:
        taken.add(("radmod_namelist", "NSTARTEMP"))
        taken.add(("radmod_namelist", "STARBBTEMP"))
        on = namelist_number(rad["NSTARTEMP"]) != 0
        cfg["starTemperatureK"] = namelist_number(rad.get("STARBBTEMP", "5772")) if on else 0.0
    ignored = sorted((name, key) for name, vals in values.items() for key in vals
                     if (name, key) not in taken and (name, key) not in _DERIVED)
    return cfg, ignored


def planet_from_files(files: dict, truncation: int, layers: int, t_init, q_init, base: dict | None = None):
    """A planets.Planet for exogcm_configure from a run's files: the
    configuration from the namelists and the boundary from
    N<NLAT>_surf_<code>.sra (172 land mask and 129 orography required; 169
    SST and 210 ice cover as 12 monthly fields when present). `t_init` and
    `q_init` [levels][NHOR] are the initial temperature and humidity.
    Returns (planet, ignored namelist keys)."""
    from . import planets  # noqa: PLC0415
    nlat = LATITUDES[truncation]
    points = 2 * nlat * nlat
    cfg, ignored = config_from_namelists(files, truncation, layers, base)
    boundary = {}
    for code in (LAND_SEA_CODE, OROGRAPHY_CODE):
        name = sra_name(nlat, code)
        if name not in files:
            raise ValueError(f"{name} is required")
        boundary[code] = read_sra(files[name], points, 1, name)[0]
    for code in (SST_CODE, ICE_COVER_CODE):
        name = sra_name(nlat, code)
        if name in files:
            boundary[code] = read_sra(files[name], points, MONTHS, name)[1:13].reshape(-1)
    land = float(np.mean(boundary[LAND_SEA_CODE] > 0.5))
    planet = planets.Planet(config=cfg, land_fraction=land, boundary=boundary,
                            t_grid=np.asarray(t_init, dtype=np.float64).reshape(layers, points),
                            q_grid=np.asarray(q_init, dtype=np.float64).reshape(layers, points))
    return planet, ignored
