"""FP64 restatement of the reference's GCM set-up, used only as a test oracle.

TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg may import this module; the product library never does.

Every function restates one routine of ryoung48/web-exoplasim's TypeScript
set-up (paths relative to src/model/climate/gcm/) in numpy float64, keeping
the reference's statement order where it changes rounding.  It produces the
tables, constants and initial state that oracle/oracle.cpp steps.

Parity of this module is pinned by analytic invariants (Gaussian weights sum
to 2, Legendre orthonormality, LU inverse identity, transform round trips) and
by the reference's documented set-up agreement levels; the reference's own
golden dumps are not in the checkout.
"""
from __future__ import annotations

import functools
import math

import numpy as np

# setup/pumamod/index.ts:9-11 -- pumamod's PI parameter and derived constants.
PI = 3.14159265359
TWOPI = PI + PI
EZ = 1.63299310207
RV = 461.51
ACPV = 1870.0
SBK = 5.67e-8
CPS = 4180.0
CO2EARTH = 330.0
RAD_EARTHSQ = 6371220.0 * 6371220.0
ICE = dict(TMELT=273.16, CRHOI=920.0, CRHOS=1030.0, CRHOSN=330.0, CPI=2070.0,
           CKAPI=2.03, CKAPSN=0.31, CLFI=3.28e5, CLFSN=3.337e5)
UNIVERSAL_GAS_CONSTANT = 8314.46261815324
NATIVE_MEAN_MOLAR_MASS = 28.970253
NATIVE_GAS_CONSTANT = UNIVERSAL_GAS_CONSTANT / NATIVE_MEAN_MOLAR_MASS
SOIL_LAYERS = 5
MONTHS = 14


def js_round(x: float) -> float:
    """JavaScript Math.round: halves go towards +infinity."""
    return math.floor(x + 0.5)


def trunc(x: float) -> int:
    return int(math.trunc(x))


# ---------------------------------------------------------------- grid
def _ql(k: int, p: float) -> float:
    """grid/index.ts:15-30 (ql): normalised Legendre polynomial of degree k."""
    angle = math.acos(p)
    factor = 1.0
    s = 0.0
    term = 0.0
    j = k
    while j >= 0:
        term = factor * math.cos(angle * j)
        s = s + term
        z4 = (k - j + 1) * (k + j) * 0.5
        factor = (factor * z4) / (z4 + (j - 1))
        j -= 2
    if k % 2 == 0:
        s = s - 0.5 * term
    norm = math.sqrt(2)
    for j in range(1, k + 1):
        norm = norm * math.sqrt(1 - 0.25 / (j * j))
    return norm * s


@functools.lru_cache(maxsize=None)
def gaussian_latitudes(count: int):
    """grid/index.ts:32-63 (inigau): sines, weights and degrees, north first."""
    inigau_pi = 3.14159265358979
    degrees = np.zeros(count)
    sines = np.zeros(count)
    weights = np.zeros(count)
    z0 = inigau_pi / (2 * count + 1)
    z1 = 1.0 / (count * count * 8)
    z4 = 2.0 / (count * count)
    for root in range(count // 2):
        guess = z0 * (2 * (root + 1) - 0.5)
        x = math.cos(guess + z1 / math.tan(guess))
        for _ in range(50):
            value = _ql(count, x)
            z = x * value - math.sqrt((count + count + 1) / (count + count - 1)) * _ql(count - 1, x)
            step = value * ((x * x - 1) / (count * z))
            x = x - step
            if abs(step) < 1e-16:
                break
        z5 = _ql(count - 1, x) / math.sqrt(count - 0.5)
        latitude = math.asin(x) * 180 / math.pi
        weight = (z4 * (1 - x * x)) / (z5 * z5)
        degrees[root] = latitude
        degrees[count - 1 - root] = -latitude
        sines[root] = x
        sines[count - 1 - root] = -x
        weights[root] = weight
        weights[count - 1 - root] = weight
    return sines, weights, degrees


def latitudes_for_truncation(truncation: int) -> int:
    """grid/index.ts:88-93 (forTruncation)."""
    return {21: 32, 42: 64, 63: 96}[truncation]


# ---------------------------------------------------------------- fourier
def fourier_tables(longitudes: int, truncation: int):
    """fourier/index.ts:19-36: forward [j][k] and inverse [k][j] tables."""
    nfc = 2 * (truncation + 1)
    forward = np.zeros((longitudes, nfc))
    inverse = np.zeros((nfc, longitudes))
    for j in range(longitudes):
        lam = (2 * math.pi * j) / longitudes
        for m in range(truncation + 1):
            c = math.cos(m * lam)
            s = math.sin(m * lam)
            forward[j, 2 * m] = c / longitudes
            forward[j, 2 * m + 1] = -s / longitudes
            weight = 1 if m == 0 else 2
            inverse[2 * m, j] = weight * c
            inverse[2 * m + 1, j] = 0 if m == 0 else -weight * s
    return forward, inverse


def fourier_analyse(values, longitudes, truncation):
    """fourier/index.ts:95-115 (analyse): gp2fc in f64, rows of NFC."""
    forward, _ = fourier_tables(longitudes, truncation)
    rows = values.reshape(-1, longitudes)
    return rows @ forward


# ---------------------------------------------------------------- legendre
def legendre_tables(sines, weights, truncation):
    """legendre/index.ts:29-108 (legini): qi qj qc qe qm qq qu qv [lat][mode]."""
    key = (truncation, tuple(np.asarray(sines).tolist()), tuple(np.asarray(weights).tolist()))
    if key not in _LEGINI:
        _LEGINI[key] = _legendre_tables(sines, weights, truncation)
    return {k: v.copy() for k, v in _LEGINI[key].items()}


_LEGINI: dict = {}


def _legendre_tables(sines, weights, truncation):
    nlat = len(sines)
    modes = (truncation + 1) * (truncation + 2) // 2
    out = {k: np.zeros((nlat, modes)) for k in ("qi", "qj", "qc", "qe", "qm", "qq", "qu", "qv")}
    pli = np.zeros(modes + 1)
    pld = np.zeros(modes + 1)
    for lat in range(nlat):
        sin = sines[lat]
        weight = weights[lat]
        cos2 = 1 - sin * sin
        wocs = weight / cos2
        f1m = math.sqrt(1.5)
        pli[1] = math.sqrt(0.5)
        pli[2] = f1m * sin
        pld[1] = 0
        lm = 2
        for m in range(truncation + 1):
            if m > 0:
                lm += 1
                f2m = -f1m * math.sqrt(cos2 / (m + m))
                f1m = f2m * math.sqrt(m + m + 3)
                pli[lm] = f2m
                if lm < modes:
                    lm += 1
                    pli[lm] = f1m * sin
                    pld[lm - 1] = -m * f2m * sin
            m2 = m * m
            for n in range(m + 2, truncation + 1):
                lm += 1
                z1 = math.sqrt(((n - 1) * (n - 1) - m2) / (4 * (n - 1) * (n - 1) - 1))
                z2 = sin * pli[lm - 1] - z1 * pli[lm - 2]
                pli[lm] = z2 * math.sqrt((4 * n * n - 1) / (n * n - m2))
                pld[lm - 1] = (1 - n) * z2 + n * z1 * pli[lm - 2]
            if lm < modes:
                z3 = math.sqrt((truncation * truncation - m2) / (4 * truncation * truncation - 1))
                pld[lm] = -truncation * sin * pli[lm] + (truncation + truncation + 1) * pli[lm - 1] * z3
            else:
                pld[lm] = -truncation * sin * pli[lm]
        w = 0
        for m in range(truncation + 1):
            for n in range(m, truncation + 1):
                inv_degree = 1.0 / (n * (n + 1)) if n > 0 else 0.0
                p = pli[w + 1]
                d = pld[w + 1]
                out["qi"][lat, w] = p
                out["qj"][lat, w] = d
                out["qc"][lat, w] = p * weight
                out["qu"][lat, w] = p * inv_degree * m
                out["qv"][lat, w] = d * inv_degree
                out["qe"][lat, w] = d * wocs
                out["qq"][lat, w] = p * wocs * n * (n + 1) * 0.5
                out["qm"][lat, w] = p * wocs * m
                w += 1
    return out


def legendre_filters(truncation, nfilter, ngptfilter, nspvfilter, filterkappa, nfilterexp, landhoskn0):
    """legendre/index.ts:111-136: skgpsp and skspgp by total wavenumber."""
    g2s = np.zeros(truncation + 1)
    s2g = np.zeros(truncation + 1)
    for degree in range(truncation + 1):
        n = degree + 1
        shapes = {
            0: 1.0,
            1: 1 - n / (truncation + 1),
            2: math.exp(-filterkappa * (n / truncation) ** nfilterexp),
            3: math.exp(-(((n * (n + 1)) / (landhoskn0 * (landhoskn0 + 1))) ** 2)),
            4: (1 - n / (truncation + 1)) ** 2,
        }
        shape = 1.0 if nfilter == 0 else shapes[nfilter]
        g2s[degree] = 1 - ngptfilter + ngptfilter * shape
        s2g[degree] = 1 - nspvfilter + nspvfilter * shape
    return g2s, s2g


def mode_mn(truncation):
    """Mode index w -> (m, n) in the m-major order of legini."""
    ms, ns = [], []
    for m in range(truncation + 1):
        for n in range(m, truncation + 1):
            ms.append(m)
            ns.append(n)
    return np.array(ms), np.array(ns)


def legendre_kernel_tables(tables, g2s, s2g, truncation):
    """legendre/index.ts:138-155 + 200-221: filtered tables named legendre_<q>.

    filtered() indexes the filter by m + w_local = n (legendre/index.ts:138-155).
    """
    _, ns = mode_mn(truncation)
    out = {}
    for name in ("qc", "qe", "qm", "qq"):
        out["legendre_" + name] = tables[name] * g2s[ns][None, :]
    for name in ("qi", "qj", "qu", "qv"):
        out["legendre_" + name] = tables[name] * s2g[ns][None, :]
    return out


def legendre_analyse(fourier, qc, filt, latitudes, truncation):
    """legendre/index.ts:334-361 (analyse): fc2sp in f64, (re, im) per mode."""
    modes = (truncation + 1) * (truncation + 2) // 2
    nfc = 2 * (truncation + 1)
    f = fourier.reshape(latitudes, nfc)
    sp = np.zeros(2 * modes)
    for l in range(latitudes // 2):
        north = f[l]
        south = f[latitudes - 1 - l]
        w = 0
        for m in range(truncation + 1):
            for n in range(m, truncation + 1):
                sign = 1 if (m + n) % 2 == 0 else -1
                weight = qc[l, w]
                for part in range(2):
                    row = north[2 * m + part] + sign * south[2 * m + part]
                    sp[2 * w + part] = sp[2 * w + part] + weight * row * filt[n]
                w += 1
    return sp


# ---------------------------------------------------------------- namelists
BASE_NAMELISTS = {
    # public/gcm/t21/namelists.json: the values the set-up reads.
    "planet_namelist": dict(ECCEN=0.0, MVELP=102.7, OBLIQ=0.0, GSOL0=1367.0, NFIXORB=1),
    "plasim_namelist": dict(N_START_YEAR=1, N_DAYS_PER_YEAR=360, KICK=1, MPSTEP=30.0, NQSPEC=1,
                            NVEG=0, NWPD=0, NLOWIO=1, NSTPW=160, NFILTER=0, NGPTFILTER=1,
                            NSPVFILTER=1, PSURF=100040.0,
                            SEED=[14963991, 2, 3, 4, 5, 6, 7, 8]),
    "carbonmod_namelist": dict(NCARBON=1, KACT=0.09, BETA=0.5, FREQUENCY=4, PEARTH=79.0,
                               NSUPPLY=0, WMAX=80.9),
    "glacier_namelist": dict(NGLACIER=0, GLACELIM=2.0),
    "icemod_namelist": dict(NICE=1),
    "radmod_namelist": dict(CO2=360.0),
    "hurricane_namelist": dict(NSTORMDIAG=0),
}

DEFAULT_CONFIG = dict(
    # index.ts:4-44 (GCM.DEFAULT_CONFIG) with the atmosphere resolved.
    layers=10, truncation=21, radiusEarth=1.0, gravityMs2=9.80665, synchronous=False,
    substellarLongitudeDeg=180.0, oceanDepthM=50.0, fluxWm2=1367.0, starTemperatureK=0.0,
    yearDays=360, eccentricity=0.016715, rotationPeriodDays=1.0, obliquityDeg=23.5,
    fixedOrbit=True, keplerian=False, wetSoil=False, vegetation=2, initialGrowth=0.5,
    glaciersEnabled=True, glaciersMinDepthM=2.0, glaciersInitialHeightM=-1.0,
    physicsFilter=("gp", "exp", "sp"), timestepMinutes=45.0, pressureBar=1.011,
    gasConstant=NATIVE_GAS_CONSTANT, co2Ppm=300.0, ozone=True, soilDepthScale=1.0,
)

FILTER_SWITCHES = {"gp": ("NGPTFILTER", 1), "sp": ("NSPVFILTER", 1), "none": ("NFILTER", 0),
                   "cesaro": ("NFILTER", 1), "exp": ("NFILTER", 2), "lh": ("NFILTER", 3)}


def namelist_edits(config):
    """namelist/index.ts:40-182 (edits) for the config keys this build exposes."""
    planet = dict(GA=config["gravityMs2"], PLARAD=config["radiusEarth"] * 6371220.0,
                  GSOL0=config["fluxWm2"], ECCEN=config["eccentricity"], OBLIQ=config["obliquityDeg"],
                  NFIXORB=1 if config["fixedOrbit"] else 0, NGENKEPLERIAN=1 if config["keplerian"] else 0,
                  GASCON=config["gasConstant"], SIDEREAL_YEAR=config["yearDays"] * 86400.0)
    tsm = config["timestepMinutes"]
    plasim = dict(FIXEDLON=config["substellarLongitudeDeg"], N_DAYS_PER_YEAR=config["yearDays"],
                  PSURF=config["pressureBar"] * 1e5, NVEG=config["vegetation"], NEQSIG=0,
                  MPSTEP=tsm, NSTPW=math.floor(7200 / tsm), FILTERKAPPA=8, NFILTEREXP=8,
                  LANDHOSKN0=15)
    if config["rotationPeriodDays"] != 1:
        planet["ROTSPD"] = 1 / config["rotationPeriodDays"]
        plasim["N_DAYS_PER_YEAR"] = max(
            math.floor(config["yearDays"] / config["rotationPeriodDays"] / 12 + 0.5), 1) * 12
    plasim["N_START_YEAR"] = 1 if plasim["N_DAYS_PER_YEAR"] == 365 else 0
    for f in config["physicsFilter"]:
        key, value = FILTER_SWITCHES[f]
        plasim[key] = value
    land = dict(NWETSOIL=1 if config["wetSoil"] else 0,
                DSOILZ=[d * config["soilDepthScale"] for d in (0.4, 0.8, 1.6, 3.2, 6.4)])
    radmod = dict(NFIXED=1 if config["synchronous"] else 0, NO3=1 if config["ozone"] else 0,
                  CO2=config["co2Ppm"])
    if config["starTemperatureK"] > 0:
        raise NotImplementedError("stellar spectrum split (nstartemp) is not restated")
    return {
        "planet_namelist": planet,
        "plasim_namelist": plasim,
        "radmod_namelist": radmod,
        "landmod_namelist": land,
        "oceanmod_namelist": dict(MLDEPTH=config["oceanDepthM"]),
        "vegmod_namelist": dict(NCVEG=1, FORGROW=1.0, RINIDSC=1.0, RINIDMR=2.0, RINISOIL=0.0,
                                RINIVEG=0.0, RINIDAGG=config["initialGrowth"]),
        # namelist/index.ts:175: NSTORMDIAG = flag(config.stormclim); CKCD and
        # VITHRESH only through namelist text, here config overrides.
        "hurricane_namelist": dict(NSTORMDIAG=1 if config.get("stormclim") else 0,
                                   **({"CKCD": config["stormCkcd"]} if config.get("stormCkcd") else {}),
                                   **({"VITHRESH": config["stormVithresh"]} if config.get("stormVithresh") else {})),
        "glacier_namelist": dict(NGLACIER=1 if config["glaciersEnabled"] else 0,
                                 GLACELIM=config["glaciersMinDepthM"],
                                 ICESHEETH=config["glaciersInitialHeightM"]),
    }


def namelists_for(config):
    files = {k: dict(v) for k, v in BASE_NAMELISTS.items()}
    for name, values in namelist_edits(config).items():
        files.setdefault(name, {}).update(values)
    return files


def nl_read(namelist, defaults):
    """namelist/index.ts:209-231 (read): defaults overwritten by the namelist;
    arrays are filled from the front."""
    out = {}
    for key, fallback in defaults.items():
        value = namelist.get(key.upper())
        if value is None:
            out[key] = list(fallback) if isinstance(fallback, list) else fallback
            continue
        if isinstance(fallback, list):
            arr = list(fallback)
            parts = value if isinstance(value, (list, tuple)) else [value]
            for i, p in enumerate(parts):
                if i < len(arr):
                    arr[i] = p
                else:
                    arr.append(p)
            out[key] = arr
        else:
            out[key] = value[0] if isinstance(value, (list, tuple)) else value
    return out


EARTH = dict(eccen=0.016715, mvelp=102.7, obliq=23.441, rotspd=1.0, sidereal_day=86164.0916,
             solar_day=86400.0, sidereal_year=31558149.0, tropical_year=31556956.0,
             meananom0=-2.9589, akap=0.286, alr=0.0065, gascon=287.0, ra1=610.78,
             ra2=17.2693882, ra4=35.86, pnu=0.1, ga=9.80665, plarad=6371220.0, gsol0=1365.0,
             nfixorb=0, ngenkeplerian=0)


def pumamod(truncation, levels, files):
    """setup/pumamod/index.ts:94-237 (planet_ini then readnl)."""
    planet = nl_read(files.get("planet_namelist", {}), EARTH)
    day24 = 86400.0
    d = dict(psurf=101100.0, mpstep=0.0, ntspd=0, n_days_per_year=360, n_start_year=1,
             n_start_month=1, nkits=3, kick=1, ndheat=1, nveg=1, nqspec=1, nhdiff=15, nhordif=1,
             neqsig=0, nfilter=0, ngptfilter=0, nspvfilter=0, filterkappa=8.0, nfilterexp=8.0,
             landhoskn0=15.0, nwpd=0, nlowio=0, nstpw=0, dtep=0.0, dtns=0.0, dtrop=12000.0,
             dttrp=2.0, dttl=0.0, fixedlon=0.0, tgr=288.0, ptop=7500.0, frcmod=1.0,
             ndel=[2] * levels, tdissd=[0.2] * levels, tdissz=[1.1] * levels,
             tdisst=[5.6] * levels, tdissq=[0.1] * levels, restim=[0.0] * levels,
             t0=[250.0] * levels, tfrc=[0.0] * levels, seed=[0] * 8)
    if levels == 10:
        d["tfrc"] = [(20 if l == 0 else 100 if l == 1 else 0) * day24 * d["frcmod"] for l in range(levels)]
    if truncation == 42:
        d["nhdiff"] = 16
        d["ndel"] = [4] * levels
        d["tdissq"] = [0.1 * day24] * levels
        d["tdisst"] = [0.76 * day24] * levels
        d["tdissz"] = [0.3 * day24] * levels
        d["tdissd"] = [0.06 * day24] * levels
    nl = nl_read(files.get("plasim_namelist", {}), d)
    ndpy = nl["n_days_per_year"]
    solar_day = day24
    sidereal_day = (solar_day * (ndpy - 1)) / ndpy
    if planet["rotspd"] != 1:
        sidereal_day = day24 / planet["rotspd"]
        solar_day = (sidereal_day * ndpy) / (ndpy - 1) if ndpy != 1 else sidereal_day
    m_days_per_year = js_round((ndpy * sidereal_day) / day24)
    ww = TWOPI / sidereal_day
    acpd = planet["gascon"] / planet["akap"]
    cv = planet["plarad"] * ww
    mpstep = nl["mpstep"]
    if mpstep <= 0 and nl["ntspd"] <= 0:
        lat = latitudes_for_truncation(truncation)
        mpstep = 45 if lat <= 32 else 36 if lat <= 48 else trunc((30 * 64) / lat)
    mtspd = 0
    if mpstep > 0:
        mtspd = trunc(js_round(day24) / js_round(mpstep * 60))
        mtspd = mtspd + (mtspd % 2)
    mpstep = day24 / (mtspd * 60)
    ntspd = trunc(js_round(solar_day) / js_round(mpstep * 60))
    nafter = mtspd
    if 0 < nl["nwpd"] <= mtspd:
        nafter = trunc(mtspd / nl["nwpd"])
    if nl["nlowio"] > 0 and nl["nstpw"] > 0:
        nafter = nl["nstpw"]
    hordif = nl["nhordif"] != 0

    def zeroed(values):
        return list(values) if hordif else [0.0] * len(values)

    n_days_per_month = trunc(m_days_per_year / 12)
    p = dict(planet)
    p.update(
        day_24hr=day24, solar_day=solar_day, sidereal_day=sidereal_day, ww=ww, acpd=acpd,
        adv=ACPV / acpd - 1, cv=cv, ct=(cv * cv) / planet["gascon"], pnu21=1 - 2 * planet["pnu"],
        rdbrv=planet["gascon"] / RV, tmelt=273.16, alv=2.5008e6, als=2.8345e6, dawn=0.0,
        psurf=nl["psurf"], plavor=EZ, mpstep=mpstep, mtspd=mtspd, ntspd=ntspd, nafter=nafter,
        n_steps_per_year=js_round(planet["sidereal_year"] / (mpstep * 60)),
        n_days_per_year=ndpy, n_start_year=nl["n_start_year"], n_start_month=nl["n_start_month"],
        n_start_step=start_step(mtspd, nl["n_start_year"], nl["n_start_month"], ndpy, n_days_per_month),
        n_days_per_month=n_days_per_month, m_days_per_year=m_days_per_year,
        nkits=nl["nkits"], kick=nl["kick"], ndheat=nl["ndheat"], nveg=nl["nveg"], nqspec=nl["nqspec"],
        nhdiff=nl["nhdiff"], nhordif=nl["nhordif"], neqsig=nl["neqsig"], nfilter=int(nl["nfilter"]),
        ngptfilter=nl["ngptfilter"], nspvfilter=nl["nspvfilter"], filterkappa=nl["filterkappa"],
        nfilterexp=nl["nfilterexp"], landhoskn0=nl["landhoskn0"], dtep=nl["dtep"], dtns=nl["dtns"],
        dtrop=nl["dtrop"], dttrp=nl["dttrp"], dttl=nl["dttl"], fixedlon=nl["fixedlon"], tgr=nl["tgr"],
        ptop=nl["ptop"], ndel=nl["ndel"], tdissd=zeroed(nl["tdissd"]), tdissz=zeroed(nl["tdissz"]),
        tdisst=zeroed(nl["tdisst"]), tdissq=zeroed(nl["tdissq"]), restim=zeroed(nl["restim"]),
        t0=nl["t0"], tfrc=zeroed(nl["tfrc"]), seed=nl["seed"],
    )
    return p


# ---------------------------------------------------------------- calendar
MONTH_DAYS = [31, 28, 31, 30, 31, 30, 31, 31, 30, 31, 30, 31]


def _leap(y):
    return y % 4 == 0 and (y % 100 != 0 or y % 400 == 0)


def _year_start(y):
    return 365 * y + math.floor((y + 3) / 4) - math.floor((y + 99) / 100) + math.floor((y + 399) / 400)


def _month_days(y, m):
    return MONTH_DAYS[m - 1] + (1 if m == 2 and _leap(y) else 0)


def start_step(mtspd, year, month, days_per_year, days_per_month):
    """calendar/date/index.ts:30-41 (startStep)."""
    if days_per_year != 365:
        return mtspd * (year * days_per_year + (month - 1) * days_per_month)
    days = _year_start(year)
    for at in range(1, month):
        days += _month_days(year, at)
    return mtspd * days


def cal_date(step, steps_per_day, days_per_year, step_minutes):
    """calendar/date/index.ts:43-80 (date)."""
    if days_per_year == 365:
        days = trunc(step / steps_per_day)
        year = trunc(days / 365.2425)
        while _year_start(year) > days:
            year -= 1
        while _year_start(year + 1) <= days:
            year += 1
        day = days - _year_start(year) + 1
        month = 1
        while day > _month_days(year, month):
            day -= _month_days(year, month)
            month += 1
        minutes = trunc(((step % steps_per_day) * 1440) / steps_per_day)
        return year, month, day, trunc(minutes / 60), minutes % 60
    mtspd = trunc((days_per_year * steps_per_day) / 360)
    days = trunc(step / mtspd)
    doy = days % 360
    minutes = trunc((step % mtspd) * js_round(step_minutes))
    return trunc(days / 360) + 1, trunc(doy / 30) + 1, (doy % 30) + 1, trunc(minutes / 60), minutes % 60


def month_interpolation(step, steps_per_day, days_per_year, days_per_month, step_minutes, solar_day):
    """calendar/date/index.ts:82-112 (monthInterpolation, momint)."""
    year, month, day, hour, minute = cal_date(step, steps_per_day, days_per_year, step_minutes)
    fday = day + ((hour * 60 + minute) * 60) / solar_day
    current = _month_days(year, month) if days_per_year == 365 else days_per_month
    median = 0.5 * (current + 1)
    neighbour = month + 1 if fday > median else month - 1
    adjacent = _month_days(year, ((neighbour + 11) % 12) + 1) if days_per_year == 365 else days_per_month
    return month, neighbour, abs(fday - median) / (median + 0.5 * (adjacent + 1) - 1)


def orbit(fixed, eccentricity, obliquity_deg, perihelion_deg, mean_anomaly_deg):
    """calendar/index.ts:37-126 (orb_params) for a fixed orbit (nfixorb = 1)."""
    if not fixed:
        raise NotImplementedError("Berger orbit series (nfixorb = 0) is not restated")
    pi = 4 * math.atan(1)
    degrad = pi / 180
    eccen, obliq, mvelp = eccentricity, obliquity_deg, perihelion_deg
    e2 = eccen * eccen
    e3 = e2 * eccen
    mvelpp = (mvelp + 180) * degrad
    beta = math.sqrt(1 - e2)
    return dict(
        eccentricity=eccen, obliquityRad=obliq * degrad, meanAnomalyRad=mean_anomaly_deg * degrad,
        perihelionLongitudeRad=mvelpp,
        meanLongitudeAtEquinoxRad=2 * ((0.5 * eccen + 0.125 * e3) * (1 + beta) * math.sin(mvelpp)
                                       - 0.25 * e2 * (0.5 + beta) * math.sin(2 * mvelpp)
                                       + 0.125 * e3 * (1 / 3 + beta) * math.sin(3 * mvelpp)),
    )


def solar_position(step, steps_per_year, steps_per_day, step_minutes, orb, keplerian, synchronous):
    """calendar/solar/index.ts:26-89 (position)."""
    calendar_day = (step % steps_per_year) / steps_per_year
    minutes = trunc((step % steps_per_day) * step_minutes)
    e = orb["eccentricity"]
    if keplerian:
        true_anomaly = 0.0
        distance = 1.0
        if not synchronous:
            mean = calendar_day * TWOPI + orb["meanAnomalyRad"]
            while mean > TWOPI:
                mean -= TWOPI
            while mean < 0:
                mean += TWOPI
            if e > 0:
                value = mean if e < 0.5 else PI
                for _ in range(101):
                    prev = value
                    value -= (value - (mean + e * math.sin(value))) / max(1e-15, 1 - e * math.cos(value))
                    if abs(value - prev) <= 1e-14:
                        break
                tangent = math.tan(value * 0.5)
                mag = math.sqrt(((1 + e) / (1 - e)) * tangent * tangent)
                true_anomaly = 2 * math.atan(-mag if tangent < 0 else mag)
                if true_anomaly < 0:
                    true_anomaly += TWOPI
                true_anomaly = math.fmod(true_anomaly, TWOPI)
                inv = 1 / (1 - e * math.cos(value))
                distance = inv * inv
            else:
                true_anomaly = mean
        longitude = math.fmod(orb["perihelionLongitudeRad"] + true_anomaly, TWOPI)
    else:
        mean_longitude = orb["meanLongitudeAtEquinoxRad"] + (calendar_day - 80.5 / 365) * 2 * math.pi
        anomaly = mean_longitude - orb["perihelionLongitudeRad"]
        sine = math.sin(anomaly)
        longitude = mean_longitude + e * (2 * sine + e * (1.25 * math.sin(2 * anomaly)
                                                          + e * ((13 / 12) * math.sin(3 * anomaly) - 0.25 * sine)))
        inv = (1 + e * math.cos(longitude - orb["perihelionLongitudeRad"])) / (1 - e * e)
        distance = inv * inv
    return dict(calendarDay=calendar_day, minutes=minutes,
                declination=math.asin(math.sin(orb["obliquityRad"]) * math.sin(longitude)),
                distanceFactor=distance,
                rightAscension=math.atan2(math.cos(orb["obliquityRad"]) * math.sin(longitude),
                                          math.cos(longitude)))


def step_values(step, carbon_step, cal):
    """stepper/index.ts:281-334 (values) and radiation/index.ts:96-113 (step),
    surface/index.ts:49-59 (step), carbon/index.ts:23-28 (cycle)."""
    def month(at):
        return month_interpolation(at, cal["stepsPerDay"], cal["daysPerYear"], cal["daysPerMonth"],
                                   cal["stepMinutes"], cal["solarDay"])
    solar = solar_position(step, cal["stepsPerYear"], cal["stepsPerDay"], cal["stepMinutes"],
                           cal["orbit"], cal["keplerian"], cal["fixedSun"] is not None)

    def year(at):
        return cal_date(at, cal["stepsPerDay"], cal["daysPerYear"], cal["stepMinutes"])[0]
    nxt = carbon_step + 1
    weathers = nxt == cal["carbonInterval"]
    new_cstep = 0 if weathers else nxt
    fixed = cal["fixedSun"]
    declination = fixed["declinationRad"] if fixed else solar["declination"]
    phase = ((1 - fixed["longitudeDeg"] / 360) * TWOPI if fixed
             else (solar["minutes"] * cal["rotationSpeed"] * TWOPI) / 1440)
    rad = [math.sin(declination), math.cos(declination),
           phase - (solar["rightAscension"] if cal["keplerian"] else 0.0),
           solar["distanceFactor"], math.cos(TWOPI * (solar["calendarDay"] - cal["toffo3"]))]
    now = month(step)
    nx = month(step + 1)
    surf = [now[0], now[1], now[2], nx[0], nx[1], nx[2], 1.0 if year(step + 1) != year(step) else 0.0]
    return dict(radiation_step=np.array(rad), surface_step=np.array(surf, dtype=float),
                carbon_step=np.array([1.0 if weathers else 0.0]),
                snapshot_step=np.array([float(step), float(cal["outputWindowSteps"]), 0.0])), new_cstep


# ---------------------------------------------------------------- modules
def module_setup(truncation, levels, files, pm):
    """setup/modules/index.ts:1-318: each physics module's *ini values."""
    ndcycle = 1
    rad = nl_read(files.get("radmod_namelist", {}), dict(
        nfixed=0, ndcycle=1, no3=1, co2=360.0, nstartemp=0, starbbtemp=5772.0, th2oc=0.024,
        tswr1=0.077, tswr2=0.065, tswr3=0.0055, tpofmt=1.0, acllwr=0.1, a0o3=0.25, a1o3=0.11,
        aco3=0.08, bo3=20000.0, co3=5000.0, toffo3=0.25, dawn=0.0, iyrbp=1950 - pm["n_start_year"]))
    del ndcycle
    albedos = dict(dsnowalb=[0.6, 0.6], dsnowalbmn=[0.4, 0.4], dsnowalbmx=[0.8, 0.8],
                   dicealbmn=[0.5, 0.5], dicealbmx=[0.7, 0.7], dglacalbmn=[0.6, 0.6],
                   dgroundalb=[0.2, 0.2], doceanalb=[0.069, 0.069])
    rad.update(gsol0=pm["gsol0"], zsolar1=0.517, zsolar2=0.483, zsolars=[0.0, 0.0], rcoeff=1.0,
               year=1950 - rad["iyrbp"])
    rain = nl_read(files.get("rainmod_namelist", {}), dict(
        rhbeta=0.0, nbeta=3, pdeep=999999.0, pdeepth=70000.0, rkshallow=10.0,
        gamma=0.007 if (truncation == 42 and levels == 10) else 0.01, clwcrit1=-0.1, clwcrit2=0.0,
        rcritmod=1.0, rcritslope=0.0))
    c1, c2 = rain["clwcrit1"], rain["clwcrit2"]
    rain["clwfac"] = 1 / (c1 - c2) if c1 > c2 else (-1.0 if c1 < c2 else 1.0)
    flux = nl_read(files.get("fluxmod_namelist", {}), dict(zumin=1.0, vdiff_lamm=160.0, vdiff_b=5.0,
                                                              vdiff_c=5.0, vdiff_d=5.0))
    land = nl_read(files.get("landmod_namelist", {}), dict(
        nwetsoil=0, albland=0.22, albsmin=0.4, albsmax=0.8, albsminf=0.3, albsmaxf=0.4, albgmin=0.6,
        albgmax=0.8, alblandmax=0.4, drhsfull=0.4, dztop=0.2, dsmax=5.0, wsmax=0.5, rlue=3.4e-10,
        co2conv=8.3e-4, tau_veg=10.0, tau_soil=42.0, rhosnow=330.0, soildiff=1.8, sicediff=2.03,
        snowdiff=0.31, soilcap=2.4e6, sicecap=2.07e6, snowcap=0.6897e6, dsoilz=[0.4, 0.8, 1.6, 3.2, 6.4],
        rinifor=0.5, dz0land=2.0, drhsland=0.25, dzglac=-1.0, nwatcini=0, dwatcini=0.0,
        dsnowalbmn=albedos["dsnowalbmn"], dsnowalbmx=albedos["dsnowalbmx"],
        dglacalbmn=albedos["dglacalbmn"], dgroundalb=albedos["dgroundalb"]))
    a1 = 0.5 * land["dsnowalbmx"][0]
    a2 = 0.5 * land["dsnowalbmx"][1]
    land.update(wsmax=max(land["wsmax"], 0.0), albsmax1=land["dsnowalbmx"][0], albgmax1=land["dsnowalbmx"][0],
                albsmax2=land["dsnowalbmx"][1], albgmax2=land["dsnowalbmx"][1], albsmaxf1=a1, albsmaxf2=a2,
                albsmin1=land["dsnowalbmn"][0], albsmin2=land["dsnowalbmn"][1],
                albgmin1=land["dglacalbmn"][0], albgmin2=land["dglacalbmn"][1],
                albsminf1=0.75 * a1, albsminf2=0.75 * a2,
                tau_veg=land["tau_veg"] * pm["m_days_per_year"] * pm["day_24hr"],
                tau_soil=land["tau_soil"] * pm["m_days_per_year"] * pm["day_24hr"])
    sea = nl_read(files.get("seamod_namelist", {}), dict(
        albsea=0.069, albice=0.7, dz0sea=1.5e-5, dz0ice=0.001, drhssea=1.0, drhsice=1.0, charnock=0.018,
        doceanalb=albedos["doceanalb"], dicealbmn=albedos["dicealbmn"], dicealbmx=albedos["dicealbmx"]))
    ice = nl_read(files.get("icemod_namelist", {}), dict(
        nice=1, nseaice=1, xmind=0.1, xmaxd=9.0, thicec=0.5, tfreeze=271.25, cicemin=0.5))
    ice["tfreeze"] = 0.0 if ice["nseaice"] == 0 else ice["tfreeze"]
    ice["xdt"] = pm["solar_day"] / pm["ntspd"]
    veg = nl_read(files.get("vegmod_namelist", {}), dict(
        ncveg=1, forgrow=1.0, rinidagg=0.5, rinidsc=1.0, rinidmr=2.0, rinisoil=0.0, riniveg=0.0))
    carbon = nl_read(files.get("carbonmod_namelist", {}), dict(
        ncarbon=1, nsupply=0, kact=0.09, beta=0.5, frequency=4, vearth=0.05, pearth=79.0, wmax=1.0))
    freq = min(carbon["frequency"], pm["mtspd"])
    carbon.update(frequency=freq, interval=trunc(pm["mtspd"] / freq),
                  timeweight=1 / (freq * pm["m_days_per_year"]))
    ocean = nl_read(files.get("oceanmod_namelist", {}), dict(mldepth=50.0))
    surf = nl_read(files.get("surfmod_namelist", {}), dict(nspinit=0, noromax=truncation))
    glacier = nl_read(files.get("glacier_namelist", {}), dict(nglacier=1, glacelim=2.0, icesheeth=-1.0))
    # setup/index.ts:107-113: hurricane_namelist with its defaults.
    storm = nl_read(files.get("hurricane_namelist", {}), dict(nstormdiag=0, ckcd=0.9, vithresh=0.145))
    return dict(rad=rad, rain=rain, flux=flux, land=land, sea=sea, ice=ice, veg=veg, carbon=carbon,
                ocean=ocean, surf=surf, glacier=glacier, albedos=albedos, storm=storm)


# ---------------------------------------------------------------- dynamics set-up
def _seconds(values, threshold, day):
    """dynamics/setup/index.ts:19-25 (dayseccheck)."""
    largest = max(values)
    if largest < threshold and largest > 0:
        return [v * day for v in values]
    return list(values)


def initpm(truncation, levels, pm):
    """dynamics/setup/index.ts:27-110 (initpm, NEQSIG = 0) and initsi."""
    if pm["neqsig"] != 0:
        raise NotImplementedError("NEQSIG != 0")
    day = pm["day_24hr"]
    z = (np.arange(levels) + 1) / levels
    sigmah = 0.75 * z + 1.75 * z ** 3 - 1.5 * z ** 4
    dsigma = np.array([sigmah[0]] + [sigmah[l] - sigmah[l - 1] for l in range(1, levels)])
    rdsig = 0.5 / dsigma
    sigma = np.array([0.5 * sigmah[0]] + [0.5 * (sigmah[l - 1] + sigmah[l]) for l in range(1, levels)])
    threshold = day / pm["mtspd"]

    def rate(values):
        secs = _seconds(values, threshold, day)
        return np.array([day / (TWOPI * v) if v > 0 else 0.0 for v in secs])

    nrsp = (truncation + 1) * (truncation + 2)
    sak = np.zeros((levels, nrsp))
    nhdiff = pm["nhdiff"]
    for l in range(levels):
        power = pm["ndel"][l]
        scale = 1.0 / (truncation - nhdiff) ** power
        r = 0
        for m in range(truncation + 1):
            for n in range(m, truncation + 1):
                value = scale * (n - nhdiff) ** power if n >= nhdiff else 0.0
                sak[l, r] = value
                sak[l, r + 1] = value
                r += 2
    nindex = np.zeros(nrsp)
    r = 0
    for m in range(truncation + 1):
        for n in range(m, truncation + 1):
            nindex[r] = nindex[r + 1] = n
            r += 2
    ct = pm["ct"]
    s = dict(sigmah=sigmah, sigma=sigma, dsigma=dsigma, rdsig=rdsig, damp=rate(pm["restim"]),
             tfrc=rate(pm["tfrc"]), tdissd=rate(pm["tdissd"]), tdissz=rate(pm["tdissz"]),
             tdisst=rate(pm["tdisst"]), tdissq=rate(pm["tdissq"]), sak=sak, nindex=nindex,
             t0=np.array(pm["t0"], dtype=float) / ct, dtns=pm["dtns"] / ct, dtep=pm["dtep"] / ct,
             dttrp=pm["dttrp"] / ct)
    initsi(s, pm["akap"])
    return s


def initsi(s, akap):
    """dynamics/setup/index.ts:112-152 (initsi). Matrices row-major [j][i] = a(i, j)
    as the reference's column-major j*n + i."""
    t0, sigmah, dsigma, rdsig = s["t0"], s["sigmah"], s["dsigma"], s["rdsig"]
    n = len(t0)
    g = np.zeros(n * n)
    c = np.zeros(n * n)
    tau = np.zeros(n * n)

    def at(i, j):
        return j * n + i
    tkp = akap * t0
    t01s2 = np.zeros(n)
    for l in range(n - 1):
        t01s2[l] = t0[l + 1] - t0[l]
    alp = np.array([0.0] + [math.log(sigmah[l]) - math.log(sigmah[l - 1]) for l in range(1, n)])
    g[at(0, 0)] = 1
    for l in range(1, n):
        g[at(l, l)] = 1 - (alp[l] * sigmah[l - 1]) / dsigma[l]
        for k in range(l):
            g[at(l, k)] = alp[l]
    for l in range(n):
        for k in range(n):
            c[at(l, k)] = g[at(k, l)] * (dsigma[l] / dsigma[k])
    t01 = t01s2[0]
    sig = sigmah[0]
    tau[at(0, 0)] = 0.5 * t01 * (sig - 1) + tkp[0]
    for k in range(1, n):
        tau[at(k, 0)] = 0.5 * t01 * dsigma[k]
    for l in range(1, n):
        pt01 = t01
        psig = sig
        t01 = t01s2[l]
        sig = sigmah[l]
        for k in range(n):
            below = 1 if k <= l else 0
            above = 1 if k < l else 0
            value = pt01 * (psig - above)
            if l < n - 1:
                value = value + t01 * (sig - below)
            value = value * rdsig[l] * dsigma[k]
            if k <= l:
                value = value + tkp[l] * c[at(k, l)]
            tau[at(k, l)] = value
    s.update(tkp=tkp, t01s2=t01s2, g=g, c=c, tau=tau)


def invert(matrix, n):
    """dynamics/setup/index.ts:154-211 (ludcmp + lubksb, partial pivoting)."""
    a = matrix.copy()

    def at(i, j):
        return j * n + i
    scale = np.zeros(n)
    for i in range(n):
        largest = 0.0
        for j in range(n):
            largest = max(largest, abs(a[at(i, j)]))
        scale[i] = 1 / largest
    index = [0] * n
    for j in range(n):
        for i in range(1, j):
            dot = 0.0
            for k in range(i):
                dot += a[at(i, k)] * a[at(k, j)]
            a[at(i, j)] -= dot
        largest = 0.0
        pivot = j
        for i in range(j, n):
            if j > 0:
                dot = 0.0
                for k in range(j):
                    dot += a[at(i, k)] * a[at(k, j)]
                a[at(i, j)] -= dot
            size = scale[i] * abs(a[at(i, j)])
            if size >= largest:
                pivot = i
                largest = size
        if j != pivot:
            for k in range(n):
                a[at(pivot, k)], a[at(j, k)] = a[at(j, k)], a[at(pivot, k)]
            scale[pivot] = scale[j]
        index[j] = pivot
        if a[at(j, j)] == 0:
            a[at(j, j)] = 5e-324
        for i in range(j + 1, n):
            a[at(i, j)] /= a[at(j, j)]
    inverse = np.zeros(n * n)
    for column in range(n):
        b = [1.0 if i == column else 0.0 for i in range(n)]
        first = -1
        for i in range(n):
            li = index[i]
            sm = b[li]
            b[li] = b[i]
            if first >= 0:
                for j in range(first, i):
                    sm -= a[at(i, j)] * b[j]
            elif sm != 0:
                first = i
            b[i] = sm
        for i in range(n - 1, -1, -1):
            sm = b[i]
            for j in range(i + 1, n):
                sm -= a[at(i, j)] * b[j]
            b[i] = sm / a[at(i, i)]
        inverse[column * n:(column + 1) * n] = b
    return inverse


def makebm(s, truncation, delt):
    """dynamics/setup/index.ts:213-239 (makebm): bm1[n-1] = inv(I/(n(n+1)) + delt^2 B)."""
    t0, dsigma, g, tau = s["t0"], s["dsigma"], s["g"], s["tau"]
    n = len(t0)
    d2 = delt * delt
    base = np.zeros(n * n)
    for l1 in range(n):
        for l2 in range(n):
            dot = 0.0
            for k in range(n):
                dot += g[l1 * n + k] * tau[k * n + l2]
            base[l1 * n + l2] = d2 * (t0[l1] * dsigma[l2] + dot)
    bm1 = np.zeros(n * n * truncation)
    for degree in range(1, truncation + 1):
        mat = base.copy()
        for l in range(n):
            mat[l * n + l] += 1 / (degree * (degree + 1))
        bm1[(degree - 1) * n * n: degree * n * n] = invert(mat, n)
    return bm1


def latitude_factors(sines, nlon):
    """dynamics/setup/index.ts:241-254 (rcsq)."""
    return np.repeat(1 / (1 - sines * sines), nlon)


def setzt(s, truncation, pm):
    """dynamics/setup/index.ts:256-313 (setzt): restoration temperature sr."""
    sigma, t0, dtns, dtep = s["sigma"], s["t0"], s["dtns"], s["dtep"]
    gascon, ga, ct, alr, tgr, dtrop = pm["gascon"], pm["ga"], pm["ct"], pm["alr"], pm["tgr"], pm["dtrop"]
    levels = len(sigma)
    dttrp = s["dttrp"] * ct

    def profile(height):
        return (tgr - dtrop * alr + math.sqrt((0.5 * alr * (height - dtrop)) ** 2 + dttrp ** 2)
                - 0.5 * alr * (height - dtrop))
    trs = np.zeros(levels)
    sp, tp, zp = 1.0, tgr, 0.0
    for l in range(levels - 1, -1, -1):
        lr = math.log(sp / sigma[l])
        first = profile(zp + ((gascon * tp) / ga) * lr)
        t = profile(zp + ((gascon * (0.5 * (tp + first))) / ga) * lr)
        trs[l] = t
        zp = zp + ((0.5 * (t + tp) * gascon) / ga) * lr
        tp = t
        sp = sigma[l]
    tropopause = ((tgr - dtrop * alr) / tgr) ** (ga / (alr * gascon))
    substellar = (1 / 3.463843223261725 / ct) * pm["dttl"]
    subst1 = -substellar * math.cos((pm["fixedlon"] * PI) / 180)
    subst2 = substellar * math.sin((pm["fixedlon"] * PI) / 180)
    nrsp = (truncation + 1) * (truncation + 2)
    sas = 2 * (truncation + 1)
    sr = np.zeros((levels, nrsp))
    for l in range(levels):
        fac = max(math.sin((0.5 * PI * (sigma[l] - tropopause)) / (1 - tropopause)), 0)
        sr[l, 0] = math.sqrt(2) * (trs[l] / ct - t0[l])
        sr[l, 2] = (1 / math.sqrt(6)) * dtns * fac
        sr[l, 4] = (-2 / 3) * math.sqrt(0.4) * dtep * fac
        sr[l, sas] = subst1 * fac
        sr[l, sas + 1] = subst2 * fac
    return sr


# ---------------------------------------------------------------- physics tables
def surface_flux_tables(sigma, sigmah, akap, gascon, ga, lamm, vd):
    """physics/surface-flux/index.ts:30-67 (tables)."""
    levels = len(sigma)
    zlamh = lamm * math.sqrt(3 * vd * 0.5)
    out = dict(flux_sigfac=np.array([sigma[-1] ** -akap]), flux_lnsig=np.array([math.log(sigma[-1])]),
               vdiff_skap=sigma ** akap, vdiff_skaph=sigmah ** akap)
    for k in ("vdiff_mixh2", "vdiff_mixm2", "vdiff_rdsig", "vdiff_sigmah3", "vdiff_kfac"):
        out[k] = np.zeros(levels)
    for l in range(levels - 1):
        zzlev = (-gascon * 250 * math.log(sigmah[l])) / ga
        zdz = (gascon * 250 * math.log(sigma[l + 1] / sigma[l])) / ga
        zmixh = (zlamh * 0.4 * zzlev) / (zlamh + 0.4 * zzlev)
        zmixm = (lamm * 0.4 * zzlev) / (lamm + 0.4 * zzlev)
        zrdsig = 1 / (sigma[l + 1] - sigma[l])
        out["vdiff_mixh2"][l] = zmixh * zmixh
        out["vdiff_mixm2"][l] = zmixm * zmixm
        out["vdiff_rdsig"][l] = zrdsig
        out["vdiff_sigmah3"][l] = sigmah[l] * sigmah[l] * sigmah[l] * zrdsig
        ratio = (((zzlev + zdz) / zzlev) ** (1 / 3) - 1) / zdz
        out["vdiff_kfac"][l] = math.sqrt(ratio ** 3 / zzlev)
    return out


def radiation_tables(sines, sigma, sigmah, dsigma, ga, acllwr):
    """physics/radiation/index.ts:59-94 (tables)."""
    levels = len(sigma)
    lnsig = np.zeros(levels)
    lnsig[0] = math.log(sigma[0] / sigmah[0]) * 0.5
    for l in range(1, levels):
        lnsig[l] = math.log(sigmah[l - 1] / sigmah[l])
    return dict(sid=np.array(sines), cola=np.sqrt(1 - sines * sines), rad_lnsig=lnsig,
                lwr_zzf1=(sigma * dsigma) / ga / 100000, lwr_zzf3=(-1.66 * acllwr * 1000 * dsigma) / ga)


def precipitation_tables(sigma, akap, rcritmod, rcritslope):
    """physics/precipitation/index.ts:45-63 (tables)."""
    levels = len(sigma)
    rcrit = np.array([max(0.85, max(v, 1 - v)) * rcritmod * (1 - (2 * rcritslope * (levels / 2 - (l + 1))) / levels)
                      for l, v in enumerate(sigma)])
    kuo = np.array([(sigma[l] / sigma[l + 1]) ** akap for l in range(levels - 1)])
    return dict(rcrit=rcrit, kuo_zfac=kuo)


def lwr_offsets():
    """physics/radiation/index.ts:116-134 (absorptivityOffsets)."""
    zao30 = 0.209 * 7e-5 ** 0.436
    zco20 = 0.0676 * 0.01022 ** 0.421
    zh2o0a = 0.846 * 3.59e-5 ** 0.243
    zh2o0 = 0.832 * 0.0286 ** 0.26
    return dict(ZAO30=zao30, ZCO20=zco20, ZH2O0A=zh2o0a, ZH2O0=zh2o0,
                ZAO3C=0.209 * (0.01 + 7e-5) ** 0.436 - zao30 - 0.0212 * math.log10(0.01),
                ZACO2C=0.0676 * 1.01022 ** 0.421 - zco20,
                ZAH2OC=0.846 * (0.01 + 3.59e-5) ** 0.243 - zh2o0a - 0.24 * math.log10(0.02),
                ZTH2OC=1 - (0.832 * (2 + 0.0286) ** 0.26 - zh2o0) + 0.1196 * math.log(2 - 0.6931))
