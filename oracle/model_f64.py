"""FP64 restatement of the reference's surface set-up, constants and schedule.

TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg may import this module.

Follows src/model/climate/gcm/setup/surface/index.ts (surfini),
setup/index.ts (constants, dynamicsTables, schedule) and stepper/index.ts
(tables).  The model it returns is what oracle/oracle.cpp steps: a flat dict of
named constants per start-up phase, named tables and named state fields, all
float64, with the reference's field names and plane layouts.
"""
from __future__ import annotations

import math

import numpy as np

from . import setup_f64 as S

UNSET = 1e20
RUNOFF_SPEED = 4.2
RUNOFF_EXPONENT = 0.18
GRAVITY_CONSTANT = 6.67408e-11
EARTH_MASS = 5.9722e24
EARTH_RADIUS = 6.371e6
GLACIER_DENSITY = 850.0
ICE_NORTH = dict(cmin=0.1, cmax=0.9, hmin=0.25, hmax=3.0)
ICE_SOUTH = dict(cmin=0.25, hmin=0.25, hmax=0.5)
ICE_MONTH_FACTOR = [0.912, 0.942, 1, 1.058, 1.124, 1.161, 1.175, 1.058, 0.931, 0.883, 0.88, 0.876,
                    0.912, 0.942]
CODE = dict(LAND_MASK=172, OROGRAPHY=129, ROUGHNESS=173, OROGRAPHIC_ROUGHNESS=1730, GLACIER=232,
            FOREST=212, FIELD_CAPACITY=229, SOIL_TEMPERATURE=209, ALBEDO=174, ALBEDO_VISIBLE=175,
            ALBEDO_INFRARED=176, ABOVE_GROUND_GROWTH=1605, STOMATAL_CONDUCTANCE=1606,
            MAXIMUM_ROUGHNESS=1607, BIOMASS_GROWTH=1604, SURFACE_TEMPERATURE=169, ICE_COVER=210,
            ICE_THICKNESS=211)


def _read(files, code, points, months):
    """setup/surface/index.ts:72-103 (get_surf_array): 1 or 12 fields -> months."""
    data = files.get(code)
    if data is None:
        return None
    data = np.asarray(data, dtype=float).reshape(-1, points)
    found = min(months, data.shape[0])
    result = np.zeros((months, points))
    result[:found] = data[:found]
    if found == months:
        return result.reshape(-1)
    if found == 12 and months == S.MONTHS:
        for month in range(12, 0, -1):
            result[month] = result[month - 1]
        result[13] = result[1]
        result[0] = result[12]
    elif found == 1 and months == S.MONTHS:
        result[1:] = result[0]
    else:
        raise ValueError(f"surface code {code} has {found} fields, expected {months}")
    return result.reshape(-1)


def _monthly(table, step, pm, points):
    """setup/surface/index.ts:106-126 (momint at a step)."""
    month, neighbour, weight = S.month_interpolation(step, pm["ntspd"], pm["n_days_per_year"],
                                                     pm["n_days_per_month"], pm["mpstep"], pm["solar_day"])
    t = table.reshape(-1, points)
    return (1 - weight) * t[month] + weight * t[neighbour]


def _glacier_albedo(mx, mn, ts, tmelt):
    return max(mn, min(mx, mx - ((mx - mn) * (ts - 263.16)) / (tmelt - 263.16)))


def _wet_soil_albedo(bf, dry, ocean):
    aa, yy = 5.2, 4.0
    al = (1 / aa) * (max(bf, 1e-3) ** ((1 - yy) / yy) - 1) ** (1 / yy)
    dw = math.exp(-((bf * 25) ** 6))
    ww = math.exp(-(((1 - bf) * 30) ** 9))
    return dry * dw + al * (1 - dw - ww) + ocean * ww


def _saturation(temperature, pm):
    """setup/surface/index.ts:159-167 (Magnus-Tetens at namelist psurf)."""
    q = (pm["rdbrv"] * pm["ra1"] * math.exp((pm["ra2"] * (temperature - pm["tmelt"]))
                                            / (temperature - pm["ra4"]))) / pm["psurf"]
    return q / (1 - (1 / pm["rdbrv"] - 1) * q)


def _runoff(orography, mask, nlat, nlon, sines, pm):
    """setup/surface/index.ts:170-236 (oroini river directions and velocities)."""
    points = nlat * nlon
    duroff = np.zeros(points)
    dvroff = np.zeros(points)
    height = np.array([mask[h] - 1 if mask[h] < 1 else max(orography[h], 0.0) for h in range(points)])
    if (height.max() - height.min()) / pm["ga"] <= 0.01:
        return duroff, dvroff

    def neighbours(h, hgt):
        lon = h % nlon
        lat = (h - lon) // nlon
        around = [lat * nlon + ((lon + 1) % nlon), lat * nlon + ((lon + nlon - 1) % nlon)]
        if lat > 0:
            around.append(h - nlon)
        if lat < nlat - 1:
            around.append(h + nlon)
        return [hgt[a] for a in around]
    raised = True
    while raised:
        raised = False
        nxt = np.zeros(points)
        for h in range(points):
            around = neighbours(h, height)
            if mask[h] > 0 and all(height[h] <= v for v in around):
                nxt[h] = 1 + min(around)
                raised = True
            else:
                nxt[h] = height[h]
        height = nxt

    def rate(slope, spacing, sign):
        return ((sign * RUNOFF_SPEED) / spacing) * abs(slope) ** RUNOFF_EXPONENT
    for lat in range(nlat):
        dx = (S.TWOPI * math.cos(math.asin(sines[lat])) * pm["plarad"]) / nlon
        for lon in range(nlon):
            h = lat * nlon + lon
            slope = (height[lat * nlon + ((lon + 1) % nlon)] - height[h]) / dx
            duroff[h] = rate(slope, dx, -1 if slope > 0 else 1)
    for lat in range(nlat - 1):
        dy = (math.asin(sines[lat + 1]) - math.asin(sines[lat])) * pm["plarad"]
        for lon in range(nlon):
            h = lat * nlon + lon
            slope = (height[h + nlon] - height[h]) / dy
            dvroff[h] = rate(slope, dy, -1 if slope < 0 else 1)
    return duroff, dvroff


def _ice_thickness(cover, nlat, nlon):
    """setup/surface/index.ts:239-261 (make_ice_thickness)."""
    points = nlat * nlon
    c = cover.reshape(S.MONTHS, points)
    out = np.zeros_like(c)
    for month in range(S.MONTHS):
        for h in range(points):
            v = c[month, h]
            north = (h // nlon) < nlat / 2
            d = 0.0
            if north:
                f = ICE_MONTH_FACTOR[month]
                n = ICE_NORTH
                if v >= n["cmax"]:
                    d = n["hmax"] * f
                elif v >= n["cmin"]:
                    d = (n["hmin"] + ((n["hmax"] - n["hmin"]) * (v - n["cmin"])) / (n["cmax"] - n["cmin"])) * f
                elif v > 0:
                    d = n["hmin"] * f
            elif v >= ICE_SOUTH["cmin"]:
                d = ICE_SOUTH["hmax"]
            elif v > 0:
                d = ICE_SOUTH["hmin"] + v
            out[month, h] = d
    return out.reshape(-1)


def surface_initial(truncation, levels, pm, mods, files, sines, weights):
    """setup/surface/index.ts:265-647 (initial: surfini and friends)."""
    nlat = len(sines)
    nlon = 2 * nlat
    points = nlat * nlon
    land, sea, ice, veg, ocean, surf, glacier, rad = (mods[k] for k in
                                                      ("land", "sea", "ice", "veg", "ocean", "surf", "glacier", "rad"))
    tmelt = pm["tmelt"]
    step = pm["n_start_step"]

    def field(code, fallback):
        r = _read(files, code, points, 1)
        return r.copy() if r is not None else np.full(points, float(fallback))

    def clim(code, fallback):
        r = _read(files, code, points, S.MONTHS)
        return r.copy() if r is not None else np.full(S.MONTHS * points, float(fallback))
    row_w = np.repeat(weights, nlon)
    dls = (field(CODE["LAND_MASK"], 1) > 0.5).astype(float)
    orography = field(CODE["OROGRAPHY"], 0)
    dz0clim = field(CODE["ROUGHNESS"], land["dz0land"])
    dz0climo = field(CODE["OROGRAPHIC_ROUGHNESS"], 0)
    dglac = field(CODE["GLACIER"], 0)
    if land["dzglac"] > 0:
        dglac[orography > land["dzglac"] * pm["ga"]] = 1
    dglac = (dglac > 0.5).astype(float)
    dforest = field(CODE["FOREST"], land["rinifor"])
    dwmax = np.maximum(field(CODE["FIELD_CAPACITY"], land["wsmax"]), 0)
    dtclsoil = field(CODE["SOIL_TEMPERATURE"], tmelt)
    dalbcl = clim(CODE["ALBEDO"], land["albland"])
    dalbcl1 = clim(CODE["ALBEDO_VISIBLE"], land["dgroundalb"][0])
    dalbcl2 = clim(CODE["ALBEDO_INFRARED"], land["dgroundalb"][1])
    land_dts = np.full(points, UNSET)
    land_dtsm = np.full(points, UNSET)
    land_dqs = np.full(points, UNSET)
    dsoilt = np.full(S.SOIL_LAYERS * points, tmelt)
    dsnowt = np.full(points, tmelt)
    dsnowz = np.zeros(points)
    dwatc = np.zeros(points)
    for h in range(points):
        if dls[h] <= 0:
            continue
        land_dts[h] = dtclsoil[h]
        for l in range(S.SOIL_LAYERS):
            dsoilt[l * points + h] = land_dts[h]
        dwatc[h] = land["dwatcini"] if land["nwatcini"] > 0 else land["drhsland"] * land["drhsfull"] * dwmax[h]
    dalbclim = _monthly(dalbcl, step + 1, pm, points)
    dalbclim1 = _monthly(dalbcl1, step + 1, pm, points)
    dalbclim2 = _monthly(dalbcl2, step + 1, pm, points)
    if land["nwetsoil"] > 0.5:
        for h in range(points):
            if dls[h] <= 0.5:
                continue
            if land_dts[h] > 273.15:
                bf = 0 / land["wsmax"]
                dalbclim[h] = _wet_soil_albedo(bf, land["alblandmax"], sea["doceanalb"][0])
                dalbclim1[h] = dalbclim[h]
                dalbclim2[h] = _wet_soil_albedo(bf, land["alblandmax"], sea["doceanalb"][1])
            else:
                dalbclim[h] = land["albland"]
                dalbclim1[h] = land["dgroundalb"][0]
                dalbclim2[h] = land["dgroundalb"][1]
    dalb = np.zeros(points)
    dsalb = np.zeros(2 * points)
    drhs = np.zeros(points)
    dz0 = np.zeros(points)
    dsnow = np.zeros(points)
    soil = [np.zeros(points) for _ in range(5)]
    dt = np.zeros((levels + 1) * points)
    dq = np.zeros((levels + 1) * points)
    sl = levels * points
    for h in range(points):
        if dls[h] <= 0:
            continue
        ts = land_dts[h]
        land_dtsm[h] = ts
        land_dqs[h] = _saturation(ts, pm)
        dsnow[h] = dsnowz[h]
        dalb[h] = dalbclim[h]
        dsalb[h] = dalbclim1[h]
        dsalb[points + h] = dalbclim2[h]
        if dwmax[h] > 0:
            drhs[h] = min(1, dwatc[h] / (land["drhsfull"] * dwmax[h]))
        dz0[h] = dz0clim[h]
        for l in range(5):
            soil[l][h] = dsoilt[l * points + h]
        if dglac[h] > 0.5:
            dsnowz[h] = max(land["dsmax"], 0)
            dsnow[h] = dsnowz[h]
            dalb[h] = _glacier_albedo(land["albgmax"], land["albgmin"], ts, tmelt)
            dsalb[h] = _glacier_albedo(land["albgmax1"], land["albgmin1"], ts, tmelt)
            dsalb[points + h] = _glacier_albedo(land["albgmax2"], land["albgmin2"], ts, tmelt)
            drhs[h] = 1
        dt[sl + h] = ts
        dq[sl + h] = land_dqs[h]
    if glacier["icesheeth"] >= 0:
        covered = orography != 0
        dglac = covered.astype(float)
        dsnowz = np.where(covered, glacier["icesheeth"], 0.0)
    else:
        dsnowz = np.where((dglac > 0) & (dsnowz == 0), glacier["glacelim"], dsnowz)
    doro = orography.copy()
    if glacier["nglacier"] == 1:
        gm = GRAVITY_CONSTANT * EARTH_MASS
        ground = orography * 1.0
        dz = (EARTH_RADIUS * EARTH_RADIUS * ground) / (gm - EARTH_RADIUS * ground)
        snow = dsnowz / (GLACIER_DENSITY / 1000)
        gravity = gm / ((EARTH_RADIUS + dz) * (EARTH_RADIUS + dz))
        doro = ground + (gravity * snow - (gravity / (dz + EARTH_RADIUS)) * snow * snow)
    duroff, dvroff = _runoff(doro, dls, nlat, nlon, sines, pm)
    ltab = S.legendre_tables(sines, weights, truncation)
    g2s, _ = S.legendre_filters(truncation, pm["nfilter"], pm["ngptfilter"], pm["nspvfilter"],
                                pm["filterkappa"], pm["nfilterexp"], pm["landhoskn0"])
    so = S.legendre_analyse(S.fourier_analyse(doro * 1.0, nlon, truncation), ltab["qc"], g2s, nlat,
                            truncation) / (pm["cv"] * pm["cv"])
    r = 0
    for m in range(truncation + 1):
        for n in range(m, truncation + 1):
            if n > surf["noromax"]:
                so[r:r + 2] = 0
            r += 2
    if glacier["nglacier"] == 1:
        dglac[dsnowz > 30] = 1
    dpersist = (dls >= 0.5).astype(float)
    dagg = field(CODE["ABOVE_GROUND_GROWTH"], veg["rinidagg"])
    dsc = field(CODE["STOMATAL_CONDUCTANCE"], veg["rinidsc"])
    dmr = field(CODE["MAXIMUM_ROUGHNESS"], veg["rinidmr"])
    dgrow = field(CODE["BIOMASS_GROWTH"], veg["forgrow"])
    dforest[dls == 0] = 0
    xls = (field(CODE["LAND_MASK"], 0) > 0.5).astype(float)
    xclsst = clim(CODE["SURFACE_TEMPERATURE"], -999)
    xclicec = clim(CODE["ICE_COVER"], -999)
    xcliced = clim(CODE["ICE_THICKNESS"], -999)
    if ice["nseaice"] == 0:
        xclicec[:] = 0
        xcliced[:] = 0
    cover_max = xclicec.max()
    if ice["nice"] >= 0:
        if cover_max > 5:
            xclicec = xclicec * 0.01
        if cover_max < 0:
            xclicec = np.where((ice["nice"] > 0.5) & (xclsst <= ice["tfreeze"]), 1.0, 0.0)
        if xcliced[0] < 0:
            xcliced = _ice_thickness(xclicec, nlat, nlon)
    for i in range(len(xclicec)):
        if ice["nseaice"] == 0 or xls[i % points] >= 1:
            xclicec[i] = 0
            xcliced[i] = 0
    xclssto = _monthly(xclsst, step, pm, points)
    xclsst2 = _monthly(xclsst, step + 1, pm, points)
    xcliced2 = np.maximum(_monthly(xcliced, step + 1, pm, points), 0)
    xclicec2 = np.where(xcliced2 <= 0, 0.0, np.maximum(_monthly(xclicec, step + 1, pm, points), 0))
    xiced = xcliced2.copy()
    xicec = (xclicec2 >= ice["thicec"]).astype(float)
    yls = (field(CODE["LAND_MASK"], 0) > 0.5).astype(float)
    yclsst = np.maximum(clim(CODE["SURFACE_TEMPERATURE"], 0), ice["tfreeze"])
    yclsst2 = _monthly(yclsst, step + 1, pm, points)
    ymld = np.full(points, float(ocean["mldepth"]))
    sea_dts = np.zeros(points)
    sea_dqs = np.zeros(points)
    sea_dsst = np.zeros(points)
    dicec = np.zeros(points)
    diced = np.zeros(points)
    dmld = np.zeros(points)
    sea_points = points - S.js_round(dls.sum())
    if sea_points > 0:
        for h in range(points):
            if dls[h] >= 0.5:
                continue
            ts = yclsst2[h]
            sea_dts[h] = ts
            dicec[h] = xicec[h]
            diced[h] = xiced[h]
            dsnow[h] = 0
            sea_dsst[h] = ts
            dmld[h] = ymld[h]
            dt[sl + h] = ts
            sea_dqs[h] = _saturation(ts, pm)
            dq[sl + h] = sea_dqs[h]
            c = dicec[h]
            drhs[h] = sea["drhssea"] * (1 - c) + sea["drhsice"] * c
            dalb[h] = sea["albsea"] * (1 - c) + c * min(sea["albice"], 0.5 + 0.025 * (273 - ts))
            dsalb[h] = sea["doceanalb"][0] * (1 - c) + c * min(sea["dicealbmx"][0], sea["dicealbmn"][0] + 0.025 * (273 - ts))
            dsalb[points + h] = sea["doceanalb"][1] * (1 - c) + c * min(sea["dicealbmx"][1], sea["dicealbmn"][1] + 0.025 * (273 - ts))
            dz0[h] = sea["dz0sea"] * (1 - c) + sea["dz0ice"] * c
    co2 = rad["co2"]
    fields = dict(
        dls=dls, dz0=dz0, drhs=drhs, dwatc=dwatc, dqco2=np.full(levels * points, co2 if co2 > 0 else 0.0),
        co2=np.array([co2]), dalb=dalb, dsalb=dsalb, dicec=dicec, diced=diced, dmld=dmld, dforest=dforest,
        dglac=dglac, dpersist=dpersist, dwmax=dwmax, dsnow=dsnow, dtsoil=soil[0], dtd2=soil[1], dtd3=soil[2],
        dtd4=soil[3], dtd5=soil[4], dt=dt, dq=dq, land_dts=land_dts, land_dtsm=land_dtsm, land_dqs=land_dqs,
        duroff=duroff, dvroff=dvroff, darea=row_w.copy(), dsnowt=dsnowt, dsnowz=dsnowz, dz0climo=dz0climo,
        dalbclim=dalbclim, dalbclim1=dalbclim1, dalbclim2=dalbclim2, dsoilt=dsoilt, dalbcl=dalbcl,
        dalbcl1=dalbcl1, dalbcl2=dalbcl2, dagg=dagg, dgrow=dgrow, dsc=dsc, dmr=dmr, xts=yclsst2.copy(),
        xsst=yclsst2.copy(), xmld=ymld.copy(), xls=xls, xiced=xiced, xicec=xicec, xgw=row_w.copy(),
        xclsst2=xclsst2, xclicec2=xclicec2, xcliced2=xcliced2, xclssto=xclssto, xclsst=xclsst,
        xclicec=xclicec, xcliced=xcliced, ysst=yclsst2, ymld=ymld, yls=yls, yclsst2=yclsst2.copy(),
        yclsst=yclsst, sea_dts=sea_dts, sea_dqs=sea_dqs, sea_dsst=sea_dsst)
    return fields, so


def timesteps(pm, kits):
    """setup/index.ts:44-49 (timesteps)."""
    return pm["day_24hr"] / pm["mtspd"] / 2 ** kits, S.TWOPI / pm["ntspd"] / 2 ** kits


def phase_constants(pm, mods, kits, nlon):
    """setup/index.ts:53-375 (constants): every kernel constant under its WGSL
    override name, for the step with `kits` start-up steps still to run."""
    rad, rain, flux, land, sea, ice, veg, carbon, glacier = (mods[k] for k in (
        "rad", "rain", "flux", "land", "sea", "ice", "veg", "carbon", "glacier"))
    deltsec, delt = timesteps(pm, kits)
    coupled = kits == 0
    c = dict(
        PSURF=pm["psurf"], WW=pm["ww"], CV=pm["cv"], CT=pm["ct"], AKAP=pm["akap"], RDBRV=pm["rdbrv"],
        ADV=pm["adv"], ACPD=pm["acpd"], GA=pm["ga"], GASCON=pm["gascon"], PLAVOR=pm["plavor"],
        DELT=delt, DELT2=delt + delt, DELTSEC=deltsec, DELTSEC2=deltsec + deltsec, PNU=pm["pnu"],
        PNU21=pm["pnu21"], FILTER=1.0 if coupled else 0.0, RA1=pm["ra1"], RA2=pm["ra2"], RA4=pm["ra4"],
        TMELT=pm["tmelt"], ALV=pm["alv"], ALS=pm["als"], MOIST=1 / pm["rdbrv"] - 1,
        ZUMIN=flux["zumin"], VDIFF_B=flux["vdiff_b"], VDIFF_C=flux["vdiff_c"], VDIFF_D=flux["vdiff_d"],
        NDHEAT=1.0 if pm["ndheat"] > 0 else 0.0,
        NFIXED=1.0 if rad["nfixed"] == 1 else 0.0, ZRLON=S.TWOPI / nlon,
        ZDAWN=math.sin((rad["dawn"] * S.PI) / 180), OZONE=1.0 if rad["no3"] == 1 else 0.0,
        A0O3=rad["a0o3"], A1O3=rad["a1o3"], ACO3=rad["aco3"], BO3=rad["bo3"], CO3=rad["co3"],
        ZCONST=math.exp(-rad["bo3"] / rad["co3"]), GSOL0=rad["gsol0"], ZSOLAR1=rad["zsolar1"],
        ZSOLAR2=rad["zsolar2"], ZSOLARS1=rad["zsolars"][0], ZSOLARS2=rad["zsolars"][1],
        TSWR1=rad["tswr1"], TSWR2=rad["tswr2"], TSWR3=rad["tswr3"],
        ZB3=(rad["tswr1"] * math.sqrt(0.5)) / 0.5, ZB4=rad["tswr2"] * math.sqrt(0.5), ZB5=rad["tswr3"] * 0.25,
        RCOEFF=rad["rcoeff"], LN_DIFFUSE_RAYLEIGH=math.log(1 - 0.144),
        NSTARTEMP=1.0 if rad["nstartemp"] > 0 else 0.0, SBK=S.SBK, TH2OC=rad["th2oc"], TPOFMT=rad["tpofmt"],
        ZFCO2_ZZF2=(100 / 1.9635) * (0.0440098 / 0.0289644) * 1e-6,
        RHBETA=rain["rhbeta"], NBETA=float(rain["nbeta"]), PDEEP=rain["pdeep"], PDEEPTH=rain["pdeepth"],
        RKSHALLOW=rain["rkshallow"], GAMMA=rain["gamma"], ZRFAC=pm["solar_day"] * 1000,
        CLWFAC=rain["clwfac"], CLWCRIT1=rain["clwcrit1"], CLWCRIT2=rain["clwcrit2"],
        SICECAP=land["sicecap"], SOILCAP=land["soilcap"], SICEDIFF=land["sicediff"],
        SOILDIFF=land["soildiff"], SNOWCAP=land["snowcap"], SNOWDIFF=land["snowdiff"],
        RHOSNOW=land["rhosnow"], DZTOP=land["dztop"], DSMAX=land["dsmax"],
        ALBSMAX=land["albsmax"], ALBSMIN=land["albsmin"], ALBSMAXF=land["albsmaxf"], ALBSMINF=land["albsminf"],
        ALBSMAX1=land["albsmax1"], ALBSMIN1=land["albsmin1"], ALBSMAXF1=land["albsmaxf1"],
        ALBSMINF1=land["albsminf1"], ALBSMAX2=land["albsmax2"], ALBSMIN2=land["albsmin2"],
        ALBSMAXF2=land["albsmaxf2"], ALBSMINF2=land["albsminf2"], ALBGMAX=land["albgmax"],
        ALBGMIN=land["albgmin"], ALBGMAX1=land["albgmax1"], ALBGMIN1=land["albgmin1"],
        ALBGMAX2=land["albgmax2"], ALBGMIN2=land["albgmin2"], DRHSFULL=land["drhsfull"],
        NWETSOIL=float(land["nwetsoil"]), WSMAX=land["wsmax"], ALBLAND=land["albland"],
        ALBLANDMAX=land["alblandmax"], DGROUNDALB1=land["dgroundalb"][0], DGROUNDALB2=land["dgroundalb"][1],
        DOCEANALB1=sea["doceanalb"][0], DOCEANALB2=sea["doceanalb"][1],
        NVEG=float(pm["nveg"]), RLUE=land["rlue"], CO2CONV=land["co2conv"], TAU_VEG=land["tau_veg"],
        TAU_SOIL=land["tau_soil"], VWS_CRIT=0.25, Q10=2.0, ZLAIMAX=9.0, ZLAIMIN=0.1, VALB_MIN=0.12,
        VALB_MAX=0.3, VSALB_MIN=0.2, VWMAX_MAX=0.5, VWMAX_MIN=0.05, VZ0_MIN=0.05, CVEG_A=2.9,
        CVEG_C=1.570796326794897, CVEG_F=3.0, CVEG_K=0.5, CVEG_L=0.25, CT_CRIT=5.0,
        CO2_REF=360.0, CO2_COMP=0.0, CO2_SENS=0.3, CVEG_E=math.atan(-1.9), CVEG_G=math.atan(-3.0),
        NCVEG=float(veg["ncveg"]), NGLACIER=1.0 if glacier["nglacier"] > 0 else 0.0,
        GLACELIM=glacier["glacelim"],
        XDT=ice["xdt"], XMIND=ice["xmind"], XMAXD=ice["xmaxd"], CICEMIN=ice["cicemin"], THICEC=ice["thicec"],
        TFREEZE=ice["tfreeze"], CRHOI=S.ICE["CRHOI"], CRHOS=S.ICE["CRHOS"], CRHOSN=S.ICE["CRHOSN"],
        CPI=S.ICE["CPI"], CKAPI=S.ICE["CKAPI"], CKAPSN=S.ICE["CKAPSN"], CLFI=S.ICE["CLFI"],
        CLFSN=S.ICE["CLFSN"], DTMIX=pm["solar_day"] / pm["ntspd"], CPS=S.CPS,
        CHARNOCK=sea["charnock"], DZ0SEA=sea["dz0sea"], DZ0ICE=sea["dz0ice"], DRHSSEA=sea["drhssea"],
        DRHSICE=sea["drhsice"], ALBSEA=sea["albsea"], ALBICE=sea["albice"],
        DICEALBMX1=sea["dicealbmx"][0], DICEALBMX2=sea["dicealbmx"][1],
        DICEALBMN1=sea["dicealbmn"][0], DICEALBMN2=sea["dicealbmn"][1],
        ICE_COUPLED=1.0 if coupled else 0.0,
        NCARBON=1.0 if carbon["ncarbon"] else 0.0, NSUPPLY=1.0 if carbon["nsupply"] else 0.0,
        TIMEWEIGHT=carbon["timeweight"], CO2EARTH=S.CO2EARTH, BETA=carbon["beta"], KACT=carbon["kact"],
        PEARTH=carbon["pearth"], WMAX=carbon["wmax"], VEARTH=carbon["vearth"], PLARAD=pm["plarad"],
        RAD_EARTHSQ=S.RAD_EARTHSQ, NSTORMDIAG=float(mods["storm"]["nstormdiag"]), CKCD=mods["storm"]["ckcd"],
        VITHRESH=mods["storm"]["vithresh"],
    )
    c.update(S.lwr_offsets())
    return c


def build(config, boundary, t_grid, q_grid):
    """The whole FP64 model for one planet: SETUP.constants/schedule/state
    (setup/index.ts:53-477) with the synthetic initial atmosphere given as grid
    temperature (K) and humidity (kg/kg) per level."""
    truncation = config["truncation"]
    levels = config["layers"]
    files = S.namelists_for(config)
    pm = S.pumamod(truncation, levels, files)
    nlat = S.latitudes_for_truncation(truncation)
    nlon = 2 * nlat
    points = nlat * nlon
    sines, weights, _ = S.gaussian_latitudes(nlat)
    mods = S.module_setup(truncation, levels, files, pm)
    surface, so = surface_initial(truncation, levels, pm, mods, boundary, sines, weights)
    # setup/index.ts:53-62: psurf lowered to the mean surface pressure.
    mean_height = (so[0] * pm["cv"] * pm["cv"]) / math.sqrt(2)
    pm["psurf"] = math.exp(math.log(pm["psurf"]) - mean_height / pm["gascon"] / pm["tgr"])
    dyn = S.initpm(truncation, levels, pm)
    sr = S.setzt(dyn, truncation, pm)
    nkits = max(pm["nkits"], 1)
    phases = {k: phase_constants(pm, mods, k, nlon) for k in range(nkits + 1)}
    bm1 = {k: S.makebm(dyn, truncation, timesteps(pm, k)[1]) for k in range(nkits + 1)}
    g2s, s2g = S.legendre_filters(truncation, pm["nfilter"], pm["ngptfilter"], pm["nspvfilter"],
                                  pm["filterkappa"], pm["nfilterexp"], pm["landhoskn0"])
    ltab = S.legendre_tables(sines, weights, truncation)
    ffw, finv = S.fourier_tables(nlon, truncation)
    tables = dict(fourier_forward=ffw, fourier_inverse=finv)
    tables.update(S.legendre_kernel_tables(ltab, g2s, s2g, truncation))
    tables["zgw"] = np.repeat(weights, nlon)
    tables.update(S.surface_flux_tables(dyn["sigma"], dyn["sigmah"], pm["akap"], pm["gascon"], pm["ga"],
                                        mods["flux"]["vdiff_lamm"], mods["flux"]["vdiff_d"]))
    tables.update(S.radiation_tables(sines, dyn["sigma"], dyn["sigmah"], dyn["dsigma"], pm["ga"],
                                     mods["rad"]["acllwr"]))
    tables.update(S.precipitation_tables(dyn["sigma"], pm["akap"], mods["rain"]["rcritmod"],
                                         mods["rain"]["rcritslope"]))
    tables["dsoilz"] = np.array(mods["land"]["dsoilz"], dtype=float)
    for k in ("t0", "dsigma", "sigma", "sigmah", "rdsig", "t01s2", "tkp", "damp", "tdisst", "tdissq",
              "tdissd", "tdissz", "tfrc", "c", "g", "tau", "nindex"):
        tables[k] = np.asarray(dyn[k], dtype=float)
    tables["sakpp"] = dyn["sak"].reshape(-1)
    tables["rcsq"] = S.latitude_factors(sines, nlon)
    tables["sop"] = so
    tables["srp"] = sr.reshape(-1)
    tables["bm1"] = bm1[nkits]

    # Synthetic initial atmosphere, transformed to spectral in f64.
    nrsp = (truncation + 1) * (truncation + 2)
    st = np.zeros((levels, nrsp))
    sq = np.zeros((levels, nrsp))
    for l in range(levels):
        tg = np.asarray(t_grid[l], dtype=float) / pm["ct"] - dyn["t0"][l]
        st[l] = S.legendre_analyse(S.fourier_analyse(tg, nlon, truncation), ltab["qc"], g2s, nlat, truncation)
        sq[l] = S.legendre_analyse(S.fourier_analyse(np.asarray(q_grid[l], dtype=float), nlon, truncation),
                                   ltab["qc"], g2s, nlat, truncation)
    sz = np.zeros((levels, nrsp))
    sz[:, 2] = pm["plavor"]
    sp = np.zeros(nrsp)
    if mods["surf"]["nspinit"] > 0:
        sp = -so * (pm["cv"] * pm["cv"]) / (pm["gascon"] * pm["tgr"])
    state = dict(sp=sp, spm=sp.copy(), st=st.reshape(-1), stm=st.reshape(-1).copy(),
                 sz=sz.reshape(-1), szm=sz.reshape(-1).copy(), sd=np.zeros(levels * nrsp),
                 sdm=np.zeros(levels * nrsp), sq=sq.reshape(-1), sqm=sq.reshape(-1).copy())
    state.update(surface)
    orb = S.orbit(pm["nfixorb"] == 1, pm["eccen"], pm["obliq"], pm["mvelp"], pm["meananom0"])
    cal = dict(keplerian=pm["ngenkeplerian"] == 1,
               fixedSun=(dict(longitudeDeg=pm["fixedlon"], declinationRad=orb["obliquityRad"])
                         if mods["rad"]["nfixed"] == 1 else None),
               stepsPerYear=pm["n_steps_per_year"], stepsPerDay=pm["ntspd"], outputWindowSteps=pm["nafter"],
               stepMinutes=pm["mpstep"], daysPerYear=pm["n_days_per_year"],
               daysPerMonth=pm["n_days_per_month"], solarDay=pm["solar_day"], rotationSpeed=pm["rotspd"],
               toffo3=mods["rad"]["toffo3"], orbit=orb, carbonInterval=mods["carbon"]["interval"])
    return dict(truncation=truncation, levels=levels, nlat=nlat, nlon=nlon, points=points, pumamod=pm,
                modules=mods, phases=phases, bm1=bm1, nkits=nkits, tables=tables, state=state,
                calendar=cal, start_step=pm["n_start_step"], so=so, sines=sines, weights=weights)
