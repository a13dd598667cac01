"""Shared helpers for the parity tests: product state <-> oracle state."""
import importlib

import numpy as np

import oracle

pkg = importlib.import_module("web-exoplasim_b200")
planets = importlib.import_module("web-exoplasim_b200.planets")

# State fields the engine holds for the oracle to replay (every field).
def field_names(o):
    return [n for n in oracle_field_list() if o.size(n) >= 0]


def oracle_field_list():
    import re
    text = open(oracle.os.path.join(oracle.HERE, "oracle_fields.h")).read()
    return re.findall(r"X\((\w+),[SFGT],", text)


def copy_engine_to_oracle(engine, slot, o, names=None):
    for name in names or field_names(o):
        o.set(name, engine.read(slot, name).astype(np.float64))


def rel_rms(got, ref):
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    den = np.sqrt(np.mean(ref * ref))
    num = np.sqrt(np.mean((got - ref) ** 2))
    if den == 0:
        return 0.0 if num == 0 else np.inf
    return num / den


def oracle_at_phase(o, phase, step):
    """Sets the oracle's constants and host values to one step of a slot."""
    o.set_phase(phase)
    o.write_step_values(step, publish=False)


def rel_rms_without_worst_columns(got, ref, nhor, drop):
    """Relative RMS of a grid field after removing its `drop` columns with
    the largest squared error (summed over the field's planes)."""
    got = np.asarray(got, dtype=np.float64).reshape(-1, nhor)
    ref = np.asarray(ref, dtype=np.float64).reshape(-1, nhor)
    col = ((got - ref) ** 2).sum(axis=0)
    keep = np.ones(nhor, dtype=bool)
    keep[np.argsort(col)[::-1][:drop]] = False
    return rel_rms(got[:, keep], ref[:, keep])


# The reference's V3 gate (scripts/exoplasim-webgpu/verify-dynamics.mjs:56-59,
# 179-204). A point is off when it differs from f64 by more than
# POINT_TOLERANCE of the field's RMS; a field passes when the GPU's relative
# RMS error is within twice the sequential-f32 build's and its off-point count
# within twice the f32 count plus one. A grid field that fails because one
# column holds more than OUTLIER_SHARE of the GPU's squared error is judged
# again without that one column.
POINT_TOLERANCE = 1e-5
OUTLIER_SHARE = 0.5


def _rms(values, reference=None):
    values = np.asarray(values, dtype=np.float64)
    d = values if reference is None else values - np.asarray(reference, dtype=np.float64)
    return float(np.sqrt(np.mean(d * d))) if d.size else 0.0


def count_off(values, reference, scale):
    d = np.abs(np.asarray(values, dtype=np.float64) - np.asarray(reference, dtype=np.float64))
    return int(np.count_nonzero(d > POINT_TOLERANCE * scale))


def within_gate(gpu_error, f32_error, gpu_off, f32_off, factor=2):
    return gpu_error <= factor * f32_error and gpu_off <= factor * f32_off + 1


def v3_gate(gpu, exact, f32, points=None, factor=2):
    """Judges one field as verify-dynamics.mjs does (`factor` 2). `points` is
    the grid's column count for grid fields (the outlier rule applies to them
    only).
    Returns a dict with the errors, counts, the verdict and any outlier."""
    gpu = np.asarray(gpu, dtype=np.float64).reshape(-1)
    exact = np.asarray(exact, dtype=np.float64).reshape(-1)
    f32 = np.asarray(f32, dtype=np.float64).reshape(-1)
    scale = _rms(exact)
    if scale == 0:
        ok = _rms(gpu) == 0
        return dict(gpu=0.0 if ok else np.inf, f32=0.0, gpu_off=0, f32_off=0, ok=ok, outlier=None)
    r = dict(gpu=_rms(gpu, exact) / scale, f32=_rms(f32, exact) / scale,
             gpu_off=count_off(gpu, exact, scale), f32_off=count_off(f32, exact, scale), outlier=None)
    r["ok"] = within_gate(r["gpu"], r["f32"], r["gpu_off"], r["f32_off"], factor)
    if not r["ok"] and points and gpu.size % points == 0:
        sq = ((gpu - exact) ** 2).reshape(-1, points).sum(axis=0)
        total = sq.sum()
        column = int(np.argmax(sq))
        if total > 0 and sq[column] / total > OUTLIER_SHARE:
            keep = np.arange(gpu.size) % points != column
            g, e, s = gpu[keep], exact[keep], f32[keep]
            out = dict(column=column, share=float(sq[column] / total), gpu=_rms(g, e) / scale,
                       f32=_rms(s, e) / scale, gpu_off=count_off(g, e, scale), f32_off=count_off(s, e, scale))
            r["outlier"] = out
            r["ok"] = within_gate(out["gpu"], out["f32"], out["gpu_off"], out["f32_off"], factor)
    return r


def carbon_counter(model, main_steps):
    """The host's carbon-cycle counter (carbonmod's cstep) after the start-up
    steps and `main_steps` main-loop steps of a run, as the engine and
    Oracle.advance carry it (physics/carbon/index.ts:23-28)."""
    from oracle import setup_f64
    c = 0
    start = model["start_step"]
    for _ in range(model["nkits"]):
        _, c = setup_f64.step_values(start, c, model["calendar"])
    for k in range(main_steps):
        _, c = setup_f64.step_values(start + k, c, model["calendar"])
    return c


# The storm diagnostics' synthetic columns (the reference's
# scripts/exoplasim-webgpu/verify-storm.mjs:48-66 recipe): eleven climates at
# one gas constant over the model's sigma levels; `t` and `r` carry the
# surface value after the L levels, `u`, `v`, `z` only the L levels.
STORM_CLIMATES = ("tropical", "warm", "cold", "hot", "dry", "stable", "thin", "humid", "cold-profile",
                  "reversed-vorticity", "zero-shear")
STORM_FIELDS = ("capen", "lnb", "mpoti", "chim", "laav", "venti", "vrmpi", "gpi", "shear")
# verify-storm.mjs:126-129: |got - expected| <= absolute + 0.5 % |expected|.
STORM_ABSOLUTE = (5.0, 1.0, 0.2, 0.005, 1e-9, 0.005, 0.005, 0.005, 1e-4)


def storm_columns(sigma, rd):
    import math
    rows = []
    for climate in STORM_CLIMATES:
        msl = 500.0 if climate == "thin" else 1000.0
        sst = {"cold": 270.0, "hot": 330.0, "warm": 300.0}.get(climate, 305.0)
        t = [290.0 if climate == "stable" else 95 + 150 * s if climate == "cold-profile" else 195 + 108 * math.sqrt(s)
             for s in sigma]

        def e_of(temp):
            return 6.112 * math.exp(17.67 * (temp - 273.15) / (temp - 29.65))
        r = [0.0 if climate == "dry" else rd / 461.5 * e_of(tl) / (msl * sl - e_of(tl)) *
             (0.98 if climate == "humid" else 0.7) for tl, sl in zip(t, sigma)]
        es = e_of(sst)
        r.append(0.0 if climate == "dry" else 0.8 * (rd / 461.5) * es / (msl - es))
        rows.append(dict(climate=climate, msl=msl, sst=sst, t=t + [sst], r=r,
                         u=[5.0 if climate == "zero-shear" else 3 + 20 * (1 - s) for s in sigma],
                         v=[4.0] * len(sigma), z=[-1.2 if climate == "reversed-vorticity" else 1.2] * len(sigma)))
    return rows


def storm_state(rows, levels, nhor):
    """Fields dt, dq (L + 1 levels), du, dv (L + 1, the last zero), gz (L)
    and dp (Pa) with column h holding rows[h % len(rows)]."""
    pick = [rows[h % len(rows)] for h in range(nhor)]
    out = {}
    for key, name, count in (("t", "dt", levels + 1), ("r", "dq", levels + 1), ("u", "du", levels + 1),
                             ("v", "dv", levels + 1), ("z", "gz", levels)):
        arr = np.zeros((count, nhor))
        for h, row in enumerate(pick):
            vals = row[key]
            arr[:len(vals), h] = vals[:count]
        out[name] = arr
    out["dp"] = np.array([row["msl"] * 100.0 for row in pick])
    return out


def storm_within(got, expected):
    """Per field, the columns outside the reference's storm tolerance."""
    bad = {}
    for i, name in enumerate(STORM_FIELDS):
        g, e = np.asarray(got[name], float), np.asarray(expected[name], float)
        off = ~(np.isfinite(g) & (np.abs(g - e) <= STORM_ABSOLUTE[i] + 0.005 * np.abs(e)))
        if off.any():
            bad[name] = np.flatnonzero(off)
    return bad
