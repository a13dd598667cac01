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
