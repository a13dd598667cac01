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
