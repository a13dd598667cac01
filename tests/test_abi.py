"""The C-ABI library loads without a GPU and exports every declared symbol;
its host-side FP64 set-up matches the oracle's (no device calls here)."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from tests.helpers import pkg, planets

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "exogcm.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void\*?|void)\s+\**(exogcm_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = pkg.load_library()
    names = declared()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
        assert name in pkg.SIGNATURES, name


def test_invalid_arguments_fail_without_a_device():
    lib = pkg.load_library()
    h = ctypes.c_void_p()
    assert lib.exogcm_create(30, 10, 1, 0, ctypes.byref(h)) == -1
    buf = ctypes.create_string_buffer(256)
    lib.exogcm_last_error(buf, 256)
    assert b"truncation" in buf.value
    assert lib.exogcm_create(21, 7, 1, 0, ctypes.byref(h)) == -1


@pytest.mark.parametrize("truncation,levels,seed", [(21, 10, 3), (42, 10, 4), (21, 5, 5), (63, 10, 6)])
def test_setup_matches_oracle(truncation, levels, seed):
    p = planets.make_planet(seed, truncation=truncation, levels=levels,
                            rotationPeriodDays=1.0 if seed % 2 else 2.5, pressureBar=1.011 if seed < 5 else 3.0)
    m = oracle.model_for(p)
    for name, ref in m["tables"].items():
        if name in ("fourier_forward", "fourier_inverse", "zgw", "sid", "cola", "rcsq", "nindex") or \
                name.startswith("legendre_"):
            continue
        ref = np.concatenate([m["bm1"][k] for k in range(4)]) if name == "bm1" else np.asarray(ref).reshape(-1)
        got = pkg.setup_preview(p, "table:" + name)[:ref.size]
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(got - ref).max() / scale < 1e-12, name
    for name, ref in m["state"].items():
        got = pkg.setup_preview(p, "state:" + name)
        ref = np.asarray(ref, dtype=float).reshape(-1)
        assert got.shape == ref.shape, name
        assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0), name
    for k, v in m["phases"][0].items():
        if k in ("DELT", "DELT2", "DELTSEC", "DELTSEC2", "FILTER", "ICE_COUPLED"):
            continue
        got = pkg.setup_preview(p, "const:" + k)[0]
        assert abs(got - v) <= 1e-12 * max(abs(v), 1.0), k
    for q in ("qi", "qj", "qc", "qe", "qm", "qq", "qu", "qv"):
        got = pkg.setup_preview(p, "shared:" + q)
        assert np.abs(got - m["tables"]["legendre_" + q].reshape(-1)).max() < 1e-13, q


@pytest.mark.parametrize("rotation", [1.0, 0.25, 37.0])
def test_calendar_matches_oracle(rotation):
    p = planets.make_planet(7, truncation=21, levels=5, rotationPeriodDays=rotation)
    m = oracle.model_for(p)
    for step in (0, 1, 31, 47, 500, 11519, 23040):
        got = pkg.setup_preview(p, f"calendar:{step}")
        vals, cs = oracle.setup_f64.step_values(step, 0, m["calendar"])
        ref = np.concatenate([vals["radiation_step"], vals["surface_step"], vals["carbon_step"], [cs]])
        np.testing.assert_allclose(got[:14], ref, atol=1e-12)
    assert pkg.setup_preview(p, "calendar:0")[14] == m["start_step"]


def test_setup_rejects_unsupported_inputs():
    p = planets.make_planet(1, truncation=21, levels=10, starTemperatureK=5780.0)
    with pytest.raises(pkg.ExogcmError):
        pkg.setup_preview(p, "table:t0")
