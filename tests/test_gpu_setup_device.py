"""The FP64 set-up loops on the device (legini with the filters, the grid ->
spectral analysis of the orography and initial state, makebm's LU inverses;
legendre/index.ts:29-136 and 334-361, dynamics/setup/index.ts:154-239):
bit for bit the host set-up's numbers, within 1e-12 of the oracle, and an
engine configured either way holds the same state."""
import numpy as np
import pytest

import oracle
from tests.helpers import field_names, pkg, planets

pytestmark = pytest.mark.gpu

CASES = [(21, 10, 3), (42, 10, 4), (21, 5, 5), (63, 10, 6)]
DEVICE_ARRAYS = ["shared:" + q for q in ("qi", "qj", "qc", "qe", "qm", "qq", "qu", "qv")] + \
    ["table:bm1", "table:sop", "state:st", "state:stm", "state:sq", "state:sqm", "state:sz"]


def planet_for(truncation, levels, seed):
    return planets.make_planet(seed, truncation=truncation, levels=levels,
                               rotationPeriodDays=1.0 if seed % 2 else 2.5,
                               pressureBar=1.011 if seed < 5 else 3.0)


@pytest.mark.parametrize("truncation,levels,seed", CASES)
def test_device_setup_equals_host_bitwise(truncation, levels, seed):
    p = planet_for(truncation, levels, seed)
    for name in DEVICE_ARRAYS:
        host = pkg.setup_preview(p, name)
        dev = pkg.setup_preview(p, name, on_device=True)
        assert dev.shape == host.shape, name
        np.testing.assert_array_equal(dev, host, err_msg=name)


@pytest.mark.parametrize("truncation,levels,seed", CASES)
def test_device_setup_matches_oracle(truncation, levels, seed):
    p = planet_for(truncation, levels, seed)
    m = oracle.model_for(p)
    for q in ("qi", "qj", "qc", "qe", "qm", "qq", "qu", "qv"):
        got = pkg.setup_preview(p, "shared:" + q, on_device=True)
        ref = m["tables"]["legendre_" + q].reshape(-1)
        assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0), q
    ref = np.concatenate([m["bm1"][k] for k in range(4)])
    got = pkg.setup_preview(p, "table:bm1", on_device=True)[:ref.size]
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
    for name in ("st", "stm", "sq", "sqm", "sz"):
        got = pkg.setup_preview(p, "state:" + name, on_device=True)
        ref = np.asarray(m["state"][name], dtype=float).reshape(-1)
        assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0), name
    ref = np.asarray(m["tables"]["sop"], dtype=float).reshape(-1)
    got = pkg.setup_preview(p, "table:sop", on_device=True)[:ref.size]
    assert np.abs(got - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1.0)


@pytest.mark.parametrize("mode", [0, 1])
def test_engine_state_is_the_same_with_host_or_device_setup(mode):
    p = planets.make_planet(8, truncation=21, levels=10)
    q = planets.make_planet(9, truncation=21, levels=10, rotationPeriodDays=3.0)
    dev = pkg.Engine(21, 10, 2, mode=mode)
    host = pkg.Engine(21, 10, 2, mode=mode)
    host.setup_on_device(False)
    try:
        for e in (dev, host):
            e.configure(0, p)
            e.configure(1, q)
        o = oracle.Oracle(oracle.model_for(p))
        for slot in (0, 1):
            for name in field_names(o):
                np.testing.assert_array_equal(dev.read(slot, name), host.read(slot, name), err_msg=name)
        # Both step to the same state.
        dev.step(2, 1000)
        host.step(2, 1000)
        for name in ("st", "sz", "sq", "dt"):
            np.testing.assert_array_equal(dev.read(1, name), host.read(1, name), err_msg=name)
    finally:
        dev.close()
        host.close()
