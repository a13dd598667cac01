"""The allocation-free sums entry point against the engine's own sums.

Callers that cannot allocate device memory (a host inside another
framework's memory pool, a runtime with a fixed device footprint) get the
per-planet FP64 sums through exogcm_slot_sums_noalloc, whose scratch is a
static device array. This checks, through the C ABI, that two calls in a row
reproduce what the engine's fixer and getiflx reductions wrote, that a call
after the first leaves the device's free memory unchanged, and that every
slot is summed, an uncoupled one included, which the step's getiflx skips.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import pkg, planets


def _sums(lib, a, b, slots, nhor, out):
    rc = lib.exogcm_slot_sums_noalloc(ctypes.c_void_p(a), ctypes.c_void_p(b), slots, nhor,
                                      ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 0


@pytest.mark.gpu
def test_noalloc_sums_match_engine_sums_on_two_calls():
    import torch

    lib = pkg.load_library()
    slots = 3
    engine = pkg.Engine(21, 5, slots)
    for s in range(slots):
        engine.configure(s, planets.make_planet(81 + s, truncation=21, levels=5, land_fraction=0.2 + 0.1 * s))
    engine.step(3)  # start-up steps
    engine.step(2)  # main loop: icestep and getiflx run
    nhor = 32 * 64
    out = torch.full((2 * slots,), -1.0, dtype=torch.float32, device="cuda")
    cases = [("fixer", "fixneg", "fixpos", "fixsum"), ("surface", "ice_part1", "ice_part2", "ice_sums")]
    # the first call on the device commits the static scratch (lazy module loading)
    a, _ = engine.device_field("fixneg")
    _sums(lib, a, a, slots, nhor, out)
    torch.cuda.synchronize()
    for stage, first, second, sums in cases:
        engine.run_stage(stage)  # the existing entry point writes its sums into the state
        want = np.stack([engine.read(s, sums) for s in range(slots)], axis=1)  # [2][slots]
        a, _ = engine.device_field(first)
        b, _ = engine.device_field(second)
        torch.cuda.synchronize()
        free_before, _ = torch.cuda.mem_get_info()
        _sums(lib, a, b, slots, nhor, out)
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before, "the call changed the device's free memory"
        got = out.cpu().numpy().reshape(2, slots)
        # same FP64 summation order: equal to the last bit (tolerance 0)
        np.testing.assert_array_equal(got, want)
        assert np.abs(want).max() > 0


@pytest.mark.gpu
def test_noalloc_sums_every_slot_including_uncoupled():
    """The step's getiflx sum skips slots without sea-ice coupling (their
    ice_sums stay as they were); the allocation-free entry point sums every
    slot it is given. Checked against a float64 sum of the same inputs."""
    import torch

    lib = pkg.load_library()
    engine = pkg.Engine(21, 5, 2)
    engine.configure(0, planets.make_planet(91, truncation=21, levels=5))
    engine.step(3)
    # slot 1 joins now: its next step is a start-up step, without icestep, so
    # the step's getiflx leaves its ice_sums alone while slot 0's are summed
    engine.configure(1, planets.make_planet(92, truncation=21, levels=5))
    engine.step(1)
    assert engine.slot_info(1)["startup_left"] > 0
    nhor = 32 * 64
    a, _ = engine.device_field("ice_part1")
    b, _ = engine.device_field("ice_part2")
    out = torch.zeros(4, dtype=torch.float32, device="cuda")
    _sums(lib, a, b, 2, nhor, out)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(2, 2)
    for s in range(2):
        for k, name in enumerate(("ice_part1", "ice_part2")):
            want = np.float32(engine.read(s, name).astype(np.float64).sum())
            assert abs(got[k, s] - want) <= 1e-6 * max(abs(want), 1.0), (s, name)


@pytest.mark.gpu
def test_noalloc_rejects_too_many_slots():
    import torch

    lib = pkg.load_library()
    buf = torch.zeros(4, device="cuda")
    rc = lib.exogcm_slot_sums_noalloc(ctypes.c_void_p(buf.data_ptr()), ctypes.c_void_p(buf.data_ptr()), 257, 1,
                                      ctypes.c_void_p(buf.data_ptr()), None)
    assert rc == -1
    msg = ctypes.create_string_buffer(256)
    lib.exogcm_last_error(msg, 256)
    assert b"256" in msg.value
