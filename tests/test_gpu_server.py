"""The C ABI's batched server (exogcm_server_*): runs served together equal
the same runs stepped alone, bit for bit; a budget too small for one block
rejects; a budget for one block at a time serves two resolutions in turn by
destroying the empty block."""
import ctypes

import numpy as np
import pytest

from tests.helpers import pkg, planets


def slot_bytes(T, L):
    """Device bytes of one engine slot as the server counts them: every
    state field of the layout (csrc/fields.h) in f32, plus 64 KiB of tables."""
    import os
    import re
    src = os.path.join(os.path.dirname(pkg.__file__), "csrc", "fields.h")
    text = open(src).read()
    text = text[text.index("#define EXOGCM_FIELDS"):text.index("// clang-format on")]
    nlat = {21: 32, 42: 64, 63: 96}[T]
    plane = {"S": (T + 1) * (T + 2), "F": nlat * 2 * (T + 1), "G": 2 * nlat * nlat}
    count = {"L": L, "H": L + 1, "P": 51 + 5 * L}
    total = 0
    for _, shape, n in re.findall(r"X\((\w+),([SFGT]),(\w+)\)", text):
        n = count[n] if n in count else int(n)
        total += n if shape == "T" else plane[shape] * n
    return total * 4 + 64 * 1024


def alone(p, steps):
    """The run stepped by itself in a one-slot engine, stopped at `steps` main-loop steps."""
    T, L = p.config["truncation"], p.config["layers"]
    e = pkg.Engine(T, L, 1, mode=1)
    try:
        e.configure(0, p)
        start = e.slot_info(0)["step"]
        e.set_stop(0, start + steps)
        while True:
            info = e.slot_info(0)
            if info["startup_left"] == 0 and info["step"] >= start + steps:
                break
            e.step(16)
        return {n: e.read(0, n) for n in ("st", "sz", "sd", "sq", "sp")}, {n: e.field_size(n) for n in ("st", "sp")}
    finally:
        e.close()


def test_invalid_options_fail_without_a_device():
    lib = pkg.load_library()
    h = ctypes.c_void_p()
    bad = pkg.ServerOptions(budget_bytes=0.0, block_slots=4, chunk_steps=8, mode=1)
    assert lib.exogcm_server_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    bad = pkg.ServerOptions(budget_bytes=1e9, block_slots=4, chunk_steps=100, mode=1)
    assert lib.exogcm_server_create(ctypes.byref(bad), ctypes.byref(h)) == -1
    ok = pkg.ServerOptions(budget_bytes=1e9, block_slots=4, chunk_steps=8, mode=1)
    assert lib.exogcm_server_create(ctypes.byref(ok), ctypes.byref(h)) == 0
    rid = ctypes.c_long()
    p = pkg.planet_struct(planets.BASE_CONFIG)
    b = pkg.Boundary()  # no land mask: rejected before any device work
    assert lib.exogcm_server_submit(h, ctypes.byref(p), ctypes.byref(b), 10, ctypes.byref(rid)) == -1
    lib.exogcm_server_destroy(h)


@pytest.mark.gpu
def test_served_runs_equal_runs_alone():
    runs = [(planets.make_planet(301, truncation=21, levels=5), 40),
            (planets.make_planet(302, truncation=21, levels=5), 70),
            (planets.make_planet(303, truncation=42, levels=10), 24)]
    server = pkg.NativeServer(budget_bytes=8e9, block_slots=4, chunk_steps=16, mode=1)
    try:
        ids = [server.submit(p, steps) for p, steps in runs]
        assert server.poll(ids[0]) == ("queued", 0)
        for _ in range(200):
            if server.pump() == 0:
                break
        for rid, (p, steps) in zip(ids, runs):
            status, done = server.poll(rid)
            assert status == "finished" and done == steps, (rid, status, done)
            ref, sizes = alone(p, steps)
            for name, want in ref.items():
                got = server.result(rid, name, want.size)
                np.testing.assert_array_equal(got, want, err_msg=name)
            server.release(rid)
        with pytest.raises(pkg.ExogcmError):
            server.poll(ids[0])
    finally:
        server.close()


@pytest.mark.gpu
def test_budget_rejects_and_evicts():
    small = pkg.NativeServer(budget_bytes=1e6, block_slots=4, chunk_steps=8, mode=1)
    try:
        rid = small.submit(planets.make_planet(311, truncation=21, levels=5), 8)
        small.pump()
        assert small.poll(rid)[0] == "rejected"
    finally:
        small.close()
    # room for the one-slot T42 L10 block, not for it and the T21 L5 block together
    budget = slot_bytes(42, 10) + 0.5 * slot_bytes(21, 5)
    server = pkg.NativeServer(budget_bytes=budget, block_slots=1, chunk_steps=8, mode=1)
    try:
        a = server.submit(planets.make_planet(312, truncation=21, levels=5), 16)
        b = server.submit(planets.make_planet(313, truncation=42, levels=10), 8)
        seen_b_queued_while_a_runs = False
        for _ in range(200):
            active = server.pump()
            if server.poll(a)[0] == "running" and server.poll(b)[0] == "queued":
                seen_b_queued_while_a_runs = True
            if active == 0:
                break
        assert server.poll(a)[0] == "finished" and server.poll(b)[0] == "finished"
        assert seen_b_queued_while_a_runs
    finally:
        server.close()


@pytest.mark.gpu
def test_unstable_and_rejected_set_up_runs_fail_alone():
    good = planets.make_planet(321, truncation=21, levels=5)
    nan = planets.make_planet(322, truncation=21, levels=5)
    nan.t_grid[:] = np.nan  # a state that cannot be stepped
    bad = planets.make_planet(323, truncation=21, levels=5, starTemperatureK=5000.0)  # set-up refuses it
    server = pkg.NativeServer(budget_bytes=4e9, block_slots=4, chunk_steps=8, mode=1)
    try:
        ids = [server.submit(p, 16) for p in (good, nan, bad)]
        for _ in range(100):
            if server.pump() == 0:
                break
        assert [server.poll(i)[0] for i in ids] == ["finished", "failed", "failed"]
        ref, _ = alone(good, 16)
        np.testing.assert_array_equal(server.result(ids[0], "st", ref["st"].size), ref["st"])
        with pytest.raises(pkg.ExogcmError):
            server.result(ids[1], "st", ref["st"].size)
    finally:
        server.close()
