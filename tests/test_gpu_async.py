"""exogcm_step_async / exogcm_poll / exogcm_wait: the worker's pipelined
submit (runner/webgpu/gcm.worker.ts:215-346, IN_FLIGHT = 2) through the C ABI."""
import numpy as np
import pytest

from tests.helpers import pkg, planets


def _engine(seed=101, slots=2):
    e = pkg.Engine(21, 10, slots, mode=1)
    for s in range(slots):
        e.configure(s, planets.make_planet(seed + s, truncation=21, levels=10))
    return e


@pytest.mark.gpu
def test_async_batches_equal_synchronous_steps():
    sync, pipe = _engine(), _engine()
    sync.step(3)
    pipe.step(3)
    for _ in range(3):
        sync.step(8)
    # three batches: the third submission waits for the first (two in flight)
    for _ in range(3):
        pipe.step_async(8)
    pipe.wait()
    assert pipe.poll()
    for name in ("st", "sz", "sd", "sq", "sp", "dt", "xsst"):
        for s in range(2):
            assert np.array_equal(sync.read(s, name), pipe.read(s, name)), (name, s)
    assert pipe.slot_info(0)["step"] == sync.slot_info(0)["step"]


@pytest.mark.gpu
def test_poll_reports_pending_then_done():
    e = _engine(slots=8)
    e.step(3)
    e.step_async(32)
    e.step_async(32)
    # 64 steps of 8 planets take milliseconds of device time; the host gets
    # here in microseconds, so the batches are still in flight
    assert not e.poll()
    for _ in range(200000):
        if e.poll():
            break
    assert e.poll()
    assert e.last_step_ms() > 0


@pytest.mark.gpu
def test_configure_during_async_batch_waits_and_keeps_results():
    """A planet configured while a batch is in flight is uploaded after the
    batch; the slots already stepping match a run without the new planet."""
    a = planets.make_planet(111, truncation=21, levels=10)
    b = planets.make_planet(112, truncation=21, levels=10)
    e = pkg.Engine(21, 10, 2, mode=1)
    ref = pkg.Engine(21, 10, 1, mode=1)
    e.configure(0, a)
    ref.configure(0, a)
    e.step(3)
    ref.step(3)
    e.step_async(8)
    e.configure(1, b)
    e.step(8)
    ref.step(16)
    assert np.array_equal(e.read(0, "st"), ref.read(0, "st"))
    assert e.slot_info(1)["step"] > 0 or e.slot_info(1)["startup_left"] < 3


@pytest.mark.gpu
def test_group_step_runs_mixed_resolutions_as_one_graph():
    """exogcm_group_step: engines of three resolutions stepped by one graph
    launch give each engine's own exogcm_step results bit for bit, with
    per-engine step counts (T63 at 30-minute steps takes more steps per day)."""
    specs = [(21, 5, 2, 45.0, 16), (42, 10, 1, 45.0, 16), (63, 10, 1, 30.0, 24)]

    def make():
        out = []
        for t, l, n, minutes, _ in specs:
            e = pkg.Engine(t, l, n, mode=1)
            for s in range(n):
                e.configure(s, planets.make_planet(120 + s + t, truncation=t, levels=l, timestepMinutes=minutes))
            e.step(3)
            out.append(e)
        return out

    grouped, alone = make(), make()
    steps = [k for *_, k in specs]
    for _ in range(2):
        ms = pkg.group_step(grouped, steps)
        assert ms > 0
        for e, k in zip(alone, steps):
            e.step(k)
    for (t, l, n, *_), g, a in zip(specs, grouped, alone):
        for s in range(n):
            for name in ("st", "sz", "sd", "sq", "sp", "dt"):
                assert np.array_equal(g.read(s, name), a.read(s, name)), (t, l, s, name)
        assert g.slot_info(0)["step"] == a.slot_info(0)["step"]


@pytest.mark.gpu
def test_snapshots_of_pipelined_days_equal_synchronous_days():
    """exogcm_snapshots_begin does not wait for batches in flight: it copies
    the snapshot the last submitted batch leaves. Days submitted with
    step_async (two in flight) and a bulk snapshot copy after each give the
    snapshots and states of exogcm_step day by day, bit for bit."""
    sync, pipe = _engine(slots=3), _engine(slots=3)
    for e in (sync, pipe):
        e.step(3)
    planes = sync.field_size("snapshot")
    ref = []
    for _ in range(3):
        sync.step(32, publish_every=32)
        out = np.zeros(planes * 3, dtype=np.float32)
        sync.snapshots_begin(out)
        sync.snapshots_wait()
        ref.append(out)
    got = [np.zeros(planes * 3, dtype=np.float32) for _ in range(3)]
    for day in range(3):
        pipe.step_async(32, publish_every=32)
        pipe.snapshots_begin(got[day])
    pipe.snapshots_wait()
    assert pipe.poll()
    for day in range(3):
        assert np.array_equal(ref[day], got[day]), day
    assert not np.array_equal(ref[0], ref[2])
    for name in ("st", "sq", "sp"):
        for s in range(3):
            assert np.array_equal(sync.read(s, name), pipe.read(s, name)), (name, s)
