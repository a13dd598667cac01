"""Serving (continuous batching) and the GCM_RUNNER mirror on the GPU."""
import importlib
import threading

import numpy as np
import pytest

serving = importlib.import_module("web-exoplasim_b200.serving")
runner = importlib.import_module("web-exoplasim_b200.runner")
checkpoint = importlib.import_module("web-exoplasim_b200.checkpoint")
planets = importlib.import_module("web-exoplasim_b200.planets")


def _request(i, seed, days, arrival=0.0, truncation=21, levels=5):
    return serving.Request(id=i, truncation=truncation, levels=levels, days=days, seed=seed, arrival=arrival)


@pytest.mark.gpu
def test_result_is_the_same_alone_and_in_the_mix():
    target = dict(seed=901, days=1.5)
    alone = serving.Server({(21, 5): 1}, chunk=8)
    a = _request(0, **target)
    alone.run([a], window=120, drain=True)
    assert a.status == "finished"
    mix = [_request(1, 902, 2.0), _request(2, 903, 0.5, truncation=21, levels=10), _request(3, 904, 1.0, arrival=0.05)]
    b = _request(4, **target, arrival=0.1)  # arrives while others run
    busy = serving.Server({(21, 5): 3, (21, 10): 1}, chunk=8)
    report = busy.run(mix + [b], window=120, drain=True)
    assert b.status == "finished" and report["completed"] == len(mix) + 1
    for name in ("st", "sz", "sd", "sq", "sp"):
        assert np.array_equal(a.result[name], b.result[name]), name


@pytest.mark.gpu
def test_continuous_batching_admits_into_freed_slots():
    # five requests at once for two slots: three wait and enter as slots free
    reqs = [_request(i, 950 + i, days=0.5 + 0.25 * i) for i in range(5)]
    server = serving.Server({(21, 5): 2}, chunk=8)
    report = server.run(reqs, window=300, drain=True)
    assert report["completed"] == 5
    assert report["queue_depth_max"] == 3
    spans = sorted((r.admitted, r.finished) for r in reqs)
    overlaps = sum(1 for (s1, e1), (s2, e2) in zip(spans, spans[1:]) if s2 < e1)
    assert overlaps >= 1
    assert report["p99_s"] >= report["p50_s"] > 0


@pytest.mark.gpu
def test_runner_publishes_pauses_checkpoints_and_stops():
    planet = planets.make_planet(911, truncation=21, levels=5)
    snaps, statuses, saved = [], [], []
    done = threading.Event()

    def status(update):
        statuses.append(update.status)
        if update.status in ("finished", "failed"):
            done.set()

    run = runner.GCM_RUNNER.start(runner.GcmRunRequest(
        planet=planet, publish_every=8, max_steps=40, on_snapshot=snaps.append, on_status=status,
        on_checkpoint=saved.append))
    run.checkpoint()
    assert done.wait(120)
    run.join(10)
    assert statuses[-1] == "finished", statuses
    assert [s.step for s in snaps][:3] == [0, 8, 16]
    assert all(np.all(np.isfinite(s.values)) for s in snaps)
    # the format-21 container around the engine's restart file
    assert saved and saved[0].startswith(checkpoint.MAGIC)
    ckpt = checkpoint.decode(saved[0])
    assert ckpt["meta"]["format"] == 21 and ckpt["restart"].startswith(b"GCM-WEBGPU-STATE\n")


@pytest.mark.gpu
def test_runner_reports_instability():
    planet = planets.make_planet(912, truncation=21, levels=5)
    planet.t_grid[:] = np.nan  # a state that cannot be stepped
    statuses = []
    done = threading.Event()

    def status(update):
        statuses.append((update.status, update.message))
        if update.status in ("finished", "failed"):
            done.set()

    run = runner.GCM_RUNNER.start(runner.GcmRunRequest(planet=planet, publish_every=4, max_steps=8,
                                                       on_status=status))
    assert done.wait(120)
    assert statuses[-1][0] == "failed"
    assert "unstable" in statuses[-1][1]
