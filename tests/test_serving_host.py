"""Host-side logic of the serving loop that needs no GPU: the Poisson request
stream and the latency report."""
import importlib

import numpy as np

serving = importlib.import_module("web-exoplasim_b200.serving")


def test_poisson_requests_are_seeded_ordered_and_bounded():
    resolutions = ((21, 5), (42, 10))
    reqs = serving.poisson_requests(8.0, 500.0, seed=3, max_days=2.0, min_days=0.5, resolutions=resolutions)
    again = serving.poisson_requests(8.0, 500.0, seed=3, max_days=2.0, min_days=0.5, resolutions=resolutions)
    assert [(r.arrival, r.days, r.seed, r.truncation, r.levels) for r in reqs] == \
           [(r.arrival, r.days, r.seed, r.truncation, r.levels) for r in again]
    arrivals = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arrivals) > 0) and 0 < arrivals[0] and arrivals[-1] <= 500.0
    # 4000 arrivals expected; a Poisson count stays within a few standard deviations (63)
    assert abs(len(reqs) - 4000) < 300
    assert [r.id for r in reqs] == list(range(len(reqs)))
    assert all(0.5 <= r.days <= 2.0 for r in reqs)
    assert {(r.truncation, r.levels) for r in reqs} == set(resolutions)
    assert all(r.status == "queued" and r.admitted is None for r in reqs)
    other = serving.poisson_requests(8.0, 500.0, seed=4, max_days=2.0, min_days=0.5, resolutions=resolutions)
    assert [r.arrival for r in other[:5]] != [r.arrival for r in reqs[:5]]


def test_report_gives_latency_percentiles_of_finished_runs():
    server = serving.Server({})
    latencies = []
    for i in range(101):
        r = serving.Request(id=i, truncation=21, levels=5, days=1.0, seed=i, arrival=float(i))
        r.finished = r.arrival + 0.01 * (i + 1)
        r.status = "finished"
        latencies.append(0.01 * (i + 1))
        server.done.append(r)
    failed = serving.Request(id=101, truncation=21, levels=5, days=1.0, seed=0, arrival=0.0)
    failed.status = "failed"
    server.done.append(failed)
    rep = server.report(elapsed=50.0)
    assert rep["completed"] == 101 and rep["failed"] == 1
    assert abs(rep["p50_s"] - np.percentile(latencies, 50)) < 1e-12
    assert abs(rep["p99_s"] - np.percentile(latencies, 99)) < 1e-12
    assert abs(rep["sim_days_per_s"] - 101 / 50.0) < 1e-12
    assert rep["slots"] == {} and rep["window_s"] == 50.0
