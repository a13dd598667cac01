"""Per-planet FP64 global budgets and the device-side monthly means
(exogcm_budgets, exogcm_averages_*), against FP64 sums of the engine's own
fields on the host."""
import numpy as np
import pytest

from oracle import setup_f64
from tests.helpers import pkg, planets


def _weights(nlat):
    _, w, _ = setup_f64.gaussian_latitudes(nlat)
    return np.repeat(np.asarray(w, dtype=np.float64), 2 * nlat)


def _host_budgets(e, slot, w, L):
    nhor = w.size
    r = lambda n: e.read(slot, n).astype(np.float64)
    dswfl, dlwfl, dt = r("dswfl").reshape(L + 1, nhor), r("dlwfl").reshape(L + 1, nhor), r("dt").reshape(L + 1, nhor)
    q = [r("dp"), dswfl[0] + dlwfl[0], r("dsmelt") * -333700000.0 + dswfl[L] + dlwfl[L] + r("dshfl") + r("dlhfl"),
         dt[L], r("dprc") + r("dprl"), -r("devap"), r("dqvi"), np.ones(nhor)]
    return np.array([np.sum(w * x) / np.sum(w) for x in q])


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_budgets_are_fp64_global_means_of_the_published_step(mode):
    L = 10
    e = pkg.Engine(21, L, 2, mode=mode)
    e.configure(0, planets.make_planet(141, truncation=21, levels=L))
    e.configure(1, planets.make_planet(142, truncation=21, levels=L, co2Ppm=2000.0))
    w = _weights(32)
    # the start-up steps and main-loop step 0 (both at step number 0, a
    # multiple of every publish interval) publish: leave those samples out
    e.step(4)
    for s in range(2):
        e.budgets(s, reset=True)
    seen = []
    for _ in range(3):
        # the budgets are those of the step that published: make it the
        # last one run, so the fields read back are that step's
        e.step(3)
        e.step(1, publish_every=1)
        for s in range(2):
            b = e.budgets(s)
            host = _host_budgets(e, s, w, L)
            got = np.array([b["last"][k] for k in pkg.Engine.BUDGETS])
            np.testing.assert_allclose(got, host, rtol=1e-12, atol=1e-300)
            seen.append((s, host))
    for s in range(2):
        b = e.budgets(s, reset=True)
        assert b["samples"] == 3
        want = np.mean([h for t, h in seen if t == s], axis=0)
        np.testing.assert_allclose([b["mean"][k] for k in pkg.Engine.BUDGETS], want, rtol=1e-12)
        assert abs(b["last"]["weight"] - 1.0) < 1e-14
        assert 5e4 < b["last"]["surface_pressure"] < 2e5 and 150 < b["last"]["surface_temperature"] < 350
        assert e.budgets(s)["samples"] == 0


@pytest.mark.gpu
def test_monthly_means_on_device_equal_the_mean_of_published_snapshots():
    e = pkg.Engine(21, 5, 2, mode=1)
    for s in range(2):
        e.configure(s, planets.make_planet(151 + s, truncation=21, levels=5))
    e.step(3)
    e.averages_enable(True)
    snaps = {0: [], 1: []}
    for _ in range(4):
        e.step(4, publish_every=4)
        for s in range(2):
            step, snap = e.snapshot(s)
            assert step >= 0
            snaps[s].append(snap.astype(np.float64))
    for s in range(2):
        mean, n = e.averages_read(s, reset=True)
        assert n == 4
        want = np.mean(snaps[s], axis=0).astype(np.float32)
        np.testing.assert_array_equal(mean, want.reshape(mean.shape))
        _, n = e.averages_read(s)
        assert n == 0
    e.step(4, publish_every=4)
    mean, n = e.averages_read(0)
    assert n == 1
    np.testing.assert_array_equal(mean, e.snapshot(0)[1].reshape(mean.shape))
    e.averages_enable(False)
    with pytest.raises(pkg.ExogcmError):
        e.averages_read(0)
