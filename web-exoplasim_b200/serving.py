"""Serving: continuous batching of many planet runs on one GPU.

Requests (a seeded planet, a resolution and a duration in simulated days)
arrive over time. Runs of one resolution (T, L) share batched engines
("blocks" of slots). A request is admitted into a free slot of its
resolution, or, when none is free, into a new block if the HBM budget has
room for it: every resolution draws on one byte budget by its per-slot state
footprint, blocks are created as requests need them and destroyed when they
empty while another resolution waits for room. An admitted run is configured
into its slot while the other slots keep their state on the device, steps
with everyone else in the same launches, and leaves when its last step is
done: the engine stops a slot exactly at its final step (exogcm_set_stop), so
a result does not depend on what else was running.

Every block with running slots is submitted with exogcm_step_async, so the
blocks' batches run concurrently on their own streams while the host admits
new arrivals (their host set-up overlaps the device work); the loop then
waits for the batches and collects finished runs.

Reported: time-to-result p50/p99, admission queue depth, and aggregate
simulated days per second over the window.
"""
from __future__ import annotations

import importlib
import math
import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

pkg = importlib.import_module("web-exoplasim_b200")
planets_mod = importlib.import_module("web-exoplasim_b200.planets")

# Model timestep per truncation: 45 minutes, and 30 at T63 where the
# reference documents 45-minute runs going unstable.
STEP_MINUTES = {21: 45.0, 42: 45.0, 63: 30.0}


@dataclass
class Request:
    id: int
    truncation: int
    levels: int
    days: float
    seed: int
    arrival: float = 0.0
    overrides: dict = field(default_factory=dict)
    planet: object = None  # a prebuilt planets.Planet (the client's input); else made from the seed
    # filled in by the server
    admitted: float | None = None
    finished: float | None = None
    steps: int = 0
    status: str = "queued"
    result: dict | None = None


def slot_bytes(truncation: int, levels: int) -> int:
    """Device bytes one slot of a (T, L) engine holds (state plus tables)."""
    e = pkg.Engine(truncation, levels, 1)
    try:
        names = [n for n in FIELD_NAMES]
        return sum(e.field_size(n) for n in names) * 4 + 64 * 1024
    finally:
        e.close()


FIELD_NAMES: list[str] = []


def _field_names():
    import os
    import re
    src = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "fields.h")
    return re.findall(r"X\((\w+),[SFGT],", open(src).read())


class Group:
    """One batched engine (a block of slots of one resolution)."""

    def __init__(self, truncation, levels, slots, chunk, mode=1, setup_on_device=True):
        self.truncation, self.levels, self.slots, self.chunk = truncation, levels, slots, chunk
        self.engine = pkg.Engine(truncation, levels, slots, mode=mode)
        self.engine.setup_on_device(setup_on_device)
        self.configure_s: list[float] = []  # wall time of each exogcm_configure (set-up + upload)
        self.free = deque(range(slots))
        self.running: dict[int, Request] = {}
        self.stop_step: dict[int, int] = {}
        self.sim_days = 0.0
        self.in_flight = False

    def admit(self, req: Request, now: float):
        slot = self.free.popleft()
        planet = req.planet
        if planet is None:
            planet = planets_mod.make_planet(req.seed, truncation=req.truncation, levels=req.levels,
                                             timestepMinutes=STEP_MINUTES[req.truncation], **req.overrides)
        t = time.perf_counter()
        self.engine.configure(slot, planet)
        self.configure_s.append(time.perf_counter() - t)
        steps_per_day = 1440.0 / STEP_MINUTES[req.truncation]
        req.steps = max(1, int(round(req.days * steps_per_day)))
        start = self.engine.slot_info(slot)["step"]
        self.stop_step[slot] = start + req.steps
        self.engine.set_stop(slot, start + req.steps)
        req.admitted = now
        req.status = "running"
        self.running[slot] = req

    def submit(self):
        if self.running:
            self.engine.step_async(self.chunk, publish_every=1 << 30)
            self.in_flight = True

    def wait(self):
        if self.in_flight:
            self.engine.wait()
            self.in_flight = False

    def step(self):
        self.submit()
        self.wait()

    def collect(self, now: float, done: list):
        unstable = self.engine.unstable() if self.running else None
        for slot, req in list(self.running.items()):
            info = self.engine.slot_info(slot)
            failed = unstable is not None and unstable[slot]
            if failed or (info["startup_left"] == 0 and info["step"] >= self.stop_step[slot]):
                req.finished = now
                req.status = "failed" if failed else "finished"
                if not failed:
                    self.sim_days += req.days
                    req.result = {name: self.engine.read(slot, name) for name in ("st", "sz", "sd", "sq", "sp")}
                self.engine.release(slot)
                del self.running[slot]
                self.free.append(slot)
                done.append(req)

    def close(self):
        self.wait()
        self.engine.close()


class Server:
    """Continuous-batching loop over blocks of batched engines.

    Server(capacity): one fixed block per (T, L) with the given slot counts.
    Server(budget_bytes=B, block=n): blocks of n slots (fewer at the larger
    resolutions, see `block_slots`) created and destroyed on demand within an
    HBM budget of B bytes shared by every resolution."""

    def __init__(self, capacity: dict | None = None, chunk: int = 16, keep_results: bool = True,
                 budget_bytes: float | None = None, block: int = 32, mode: int = 1, setup_on_device: bool = True):
        self.chunk, self.mode, self.block = chunk, mode, block
        self.setup_on_device = setup_on_device
        self.blocks: list[Group] = [Group(key[0], key[1], n, chunk, mode, setup_on_device)
                                    for key, n in (capacity or {}).items() if n > 0]
        self.configure_s: list[float] = []  # of blocks already destroyed
        self.elastic = budget_bytes is not None
        self.budget = float(budget_bytes or 0.0)
        self.queue: deque[Request] = deque()
        self.done: list[Request] = []
        self.queue_depth: list[int] = []
        self.keep_results = keep_results
        self.peak_bytes = 0
        self.blocks_created = 0
        self.blocks_destroyed = 0

    # kept for callers that address one block per resolution
    @property
    def groups(self) -> dict:
        return {(b.truncation, b.levels): b for b in self.blocks}

    @staticmethod
    def capacity_for(budget_bytes: float, mix: dict, max_slots: int = 256) -> dict:
        """Slots per (T, L) from an HBM budget split by the expected mix of
        work (fraction of requests per resolution times its per-slot bytes)."""
        sizes = {key: slot_bytes_cached(*key) for key in mix}
        weight = sum(mix[k] * sizes[k] for k in mix)
        return {k: int(min(max_slots, max(1, budget_bytes * mix[k] / weight))) for k in mix}

    def block_slots(self, truncation: int, levels: int) -> int:
        """Slots of a new block: `block` at T21, scaled down by the footprint
        so a block's bytes stay about the same at every resolution."""
        ratio = slot_bytes_cached(21, 5) / slot_bytes_cached(truncation, levels)
        return max(1, int(round(self.block * min(1.0, 4 * ratio))))

    def used_bytes(self) -> int:
        return sum(b.slots * slot_bytes_cached(b.truncation, b.levels) for b in self.blocks)

    def submit(self, req: Request):
        self.queue.append(req)

    def _free_slot(self, key):
        for b in self.blocks:
            if (b.truncation, b.levels) == key and b.free:
                return b
        return None

    def _grow(self, key):
        """A new block for `key` if the budget holds it, destroying empty
        blocks of other resolutions to make room."""
        if not self.elastic:
            return None
        n = self.block_slots(*key)
        need = n * slot_bytes_cached(*key)
        while self.used_bytes() + need > self.budget:
            empty = [b for b in self.blocks if not b.running and (b.truncation, b.levels) != key]
            if not empty:
                return None
            b = empty[0]
            self.configure_s.extend(b.configure_s)
            b.close()
            self.blocks.remove(b)
            self.blocks_destroyed += 1
        block = Group(key[0], key[1], n, self.chunk, self.mode, self.setup_on_device)
        self.blocks.append(block)
        self.blocks_created += 1
        self.peak_bytes = max(self.peak_bytes, self.used_bytes())
        return block

    def _admit(self, now: float):
        waiting = deque()
        while self.queue:
            req = self.queue.popleft()
            key = (req.truncation, req.levels)
            if not self.elastic and key not in self.groups:
                req.status = "rejected"
                req.finished = now
                self.done.append(req)
                continue
            if req.arrival > now:
                waiting.append(req)
                continue
            block = self._free_slot(key) or self._grow(key)
            if block is not None:
                block.admit(req, now)
            else:
                waiting.append(req)
        self.queue = waiting

    def run(self, requests: list[Request], window: float, drain: bool = False, clock=time.perf_counter):
        """Serves `requests` (arrival times relative to the start) for
        `window` seconds of wall time, or until all finish with `drain`."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        t0 = clock()
        while True:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                self.queue.append(pending.popleft())
            active = [b for b in self.blocks if b.running]
            for b in active:
                b.submit()
            # arrivals are admitted while the submitted batches run
            self._admit(now)
            self.queue_depth.append(len(self.queue))
            if not active:
                if not pending and not self.queue and not any(b.running for b in self.blocks):
                    break
                if now > window and not drain:
                    break
                if not any(b.running for b in self.blocks):
                    time.sleep(0.001)
                continue
            for b in active:
                b.wait()
            now = clock() - t0
            for b in active:
                b.collect(now, self.done)
            if not self.keep_results:
                for r in self.done:
                    r.result = None
            if now > window and not drain:
                break
        elapsed = clock() - t0
        return self.report(elapsed)

    def report(self, elapsed: float) -> dict:
        finished = [r for r in self.done if r.status == "finished"]
        latency = np.array([r.finished - r.arrival for r in finished]) if finished else np.array([np.nan])
        days = sum(r.days for r in finished)
        partial = 0.0
        for g in self.blocks:
            for slot, req in g.running.items():
                info = g.engine.slot_info(slot)
                done_steps = req.steps - max(0, g.stop_step[slot] - info["step"])
                partial += done_steps * STEP_MINUTES[g.truncation] / 1440.0
        configure = np.array(self.configure_s + [t for b in self.blocks for t in b.configure_s])
        slots: dict = {}
        for b in self.blocks:
            k = f"T{b.truncation}L{b.levels}"
            slots[k] = slots.get(k, 0) + b.slots
        return {
            "completed": len(finished),
            "failed": sum(r.status == "failed" for r in self.done),
            "p50_s": float(np.nanpercentile(latency, 50)),
            "p99_s": float(np.nanpercentile(latency, 99)),
            "queue_depth_mean": float(np.mean(self.queue_depth)) if self.queue_depth else 0.0,
            "queue_depth_max": int(max(self.queue_depth)) if self.queue_depth else 0,
            "sim_days_per_s": (days + partial) / elapsed,
            "window_s": elapsed,
            "slots": slots,
            "blocks_created": self.blocks_created,
            "blocks_destroyed": self.blocks_destroyed,
            "peak_bytes": self.peak_bytes,
            "setup_on_device": self.setup_on_device,
            "configure_ms_p50": float(np.percentile(configure, 50)) * 1e3 if configure.size else None,
            "configure_ms_p99": float(np.percentile(configure, 99)) * 1e3 if configure.size else None,
        }

    def prewarm(self, resolutions=((21, 5), (21, 10), (42, 5), (42, 10), (63, 5), (63, 10)), seed: int = 1):
        """Creates one block per resolution before serving and configures (then
        releases) a planet in it, so the shared tables and the autotuned launch
        shapes of each block shape exist before the first request: a warm pool.
        The blocks stay and take the first requests; returns the seconds taken."""
        t0 = time.perf_counter()
        for key in resolutions:
            block = self._free_slot(key) or self._grow(key)
            if block is None:
                continue
            planet = planets_mod.make_planet(seed, truncation=key[0], levels=key[1],
                                             timestepMinutes=STEP_MINUTES[key[0]])
            block.engine.configure(0, planet)
            block.engine.release(0)
        return time.perf_counter() - t0

    def close(self):
        for b in self.blocks:
            b.close()
        self.blocks = []


_SLOT_BYTES: dict = {}


def slot_bytes_cached(truncation: int, levels: int) -> int:
    global FIELD_NAMES
    key = (truncation, levels)
    if key not in _SLOT_BYTES:
        if not FIELD_NAMES:
            FIELD_NAMES = _field_names()
        _SLOT_BYTES[key] = slot_bytes(truncation, levels)
    return _SLOT_BYTES[key]


def poisson_requests(rate: float, window: float, seed: int, max_days: float = 365.0, min_days: float = 1.0,
                     resolutions=((21, 5), (21, 10), (42, 5), (42, 10), (63, 5), (63, 10))) -> list[Request]:
    """Poisson arrivals at `rate` per second over `window` seconds, each with a
    resolution drawn uniformly and a duration uniform in [min_days, max_days]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    i = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > window:
            break
        tr, lv = resolutions[rng.integers(len(resolutions))]
        out.append(Request(id=i, truncation=int(tr), levels=int(lv), days=float(rng.uniform(min_days, max_days)),
                           seed=int(rng.integers(1 << 30)), arrival=t))
        i += 1
    return out


if __name__ == "__main__":
    import argparse
    import json

    ap = argparse.ArgumentParser(description="Serve Poisson planet-run requests on one GPU")
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--window", type=float, default=600.0)
    ap.add_argument("--max-days", type=float, default=365.0)
    ap.add_argument("--budget-gb", type=float, default=60.0)
    ap.add_argument("--drain", action="store_true")
    args = ap.parse_args()
    reqs = poisson_requests(args.rate, args.window, seed=5, max_days=args.max_days)
    mix = {}
    for r in reqs:
        mix[(r.truncation, r.levels)] = mix.get((r.truncation, r.levels), 0) + r.days
    total = sum(mix.values())
    mix = {k: v / total for k, v in mix.items()}
    server = Server(budget_bytes=args.budget_gb * 1e9, keep_results=False)
    print(json.dumps(server.run(reqs, args.window, drain=args.drain)))
